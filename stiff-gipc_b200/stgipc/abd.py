"""Affine bodies (ABD) on the GPU: the body inertia + orthogonality terms
(stg_abd_body_system), body-point positions (stg_abd_points), the mapping of point-level
contact triplets onto body DOFs (stg_abd_map_triplets) and the body gradient
(stg_abd_gather_gradient) -- GIPC's ABDSystem::setup_abd_system_gradient_hessian
(abd_system/abd_system_function/setup_abd_system_gradient_and_hessian.cu)."""
from __future__ import annotations

from . import _lib as _L
from ._lib import check


def _p(t):
    return None if t is None else t.data_ptr()


def _s(stream):
    return None if stream is None else stream.cuda_stream


def body_system(q, q_tilde, mass, volume, kappa, dt, fixed=None, stream=None):
    """(rows, cols, blocks [10 N, 9] column-major, grad [N, 12]) device tensors."""
    import torch
    N, dev = q.shape[0], q.device
    rows = torch.empty(10 * N, dtype=torch.int32, device=dev)
    cols = torch.empty(10 * N, dtype=torch.int32, device=dev)
    blocks = torch.empty(10 * N, 9, dtype=torch.float64, device=dev)
    grad = torch.empty(N, 12, dtype=torch.float64, device=dev)
    check(_L.lib().stg_abd_body_system(N, _p(q), _p(q_tilde), _p(mass), _p(volume), _p(fixed), float(kappa),
                                       float(dt), _p(rows), _p(cols), _p(blocks), _p(grad), _s(stream)),
          "stg_abd_body_system")
    return rows, cols, blocks, grad


def map_triplets(rows, cols, blocks, abd_points, point_body, xbar, bodies, stream=None):
    """16 global triplets per point-level triplet; returns (rows, cols, blocks [16 T, 9], bad)."""
    import torch
    T, dev = rows.numel(), rows.device
    orow = torch.empty(16 * T, dtype=torch.int32, device=dev)
    ocol = torch.empty(16 * T, dtype=torch.int32, device=dev)
    oblk = torch.empty(16 * T, 9, dtype=torch.float64, device=dev)
    bad = torch.zeros(1, dtype=torch.int32, device=dev)
    check(_L.lib().stg_abd_map_triplets(T, _p(rows), _p(cols), _p(blocks), int(abd_points), _p(point_body),
                                        _p(xbar), int(bodies), _p(orow), _p(ocol), _p(oblk), _p(bad), _s(stream)),
          "stg_abd_map_triplets")
    return orow, ocol, oblk, bad


def points(point_body, xbar, q, stream=None):
    import torch
    P = point_body.numel()
    x = torch.empty(P, 3, dtype=torch.float64, device=q.device)
    check(_L.lib().stg_abd_points(P, _p(point_body), _p(xbar), _p(q), _p(x), _s(stream)), "stg_abd_points")
    return x


def gather_gradient(body_point_start, xbar, point_grad, body_grad, stream=None):
    """body_grad += sum_i J_i^T g_i per body (in place)."""
    N = body_point_start.numel() - 1
    check(_L.lib().stg_abd_gather_gradient(N, _p(body_point_start), _p(xbar), _p(point_grad), _p(body_grad),
                                           _s(stream)), "stg_abd_gather_gradient")
    return body_grad


def coupled_system(scene, device="cuda", stream=None):
    """The triplets and right-hand side of an AbdScene's Newton iteration, built on the device:
    body terms (10 triplets per body), contact barrier triplets over the point numbering mapped
    onto body DOFs (16 per contact triplet), and the FEM triplets shifted past the body rows.
    Returns (rows, cols, blocks [T, 9], b) device tensors; block row 4 N + v is FEM vertex v."""
    import numpy as np
    import torch
    from . import contact
    dev = torch.device(device)
    t = lambda a, dt_: torch.from_numpy(np.ascontiguousarray(a, dt_)).to(dev)
    N, P, V = scene.bodies, scene.abd_points, scene.fem.num_verts
    q, qt = t(scene.q, np.float64), t(scene.q_tilde, np.float64)
    pb, xbar = t(scene.point_body, np.int32), t(scene.xbar, np.float64)
    br, bc, bb, bg = body_system(q, qt, t(scene.mass, np.float64), t(scene.volume, np.float64), scene.kappa,
                                 scene.dt, stream=stream)
    xa = points(pb, xbar, q, stream=stream)
    allpos = torch.cat([xa, t(scene.fem.pos, np.float64)])
    pairs = t(scene.contacts, np.int32)
    cr, cc, cb, cg, sk = contact.barrier(pairs, allpos, scene.dhat, scene.kappa_contact, stream=stream)
    mr, mc, mb, bad = map_triplets(cr, cc, cb, P, pb, xbar, N, stream=stream)
    pg = contact.scatter_gradient(pairs, cg, P + V)
    gather_gradient(t(scene.body_point_start, np.int32), xbar, pg[:P].contiguous(), bg, stream=stream)
    b = torch.cat([bg.reshape(-1), t(scene.fem.b, np.float64) + pg[P:].reshape(-1)])
    rows = torch.cat([br, mr, t(scene.fem.rows + 4 * N, np.int32)])
    cols = torch.cat([bc, mc, t(scene.fem.cols + 4 * N, np.int32)])
    blocks = torch.cat([bb, mb, t(scene.fem.blocks, np.float64)])
    if int(sk.item()) or int(bad.item()):
        raise ValueError(f"coupled_system: {int(sk.item())} contacts skipped, {int(bad.item())} bad triplets")
    return rows, cols, blocks, b
