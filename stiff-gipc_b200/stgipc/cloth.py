"""Cloth terms on the GPU: the Baraff-Witkin membrane (stg_cloth_membrane) and quadratic
bending (stg_cloth_bending) of StiffGIPC's triangle FEM (femEnergy.cu:2146-2216, 2620-2755),
and the assembly of the cloth-on-ball Newton system."""
from __future__ import annotations

import numpy as np

from . import _lib as _L
from ._lib import check


def _p(t):
    return None if t is None else t.data_ptr()


def membrane(tris, dminv, area, x, stretch, shear, strain_rate, dt, block_offset=0, stream=None):
    """(rows, cols, blocks [6 T, 9], grad [T, 9], bad) device tensors."""
    import torch
    T, dev = tris.shape[0], x.device
    rows = torch.empty(6 * T, dtype=torch.int32, device=dev)
    cols = torch.empty(6 * T, dtype=torch.int32, device=dev)
    blocks = torch.empty(6 * T, 9, dtype=torch.float64, device=dev)
    grad = torch.empty(T, 9, dtype=torch.float64, device=dev)
    bad = torch.zeros(1, dtype=torch.int32, device=dev)
    check(_L.lib().stg_cloth_membrane(T, _p(tris), _p(dminv), _p(area), _p(x), x.numel() // 3, float(stretch),
                                      float(shear), float(strain_rate), float(dt), int(block_offset), _p(rows),
                                      _p(cols), _p(blocks), _p(grad), _p(bad),
                                      None if stream is None else stream.cuda_stream), "stg_cloth_membrane")
    return rows, cols, blocks, grad, bad


def bending(stencil, Q, length, x, bend, dt, block_offset=0, stream=None):
    """(rows, cols, blocks [10 E, 9], grad [E, 12], bad) device tensors."""
    import torch
    E, dev = stencil.shape[0], x.device
    rows = torch.empty(10 * E, dtype=torch.int32, device=dev)
    cols = torch.empty(10 * E, dtype=torch.int32, device=dev)
    blocks = torch.empty(10 * E, 9, dtype=torch.float64, device=dev)
    grad = torch.empty(E, 12, dtype=torch.float64, device=dev)
    bad = torch.zeros(1, dtype=torch.int32, device=dev)
    check(_L.lib().stg_cloth_bending(E, _p(stencil), _p(Q), _p(length), _p(x), x.numel() // 3, float(bend),
                                     float(dt), int(block_offset), _p(rows), _p(cols), _p(blocks), _p(grad), _p(bad),
                                     None if stream is None else stream.cuda_stream), "stg_cloth_bending")
    return rows, cols, blocks, grad, bad


def _scatter(idx, g, V):
    """Sum per-element gradients [K, k * 3] over their vertex ids [K, k] (negative ids skipped)."""
    import torch
    idx = idx.long()
    g = g.view(idx.shape[0], idx.shape[1], 3)
    ok = idx >= 0
    out = torch.zeros(V, 3, dtype=g.dtype, device=g.device)
    out.index_add_(0, idx[ok], g[ok])
    return out


def cloth_system(scene, device="cuda", stream=None):
    """The triplets and right-hand side of a ClothScene's Newton iteration, built on the device:
    the ball's and the masses' triplets (scene.base), the cloth membrane (6 per triangle) and
    bending (10 per stencil) triplets, and the contact barriers.  Returns (rows, cols,
    blocks [T, 9], b, contacts) device tensors."""
    import torch
    from . import contact
    dev = torch.device(device)
    t = lambda a, dt_: torch.from_numpy(np.ascontiguousarray(a, dt_)).to(dev)
    base = scene.base
    V = base.num_verts
    x = t(base.pos, np.float64)
    tris = t(scene.tris, np.int32)
    mr, mc, mb, mg, bad1 = membrane(tris, t(scene.dminv, np.float64), t(scene.area, np.float64), x, scene.stretch,
                                    scene.shear, scene.strain_rate, scene.dt, stream=stream)
    st = t(scene.stencil, np.int32)
    br, bc, bb, bg, bad2 = bending(st, t(scene.Q, np.float64), t(scene.elen, np.float64), x, scene.bend, scene.dt,
                                   stream=stream)
    P = t(scene.contacts, np.int32)
    cr, cc, cb, cg, sk = contact.barrier(P, x, scene.dhat, scene.kappa, stream=stream)
    if int(bad1.item()) or int(bad2.item()) or int(sk.item()):
        raise ValueError("cloth_system: invalid elements or contacts")
    b = (t(base.b, np.float64).view(V, 3) + _scatter(tris, mg, V) + _scatter(st, bg, V)
         + contact.scatter_gradient(P, cg, V)).reshape(-1)
    rows = torch.cat([t(base.rows, np.int32), mr, br, cr])
    cols = torch.cat([t(base.cols, np.int32), mc, bc, cc])
    blocks = torch.cat([t(base.blocks, np.float64), mb, bb, cb])
    return rows, cols, blocks, b, P
