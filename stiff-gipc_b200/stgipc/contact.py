"""Contact barrier gradients and Hessians on the GPU (stg_contact_barrier): the triplets
GIPC's _calBarrierGradientAndHessian (GIPC.cu:3149-4988) adds to the Newton system for the
point-point, point-edge, point-triangle and edge-edge pairs of the collision detection."""
from __future__ import annotations

import numpy as np

from . import _lib as _L
from ._lib import check

PP, PE, PT, EE = range(4)


def encode(kind: int, verts) -> tuple:
    """The reference's sign-encoded int4 (GIPC.cuh:49-66) of an unmollified pair: verts are
    (point, other) for PP, (point, e0, e1) for PE, (point, t0, t1, t2) for PT and
    (a0, a1, b0, b1) for EE."""
    v = [int(i) for i in verts]
    if kind == EE:
        return (v[0], v[1], v[2], v[3])
    if kind == PP:
        return (-v[0] - 1, v[1], -1, -1)
    if kind == PE:
        return (-v[0] - 1, v[1], v[2], -1)
    if kind == PT:
        return (-v[0] - 1, v[1], v[2], v[3])
    raise ValueError(f"unknown pair kind {kind}")


def barrier(pairs, x, dhat: float, kappa: float, block_offset: int = 0, stream=None):
    """(rows, cols, blocks [10 P, 9] column-major, grad [P, 12], skipped) for the device
    int32 pairs [P, 4] at the device positions x [V, 3] (float64)."""
    import torch
    if pairs.dtype != torch.int32 or x.dtype != torch.float64 or not (pairs.is_cuda and x.is_cuda):
        raise ValueError("pairs must be a CUDA int32 tensor and x a CUDA float64 tensor")
    pairs, x = pairs.contiguous().view(-1, 4), x.contiguous().view(-1, 3)
    P, dev = pairs.shape[0], x.device
    rows = torch.empty(10 * P, dtype=torch.int32, device=dev)
    cols = torch.empty(10 * P, dtype=torch.int32, device=dev)
    blocks = torch.empty(10 * P, 9, dtype=torch.float64, device=dev)
    grad = torch.empty(P, 12, dtype=torch.float64, device=dev)
    skipped = torch.zeros(1, dtype=torch.int32, device=dev)
    s = None if stream is None else stream.cuda_stream
    check(_L.lib().stg_contact_barrier(P, pairs.data_ptr(), x.data_ptr(), x.shape[0], int(block_offset),
                                       float(dhat), float(kappa), rows.data_ptr(), cols.data_ptr(),
                                       blocks.data_ptr(), grad.data_ptr(), skipped.data_ptr(), s),
          "stg_contact_barrier")
    return rows, cols, blocks, grad, skipped


def scatter_gradient(pairs, grad, num_verts: int):
    """Sum the per-pair gradients [P, 12] into a per-vertex gradient [V, 3] (the reference's
    atomicAdd into _gradient, GIPC.cu:3368-3380), on the device."""
    import torch
    pairs = pairs.view(-1, 4).long()
    x0 = pairs[:, 0]
    pt = x0 < 0
    vid = torch.stack([torch.where(pt, -x0 - 1, x0), pairs[:, 1], pairs[:, 2], pairs[:, 3]], 1)
    g = grad.view(-1, 4, 3)
    valid = (vid >= 0) & (vid < num_verts)
    out = torch.zeros(num_verts, 3, dtype=grad.dtype, device=grad.device)
    out.index_add_(0, vid[valid], g[valid])
    return out


def energy(pairs, x, dhat: float, kappa: float, stream=None):
    """Per-pair barrier energies [P] (device float64) of the pairs at positions x."""
    import torch
    pairs, x = pairs.contiguous().view(-1, 4), x.contiguous().view(-1, 3)
    e = torch.empty(pairs.shape[0], dtype=torch.float64, device=x.device)
    s = None if stream is None else stream.cuda_stream
    check(_L.lib().stg_contact_energy(pairs.shape[0], pairs.data_ptr(), x.data_ptr(), x.shape[0], float(dhat),
                                      float(kappa), e.data_ptr(), s), "stg_contact_energy")
    return e
