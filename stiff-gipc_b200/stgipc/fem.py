"""The Hessian producer on the GPU (stg_fem_newton_system): the triplets and gradient of one
implicit-Euler Newton iteration of a tet mesh, as GIPC hands them to the linear solve."""
from __future__ import annotations

import numpy as np

from . import _lib as _L
from ._lib import check


def newton_system(rest, pos, vel, tets, E, nu, rho, dt, barriers=(), gravity_y=-9.8, device="cuda", stream=None):
    """(rows, cols, blocks [T, 9] column-major, b) device tensors for 10 tets + verts
    triplets.  barriers: (normal, offset, dhat, kappa) planes n.x = offset."""
    import torch
    dev = torch.device(device)
    t = lambda a, dt_: torch.from_numpy(np.ascontiguousarray(a, dt_)).to(dev)
    V, T = int(rest.shape[0]), int(tets.shape[0])
    planes = np.array([[*n, o, dh, k] for (n, o, dh, k) in barriers], np.float64).reshape(-1, 6)
    d_rest, d_pos, d_vel = t(rest, np.float64), t(pos, np.float64), t(vel, np.float64)
    d_tets, d_E = t(tets, np.int32), t(E, np.float64)
    d_planes = t(planes, np.float64) if len(planes) else None
    n = 10 * T + V
    rows = torch.empty(n, dtype=torch.int32, device=dev)
    cols = torch.empty(n, dtype=torch.int32, device=dev)
    blocks = torch.empty(n * 9, dtype=torch.float64, device=dev)
    b = torch.empty(3 * V, dtype=torch.float64, device=dev)
    nb = int(_L.lib().stg_fem_scratch_bytes(V, T))
    scratch = torch.empty(nb, dtype=torch.uint8, device=dev)
    s = None if stream is None else stream.cuda_stream
    ptr = lambda x: None if x is None else x.data_ptr()
    check(_L.lib().stg_fem_newton_system(V, ptr(d_rest), ptr(d_pos), ptr(d_vel), T, ptr(d_tets), ptr(d_E), float(nu),
                                         float(rho), float(dt), float(gravity_y), len(planes), ptr(d_planes), ptr(rows),
                                         ptr(cols), ptr(blocks), ptr(b), ptr(scratch), nb, s), "stg_fem_newton_system")
    return rows, cols, blocks.view(n, 9), b
