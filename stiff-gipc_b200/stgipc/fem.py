"""The Hessian producer on the GPU (stg_fem_newton_system): the triplets and gradient of one
implicit-Euler Newton iteration of a tet mesh, as GIPC hands them to the linear solve."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as _L
from ._lib import check


def newton_system(rest, pos, vel, tets, E, nu, rho, dt, barriers=(), gravity_y=-9.8, device="cuda", stream=None):
    """(rows, cols, blocks [T, 9] column-major, b) device tensors for 10 tets + verts
    triplets, from host arrays.  barriers: (normal, offset, dhat, kappa) planes n.x = offset."""
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
    check(_L.lib().stg_fem_newton_system(V, ptr(d_rest), ptr(d_pos), ptr(d_vel), None, T, ptr(d_tets), ptr(d_E), float(nu),
                                         float(rho), float(dt), float(gravity_y), len(planes), ptr(d_planes), ptr(rows),
                                         ptr(cols), ptr(blocks), ptr(b), ptr(scratch), nb, s), "stg_fem_newton_system")
    return rows, cols, blocks.view(n, 9), b


class FemScene:
    """A tet mesh on the device for Newton steps: rest / current positions, velocities,
    connectivity, per-tet Young's modulus, barrier planes, and the reusable buffers of the
    Hessian producer and energy kernels."""

    def __init__(self, state: dict, gravity_y=-9.8, device="cuda"):
        import torch
        dev = self.device = torch.device(device)
        t = lambda a, dt_: torch.from_numpy(np.ascontiguousarray(a, dt_)).to(dev)
        self.rest = t(state["pos_rest"], np.float64)
        self.pos = t(state["pos"], np.float64)
        self.vel = t(state["vel"], np.float64)
        self.tets = t(state["tets"], np.int32)
        self.E = t(state["E"], np.float64)
        self.nu, self.rho, self.dt, self.gy = float(state["nu"]), float(state["rho"]), float(state["dt"]), float(gravity_y)
        pl = np.array([[*n, o, dh, k] for (n, o, dh, k) in state["barriers"]], np.float64).reshape(-1, 6)
        self.nplanes = len(pl)
        self.planes = t(pl, np.float64) if len(pl) else None
        self.V, self.T = int(self.rest.shape[0]), int(self.tets.shape[0])
        n = 10 * self.T + self.V
        self.rows = torch.empty(n, dtype=torch.int32, device=dev)
        self.cols = torch.empty(n, dtype=torch.int32, device=dev)
        self.blocks = torch.empty(n * 9, dtype=torch.float64, device=dev)
        self.b = torch.empty(3 * self.V, dtype=torch.float64, device=dev)
        nb = int(_L.lib().stg_fem_scratch_bytes(self.V, self.T))
        self.scratch = torch.empty(nb, dtype=torch.uint8, device=dev)

    def _p(self, x):
        return None if x is None else x.data_ptr()

    def assemble(self, x, xtilde):
        """Triplets and gradient of the incremental potential at x (device [V, 3])."""
        p = self._p
        check(_L.lib().stg_fem_newton_system(self.V, p(self.rest), p(x), None, p(xtilde), self.T, p(self.tets), p(self.E),
                                             self.nu, self.rho, self.dt, self.gy, self.nplanes, p(self.planes),
                                             p(self.rows), p(self.cols), p(self.blocks), p(self.b), p(self.scratch),
                                             self.scratch.numel(), None), "stg_fem_newton_system")

    def energy(self, x, xtilde):
        """(incremental potential at x, vertices on or behind a plane)."""
        p = self._p
        e, v = C.c_double(), C.c_int()
        check(_L.lib().stg_fem_energy(self.V, p(self.rest), p(x), p(xtilde), self.T, p(self.tets), p(self.E), self.nu,
                                      self.rho, self.dt, self.nplanes, p(self.planes), p(self.scratch),
                                      self.scratch.numel(), C.byref(e), C.byref(v), None), "stg_fem_energy")
        return e.value, v.value
