"""Implicit-Euler time steps driven by the B200 linear solve: the caller's role of
GIPC::calculateMovingDirection and its line search (GIPC.cu:10730-10741, 10828-10931).

Each Newton iteration builds the incremental potential's triplets and gradient on the GPU
(stgipc.fem, stg_fem_newton_system), solves for the direction with the handle's PCG
(stg_solve_linear_system), bounds the step by continuous collision detection against the
barrier planes (vertex-plane time of impact, scaled by 0.8 as IPC's CCD does), and
backtracks until the potential decreases and no vertex reaches a plane.  A step ends when
the direction's largest entry, divided by dt, falls below tol (IPC's Newton criterion).
Only plane barriers are modelled: the synthetic scenes have no triangle contacts.
"""
from __future__ import annotations

import dataclasses
from typing import List, Optional

import numpy as np

from .fem import FemScene


@dataclasses.dataclass
class StepStats:
    newton_iterations: int
    pcg_iterations: List[int]
    line_search_halvings: int
    min_plane_distance: float


def plane_step_bound(scene: FemScene, x, p) -> float:
    """Largest alpha <= 1 such that x + alpha p keeps every vertex in front of every plane,
    times 0.8 (exact for vertex-plane pairs; the ccd of GIPC.cu:10828-10931 limited to the
    barriers modelled here)."""
    import torch
    if scene.nplanes == 0:
        return 1.0
    n = scene.planes[:, :3]                                    # [P, 3]
    d = x @ n.T - scene.planes[:, 3][None, :]                  # [V, P] distances
    rate = p @ n.T                                             # [V, P] approach rates
    toi = torch.where(rate < 0, d / (-rate), torch.full_like(d, float("inf")))
    a = float(torch.clamp(toi.min(), max=1.25))
    return min(1.0, 0.8 * a)


def min_plane_distance(scene: FemScene, x) -> float:
    if scene.nplanes == 0:
        return float("inf")
    d = x @ scene.planes[:, :3].T - scene.planes[:, 3][None, :]
    return float(d.min())


def step(scene: FemScene, solver, tol: float = 1e-6, max_newton: int = 30) -> StepStats:
    """One implicit-Euler step of `scene` (positions and velocities updated in place) with
    the linear solves of `solver` (stgipc.Solver, MAS initialised for the mesh)."""
    import torch
    dt = scene.dt
    g = torch.tensor([0.0, scene.gy, 0.0], dtype=torch.float64, device=scene.device)
    x_n = scene.pos.clone()
    xtilde = (x_n + dt * scene.vel + dt * dt * g).contiguous()
    x = x_n.clone()
    dx = torch.zeros(3 * scene.V, dtype=torch.float64, device=scene.device)
    pcg, halvings, it = [], 0, 0
    for it in range(1, max_newton + 1):
        scene.assemble(x, xtilde)
        dx.zero_()
        st = solver.solve_linear_system(scene.rows, scene.cols, scene.blocks, scene.b, dx)
        pcg.append(st["iterations"])
        p = (-dx).view(scene.V, 3)
        if float(p.abs().max()) / dt < tol:
            break
        alpha = plane_step_bound(scene, x, p)
        e0, _ = scene.energy(x, xtilde)
        for _ in range(40):
            xn = (x + alpha * p).contiguous()
            e1, viol = scene.energy(xn, xtilde)
            if viol == 0 and e1 <= e0:
                break
            alpha *= 0.5
            halvings += 1
        x = xn
    scene.vel = ((x - x_n) / dt).contiguous()
    scene.pos = x.contiguous()
    return StepStats(it, pcg, halvings, min_plane_distance(scene, x))


def save_checkpoint(path: str, positions, velocities, step: int):
    """A trajectory checkpoint: positions and velocities after each step so far (FP64,
    [steps][V][3]) and the number of steps they cover."""
    np.savez(path, pos=np.asarray(positions), vel=np.asarray(velocities), step=np.int64(step))


def resume_state(state: dict, path: str, step: Optional[int] = None) -> dict:
    """The scene state after step `step` (default: the last one) of a checkpoint: the
    material, mesh and barriers of `state`, positions and velocities from the file."""
    z = np.load(path)
    k = int(z["step"]) if step is None else int(step)
    out = dict(state)
    out["pos"] = z["pos"][k - 1].copy()
    out["vel"] = z["vel"][k - 1].copy()
    return out


def trajectory(state: dict, steps: int, config=None, tol: float = 1e-6, device="cuda", bank: int = 16,
               solver_hook=None, checkpoint: Optional[str] = None):
    """Run `steps` implicit-Euler steps from a scene state (stgipc.scenes ..., state_only=True);
    returns (positions after each step as host arrays, step statistics).  With
    `checkpoint`, positions and velocities of every step are written there after each step
    (resume with resume_state)."""
    from . import scenes
    from .linear_system import PCGSolverConfig, Solver
    scene = FemScene(state, device=device)
    V = scene.V
    start, num, nlist = scenes.vert_neighbors(V, state["tets"])
    pm, rm = scenes.mas_partition_morton(V, bank)
    solver = Solver(config or PCGSolverConfig(bank_size=bank, stop_rule="relative_residual"))
    solver.mas_init(V, start, num, nlist, pm, rm)
    if solver_hook:
        solver_hook(solver)
    out, vels, stats = [], [], []
    for k in range(steps):
        stats.append(step(scene, solver, tol))
        out.append(scene.pos.cpu().numpy().copy())
        vels.append(scene.vel.cpu().numpy().copy())
        if checkpoint:
            save_checkpoint(checkpoint, out, vels, k + 1)
    solver.close()
    return out, stats
