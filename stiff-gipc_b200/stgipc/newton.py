"""Implicit-Euler time steps driven by the B200 linear solve: the caller's role of
GIPC::calculateMovingDirection and its line search (GIPC.cu:10730-10741, 10828-10931).

Each Newton iteration builds the incremental potential's triplets and gradient on the GPU
(stgipc.fem, stg_fem_newton_system), solves for the direction with the handle's PCG
(stg_solve_linear_system), bounds the step by continuous collision detection against the
barrier planes (vertex-plane time of impact, scaled by 0.8 as IPC's CCD does), and
backtracks until the potential decreases and no vertex reaches a plane.  A step ends when
the direction's largest entry, divided by dt, falls below tol (IPC's Newton criterion).
With a ContactModel the potential also carries the IPC barrier of the point-triangle /
edge-edge / point-edge / point-point pairs between the surfaces (stgipc.contact: its
triplets join the system, its pairs the MAS connectivity), and the step is also bounded by
the additive CCD of the swept surface pairs (stgipc.ccd, GIPC::self_largestFeasibleStepSize
with slackness 0.8).  The pair sets come from the host-side search of stgipc.scenes.
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
    min_contact_distance: float = float("inf")
    contacts: int = 0
    ccd_alpha: float = 1.0


@dataclasses.dataclass
class ContactModel:
    """Surface contact between bodies: surface triangles (vertex ids), a body id per vertex
    (pairs within one body are ignored; None: every pair sharing no vertex), the squared
    activation distance dhat and the barrier stiffness kappa."""
    tris: np.ndarray
    body: Optional[np.ndarray]
    dhat: float
    kappa: float

    def pairs(self, x_host):
        from . import scenes
        body = self.body if self.body is not None else np.arange(x_host.shape[0])
        return scenes.contact_pairs(x_host, self.tris, body, self.dhat, return_d2=True)

    def energy(self, x):
        """The barrier energy at device positions x [V, 3] (pairs searched at x)."""
        import torch
        from . import contact
        p, _ = self.pairs(x.cpu().numpy())
        if p.shape[0] == 0:
            return 0.0
        return float(contact.energy(torch.from_numpy(p).to(x.device), x, self.dhat, self.kappa).sum())


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


def step(scene: FemScene, solver, tol: float = 1e-6, max_newton: int = 30,
         contact: Optional[ContactModel] = None) -> StepStats:
    """One implicit-Euler step of `scene` (positions and velocities updated in place) with
    the linear solves of `solver` (stgipc.Solver, MAS initialised for the mesh)."""
    import torch
    from . import ccd
    from . import contact as cmod
    from . import scenes
    dt = scene.dt
    dev = scene.device
    g = torch.tensor([0.0, scene.gy, 0.0], dtype=torch.float64, device=dev)
    x_n = scene.pos.clone()
    xtilde = (x_n + dt * scene.vel + dt * dt * g).contiguous()
    x = x_n.clone()
    dx = torch.zeros(3 * scene.V, dtype=torch.float64, device=dev)
    pcg, halvings, it, ncont, amin = [], 0, 0, 0, 1.0

    def potential(xx):
        e, viol = scene.energy(xx, xtilde)
        return (e + (contact.energy(xx) if contact is not None else 0.0)), viol

    for it in range(1, max_newton + 1):
        scene.assemble(x, xtilde)
        rows, cols, blocks, b, P = scene.rows, scene.cols, scene.blocks, scene.b, None
        if contact is not None:
            pairs, _ = contact.pairs(x.cpu().numpy())
            ncont = max(ncont, pairs.shape[0])
            if pairs.shape[0]:
                P = torch.from_numpy(pairs).to(dev)
                cr, cc, cb, cg, sk = cmod.barrier(P, x, contact.dhat, contact.kappa)
                rows, cols = torch.cat([rows, cr]), torch.cat([cols, cc])
                blocks = torch.cat([blocks, cb.reshape(-1)])
                b = b + cmod.scatter_gradient(P, cg, scene.V).reshape(-1)
        dx.zero_()
        st = solver.solve_linear_system(rows, cols, blocks, b, dx, contacts=P)
        pcg.append(st["iterations"])
        p = (-dx).view(scene.V, 3)
        if float(p.abs().max()) / dt < tol:
            break
        alpha = plane_step_bound(scene, x, p)
        if contact is not None:
            cp = scenes.ccd_candidates(x.cpu().numpy(), p.cpu().numpy(), contact.tris, contact.body,
                                       pad=float(np.sqrt(contact.dhat)))
            if cp.shape[0]:
                a_ccd = float(ccd.step_size(torch.from_numpy(cp).to(dev), x, p.contiguous(), slackness=0.8).item())
                amin = min(amin, a_ccd)
                alpha = min(alpha, a_ccd)
        e0, _ = potential(x)
        for _ in range(40):
            xn = (x + alpha * p).contiguous()
            e1, viol = potential(xn)
            if viol == 0 and e1 <= e0:
                break
            alpha *= 0.5
            halvings += 1
        x = xn
    scene.vel = ((x - x_n) / dt).contiguous()
    scene.pos = x.contiguous()
    dmin = float("inf")
    if contact is not None:
        _, d2 = contact.pairs(x.cpu().numpy())
        if d2.size:
            dmin = float(np.sqrt(d2.min()))
    return StepStats(it, pcg, halvings, min_plane_distance(scene, x), dmin, ncont, amin)


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
               solver_hook=None, checkpoint: Optional[str] = None, contact: Optional[ContactModel] = None):
    """Run `steps` implicit-Euler steps from a scene state (stgipc.scenes ..., state_only=True);
    returns (positions after each step as host arrays, step statistics).  With
    `checkpoint`, positions and velocities of every step are written there after each step
    (resume with resume_state).  contact: surface contact (ContactModel)."""
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
        stats.append(step(scene, solver, tol, contact=contact))
        out.append(scene.pos.cpu().numpy().copy())
        vels.append(scene.vel.cpu().numpy().copy())
        if checkpoint:
            save_checkpoint(checkpoint, out, vels, k + 1)
    solver.close()
    return out, stats
