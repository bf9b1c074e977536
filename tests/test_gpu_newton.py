"""GPU: the incremental potential (stg_fem_energy) against a numpy evaluation and against
the Hessian producer's gradient (central differences), and multi-step implicit-Euler
trajectories driven by the linear solve (stgipc.newton): the FP32 path's positions match
the FP64 path's within 1e-6 m, and no vertex ever reaches the ground (CCD + line search)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _energy_numpy(st, x, xtilde, gy=-9.8):
    rest, tets, E, nu, rho, dt = st["pos_rest"], st["tets"], st["E"], st["nu"], st["rho"], st["dt"]
    Dm = np.transpose(rest[tets[:, 1:]] - rest[tets[:, :1]], (0, 2, 1))
    vol = np.abs(np.linalg.det(Dm)) / 6.0
    F = np.transpose(x[tets[:, 1:]] - x[tets[:, :1]], (0, 2, 1)) @ np.linalg.inv(Dm)
    mu = E / (2 * (1 + nu))
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    J = np.linalg.det(F)
    psi = 0.5 * mu * ((F ** 2).sum(axis=(1, 2)) - 3) + 0.5 * lam * (J - 1 - mu / lam) ** 2
    e = (dt * dt * vol * psi).sum()
    m = np.zeros(x.shape[0])
    for a in range(4):
        np.add.at(m, tets[:, a], rho * vol / 4)
    e += 0.5 * (m * ((x - xtilde) ** 2).sum(axis=1)).sum()
    for n, o, dh, k in st["barriers"]:
        d = x @ np.asarray(n) - o
        act = d < dh
        s = d[act] ** 2
        e += (k * (-(s - dh * dh) ** 2 * np.log(s / (dh * dh)))).sum()
    return e


def test_energy_matches_numpy_and_gradient(dev):
    import torch
    from stgipc import fem, scenes
    st = scenes.make_heterogeneous_cube(n=5, seed=2500, state_only=True)
    sc = fem.FemScene(st, device=dev)
    g = np.array([0.0, -9.8, 0.0])
    xt = st["pos"] + st["dt"] * st["vel"] + st["dt"] ** 2 * g
    xtilde = torch.from_numpy(xt).to(dev)
    x = sc.pos.clone()
    e_gpu, viol = sc.energy(x, xtilde)
    assert viol == 0
    e_np = _energy_numpy(st, st["pos"], xt)
    assert abs(e_gpu - e_np) <= 1e-11 * abs(e_np)
    # the producer's gradient is the potential's: central differences along a random direction
    sc.assemble(x, xtilde)
    grad = sc.b.cpu().numpy()
    rng = np.random.default_rng(0)
    d = rng.standard_normal(x.shape) * 1e-7
    dd = torch.from_numpy(d).to(dev)
    ep, _ = sc.energy((x + dd).contiguous(), xtilde)
    em, _ = sc.energy((x - dd).contiguous(), xtilde)
    fd = (ep - em) / 2
    assert abs(fd - grad @ d.reshape(-1)) <= 1e-5 * abs(fd) + 1e-14


def test_trajectory_fp32_matches_fp64_without_interpenetration(dev):
    from stgipc import PCGSolverConfig, newton, scenes
    st = scenes.make_cube_drop(n=6, seed=2501, state_only=True)
    steps = 8
    cfg64 = PCGSolverConfig(precision="fp64", stop_rule="relative_residual", global_tol_rate=1e-4)
    cfg32 = PCGSolverConfig(precision="fp32", stop_rule="relative_residual", global_tol_rate=1e-4)
    x64, s64 = newton.trajectory(st, steps, cfg64, device=dev)
    x32, s32 = newton.trajectory(st, steps, cfg32, device=dev)
    for k in range(steps):
        assert np.abs(x32[k] - x64[k]).max() <= 1e-6, (k, np.abs(x32[k] - x64[k]).max())
        assert s64[k].min_plane_distance > 0 and s32[k].min_plane_distance > 0
    # the cube reached the ground: the barrier was active (within dhat) at some step
    assert min(s.min_plane_distance for s in s64) < 1e-3
    assert all(s.newton_iterations < 30 for s in s64 + s32)


def test_trajectory_checkpoint_resume(dev, tmp_path):
    """A trajectory resumed from the checkpoint after step 2 reproduces the uninterrupted
    run's later steps bit for bit (the solve and the producer are deterministic)."""
    from stgipc import PCGSolverConfig, newton, scenes
    st = scenes.make_cube_drop(n=5, seed=2502, state_only=True)
    cfg = PCGSolverConfig(precision="fp32", stop_rule="relative_residual", global_tol_rate=1e-4)
    ck = str(tmp_path / "traj.npz")
    full, _ = newton.trajectory(st, 4, cfg, device=dev, checkpoint=ck)
    z = np.load(ck)
    assert int(z["step"]) == 4 and z["pos"].shape == (4, st["pos"].shape[0], 3)
    rest, _ = newton.trajectory(newton.resume_state(st, ck, step=2), 2, cfg, device=dev)
    np.testing.assert_array_equal(rest[0], full[2])
    np.testing.assert_array_equal(rest[1], full[3])
