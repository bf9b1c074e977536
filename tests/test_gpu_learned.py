"""GPU: the learned coarse correction through the C ABI against the CPU oracle
(oracle/net_oracle.py): the coarse level's graph against the Galerkin operator P A P^T,
the forward pass, the gradient of the training step and the Adam update, the sample
recorder, and the flexible PCG with the network inside (convergence, the FP64-residual
fallback, and what a trained network gains over plain MAS)."""
import numpy as np
import pytest

from conftest import cube_system

pytestmark = pytest.mark.gpu


def _t(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def _solver(s, level, dev, **kw):
    from stgipc import PCGSolverConfig, Solver
    cfg = dict(stop_rule="relative_residual", global_tol_rate=1e-4)
    cfg.update(kw)
    solver = Solver(PCGSolverConfig(**cfg))
    solver.mas_init(s.num_verts, s.neighbor_start, s.neighbor_num, s.neighbor_list, *s.slot_maps(16))
    solver.net_configure(level)
    return solver


def _solve(solver, s, dev):
    x = _t(np.zeros(s.n), dev)
    st = solver.solve_linear_system(_t(s.rows, dev), _t(s.cols, dev), _t(s.blocks.reshape(-1), dev), _t(s.b, dev), x)
    return st, x


def _galerkin(s, solver, level):
    """Dense P A P^T of the level from the oracle's converted BCOO and the exported
    hierarchy (vertex -> level node)."""
    from oracle import oracle as orc
    r, c, bl = orc.convert(s.rows, s.cols, s.blocks)
    pm, _ = s.slot_maps(16)
    hier = solver.export_hierarchy(len(pm))
    ls = hier["level_size"]
    n_l, begin = int(ls[level][0]), int(ls[level][1])
    node = hier["coarse_table"][:, level - 1] - begin
    A = np.zeros((3 * n_l, 3 * n_l))
    for k in range(r.size):
        B = bl[k].reshape(3, 3).T
        I, J = node[r[k]], node[c[k]]
        A[3 * I:3 * I + 3, 3 * J:3 * J + 3] += B
        if r[k] != c[k]:
            A[3 * J:3 * J + 3, 3 * I:3 * I + 3] += B.T
    return A, n_l, node


def test_graph_is_galerkin_operator(dev):
    from oracle import net_oracle as no
    s = cube_system(8)
    level = 1
    solver = _solver(s, level, dev)
    _solve(solver, s, dev)
    g = solver.net_graph().numpy()
    A, n_l, _ = _galerkin(s, solver, level)
    assert g["n"] == n_l
    scale = np.abs(A).max()
    for i in range(n_l):
        np.testing.assert_allclose(g["dblk"][i], A[3 * i:3 * i + 3, 3 * i:3 * i + 3], atol=1e-6 * scale, rtol=1e-5)
        cols = g["col"][g["row"][i]:g["row"][i + 1]]
        assert np.all(np.diff(cols) > 0)
        for e in range(g["row"][i], g["row"][i + 1]):
            j = g["col"][e]
            np.testing.assert_allclose(g["oblk"][e], A[3 * i:3 * i + 3, 3 * j:3 * j + 3], atol=1e-6 * scale, rtol=1e-5)
    # every nonzero off-diagonal block is an entry
    nz = sum(1 for i in range(n_l) for j in range(n_l)
             if i != j and np.abs(A[3 * i:3 * i + 3, 3 * j:3 * j + 3]).max() > 0)
    assert nz == g["row"][-1]
    # weights and features as the oracle's graph builder makes them from the same operator
    keys = [(i, j) for i in range(n_l) for j in range(i, n_l)
            if i == j or np.abs(A[3 * i:3 * i + 3, 3 * j:3 * j + 3]).max() > 0]
    ub = np.array([A[3 * i:3 * i + 3, 3 * j:3 * j + 3].T.reshape(9) for i, j in keys])
    go = no.build_graph(n_l, np.array([k[0] for k in keys]), np.array([k[1] for k in keys]), ub)
    np.testing.assert_allclose(g["w"], go["w"], rtol=1e-5)
    np.testing.assert_allclose(g["feat"], go["feat"], atol=1e-5)


def _level_case(dev, level=1, S=3, seed=11, wscale=0.15):
    from oracle import net_oracle as no
    s = cube_system(8)
    solver = _solver(s, level, dev)
    _solve(solver, s, dev)
    G = solver.net_graph()
    g = G.numpy()
    rng = np.random.default_rng(seed)
    n = g["n"]
    rcs = [rng.standard_normal((n, 3)).astype(np.float32) for _ in range(S)]
    D = g["dblk"].astype(np.float64)
    zcs = [(np.linalg.solve(D, r[..., None].astype(np.float64))[..., 0] * (0.5 + 0.5 * rng.random())).astype(np.float32)
           for r in rcs]
    p = (rng.standard_normal(no.COUNT) * wscale).astype(np.float32)
    pad = lambda a: np.concatenate([a, np.zeros((a.shape[0], 1), np.float32)], axis=1)
    rc = _t(np.stack([pad(r) for r in rcs]), dev)
    zc = _t(np.stack([pad(z) for z in zcs]), dev)
    return G, g, rcs, zcs, p, rc, zc


def _rel(a, b):
    return np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30)


def test_forward_matches_oracle(dev):
    from oracle import net_oracle as no
    from stgipc import learned
    G, g, rcs, zcs, p, rc, zc = _level_case(dev)
    d = learned.forward(G, rc, zc, _t(p, dev), len(rcs)).cpu().numpy()
    for s_ in range(len(rcs)):
        de, _ = no.forward(g, rcs[s_], zcs[s_], p.astype(np.float64))
        assert _rel(d[s_, :, :3], de) < 5e-3
        assert np.all(d[s_, :, 3] == 0)


def test_gradient_and_adam_match_oracle(dev):
    from oracle import net_oracle as no
    from stgipc import learned
    G, g, rcs, zcs, p, rc, zc = _level_case(dev, S=2, seed=12)
    tr = learned.Trainer(p, dev)
    loss = tr.step(G, rc, zc, 2, 0.0).cpu().numpy()
    grad = tr.grad.cpu().numpy().astype(np.float64)
    le, ge = no.batch_loss_grad(g, rcs, zcs, p.astype(np.float64))
    np.testing.assert_allclose(loss, le, rtol=1e-4, atol=1e-6)
    for name, (o, shp) in no.P.items():
        k = int(np.prod(shp))
        if name in ("Wo", "bo"):
            k = 3 * (shp[1] if name == "Wo" else 1)  # outputs 3..7 carry no gradient
            assert np.all(grad[o + k:o + int(np.prod(shp))] == 0)
        assert _rel(grad[o:o + k], ge[o:o + k]) < 5e-3, name
    # one Adam step from zero moments on the gradient the kernels computed
    lr = 1e-3
    tr2 = learned.Trainer(p, dev)
    tr2.step(G, rc, zc, 2, lr)
    g2 = tr2.grad.cpu().numpy().astype(np.float64)
    pe, _, _ = no.adam(p.astype(np.float64), g2, np.zeros(no.COUNT), np.zeros(no.COUNT), 1, lr)
    np.testing.assert_allclose(tr2.params.cpu().numpy(), pe, rtol=1e-5, atol=1e-7)


def test_recorder_restricts_the_residual(dev):
    """Sample 0 is r0 = b restricted to the level (sums over the level's aggregates)."""
    s = cube_system(8)
    level = 2
    solver = _solver(s, level, dev)
    _solve(solver, s, dev)
    G = solver.net_graph()
    import torch
    cap = 8
    rc = torch.zeros(cap * G.nodes * 4, dtype=torch.float32, device=dev)
    zc = torch.zeros_like(rc)
    solver.net_record(rc, zc, cap, 3)
    st, _ = _solve(solver, s, dev)
    cnt = solver.net_recorded()
    assert cnt == min(cap, (st["iterations"] - 1) // 3 + 1) or cnt == min(cap, st["iterations"] // 3 + 1)
    _, n_l, node = _galerkin(s, solver, level)
    want = np.zeros((n_l, 3))
    np.add.at(want, node, s.b.reshape(-1, 3))
    got = rc.view(cap, G.nodes, 4)[0, :, :3].cpu().numpy()
    np.testing.assert_allclose(got, want, rtol=1e-4, atol=1e-5 * np.abs(want).max())
    assert np.isfinite(zc.cpu().numpy()).all()


@pytest.mark.parametrize("prec,loop", [("fp64", "graph"), ("fp32", "graph"), ("fp32", "host")])
def test_learned_solve_converges(dev, prec, loop):
    """Untrained network inside the flexible PCG: same tolerance reached, graph and host
    loops identical."""
    from stgipc import learned
    s = cube_system(10)
    solver = _solver(s, 1, dev, precision=prec, loop=loop, learned=True)
    solver.net_set_params(_t(learned.init_params(0, head_scale=0.05), dev))
    st, x = _solve(solver, s, dev)
    assert st["status"] == 0
    assert st["rel_residual"] <= 1.2e-4
    plain = _solver(s, 1, dev, precision=prec, loop=loop)
    stp, _ = _solve(plain, s, dev)
    assert st["iterations"] <= 2 * stp["iterations"] + 5


def test_fallback_to_plain_mas(dev):
    """A harmful network is switched off by the FP64 residual judge and the solve still
    converges."""
    from stgipc import learned
    s = cube_system(10)
    p = learned.init_params(1, head_scale=0.0)
    p[learned.OFF["bo"]:learned.OFF["bo"] + 3] = 50.0  # a large constant correction
    solver = _solver(s, 1, dev, precision="fp32", learned=True, refine_interval=1)
    solver.net_set_params(_t(p, dev))
    st, _ = _solve(solver, s, dev)
    assert st["status"] == 0 and st["rel_residual"] <= 1.2e-4
    assert st["learned_rejected"] == 1


@pytest.mark.parametrize("level", [1, 2])
def test_fused_apply_matches_layered_forward(dev, level):
    """The single-launch cluster kernel (the in-loop path) against the layered forward:
    z + theta s_z d with theta from the layered d."""
    import torch
    from stgipc import learned
    s = cube_system(12)
    solver = _solver(s, level, dev)
    _solve(solver, s, dev)
    G = solver.net_graph()
    rng = np.random.default_rng(21)
    n = G.nodes
    r = np.zeros((n, 4), np.float32)
    r[:, :3] = rng.standard_normal((n, 3))
    z = np.zeros((n, 4), np.float32)
    z[:, :3] = r[:, :3] * rng.uniform(0.5, 2.0, (n, 1))
    p = learned.init_params(3, head_scale=0.3)
    P = _t(p, dev)
    d = learned.forward(G, _t(r, dev), _t(z, dev), P, 1)[0].cpu().numpy().astype(np.float64)
    sz = np.sqrt((z[:, :3].astype(np.float64) ** 2).sum() / n)
    a = (r[:, :3] * z[:, :3]).astype(np.float64).sum()
    b = sz * (r[:, :3] * d[:, :3]).sum()
    th = -0.5 * a / b if b < -0.5 * a else 1.0
    want = z[:, :3] + th * sz * d[:, :3]
    zt = _t(z, dev)
    cl = learned.apply(G, _t(r, dev), zt, P)
    got = zt.cpu().numpy()
    assert cl in (8, 16), "the level fits the fused kernel"
    corr = want - z[:, :3]
    assert np.linalg.norm(got[:, :3] - want) <= 5e-3 * np.linalg.norm(corr) + 1e-7
    assert np.all(got[:, 3] == 0)


def test_training_lowers_the_energy_loss(dev):
    """From-scratch training on the GPU kernels: samples recorded by the plain FP64 solver on
    two seeds, a few hundred Adam steps, the mean energy loss falls well below the bank
    solve's (-1)."""
    from stgipc import learned, scenes
    data = []
    for sd in (2300, 2301):
        sysm = scenes.make_heterogeneous_cube(n=16, seed=sd)
        solver = _solver(sysm, 1, dev, precision="fp64")
        d, st = learned.record_samples(solver, sysm, capacity=200, every=1)
        assert d.samples == min(200, st["iterations"])
        data.append(d)
    tr = learned.Trainer(learned.init_params(0), dev)
    ev = lambda: np.mean([tr.evaluate(d.graph, d.rc[:32].contiguous(), d.zc[:32].contiguous(), min(32, d.samples))
                          for d in data])
    before = ev()
    learned.train(tr, data, 400, batch=8, lr=1e-3, lr_final=1e-4)
    after = ev()
    assert abs(before + 1.0) < 0.05
    assert after < before - 0.15, (before, after)


def test_shipped_network_gain_on_held_out_scene(dev):
    """What the shipped network (trained on heterogeneous-cube seeds 2000-2007) gains over
    plain MAS on the held-out benchmark scene (352,947 DOF, seed 1005): fewer PCG iterations
    at the same FP64 relative residual, in FP32 and in FP64."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    from stgipc import learned
    params, level, meta = learned.load_weights(learned.default_weights())
    assert 1005 not in meta["seeds"]
    sysm, _ = bench.load_system("hetcube48")
    P = _t(params, dev)
    out = {}
    for prec in ("fp32", "fp64"):
        plain = _solver(sysm, level, dev, precision=prec)
        stp, _ = _solve(plain, sysm, dev)
        lrn = _solver(sysm, level, dev, precision=prec, learned=True)
        lrn.net_set_params(P)
        stl, _ = _solve(lrn, sysm, dev)
        out[prec] = (stp["iterations"], stl["iterations"])
        assert stl["status"] == 0 and stl["rel_residual"] <= 1e-4
        assert stl["learned_rejected"] == 0
        assert stl["iterations"] <= 0.9 * stp["iterations"], out
    print("iterations plain -> learned:", out)
