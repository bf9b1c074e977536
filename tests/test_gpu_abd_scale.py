"""GPU: the affine-body path at the stiff-affine hybrid configuration -- 512 affine cubes
(12 DOF each) in an 8x8x8 lattice with random rotations, the bottom layer touching a soft slab
of 64 x 64 x 8 hexes (196,608 tets): 6,144 + 114,075 DOF, coupled 3x3 and 12x12 BCOO blocks.

Bars: the ABD producers (body system, point positions, contact mapping, body gradient) against
oracle/abd_oracle.py (rows / cols bit-exact, values to 1e-12 of their block's scale; the PSD
projection's eigen-solvers differ, 1e-9 there); the coupled FP64 MAS-PCG solve, with the ABD
block-Jacobi built on the device from the BCOO, at the oracle's iteration count and within
1e-8 of its x; the FP32-storage solve (relative-residual stop at 1e-4) to an FP64 true residual
<= 1.5e-4, with an error against the converged x no more than 3x that of the oracle's FP64 solve
stopped at the same relative residual (the error at a 1e-4 residual is set by the system's
conditioning, not by the storage precision), and an iteration count within 20 % of it.
"""
import functools

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@functools.lru_cache(maxsize=None)
def _scene():
    from stgipc import scenes
    return scenes.make_abd_slab()


def _t(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_abd_producers_match_oracle(dev):
    from oracle import abd_oracle as abd, oracle as orc
    from stgipc import abd as gabd
    sc = _scene()
    N, P = sc.bodies, sc.abd_points
    er, ec, eb, eg = abd.body_system(sc.q, sc.q_tilde, sc.mass, sc.volume, sc.kappa, sc.dt)
    r, c, b, g = gabd.body_system(_t(sc.q, dev), _t(sc.q_tilde, dev), _t(sc.mass, dev), _t(sc.volume, dev),
                                  sc.kappa, sc.dt)
    assert np.array_equal(r.cpu().numpy(), er) and np.array_equal(c.cpu().numpy(), ec)
    b = b.cpu().numpy()
    for k in range(N):
        assert _rel(b[10 * k:10 * k + 10], eb[10 * k:10 * k + 10]) <= 1e-9
    assert _rel(g.cpu().numpy(), eg) <= 1e-12
    xa = gabd.points(_t(sc.point_body, dev), _t(sc.xbar, dev), _t(sc.q, dev)).cpu().numpy()
    assert _rel(xa, abd.points(sc.point_body, sc.xbar, sc.q)) <= 1e-15
    allpos = np.concatenate([xa, sc.fem.pos])
    cr, cc, cb, cg, sk = orc.contact_barrier(sc.contacts, allpos, sc.dhat, sc.kappa_contact)
    assert sk == 0
    mr, mc, mb = abd.map_triplets(cr, cc, cb, P, sc.point_body, sc.xbar, N)
    gr, gc, gb, bad = gabd.map_triplets(_t(cr, dev), _t(cc, dev), _t(cb, dev), P, _t(sc.point_body, dev),
                                        _t(sc.xbar, dev), N)
    assert int(bad.item()) == 0
    assert np.array_equal(gr.cpu().numpy(), mr) and np.array_equal(gc.cpu().numpy(), mc)
    gb = gb.cpu().numpy()
    for t in range(cr.size):
        s = slice(16 * t, 16 * t + 16)
        assert np.abs(gb[s] - mb[s]).max() <= 1e-12 * max(np.abs(mb[s]).max(), 1e-300)
    pg = np.random.default_rng(3).normal(size=(P, 3))
    bg0 = np.random.default_rng(4).normal(size=(N, 12))
    want = abd.gather_gradient(sc.body_point_start, sc.xbar, pg, bg0)
    got = gabd.gather_gradient(_t(sc.body_point_start, dev), _t(sc.xbar, dev), _t(pg, dev), _t(bg0, dev))
    assert _rel(got.cpu().numpy(), want) <= 1e-13


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_abd512_slab_coupled_solve(dev, precision):
    import torch
    from oracle import abd_oracle as abd, oracle as orc
    from stgipc import PCGSolverConfig, Solver
    from stgipc.abd import coupled_system
    sc = _scene()
    N, s = sc.bodies, sc.fem
    rows, cols, blocks, b = coupled_system(sc, dev)
    R, C, B, bh = rows.cpu().numpy(), cols.cpu().numpy(), blocks.cpu().numpy(), b.cpu().numpy()
    r, c, bl = orc.convert(R, C, B)
    om = orc.Mas(16, s.num_verts, s.neighbor_start, s.neighbor_num, s.neighbor_list, *s.slot_maps(16))
    om.build()
    om.assemble(r, c, bl, fem_offset=4 * N)
    ai = abd.block_jacobi(r, c, bl, N).reshape(-1)
    if precision == "fp64":
        solver = Solver(PCGSolverConfig(precision=precision))
    else:
        solver = Solver(PCGSolverConfig(precision=precision, stop_rule="relative_residual", global_tol_rate=1e-4,
                                        refine_interval=8))
    solver.mas_init(s.num_verts, s.neighbor_start, s.neighbor_num, s.neighbor_list, *s.slot_maps(16))
    X = torch.zeros(b.numel(), dtype=torch.float64, device=dev)
    st = solver.solve_linear_system(rows, cols, blocks.reshape(-1), b, X, fem_block_offset=4 * N, abd_bodies=N)
    assert st["status"] == 0
    assert st["nnzb"] == r.size
    xg = X.cpu().numpy()
    if precision == "fp64":
        xe, st_e = orc.pcg(r, c, bl, bh, mas=om, fem_offset=4 * N, abd_bodies=N, abd_inv=ai)
        assert st["iterations"] == st_e["iterations"]
        assert np.linalg.norm(xg - xe) <= 1e-8 * np.linalg.norm(xe)
    else:
        # FP32 storage, FP64 dots and residual replacement: the FP64 true residual
        assert st["rel_residual"] <= 1.5e-4
        # as accurate as the oracle's FP64 solve stopped at the same relative residual
        xt, _ = orc.pcg(r, c, bl, bh, mas=om, fem_offset=4 * N, abd_bodies=N, abd_inv=ai, tol=1e-12)
        x64, st64, _, done = orc.pcg_timed(r, c, bl, bh, mas=om, fem_offset=4 * N, tol=1e-4, stop_rule="relative",
                                           abd_bodies=N, abd_inv=ai)
        assert done
        e64 = np.linalg.norm(x64 - xt)
        assert np.linalg.norm(xg - xt) <= 3.0 * e64 + 1e-6 * np.linalg.norm(xt)
        assert abs(st["iterations"] - st64["iterations"]) <= max(4, st64["iterations"] // 5)
