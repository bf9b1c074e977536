"""GPU: the cloth producers (stg_cloth_membrane, stg_cloth_bending) against
oracle/cloth_oracle.py, and the cloth-on-ball Newton solve (64 x 64 cloth over a 10^3-hex
ball; membrane, bending, ball elasticity, masses and contact barriers) against the oracle's
PCG on the same triplets.

Bars: rows / cols bit-exact; gradients within 1e-12 of the set's largest entry; the
membrane blocks within 1e-12 (both evaluate the reference's closed-form projections, in a
different operation order), bending blocks 1e-14; the FP64 MAS-PCG solve at the
oracle's iteration count and within 1e-8 of its x; the FP32-storage solve to an FP64 true
residual <= 1.5e-4.
"""
import functools

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@functools.lru_cache(maxsize=None)
def _scene():
    from stgipc import scenes
    return scenes.make_cloth_sphere(n=64, ball_n=10)


def _t(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def _per_element(got, want, k, tol):
    g, w = got.reshape(-1, k), want.reshape(-1, k)
    scale = np.maximum(np.abs(w).max(axis=1), 1e-300)
    assert np.all(np.abs(g - w).max(axis=1) <= tol * scale)


def _global(got, want, tol):
    """Against the set's largest entry (a nearly unstretched triangle's gradient is ~1e-12 of
    the others and carries their rounding)."""
    assert np.abs(got - want).max() <= tol * np.abs(want).max()


def test_cloth_producers_match_oracle(dev):
    from oracle import cloth_oracle as co
    from stgipc import cloth
    sc = _scene()
    x = sc.base.pos
    er, ec, eb, eg = co.membrane(sc.tris, sc.dminv, sc.area, x, sc.stretch, sc.shear, sc.strain_rate, sc.dt)
    r, c, b, g, bad = cloth.membrane(_t(sc.tris, dev), _t(sc.dminv, dev), _t(sc.area, dev), _t(x, dev), sc.stretch,
                                     sc.shear, sc.strain_rate, sc.dt)
    assert int(bad.item()) == 0
    assert np.array_equal(r.cpu().numpy(), er) and np.array_equal(c.cpu().numpy(), ec)
    _per_element(b.cpu().numpy(), eb, 54, 1e-12)
    _global(g.cpu().numpy(), eg, 1e-12)
    er, ec, eb, eg = co.bending(sc.stencil, sc.Q, sc.elen, x, sc.bend, sc.dt)
    r, c, b, g, bad = cloth.bending(_t(sc.stencil, dev), _t(sc.Q, dev), _t(sc.elen, dev), _t(x, dev), sc.bend, sc.dt)
    assert int(bad.item()) == 0
    assert np.array_equal(r.cpu().numpy(), er) and np.array_equal(c.cpu().numpy(), ec)
    _per_element(b.cpu().numpy(), eb, 90, 1e-14)
    _global(g.cpu().numpy(), eg, 1e-12)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_cloth_ball_solve(dev, precision):
    import torch
    from oracle import oracle as orc
    from stgipc import PCGSolverConfig, Solver
    from stgipc.cloth import cloth_system
    sc = _scene()
    s = sc.base
    rows, cols, blocks, b, P = cloth_system(sc, dev)
    R, C, B, bh = rows.cpu().numpy(), cols.cpu().numpy(), blocks.cpu().numpy(), b.cpu().numpy()
    r, c, bl = orc.convert(R, C, B)
    om = orc.Mas(16, s.num_verts, s.neighbor_start, s.neighbor_num, s.neighbor_list, *s.slot_maps(16))
    om.build(sc.contacts)
    om.assemble(r, c, bl)
    if precision == "fp64":
        solver = Solver(PCGSolverConfig(precision="fp64"))
    else:
        solver = Solver(PCGSolverConfig(precision="fp32", stop_rule="relative_residual", global_tol_rate=1e-4,
                                        refine_interval=8))
    solver.mas_init(s.num_verts, s.neighbor_start, s.neighbor_num, s.neighbor_list, *s.slot_maps(16))
    X = torch.zeros(b.numel(), dtype=torch.float64, device=dev)
    st = solver.solve_linear_system(rows, cols, blocks.reshape(-1), b, X, contacts=P)
    assert st["status"] == 0 and st["nnzb"] == r.size
    assert st["total_clusters"] == om.total
    xg = X.cpu().numpy()
    if precision == "fp64":
        xe, st_e = orc.pcg(r, c, bl, bh, mas=om)
        assert st["iterations"] == st_e["iterations"]
        assert np.linalg.norm(xg - xe) <= 1e-8 * np.linalg.norm(xe)
    else:
        assert st["rel_residual"] <= 1.5e-4
