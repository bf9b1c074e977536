"""GPU: the kernels of the in-loop SpMV and their autotuner (stg_spmv_tiles): every tile shape
of the full-copy kernel, the halo kernel and the upper kernel give the same solve up to
summation order, the tuner picks the fastest of the timed candidates and keeps it, and
unsupported shapes are rejected."""
import numpy as np
import pytest

from conftest import cube_system

pytestmark = pytest.mark.gpu


def _solve(s, dev, prec, tiles=None):
    import torch
    from stgipc import PCGSolverConfig, Solver
    solver = Solver(PCGSolverConfig(precision=prec, stop_rule="relative_residual", global_tol_rate=1e-6))
    solver.mas_init(s.num_verts, s.neighbor_start, s.neighbor_num, s.neighbor_list, *s.slot_maps(16))
    if tiles is not None:
        solver.spmv_tiles(tiles)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    x = t(np.zeros(s.n))
    st = solver.solve_linear_system(t(s.rows), t(s.cols), t(s.blocks.reshape(-1)), t(s.b), x)
    return solver, st, x.cpu().numpy()


@pytest.mark.parametrize("prec,alt,tol", [("fp32", 32, 2e-4), ("fp64", 16, 1e-7)])
def test_tile_shapes_agree(dev, prec, alt, tol):
    """Both tile shapes, the halo kernel (operands staged in shared memory) and the upper
    kernel (transposed products spilled to their rows) give the same solve up to summation
    order."""
    s = cube_system(16)
    s0, st0, x0 = _solve(s, dev, prec, -1)
    default = s0.spmv_tiles_info()[0]
    assert default in ((64 if prec == "fp32" else 32), -3)
    for shape in (64 if prec == "fp32" else 32, alt, -2, -3):
        s1, st1, x1 = _solve(s, dev, prec, shape)
        assert s1.spmv_tiles_info()[0] == shape
        assert abs(st0["iterations"] - st1["iterations"]) <= 1
        assert np.linalg.norm(x1 - x0) <= tol * np.linalg.norm(x0)


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_autotuner_picks_fastest_and_keeps_it(dev, prec):
    s = cube_system(16)
    solver, st, _ = _solve(s, dev, prec, 0)
    rt, us_a, us_b, us_h, us_u = solver.spmv_tiles_info()
    cand = ((64, 32) if prec == "fp32" else (32, 16)) + (-2, -3)
    assert us_a > 0 and us_b > 0 and us_h > 0 and us_u > 0
    us = (us_a, us_b, us_h, us_u)
    assert rt == cand[int(np.argmin(us))]
    import torch
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    x = t(np.zeros(s.n))
    st2 = solver.solve_linear_system(t(s.rows), t(s.cols), t(s.blocks.reshape(-1)), t(s.b), x)
    assert solver.spmv_tiles_info() == (rt, us_a, us_b, us_h, us_u)  # same shape: not re-timed
    assert st2["iterations"] == st["iterations"]
    # another handle on the same shape class reuses the process's choice without timing
    other, st3, _ = _solve(s, dev, prec, 0)
    assert other.spmv_tiles_info() == (rt, us_a, us_b, us_h, us_u)


def test_unsupported_tile_shape_rejected(dev):
    from stgipc import PCGSolverConfig, Solver, StgError
    solver = Solver(PCGSolverConfig(precision="fp32"))
    with pytest.raises(StgError):
        solver.spmv_tiles(16)
    solver.spmv_tiles(-1)
