"""GPU: the bounded device waits give up instead of hanging, report STG_ERR_TIMEOUT, and
leave the context usable (no fault, trap or endless loop is involved: the waited-on
mbarrier is simply never completed)."""
import ctypes as C

import numpy as np
import pytest

from conftest import cube_system

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_context_stays_usable(dev):
    import torch
    from stgipc import GlobalLinearSystem, PCGSolverConfig, _lib
    L = _lib.lib()
    status, seconds = C.c_int(-1), C.c_double(-1.0)
    assert L.stg_selftest_wait_timeout(C.byref(status), C.byref(seconds)) == _lib.STG_OK
    assert status.value == _lib.STG_ERR_TIMEOUT
    # every bounded wait gives up after 1 s of the device's global timer
    assert 0.9 < seconds.value < 3.0, seconds.value
    # the device still works: a normal solve afterwards
    gls = GlobalLinearSystem(cube_system(8), PCGSolverConfig(), device=dev)
    st = gls.solve_linear_system()
    assert st["status"] == _lib.STG_OK and np.isfinite(gls.x.cpu().numpy()).all()
    torch.cuda.synchronize()


@pytest.mark.parametrize("where,prec,loop", [("b", "fp64", "graph"), ("b", "fp32", "graph"),
                                             ("block", "fp32", "host"), ("block", "fp64", "graph")])
def test_nan_input_reports_breakdown(dev, where, prec, loop):
    """A NaN in the right-hand side or in one Hessian block (a corrupted input, injected on
    the host) ends the solve at once with STG_BREAKDOWN instead of iterating on NaNs; the
    handle then solves a clean system normally."""
    import numpy as np
    import torch
    from conftest import cube_system
    from stgipc import PCGSolverConfig, Solver, StgError, _lib
    s = cube_system(8)
    solver = Solver(PCGSolverConfig(precision=prec, loop=loop, stop_rule="relative_residual"))
    solver.mas_init(s.num_verts, s.neighbor_start, s.neighbor_num, s.neighbor_list, *s.slot_maps(16))
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    b = s.b.copy()
    blocks = s.blocks.copy()
    if where == "b":
        b[17] = np.nan
    else:
        blocks[len(blocks) // 2, 4] = np.nan
    x = t(np.zeros(s.n))
    with pytest.raises(StgError) as e:
        solver.solve_linear_system(t(s.rows), t(s.cols), t(blocks.reshape(-1)), t(b), x)
    assert e.value.status == _lib.STG_BREAKDOWN
    st = solver.solve_linear_system(t(s.rows), t(s.cols), t(s.blocks.reshape(-1)), t(s.b), x)
    assert st["status"] == 0 and st["rel_residual"] <= 1.2e-4
