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
    assert 0.0 < seconds.value < 60.0
    # the device still works: a normal solve afterwards
    gls = GlobalLinearSystem(cube_system(8), PCGSolverConfig(), device=dev)
    st = gls.solve_linear_system()
    assert st["status"] == _lib.STG_OK and np.isfinite(gls.x.cpu().numpy()).all()
    torch.cuda.synchronize()
