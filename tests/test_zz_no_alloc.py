"""GPU: the allocation-free SpMV entry point (stg_spmv_noalloc) against stg_spmv.

Collected last on purpose: it must give the same products whether it runs in a fresh
process (its first call resolves the shared scratch array) or after every other test.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import cube_system

pytestmark = pytest.mark.gpu


def _t(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def _case(n, seed, dev):
    from oracle import oracle as orc
    s = cube_system(n)
    r, c, bl = orc.convert(s.rows, s.cols, s.blocks)
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(s.n)
    y0 = rng.standard_normal(s.n)
    return (_t(bl.reshape(-1), dev), _t(r, dev), _t(c, dev), r.size, _t(x, dev)), y0


def test_noalloc_matches_spmv_two_calls(dev):
    """Two calls in a row (a larger system, then a smaller one, so stale scratch from the
    first would show in the second) give stg_spmv's products bit for bit: both run the same
    kernel over transpose lists sorted the same way."""
    from stgipc import PCGSolverConfig, Solver
    from stgipc.linear_system import spmv_noalloc
    solver = Solver(PCGSolverConfig())
    for n, seed, (a, b) in ((16, 11, (1.0, 0.0)), (8, 12, (-0.5, 2.0))):
        (blocks, rows, cols, nnzb, x), y0 = _case(n, seed, dev)
        y_ref = _t(y0, dev)
        solver.spmv(a, blocks, rows, cols, nnzb, x, b, y_ref)
        y_na = _t(y0, dev)
        spmv_noalloc(a, blocks, rows, cols, nnzb, x, b, y_na)
        ye, yg = y_ref.cpu().numpy(), y_na.cpu().numpy()
        assert np.array_equal(yg, ye), (n, np.max(np.abs(yg - ye)))


def test_noalloc_rejects_oversize_and_bad_input(dev):
    from stgipc import _lib
    L = _lib.lib()
    # beyond the fixed maximum: rejected before any device work
    st = L.stg_spmv_noalloc(1.0, None, None, None, 0, C.c_void_p(8), 0.0, C.c_void_p(8),
                            3 * (131072 + 1), None)
    assert st == _lib.STG_ERR_INVALID and b"maximum" in L.stg_last_error()
    # unsorted BCOO: rejected by the validation pass, output untouched
    (blocks, rows, cols, nnzb, x), y0 = _case(8, 13, dev)
    rows_bad = rows.flip(0).contiguous()
    cols_bad = cols.flip(0).contiguous()
    y = _t(y0, dev)
    st = L.stg_spmv_noalloc(1.0, blocks.data_ptr(), rows_bad.data_ptr(), cols_bad.data_ptr(), nnzb, x.data_ptr(),
                            0.0, y.data_ptr(), y.numel(), None)
    assert st == _lib.STG_ERR_INVALID and b"unsorted" in L.stg_last_error()
    assert np.array_equal(y.cpu().numpy(), y0)
    # a zero-size call only resolves the scratch array on the current device
    assert L.stg_spmv_noalloc(1.0, None, None, None, 0, None, 0.0, None, 0, None) == _lib.STG_OK
    # host memory is not device memory of the current device
    xh = np.zeros(y.numel())
    st = L.stg_spmv_noalloc(1.0, blocks.data_ptr(), rows.data_ptr(), cols.data_ptr(), nnzb, xh.ctypes.data,
                            0.0, y.data_ptr(), y.numel(), None)
    assert st == _lib.STG_ERR_INVALID and b"current device" in L.stg_last_error()
    # the Python wrapper checks dtypes and sizes before calling
    from stgipc.linear_system import spmv_noalloc
    with pytest.raises(ValueError):
        spmv_noalloc(1.0, blocks.float(), rows, cols, nnzb, x, 0.0, y)
    with pytest.raises(ValueError):
        spmv_noalloc(1.0, blocks, rows, cols, nnzb, x[:-3], 0.0, y)
