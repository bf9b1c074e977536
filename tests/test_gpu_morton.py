"""GPU: Morton keys on the device (stg_morton_keys, _calcVertMChash at GIPC.cu:453-502)
against the host restatement, bit for bit, through the C ABI."""
import numpy as np
import pytest

from conftest import cube_system

pytestmark = pytest.mark.gpu


def _device_keys(pos, dev):
    import torch
    from stgipc.linear_system import morton_keys
    k = morton_keys(torch.from_numpy(np.ascontiguousarray(pos, np.float64)).to(dev))
    return k.cpu().numpy().view(np.uint64)


def test_morton_keys_bit_exact(dev):
    from stgipc import scenes
    rng = np.random.default_rng(9)
    cases = [cube_system(16).pos, rng.uniform(-1.0, 4.0, size=(50000, 3)),
             scenes.cube_mesh(48)[0] + rng.uniform(-1e-3, 1e-3, size=(49 ** 3, 3))]
    for pos in cases:
        assert np.array_equal(_device_keys(pos, dev), scenes.morton_hash(pos))


def test_morton_keys_order_matches_renumber(dev):
    from stgipc import scenes
    pos, tets = scenes.cube_mesh(12)
    pos = pos + np.random.default_rng(4).uniform(-1e-3, 1e-3, size=pos.shape)
    keys = _device_keys(pos, dev)
    _, _, order = scenes.morton_renumber(pos, tets)
    assert np.array_equal(np.argsort(keys, kind="stable"), order)


def test_morton_keys_invalid_and_empty(dev):
    from stgipc import _lib
    L = _lib.lib()
    assert L.stg_morton_keys(0, None, None, None) == _lib.STG_OK
    assert L.stg_morton_keys(-1, None, None, None) == _lib.STG_ERR_INVALID
