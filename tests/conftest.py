import functools
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "stiff-gipc_b200"))
sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libstgipc.so")
    config.addinivalue_line("markers", "slow: larger cases")


@functools.lru_cache(maxsize=None)
def cube_system(n=16, seed=1001):
    from stgipc import scenes
    return scenes.make_cube_drop(n=n, seed=seed)


@functools.lru_cache(maxsize=None)
def fixture_system(name):
    """A Newton system on one of the reference's METIS-sorted fixture meshes (rest state,
    SNH + mass), keeping the fixture's vertex order and partition."""
    from stgipc import scenes
    z = np.load(os.path.join(GOLDEN, f"{name}_sorted16.npz"))
    pos = z["pos"].astype(np.float64)
    tets = z["tets"].astype(np.int64)
    V = pos.shape[0]
    vel = np.zeros_like(pos)
    vel[:, 1] = -1.0
    E = np.full(tets.shape[0], 1e5)
    s = scenes._assemble(name, pos, pos * 1.0, tets, E, 0.45, 1000.0, 1.0 / 60.0, vel,
                         barriers=[((0.0, 1.0, 0.0), float(pos[:, 1].min()) - 5e-4, 1e-3, 1e5)])
    return s, z["part"].astype(np.int64)


def random_contacts(V, count, seed, local=64):
    """Sign-encoded int4 collision pairs (GIPC.cuh:49-66 encodings: PT/EE with x >= 0,
    PP (2 verts), PE (3 verts), and the negative-x 4-vertex forms), vertices near each other."""
    rng = np.random.default_rng(seed)
    out = np.zeros((count, 4), np.int32)
    for i in range(count):
        base = int(rng.integers(0, max(V - local, 1)))
        v = base + rng.choice(local, size=4, replace=False)
        v = np.minimum(v, V - 1)
        kind = i % 7
        if kind == 0:      # x >= 0, 4 verts
            out[i] = v
        elif kind == 1:    # x >= 0, w < 0
            out[i] = [v[0], v[1], v[2], -v[3] - 1]
        elif kind == 2:    # PP: x < 0, z < 0, y >= 0
            out[i] = [-v[0] - 1, v[1], -1, -1]
        elif kind == 3:    # PE: x < 0, z >= 0, w < 0, y >= 0
            out[i] = [-v[0] - 1, v[1], v[2], -1]
        elif kind == 4:    # x < 0, y < 0, z < 0, w < 0: 4 verts
            out[i] = [-v[0] - 1, -v[1] - 1, -v[2] - 1, -v[3] - 1]
        elif kind == 5:    # x < 0, z >= 0, w < 0, y < 0: 4 verts
            out[i] = [-v[0] - 1, -v[1] - 1, v[2], -v[3] - 1]
        else:              # x < 0, z >= 0, w >= 0: 4 verts
            out[i] = [-v[0] - 1, v[1], v[2], v[3]]
    return out


@pytest.fixture(scope="session")
def cube16():
    return cube_system(16)


def have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def dev():
    if not have_gpu():
        pytest.skip("no CUDA device")
    import torch
    return torch.device("cuda:0")
