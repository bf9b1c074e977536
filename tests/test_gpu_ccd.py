"""GPU: the CCD step bound (stg_ccd_step_size) against the oracle: every pair's time of
impact and the bound bit for bit (both evaluate the same IEEE operations in the same order;
the device file is compiled without FMA contraction), on random pairs and on the two cubes
in contact pushed into each other."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _t(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def test_random_pairs_bitwise(dev):
    from oracle import oracle as orc
    from stgipc import ccd
    rng = np.random.default_rng(17)
    V = 5000
    x = rng.normal(size=(V, 3))
    dx = rng.normal(size=(V, 3)) * 0.5
    pairs = []
    for i in range(20000):
        v = rng.choice(V, size=4, replace=False)
        pairs.append([-v[0] - 1, v[1], v[2], v[3]] if i % 2 == 0 else list(v))
    pairs = np.array(pairs, np.int32)
    alpha, toc = ccd.step_size(_t(pairs, dev), _t(x, dev), _t(dx, dev), per_pair=True)
    toc = toc.cpu().numpy()
    want = np.array([orc.accd(0 if q[0] < 0 else 1, x[[(-q[0] - 1) if q[0] < 0 else q[0], q[1], q[2], q[3]]],
                              dx[[(-q[0] - 1) if q[0] < 0 else q[0], q[1], q[2], q[3]]], 0.2) for q in pairs])
    assert np.array_equal(toc, want)
    assert (want < 1).sum() > 1000
    assert float(alpha.item()) == orc.ccd_step_size(pairs, x, dx, 0.8)


def test_no_pairs_and_bad_ids(dev):
    import torch
    from stgipc import ccd
    x = _t(np.zeros((4, 3)), dev)
    alpha = ccd.step_size(torch.zeros((0, 4), dtype=torch.int32, device=dev), x, x)
    assert float(alpha.item()) == 1.0
    with pytest.raises(ValueError):
        ccd.step_size(_t(np.array([[-1, 1, 2, 9]], np.int32), dev), x, x)


def test_stacked_cubes_pushed_together(dev):
    """The upper cube moved down by twice the gap: the bound stops it before any pair of the
    interface crosses, and equals the oracle's."""
    from oracle import oracle as orc
    from stgipc import ccd, scenes
    s, _, body = scenes.make_stacked_cubes(8)
    tris = scenes.boundary_faces(s.tets)
    dx = np.zeros_like(s.pos)
    dx[body == 1, 1] = -2e-3
    pairs = scenes.contact_pairs(s.pos, tris, body, dhat=(3e-3) ** 2)
    # CCD pairs: point-triangle and edge-edge only (the reference's _ccd_collisonPairs)
    pt = pairs[(pairs[:, 0] < 0) & (pairs[:, 2] >= 0) & (pairs[:, 3] >= 0)]
    ee = pairs[(pairs[:, 0] >= 0) & (pairs[:, 3] >= 0)]
    cp = np.concatenate([pt, ee])
    assert cp.shape[0] > 100
    alpha = float(ccd.step_size(_t(cp, dev), _t(s.pos, dev), _t(dx, dev)).item())
    assert alpha == orc.ccd_step_size(cp, s.pos, dx, 0.8)
    assert 0.05 < alpha < 0.25   # gap 4e-4 of a 2e-3 push: contact at 0.2
    moved = s.pos + alpha * dx
    for q in cp:
        ids = [(-q[0] - 1) if q[0] < 0 else q[0], q[1], q[2], q[3]]
        d2, _ = orc.contact_d2(2 if q[0] < 0 else 3, moved[ids])
        assert d2 > 0
