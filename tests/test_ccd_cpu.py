"""CPU: the additive-CCD oracle (orc_accd, orc_ccd_step_size) pinned to the reference.

The reference's own ACCD.cu is compiled for the host (oracle/_ref/libstg_accd_ref.so,
`make -C oracle ref`), FMA contraction off; the oracle restates it with the same operand
order, so every time of impact must be bit-identical, on random pairs (both kinds, with and
without impact, thickness 0 and > 0) and on degenerate ones (no relative motion, parallel
edges, a point on an edge's line).  Independent of the reference: a point falling straight
onto a triangle stops before the plane, and stepping the CCD pairs by the bound leaves every
pair apart.
"""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import ROOT
from oracle import oracle as orc

REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libstg_accd_ref.so")
need_ref = pytest.mark.skipif(not os.path.exists(REF_LIB), reason="oracle/_ref/libstg_accd_ref.so not built "
                                                                  "(make -C oracle ref needs the reference's sources)")


def _ref():
    L = C.CDLL(REF_LIB)
    L.orc_accd_ref.restype = C.c_double
    L.orc_accd_ref.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_double]
    return lambda k, x, d, eta, th: L.orc_accd_ref(k, np.ascontiguousarray(x, np.float64).ctypes.data,
                                                  np.ascontiguousarray(d, np.float64).ctypes.data, eta, th)


@need_ref
@pytest.mark.parametrize("kind", [0, 1])
@pytest.mark.parametrize("thickness", [0.0, 0.05])
def test_toc_bit_identical_to_reference(kind, thickness):
    ref = _ref()
    rng = np.random.default_rng(11 + kind)
    hits = 0
    for _ in range(5000):
        x = rng.normal(size=(4, 3))
        dx = rng.normal(size=(4, 3)) * rng.choice([0.05, 0.5, 2.0, 5.0])
        eta = float(rng.choice([0.2, 0.1, 0.5]))
        a = ref(kind, x, dx, eta, thickness)
        b = orc.accd(kind, x, dx, eta, thickness)
        assert a == b or (np.isnan(a) and np.isnan(b)), (a, b)
        hits += a < 1.0
    assert hits > 200


@need_ref
def test_toc_degenerate_cases():
    ref = _ref()
    cases = []
    x = np.array([[0, 0.1, 0], [-1, 0, -1], [1, 0, -1], [0, 0, 1]], np.float64)
    cases.append((0, x, np.zeros((4, 3))))                                     # no motion
    cases.append((0, x, np.tile([0.3, -0.2, 0.1], (4, 1))))                    # translation only
    e = np.array([[0, 0, 0], [1, 0, 0], [0, 0.01, 0], [1, 0.01, 0]], np.float64)
    cases.append((1, e, np.array([[0, 0, 0], [0, 0, 0], [0, -0.02, 0], [0, -0.02, 0]])))  # parallel edges
    p = np.array([[2, 0.001, 0], [0, 0, 0], [1, 0, 0], [0, 0, 1]], np.float64)
    cases.append((0, p, np.array([[0, -0.01, 0], [0, 0, 0], [0, 0, 0], [0, 0, 0]])))  # beyond a vertex
    for kind, xx, dd in cases:
        for eta in (0.2, 0.5):
            assert ref(kind, xx, dd, eta, 0.0) == orc.accd(kind, xx, dd, eta, 0.0)


def test_point_falling_onto_triangle_stops_before_the_plane():
    h = 0.1
    x = np.array([[0.1, h, 0.1], [-1, 0, -1], [1, 0, -1], [0, 0, 1]], np.float64)
    dx = np.array([[0, -2 * h, 0], [0, 0, 0], [0, 0, 0], [0, 0, 0]], np.float64)
    for eta in (0.1, 0.2, 0.5):
        t = orc.accd(0, x, dx, eta)
        # contact at t = 0.5; conservative advancement stops once the gap shrank to about eta
        assert 0.5 * (1 - eta) * 0.95 <= t < 0.5


def test_step_bound_keeps_pairs_apart():
    rng = np.random.default_rng(5)
    V = 400
    x = rng.uniform(0, 1, size=(V, 3))
    dx = rng.normal(scale=0.2, size=(V, 3))
    pairs = []
    for i in range(600):
        v = rng.choice(V, size=4, replace=False)
        pairs.append([-v[0] - 1, v[1], v[2], v[3]] if i % 2 == 0 else list(v))
    pairs = np.array(pairs, np.int32)
    alpha = orc.ccd_step_size(pairs, x, dx, slackness=0.8)
    tocs = [orc.accd(0 if q[0] < 0 else 1, x[[(-q[0] - 1) if q[0] < 0 else q[0], q[1], q[2], q[3]]],
                     dx[[(-q[0] - 1) if q[0] < 0 else q[0], q[1], q[2], q[3]]], 0.2) for q in pairs]
    assert alpha == 1.0 / max(1.0 / t for t in tocs)
    assert 0 < alpha < 1
    # no pair crosses within the bound: its distance stays positive along the whole step
    for q in pairs:
        ids = [(-q[0] - 1) if q[0] < 0 else q[0], q[1], q[2], q[3]]
        for s in np.linspace(0, alpha, 21):
            d2, _ = orc.contact_d2(2 if q[0] < 0 else 3, x[ids] + s * dx[ids])
            assert d2 > 0
    assert orc.ccd_step_size(np.zeros((0, 4), np.int32), x, dx) == 1.0
