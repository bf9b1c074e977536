"""CPU: the contact barrier oracle (orc_contact_barrier), pinned to the reference.

The reference's contact Hessian (GIPC.cu:3149-4988, NEWF and RANK 2) is lambda0 g g^T and its
gradient flatten_pk1 * g, with g the last column of the symbolically generated derivative
pFpx_*2 (GIPC_PDerivative.cuh), i.e. d(d / sqrt(dhat)) / dx.  The oracle writes g in closed
form.  Bars:
- g against the reference's own generated code, compiled from its header where it lies
  (oracle/_ref/libstg_contact_ref.so, `make -C oracle ref`): relative 1e-11 per pair;
- gradient against torch autograd of the barrier energy kappa dhat^2 (s^2-1)^2 ln^2(s^2), and
  lambda0 against its second derivative in s, FP64: relative 1e-10;
- lambda0 >= 0 on (0, 1), frozen below s^2 = 1e-6;
- encodings: the mollified forms are skipped, slot layout row <= col, block_offset applied.
"""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import ROOT
from oracle import oracle as orc

REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libstg_contact_ref.so")
NV = {0: 2, 1: 3, 2: 4, 3: 4}


def _config(kind, rng, s_target):
    """k vertices of a pair of `kind` in general position and the dhat that puts it at
    s = s_target."""
    while True:
        v = rng.normal(size=(NV[kind], 3))
        d2, _ = orc.contact_d2(kind, v)
        if d2 > 1e-3:
            return v, d2 / s_target ** 2


def _energy_torch(kind, v, dhat, kappa):
    import torch
    x = torch.tensor(v, dtype=torch.float64, requires_grad=True)

    def d2f(x):
        if kind == 0:
            r = x[0] - x[1]
            return r @ r
        if kind == 1:
            c = torch.linalg.cross(x[1] - x[0], x[2] - x[0])
            e = x[2] - x[1]
            return (c @ c) / (e @ e)
        if kind == 2:
            b = torch.linalg.cross(x[2] - x[1], x[3] - x[1])
            return ((x[0] - x[1]) @ b) ** 2 / (b @ b)
        b = torch.linalg.cross(x[1] - x[0], x[3] - x[2])
        return ((x[2] - x[0]) @ b) ** 2 / (b @ b)

    s = torch.sqrt(d2f(x)) / np.sqrt(dhat)
    I = s * s
    E = kappa * dhat ** 2 * (I - 1) ** 2 * torch.log(I) ** 2
    (gx,) = torch.autograd.grad(E, x)
    (gs,) = torch.autograd.grad(torch.sqrt(d2f(x)) / np.sqrt(dhat), x)
    st = s.detach().clone().requires_grad_(True)
    Es = kappa * dhat ** 2 * (st * st - 1) ** 2 * torch.log(st * st) ** 2
    (e1,) = torch.autograd.grad(Es, st, create_graph=True)
    (e2,) = torch.autograd.grad(e1, st)
    return gx.numpy().reshape(-1), gs.numpy().reshape(-1), float(e2), float(s.detach())


def _pair(kind, k0=0):
    ids = list(range(k0, k0 + NV[kind]))
    from stgipc.contact import encode
    return encode(kind, ids)


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="oracle/_ref/libstg_contact_ref.so not built "
                                                         "(make -C oracle ref needs the reference's sources)")
@pytest.mark.parametrize("kind", [0, 1, 2, 3])
def test_distance_derivative_matches_reference_generated_code(kind):
    L = C.CDLL(REF_LIB)
    L.orc_contact_ref_grad.argtypes = [C.c_int, C.c_void_p, C.c_double, C.c_void_p]
    L.orc_contact_ref_grad.restype = C.c_int
    rng = np.random.default_rng(100 + kind)
    for _ in range(200):
        v, dhat = _config(kind, rng, rng.uniform(0.05, 0.95))
        d2, g2 = orc.contact_d2(kind, v)
        mine = g2[: 3 * NV[kind]] / (2 * np.sqrt(d2)) / np.sqrt(dhat)
        x = np.ascontiguousarray(v.reshape(-1))
        ref = np.zeros(12)
        assert L.orc_contact_ref_grad(kind, x.ctypes.data, np.sqrt(dhat), ref.ctypes.data) == 3 * NV[kind]
        ref = ref[: 3 * NV[kind]]
        assert np.abs(mine - ref).max() <= 1e-11 * np.abs(ref).max()


@pytest.mark.parametrize("kind", [0, 1, 2, 3])
def test_barrier_matches_autograd(kind):
    rng = np.random.default_rng(7 + kind)
    kappa = 1e4
    for _ in range(40):
        v, dhat = _config(kind, rng, rng.uniform(0.05, 0.95))
        rows, cols, blocks, grad, sk = orc.contact_barrier(np.array([_pair(kind)]), v, dhat, kappa)
        assert sk == 0
        gx, gs, e2, s = _energy_torch(kind, v, dhat, kappa)
        k = 3 * NV[kind]
        assert np.abs(grad[0, :k] - gx).max() <= 1e-10 * np.abs(gx).max()
        assert np.all(grad[0, k:] == 0)
        # assemble the dense Hessian from the upper blocks and compare with e2 gs gs^T
        H = np.zeros((12, 12))
        for r, c, b in zip(rows, cols, blocks):
            B = b.reshape(3, 3).T  # column-major
            H[3 * r:3 * r + 3, 3 * c:3 * c + 3] += B
            if r != c:
                H[3 * c:3 * c + 3, 3 * r:3 * r + 3] += B.T
        want = e2 * np.outer(gs, gs)
        assert np.abs(H[:k, :k] - want).max() <= 1e-10 * np.abs(want).max()
        assert np.all(H[k:, :] == 0) and np.all(H[:, k:] == 0)


def test_lambda0_nonnegative_and_frozen():
    v = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0]])
    lam = []
    for s in np.linspace(1e-4, 0.999, 400):
        dhat = 1.0 / s ** 2
        _, _, blocks, _, _ = orc.contact_barrier(np.array([_pair(0)]), v, dhat, 1.0)
        # PP along x: block (0,0) element (0,0) = lambda0 (ds/dx0)^2 = lambda0 / dhat
        lam.append(blocks[0, 0] * dhat)
    lam = np.array(lam)
    assert np.all(lam >= 0)
    # below s^2 = 1e-6 the reference evaluates lambda0 at s^2 = 1e-6 (GIPC.cu:3171, 3318)
    a = orc.contact_barrier(np.array([_pair(0)]), v, 1.0 / 1e-7, 1.0)[2][0, 0] * 1e7
    b = orc.contact_barrier(np.array([_pair(0)]), v, 1.0 / 5e-7, 1.0)[2][0, 0] * 5e7
    assert a == pytest.approx(b, rel=1e-12)


def test_encodings_slots_and_offset():
    rng = np.random.default_rng(3)
    x = rng.normal(size=(20, 3))
    pairs = np.array([
        (-3, 5, -1, -1),        # PP 2-5
        (-8, 1, 4, -1),         # PE 7 | 1-4
        (-10, 11, 2, 3),        # PT 9 | 11 2 3
        (6, 0, 12, 13),         # EE 6-0 | 12-13
        (1, 2, 3, -5),          # EE mollified: skipped
        (-2, -3, -4, -5),       # PP mollified: skipped
        (-2, -3, 4, -5),        # PE mollified: skipped
        (-2, 3, 3, 4),          # repeated vertex: skipped
        (-2, 3, 4, 25),         # out of range: skipped
    ], np.int32)
    rows, cols, blocks, grad, sk = orc.contact_barrier(pairs, x, 100.0, 1.0, block_offset=7)
    assert sk == 5
    assert np.all(rows <= cols)
    assert np.all(blocks[40:] == 0) and np.all(grad[4:] == 0)
    vids = [[2, 5], [7, 1, 4], [9, 11, 2, 3], [6, 0, 12, 13]]
    slots = [(i, j) for i in range(4) for j in range(i, 4)]
    for p, vs in enumerate(vids):
        for k, (i, j) in enumerate(slots):
            r, c = rows[10 * p + k] - 7, cols[10 * p + k] - 7
            if i < len(vs) and j < len(vs):
                assert (r, c) == (min(vs[i], vs[j]), max(vs[i], vs[j]))
            else:
                assert (r, c) == (vs[0], vs[0]) and np.all(blocks[10 * p + k] == 0)
    # a skipped pair's slots sit on vertex 0 (plus the offset)
    assert np.all(rows[40:] == 7) and np.all(cols[40:] == 7)
