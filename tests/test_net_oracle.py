"""CPU: the learned-correction oracle (oracle/net_oracle.py) pinned by finite differences,
plus its graph builder's invariants.  The CUDA kernels are checked against it in
tests/test_gpu_learned.py."""
import numpy as np

from oracle import net_oracle as no


def _setup(n=24, seed=3, samples=2):
    urow, ucol, ublk = no.random_level(n, seed)
    g = no.build_graph(n, urow, ucol, ublk)
    rng = np.random.default_rng(seed + 1)
    rcs = [rng.standard_normal((n, 3)) for _ in range(samples)]
    D = g["dblk"].astype(np.float64)
    zcs = [np.linalg.solve(D, r[..., None])[..., 0] * 0.7 for r in rcs]
    p = no.pack({k: 0 for k in no.P})
    rng2 = np.random.default_rng(seed + 2)
    p[:] = rng2.standard_normal(no.COUNT) * 0.15
    return g, rcs, zcs, p


def test_graph_is_symmetric_and_sorted():
    urow, ucol, ublk = no.random_level(30, 5)
    g = no.build_graph(30, urow, ucol, ublk)
    ent = {}
    for i in range(30):
        cols = g["col"][g["row"][i]:g["row"][i + 1]]
        assert np.all(np.diff(cols) > 0) and i not in cols
        for e in range(g["row"][i], g["row"][i + 1]):
            ent[(i, int(g["col"][e]))] = e
    for (i, j), e in ent.items():
        f = ent[(j, i)]
        assert g["w"][e] == g["w"][f]
        np.testing.assert_array_equal(g["oblk"][e], g["oblk"][f].T)
    # the full operator assembled from the graph equals the upper BCOO mirrored
    A = np.zeros((90, 90))
    for k, (r, c) in enumerate(zip(urow, ucol)):
        B = ublk[k].reshape(3, 3).T
        A[3 * r:3 * r + 3, 3 * c:3 * c + 3] = B
        A[3 * c:3 * c + 3, 3 * r:3 * r + 3] = B.T
    v = np.random.default_rng(0).standard_normal((30, 3))
    np.testing.assert_allclose(no.level_matvec(g, v).reshape(-1), A @ v.reshape(-1), rtol=1e-6, atol=1e-6)


def test_oracle_gradient_matches_finite_differences():
    g, rcs, zcs, p = _setup()
    _, grad = no.batch_loss_grad(g, rcs, zcs, p, rounding=False)
    rng = np.random.default_rng(7)
    blocks = [("W0", 0, 1024), ("b0", 1024, 1088), ("W1", 1088, 25664), ("b1", 25664, 25856), ("Wo", 25856, 26048),
              ("bo", 26368, 26371)]
    for name, a, b in blocks:
        for i in rng.choice(np.arange(a, b), size=min(4, b - a), replace=False):
            h = 1e-6
            pp, pm = p.copy(), p.copy()
            pp[i] += h
            pm[i] -= h
            fd = (no.batch_loss_grad(g, rcs, zcs, pp, rounding=False)[0].mean()
                  - no.batch_loss_grad(g, rcs, zcs, pm, rounding=False)[0].mean()) / (2 * h)
            assert abs(fd - grad[i]) <= 1e-5 * max(1.0, abs(fd)) + 1e-7, (name, i, fd, grad[i])


def test_loss_is_energy_error_left_after_correction():
    """J(g) = |e - g|_A^2 / 2 - |e|_A^2 / 2 for A e = r: the exact coarse solve gives the
    minimum -|e|_A^2 / 2 / |J(z)| and any other g more."""
    g, rcs, zcs, _ = _setup(samples=1)
    n = g["n"]
    A = np.zeros((3 * n, 3 * n))
    for i in range(n):
        A[3 * i:3 * i + 3, 3 * i:3 * i + 3] = g["dblk"][i]
        for e in range(g["row"][i], g["row"][i + 1]):
            j = g["col"][e]
            A[3 * i:3 * i + 3, 3 * j:3 * j + 3] = g["oblk"][e]
    r, z = rcs[0], zcs[0]
    e = np.linalg.solve(A, r.reshape(-1)).reshape(n, 3)
    d_exact = (e - z) / 1.0
    L_exact, grad = no.loss_grad(g, r, z, d_exact, 1.0)
    assert np.abs(grad).max() < 1e-8 * np.abs(r).max()
    L_other, _ = no.loss_grad(g, r, z, d_exact + 1e-2, 1.0)
    assert L_other > L_exact
    L_plain, _ = no.loss_grad(g, r, z, np.zeros_like(z), 1.0)
    assert abs(L_plain - np.sign(L_plain)) < 1e-12


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.0e-3, 65504.0, 1e-40], np.float32)
    y = no.bf16(x)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: to even (1.0); 1.005859375 rounds up
    assert y[0] == 1.0 and y[1] == 1.0 and y[2] == np.float32(1.0078125)
    assert np.all(np.abs(y[3:5] - x[3:5]) <= np.abs(x[3:5]) * 2 ** -8)


def test_adam_step():
    p = np.array([1.0, -2.0, 0.5])
    gr = np.array([0.1, -0.2, 0.0])
    p1, m, v = no.adam(p, gr, np.zeros(3), np.zeros(3), 1, 0.01)
    # first step: m_hat = g, v_hat = g^2: p - lr sign(g) (for g != 0)
    np.testing.assert_allclose(p1, [0.99, -1.99, 0.5], rtol=1e-6)
