"""CPU: the affine-body oracle (oracle/abd_oracle.py) against independent derivations.

- body gradient = torch autograd of 1/2 (q - q_tilde)^T M (q - q_tilde) + kappa v dt^2 S(q),
  S = ||A A^T - I||_F^2 (abd_energy.inl:9-27), and the a-block Hessian = its autograd Hessian
  wherever that is PSD (PSD-projected otherwise), FP64, relative 1e-12;
- M = sum_i m_i J_i^T J_i over the body's points (the dyadic mass);
- the point-to-body mapping, assembled, equals G^T K G with K the symmetric point-level
  matrix and G the global point-to-DOF map (rows J_i for body points, identity for FEM
  vertices), to 1e-12;
- the ABD block-Jacobi is the inverse of each body's diagonal tile;
- the stiff-affine hybrid scene has the configuration's sizes.
"""
import numpy as np
import pytest

from oracle import abd_oracle as abd


def _energy_torch(q, qt, M, k):
    import torch
    x = torch.tensor(q, dtype=torch.float64, requires_grad=True)
    Mt = torch.tensor(M)
    d = x - torch.tensor(qt)
    A = x[3:].reshape(3, 3)
    E = 0.5 * d @ Mt @ d + k * ((A @ A.T - torch.eye(3, dtype=torch.float64)) ** 2).sum()
    (g,) = torch.autograd.grad(E, x, create_graph=True)
    H = torch.stack([torch.autograd.grad(g[i], x, retain_graph=True)[0] for i in range(12)])
    return g.detach().numpy(), H.detach().numpy()


def _body(rng, warp):
    pts = rng.normal(scale=0.05, size=(27, 3)) + rng.normal(size=3)
    m = rng.uniform(0.01, 0.05, size=27)
    q = np.concatenate([rng.normal(scale=0.01, size=3), (np.eye(3) + rng.uniform(-warp, warp, (3, 3))).reshape(-1)])
    qt = q + rng.normal(scale=1e-3, size=12)
    return pts, m, q, qt


@pytest.mark.parametrize("warp", [1e-3, 0.3])
def test_body_system_matches_autograd(warp):
    rng = np.random.default_rng(41)
    for _ in range(10):
        pts, m, q, qt = _body(rng, warp)
        m13 = abd.dyadic_mass(m, pts)
        M = abd.dyadic_mass_matrix(m13)
        Mref = sum(mi * abd.jacobian(x).T @ abd.jacobian(x) for mi, x in zip(m, pts))
        assert np.abs(M - Mref).max() <= 1e-13 * np.abs(Mref).max()
        kappa, vol, dt = 1e8, 1e-3, 0.01
        k = kappa * vol * dt * dt
        rows, cols, blocks, grad = abd.body_system(q[None], qt[None], m13[None], np.array([vol]), kappa, dt)
        g, H = _energy_torch(q, qt, M, k)
        assert np.abs(grad[0] - g).max() <= 1e-12 * np.abs(g).max()
        Hd = np.zeros((12, 12))
        for r, c, b in zip(rows, cols, blocks):
            B = b.reshape(3, 3).T
            Hd[3 * r:3 * r + 3, 3 * c:3 * c + 3] = B
            Hd[3 * c:3 * c + 3, 3 * r:3 * r + 3] = B.T
        Sa = H[3:, 3:] - M[3:, 3:]
        if np.linalg.eigvalsh(Sa).min() >= 0:
            assert np.abs(Hd - H).max() <= 1e-12 * np.abs(H).max()
        else:
            # projected: PSD a-block; the translation rows are untouched
            assert np.linalg.eigvalsh(Hd[3:, 3:] - M[3:, 3:]).min() >= -1e-9 * np.abs(Sa).max()
            assert np.abs(Hd[:3, :] - H[:3, :]).max() <= 1e-12 * np.abs(H).max()


def test_fixed_body_is_mass_only():
    rng = np.random.default_rng(2)
    pts, m, q, qt = _body(rng, 0.1)
    m13 = abd.dyadic_mass(m, pts)
    rows, cols, blocks, grad = abd.body_system(q[None], qt[None], m13[None], np.array([1.0]), 1e8, 0.01,
                                               fixed=np.array([1]))
    assert np.all(grad == 0)
    M = abd.dyadic_mass_matrix(m13)
    for r, c, b in zip(rows, cols, blocks):
        assert np.array_equal(b.reshape(3, 3).T, M[3 * r:3 * r + 3, 3 * c:3 * c + 3])


def test_mapping_equals_dense_gtkg():
    """Point triplets of a symmetric K (upper blocks, some given transposed at (j, i)),
    mapped and assembled, give G^T K G."""
    rng = np.random.default_rng(5)
    N, per, F = 3, 4, 5
    P = N * per
    point_body = np.repeat(np.arange(N), per).astype(np.int32)
    xbar = rng.normal(size=(P, 3))
    npts = P + F
    trip = []
    for _ in range(40):
        i, j = sorted(rng.integers(0, npts, size=2))
        B = rng.normal(size=(3, 3))
        if i == j:
            B = B + B.T
        if rng.random() < 0.3 and i != j:
            trip.append((j, i, B.T))  # the same entry given as its transpose
        else:
            trip.append((i, j, B))
    rows = np.array([t[0] for t in trip], np.int32)
    cols = np.array([t[1] for t in trip], np.int32)
    blocks = np.array([t[2].T.reshape(9) for t in trip])
    K = np.zeros((3 * npts, 3 * npts))
    for (i, j, B) in trip:
        if i > j:
            i, j, B = j, i, B.T
        K[3 * i:3 * i + 3, 3 * j:3 * j + 3] += B
        if i != j:
            K[3 * j:3 * j + 3, 3 * i:3 * i + 3] += B.T
    nrow = 4 * N + F
    G = np.zeros((3 * npts, 3 * nrow))
    for p in range(P):
        G[3 * p:3 * p + 3, 12 * point_body[p]:12 * point_body[p] + 12] = abd.jacobian(xbar[p])
    for v in range(F):
        G[3 * (P + v):3 * (P + v) + 3, 3 * (4 * N + v):3 * (4 * N + v) + 3] = np.eye(3)
    want = G.T @ K @ G
    orow, ocol, oblk = abd.map_triplets(rows, cols, blocks, P, point_body, xbar, N)
    assert np.all(orow <= ocol)
    got = np.zeros_like(want)
    for r, c, b in zip(orow, ocol, oblk):
        B = b.reshape(3, 3).T
        got[3 * r:3 * r + 3, 3 * c:3 * c + 3] += B
        if r != c:
            got[3 * c:3 * c + 3, 3 * r:3 * r + 3] += B.T
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()


def test_points_gradient_and_block_jacobi():
    rng = np.random.default_rng(8)
    N, per = 4, 6
    point_body = np.repeat(np.arange(N), per).astype(np.int32)
    xbar = rng.normal(size=(N * per, 3))
    q = rng.normal(size=(N, 12))
    x = abd.points(point_body, xbar, q)
    for p in range(N * per):
        A = q[point_body[p], 3:].reshape(3, 3)
        assert np.allclose(x[p], A @ xbar[p] + q[point_body[p], :3], rtol=1e-14, atol=1e-14)
    pg = rng.normal(size=(N * per, 3))
    start = np.arange(0, N * per + 1, per)
    bg = abd.gather_gradient(start, xbar, pg, np.zeros((N, 12)))
    for b in range(N):
        want = sum(abd.jacobian(xbar[p]).T @ pg[p] for p in range(start[b], start[b + 1]))
        assert np.allclose(bg[b], want, rtol=1e-13, atol=1e-13)
    tiles = []
    for b in range(N):
        Q = rng.normal(size=(12, 12))
        tiles.append(Q @ Q.T + 12 * np.eye(12))
    rows, cols, blocks = [], [], []
    for b, T in enumerate(tiles):
        for (i, j) in abd.SLOTS:
            rows.append(4 * b + i), cols.append(4 * b + j)
            blocks.append(T[3 * i:3 * i + 3, 3 * j:3 * j + 3].T.reshape(9))
    inv = abd.block_jacobi(np.array(rows), np.array(cols), np.array(blocks), N)
    for b in range(N):
        assert np.allclose(inv[b] @ tiles[b], np.eye(12), atol=1e-12)


def test_abd_slab_scene_sizes():
    """A reduced lattice (2^3 bodies, 16 x 16 x 2 slab) keeps the configuration's structure:
    27 points per body, (n+1)^2 (layers+1) slab vertices, contacts at the bottom layer."""
    from stgipc import scenes
    sc = scenes.make_abd_slab(lattice=2, slab_n=16, slab_layers=2, slab_size=0.4)
    assert sc.bodies == 8 and sc.abd_points == 8 * 27
    assert sc.fem.num_verts == 17 * 17 * 3 and sc.fem.tets.shape[0] == 6 * 16 * 16 * 2
    assert sc.n == 3 * (4 * 8 + 17 * 17 * 3)
    assert sc.contacts.shape[0] > 0
    P = sc.abd_points
    # every contact joins a body point and a slab vertex
    for q in sc.contacts:
        ids = [(-q[0] - 1) if q[0] < 0 else q[0]] + [v for v in q[1:] if v >= 0]
        assert min(ids) < P <= max(ids)
    # the bottom layer touches: its lowest points are within sqrt(dhat) of the slab top
    top = sc.fem.pos[:, 1].max()
    x = abd.points(sc.point_body, sc.xbar, sc.q)
    low = np.array([x[sc.body_point_start[b]:sc.body_point_start[b + 1], 1].min() for b in range(sc.bodies)])
    bottom = low < top + 0.01
    assert bottom.sum() == 4 and np.all(low[bottom] - top < 1e-3) and np.all(low[bottom] - top > 0)
