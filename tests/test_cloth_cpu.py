"""CPU: the cloth oracle (oracle/cloth_oracle.py) against independent derivations.

- the reference's analytic Baraff-Witkin projections (stretch per direction, shear by its
  closed-form eigen-decomposition) equal the PSD clamp of the exact Hessians, 1e-12;
- the membrane gradient equals torch autograd of the energy, 1e-12; it vanishes at rest in
  the reference's triangle frame (F^T F = I);
- the quadratic bending matrix is PSD and annihilates translations; its gradient is its
  Hessian times x;
- the cloth-on-ball scene has the configuration's structure at a reduced size.
"""
import numpy as np
import pytest

from oracle import cloth_oracle as co


def _clamp(H):
    w, V = np.linalg.eigh(H)
    return (V * np.maximum(w, 0)) @ V.T


def test_projections_equal_eigen_clamp():
    rng = np.random.default_rng(0)
    S = np.zeros((6, 6))
    for i in range(3):
        S[3 + i, i] = S[i, 3 + i] = 1
    for _ in range(500):
        F = np.eye(3, 2) + rng.normal(scale=rng.choice([0.05, 0.3, 1.0]), size=(3, 2))
        g = np.concatenate([F[:, 1], F[:, 0]])
        Hx = 2 * (np.outer(g, g) + float(F[:, 0] @ F[:, 1]) * S)
        Hp = _clamp(Hx)
        assert np.abs(co._shear_projected(F) - Hp).max() <= 1e-12 * np.abs(Hp).max()
        sr = float(rng.choice([0.0, 1.0]))
        Hs = np.zeros((6, 6))
        for c in range(2):
            f = F[:, c]
            s = np.linalg.norm(f)
            fh = f / s
            d1 = 2 * (s - 1) + (3 * sr * (s - 1) ** 2 if s > 1 else 0)
            d2 = 2 + (6 * sr * (s - 1) if s > 1 else 0)
            Hs[3 * c:3 * c + 3, 3 * c:3 * c + 3] = _clamp((d1 / s) * (np.eye(3) - np.outer(fh, fh)) + d2 * np.outer(fh, fh))
        assert np.abs(co._stretch_projected(F, sr) - Hs).max() <= 1e-12 * np.abs(Hs).max()


def test_membrane_gradient_matches_autograd():
    import torch
    rng = np.random.default_rng(1)
    for _ in range(30):
        x = rng.normal(size=(3, 3))
        D = np.linalg.inv(rng.normal(size=(2, 2)) + 2 * np.eye(2))
        kst, ksh, sr, area, dt = 3.0, 0.5, float(rng.choice([0.0, 1.0])), 0.7, 0.1

        def energy(xt):
            Ds = torch.stack([xt[1] - xt[0], xt[2] - xt[0]], 1)
            F = Ds @ torch.tensor(D)
            su, sv = torch.linalg.norm(F[:, 0]), torch.linalg.norm(F[:, 1])
            e = (su - 1) ** 2 + (sv - 1) ** 2 + sr * (torch.clamp(su - 1, min=0) ** 3 + torch.clamp(sv - 1, min=0) ** 3)
            return area * dt * dt * (kst * e + ksh * (F[:, 0] @ F[:, 1]) ** 2)

        xt = torch.tensor(x, requires_grad=True)
        (g,) = torch.autograd.grad(energy(xt), xt)
        _, _, _, gr = co.membrane(np.array([[0, 1, 2]]), D.reshape(1, 4), np.array([area]), x, kst, ksh, sr, dt)
        assert np.abs(gr[0] - g.numpy().reshape(-1)).max() <= 1e-12 * np.abs(g.numpy()).max()


def test_rest_frame_and_zero_force_at_rest():
    from stgipc import scenes
    rng = np.random.default_rng(2)
    rest = rng.normal(size=(30, 3))
    tris = np.array([[3 * i, 3 * i + 1, 3 * i + 2] for i in range(10)])
    dminv, area = scenes.cloth_rest_frame(rest, tris)
    for t in range(10):
        X = rest[tris[t]]
        F = np.stack([X[1] - X[0], X[2] - X[0]], 1) @ dminv[t].reshape(2, 2)
        assert np.allclose(F.T @ F, np.eye(2), atol=1e-12)
        assert area[t] == pytest.approx(0.5 * np.linalg.norm(np.cross(X[1] - X[0], X[2] - X[0])))
    _, _, _, gr = co.membrane(tris, dminv, area, rest, 3.0, 0.5, 1.0, 0.1)
    assert np.abs(gr).max() <= 1e-13


def test_bending_matrix():
    from stgipc import scenes
    rng = np.random.default_rng(3)
    pos, tris = scenes.cube_mesh(3, 1.0)
    surf = scenes.boundary_faces(tris)
    rest = pos + rng.normal(scale=0.01, size=pos.shape)
    st, elen, Q = scenes.bending_stencils(rest, surf)
    assert st.shape[0] > 0 and np.all(st[:, 3] >= 0)
    for e in range(st.shape[0]):
        Qe = Q[e].reshape(4, 4)
        assert np.abs(Qe @ np.ones(4)).max() <= 1e-9 * np.abs(Qe).max()
        assert np.linalg.eigvalsh(Qe).min() >= -1e-9 * np.abs(Qe).max()
    x = rest + rng.normal(scale=0.05, size=rest.shape)
    rows, cols, blocks, grad = co.bending(st, Q, elen, x, 0.3, 0.1)
    for e in range(st.shape[0]):
        c = elen[e] * 0.3 * 0.01
        want = c * (Q[e].reshape(4, 4) @ x[st[e]]).reshape(-1)
        assert np.allclose(grad[e], want, rtol=1e-12, atol=1e-15)


def test_cloth_ball_scene_structure():
    from stgipc import scenes
    sc = scenes.make_cloth_sphere(n=32, ball_n=6)
    V = sc.base.num_verts
    assert sc.cloth_verts == 32 * 32 and V == 32 * 32 + 7 ** 3
    assert sc.tris.shape[0] == 2 * 31 * 31 and sc.base.tets.shape[0] == 6 * 6 ** 3
    assert sc.stencil.shape[0] == 3 * 31 * 31 - 2 * 31  # interior edges of the grid
    assert sc.contacts.shape[0] > 0 and np.all(np.isfinite(sc.Q)) and np.all(sc.area > 0)
    # every ball tet keeps a positive volume after the cube-to-ball map
    p = sc.base.pos
    t = sc.base.tets
    vol = np.einsum("ij,ij->i", np.cross(p[t[:, 1]] - p[t[:, 0]], p[t[:, 2]] - p[t[:, 0]]), p[t[:, 3]] - p[t[:, 0]])
    assert np.all(vol > 0)
