"""GPU: the coupled affine-body + FEM system (12x12 ABD blocks stored as 4x4 tiles of 3x3
blocks in the first 4 * bodies block rows, FEM vertices after them), preconditioned by the
ABD 12x12 block-Jacobi (ABDPreconditioner::apply, abd_preconditioner.cu:20-38) composed
with MAS or 3x3 block-Jacobi on the rest (GlobalLinearSystem::apply_preconditioner,
global_linear_system.cu:167-180), against the oracle through the C ABI."""
import numpy as np
import pytest

from conftest import cube_system

pytestmark = pytest.mark.gpu


def _t(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def abd_fem_system(bodies=6, n=8, seed=31):
    """Triplets (upper, column-major 3x3, unsorted with duplicates as the reference hands
    them over) of an SPD system: per-body 12x12 SPD blocks, the FEM cube Hessian shifted by
    4 * bodies block rows, and weak body-vertex couplings."""
    rng = np.random.default_rng(seed)
    s = cube_system(n)
    off = 4 * bodies
    rows, cols, blks = [s.rows + off], [s.cols + off], [s.blocks.reshape(-1, 9)]
    fem_diag = np.abs(s.blocks.reshape(-1, 3, 3)[s.rows == s.cols][:, [0, 1, 2], [0, 1, 2]]).mean()
    abd_inv = np.zeros((bodies, 12, 12))
    for b in range(bodies):
        Q = rng.standard_normal((12, 12))
        M = (Q @ Q.T + 12 * np.eye(12)) * fem_diag
        # couplings to 4 random FEM vertices; their row sums are added to both diagonals so
        # that the whole matrix stays diagonally dominant in the coupled rows
        for v in rng.choice(s.num_verts, size=4, replace=False):
            a = int(rng.integers(0, 4))
            C = rng.standard_normal((3, 3)) * 1e-2 * fem_diag
            rows.append(np.array([4 * b + a], np.int32))
            cols.append(np.array([off + v], np.int32))
            blks.append(C.T.reshape(1, 9))  # column-major
            w = np.abs(C).sum()
            M[3 * a:3 * a + 3, 3 * a:3 * a + 3] += w * np.eye(3)
            rows.append(np.array([off + v], np.int32))
            cols.append(np.array([off + v], np.int32))
            blks.append((w * np.eye(3)).reshape(1, 9))
        abd_inv[b] = np.linalg.inv(M)
        for a in range(4):
            for cc in range(a, 4):
                Bk = M[3 * a:3 * a + 3, 3 * cc:3 * cc + 3]
                rows.append(np.array([4 * b + a], np.int32))
                cols.append(np.array([4 * b + cc], np.int32))
                blks.append(Bk.T.reshape(1, 9))
    R = np.concatenate(rows).astype(np.int32)
    Cc = np.concatenate(cols).astype(np.int32)
    Bl = np.concatenate(blks).astype(np.float64)
    perm = rng.permutation(R.size)
    nrow = off + s.num_verts
    b = rng.standard_normal(3 * nrow)
    return s, R[perm], Cc[perm], Bl[perm], b, abd_inv, off


@pytest.mark.parametrize("precond,loop", [("mas", "graph"), ("mas", "host"), ("diag", "graph"), ("diag", "persistent")])
def test_abd_fem_coupled_vs_oracle(dev, precond, loop):
    from oracle import oracle as orc
    from stgipc import PCGSolverConfig, Solver
    bodies = 6
    s, R, Cc, Bl, b, abd_inv, off = abd_fem_system(bodies)
    r, c, bl = orc.convert(R, Cc, Bl)
    ai = abd_inv.reshape(-1)
    if precond == "mas":
        om = orc.Mas(16, s.num_verts, s.neighbor_start, s.neighbor_num, s.neighbor_list, *s.slot_maps(16))
        om.build()
        om.assemble(r, c, bl, fem_offset=off)
        xe, st_e = orc.pcg(r, c, bl, b, mas=om, fem_offset=off, abd_bodies=bodies, abd_inv=ai)
    else:
        xe, st_e = orc.pcg(r, c, bl, b, use_diag=True, abd_bodies=bodies, abd_inv=ai)
    solver = Solver(PCGSolverConfig(preconditioner=precond, loop=loop))
    if precond == "mas":
        solver.mas_init(s.num_verts, s.neighbor_start, s.neighbor_num, s.neighbor_list, *s.slot_maps(16))
    X = _t(np.zeros(b.size), dev)
    st = solver.solve_linear_system(_t(R, dev), _t(Cc, dev), _t(Bl.reshape(-1), dev), _t(b, dev), X,
                                    fem_block_offset=off, abd_inv=_t(ai, dev), abd_bodies=bodies)
    xg = X.cpu().numpy()
    # r0.z0 includes the ABD rows' 12x12 solves: it pins the ABD application directly
    if precond == "diag":
        assert st["iterations"] == st_e["iterations"]
        assert np.linalg.norm(xg - xe) <= 1e-8 * np.linalg.norm(xe)
        assert abs(st["rz0"] - st_e["rz0"]) <= 1e-12 * abs(st_e["rz0"])
    else:
        assert abs(st["iterations"] - st_e["iterations"]) <= 2
        assert np.linalg.norm(xg - xe) <= 1e-4 * np.linalg.norm(xe)
        assert abs(st["rz0"] - st_e["rz0"]) <= 1e-5 * abs(st_e["rz0"])
