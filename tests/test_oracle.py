"""CPU: the oracle against independent restatements, the reference's fixtures and invariants."""
import os

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import GOLDEN, cube_system, fixture_system, random_contacts


def _dense_sym(rows, cols, blocks, n):
    """Full symmetric sparse matrix from unique upper blocks (column-major 3x3)."""
    B = blocks.reshape(-1, 3, 3).transpose(0, 2, 1)  # row-major
    r, c, v = [], [], []
    for a in range(3):
        for b in range(3):
            r.append(3 * rows + a)
            c.append(3 * cols + b)
            v.append(B[:, a, b])
            off = rows != cols
            r.append(3 * cols[off] + b)
            c.append(3 * rows[off] + a)
            v.append(B[off, a, b])
    return sp.coo_matrix((np.concatenate(v), (np.concatenate(r), np.concatenate(c))), shape=(n, n)).tocsr()


def test_convert_matches_numpy():
    from oracle import oracle as orc
    s = cube_system(8)
    r, c, b = orc.convert(s.rows, s.cols, s.blocks)
    key = s.rows.astype(np.int64) * (1 << 32) + s.cols
    uk, inv = np.unique(key, return_inverse=True)
    sums = np.zeros((uk.size, 9))
    np.add.at(sums, inv, s.blocks)
    assert np.array_equal(r, (uk >> 32).astype(np.int32))
    assert np.array_equal(c, (uk & 0xffffffff).astype(np.int32))
    assert np.allclose(b, sums, rtol=1e-14, atol=0)


def test_spmv_matches_scipy():
    from oracle import oracle as orc
    s = cube_system(8)
    r, c, b = orc.convert(s.rows, s.cols, s.blocks)
    A = _dense_sym(r, c, b, s.n)
    x = np.random.default_rng(0).standard_normal(s.n)
    y = orc.spmv(r, c, b, x)
    assert np.allclose(y, A @ x, rtol=1e-12, atol=1e-12 * np.abs(A @ x).max())
    y2 = orc.spmv(r, c, b, x, a=-2.0, b=0.5, y=np.ones(s.n))
    assert np.allclose(y2, -2.0 * (A @ x) + 0.5, rtol=1e-12, atol=1e-12 * np.abs(A @ x).max())


def test_system_counts_match_configs():
    s = cube_system(16)
    assert s.num_verts == 4913 and s.tets.shape[0] == 24576 and s.n == 14739
    key = s.rows.astype(np.int64) * (1 << 32) + s.cols
    assert np.unique(key).size == 35937
    assert (s.rows <= s.cols).all()


def test_morton_code_known_answers():
    from stgipc import scenes
    # interleave by hand: code = sum over bits of x<<(3i+2) | y<<(3i+1) | z<<(3i)
    rng = np.random.default_rng(1)
    q = rng.integers(0, 1024, size=(200, 3)).astype(np.uint32)
    got = ((scenes.expand_bits(q[:, 0]).astype(np.uint64) << 2) + (scenes.expand_bits(q[:, 1]).astype(np.uint64) << 1)
           + scenes.expand_bits(q[:, 2]).astype(np.uint64))
    want = np.zeros(200, np.uint64)
    for i in range(10):
        for a, sh in ((0, 2), (1, 1), (2, 0)):
            want |= ((q[:, a].astype(np.uint64) >> np.uint64(i)) & np.uint64(1)) << np.uint64(3 * i + sh)
    assert np.array_equal(got, want)
    assert int(scenes.expand_bits(np.array([1023], np.uint32))[0]) == 0x09249249


def _scalar_morton_keys(pos):
    """_calcVertMChash + hash_code(type -1) + expand_bits (GIPC.cu:183-208, 453-502) written
    out per vertex with Python floats and 32-bit integer arithmetic."""
    def spread(v):
        for mul, mask in ((0x00010001, 0xFF0000FF), (0x00000101, 0x0F00F00F), (0x00000011, 0xC30C30C3),
                          (0x00000005, 0x49249249)):
            v = ((v * mul) & 0xFFFFFFFF) & mask
        return v
    lo = [min(float(p[a]) for p in pos) for a in range(3)]
    hi = [max(float(p[a]) for p in pos) for a in range(3)]
    keys = []
    for i, p in enumerate(pos):
        cells = []
        for a in range(3):
            v = (float(p[a]) - lo[a]) / (hi[a] - lo[a]) * 1024.0
            v = 0.0 if v < 0.0 else v
            v = 1023.0 if 1023.0 < v else v
            cells.append(int(v))
        code = ((spread(cells[0]) << 2) + (spread(cells[1]) << 1) + spread(cells[2])) & 0xFFFFFFFF
        keys.append((code << 32) | i)
    return np.array(keys, dtype=np.uint64)


def test_morton_whole_keys_and_order():
    """Whole 64-bit keys of scenes.morton_hash against the per-vertex restatement, on a
    jittered cube and on a random cloud; morton_renumber's order against an independent sort
    by (code, index)."""
    from stgipc import scenes
    s = cube_system(8)
    rng = np.random.default_rng(3)
    for pos in (s.pos, rng.uniform(-2.0, 3.0, size=(700, 3))):
        want = _scalar_morton_keys(pos)
        assert np.array_equal(scenes.morton_hash(pos), want)
    pos, tets = scenes.cube_mesh(6)
    pos = pos + rng.uniform(-1e-3, 1e-3, size=pos.shape)
    keys = _scalar_morton_keys(pos)
    order_want = np.array(sorted(range(pos.shape[0]), key=lambda i: (int(keys[i]) >> 32, i)))
    pos2, tets2, order = scenes.morton_renumber(pos, tets)
    assert np.array_equal(order, order_want)
    assert np.array_equal(pos2, pos[order_want])
    new_of_old = np.empty_like(order)
    new_of_old[order] = np.arange(order.size)
    assert np.array_equal(tets2, new_of_old[tets])


def test_neighbor_lists_symmetric_and_complete():
    s = cube_system(8)
    V = s.num_verts
    nb = [set(s.neighbor_list[s.neighbor_start[v]:s.neighbor_start[v] + s.neighbor_num[v]].tolist()) for v in range(V)]
    for v in range(V):
        for u in nb[v]:
            assert v in nb[u]
    edges = set()
    for t in s.tets:
        for a in range(4):
            for b in range(a + 1, 4):
                edges.add((min(t[a], t[b]), max(t[a], t[b])))
    assert sum(len(x) for x in nb) == 2 * len(edges)


def test_fixture_partitions_are_mas_ready():
    """The reference's METIS fixtures: parts of <= 16 vertices, vertices grouped by part,
    and set_mas_partition's maps are mutually inverse."""
    from stgipc import scenes
    for name in ("cube", "bunny2", "cloth_high"):
        z = np.load(os.path.join(GOLDEN, f"{name}_sorted16.npz"))
        part = z["part"]
        assert (np.diff(part) >= 0).all()
        assert np.bincount(part).max() <= 16
        pm, rm = scenes.slot_maps_from_parts(part, 16)
        assert pm.size == 16 * (part.max() + 1)
        assert np.array_equal(pm[rm], np.arange(part.size))
        assert (rm // 16 == part).all()


def test_mas_hierarchy_invariants():
    from oracle import oracle as orc
    s, part = fixture_system("bunny2")
    from stgipc import scenes
    pm, rm = scenes.slot_maps_from_parts(part, 16)
    cp = random_contacts(s.num_verts, 500, seed=2)
    m = orc.Mas(16, s.num_verts, s.neighbor_start, s.neighbor_num, s.neighbor_list, pm, rm)
    total = m.build(cp)
    h = m.hierarchy()
    L, V = m.L, s.num_verts
    ls = h["level_size"]
    assert ls[L, 1] == total and total % 16 == 0
    # level sizes shrink and begins are bank aligned
    for l in range(1, L):
        assert ls[l + 1, 0] <= ls[l, 0]
        assert ls[l, 1] % 16 == 0
    # every vertex's closed mask contains its own lane; coarse ids are in range
    lanes = rm % 16
    assert ((h["fine_mask"] >> lanes) & 1).all()
    for l in range(L):
        assert (h["coarse_tables"][l] >= 0).all() and (h["coarse_tables"][l] < ls[l + 1, 0]).all()
    # components at level 0 never span two banks
    g1 = h["coarse_tables"][0]
    for cid in np.unique(g1)[:200]:
        members = np.nonzero(g1 == cid)[0]
        assert np.unique(rm[members] // 16).size == 1
    # the coarse table follows going_next
    if L > 1:
        assert np.array_equal(h["coarse_table"][:, 0], h["going_next"][:V])


def test_mas_inverse_is_inverse():
    from oracle import oracle as orc
    s = cube_system(8)
    r, c, b = orc.convert(s.rows, s.cols, s.blocks)
    m = orc.Mas(16, s.num_verts, s.neighbor_start, s.neighbor_num, s.neighbor_list, *s.slot_maps(16))
    m.build()
    m.assemble(r, c, b)
    mat, inv = m.matrices()

    def dense(P, B=16):
        N = 3 * B
        D = np.zeros((N, N))
        k = 0
        for a in range(B):
            for cc in range(a, B):
                blk = P[k].reshape(3, 3).T  # column-major -> row-major
                D[3 * a:3 * a + 3, 3 * cc:3 * cc + 3] = blk
                if cc != a:
                    D[3 * cc:3 * cc + 3, 3 * a:3 * a + 3] = blk.T
                k += 1
        return D

    for bk in range(0, mat.shape[0], max(1, mat.shape[0] // 8)):
        A = dense(mat[bk])
        d = np.diag(A).copy()
        A[np.arange(48), np.arange(48)] = np.where(d == 0, 1.0, d)
        P = dense(inv[bk].astype(np.float64))
        err = np.abs(P @ A - np.eye(48)).max()
        assert err < 1e-3, (bk, err)


@pytest.mark.parametrize("case", ["cube16_b16", "cube16_b32", "bunny2_contacts"])
def test_fixed_order_matches_reference_walk(case):
    """The oracle's fixed summation order (the GPU's) against the literal walk of the
    reference's loops (PrepareHessian_bcoo's lambdas, per-element pivot division, fine
    residuals added to every level): the same operator up to rounding.  Bank matrices to
    1e-11 of each bank's largest entry, inverses to 1e-5 of it, one application to 1e-5 of
    its largest entry, and the reference-rule PCG to the same iterations and 1e-6."""
    from oracle import oracle as orc
    from stgipc import scenes
    if case == "bunny2_contacts":
        s, part = fixture_system("bunny2")
        bank, cp = 16, random_contacts(s.num_verts, 2000, seed=13)
        pm, rm = scenes.slot_maps_from_parts(part, bank)
    else:
        s = cube_system(16)
        bank, cp = int(case[-2:]), None
        pm, rm = s.slot_maps(bank)
    r, c, b = orc.convert(s.rows, s.cols, s.blocks)
    out = {}
    for order in (orc.ORDER_WALK, orc.ORDER_FIXED):
        m = orc.Mas(bank, s.num_verts, s.neighbor_start, s.neighbor_num, s.neighbor_list, pm, rm, order=order)
        m.build(cp)
        m.assemble(r, c, b)
        mat, inv = m.matrices()
        z = m.apply(np.random.default_rng(5).standard_normal(s.n))
        x, st = orc.pcg(r, c, b, s.b, mas=m)
        out[order] = (mat, inv, z, x, st["iterations"])
    (m0, i0, z0, x0, k0), (m1, i1, z1, x1, k1) = out[orc.ORDER_WALK], out[orc.ORDER_FIXED]
    assert np.max(np.abs(m1 - m0) / (np.abs(m0).max(axis=(1, 2), keepdims=True) + 1e-300)) <= 1e-11
    assert np.max(np.abs(i1 - i0) / (np.abs(i0).max(axis=(1, 2), keepdims=True) + 1e-30)) <= 1e-5
    assert np.max(np.abs(z1 - z0)) <= 1e-5 * np.max(np.abs(z0))
    assert k1 == k0
    assert np.linalg.norm(x1 - x0) <= 1e-6 * np.linalg.norm(x0)


def test_pcg_matches_scipy_solution():
    from oracle import oracle as orc
    s = cube_system(8)
    r, c, b = orc.convert(s.rows, s.cols, s.blocks)
    A = _dense_sym(r, c, b, s.n)
    m = orc.Mas(16, s.num_verts, s.neighbor_start, s.neighbor_num, s.neighbor_list, *s.slot_maps(16))
    m.build()
    m.assemble(r, c, b)
    x, st = orc.pcg(r, c, b, s.b, mas=m, tol=1e-12, max_iter_ratio=1.0)
    xs = sp.linalg.spsolve(A.tocsc(), s.b)
    assert np.linalg.norm(x - xs) <= 1e-5 * np.linalg.norm(xs)
    assert st["rel_residual"] < 1e-5


def test_pcg_reference_stop_rule_and_max_iter():
    from oracle import oracle as orc
    s = cube_system(8)
    r, c, b = orc.convert(s.rows, s.cols, s.blocks)
    x, st = orc.pcg(r, c, b, s.b, use_diag=True)
    assert abs(st["rz_final"]) <= 1e-4 * st["rz0"] * 1e4  # sanity: finite
    # a tiny max_iter_ratio stops at max_iter = (long)(ratio * n)
    x, st = orc.pcg(r, c, b, s.b, use_diag=True, max_iter_ratio=3.0 / s.n)
    assert st["iterations"] == 3


def test_threaded_timing_pcg_matches_serial():
    """The OpenMP timing variant (CPU baseline) follows the same recurrence: same iteration
    count and the same solution up to summation order."""
    from oracle import oracle as orc
    s = cube_system(8)
    r, c, b = orc.convert(s.rows, s.cols, s.blocks)
    m = orc.Mas(16, s.num_verts, s.neighbor_start, s.neighbor_num, s.neighbor_list, *s.slot_maps(16))
    m.build()
    m.assemble(r, c, b)
    x1, st1, _, done1 = orc.pcg_timed(r, c, b, s.b, mas=m, tol=1e-6, stop_rule="relative_residual")
    x2, k2, _, _, done2, threads, rel = orc.pcg_timed_mt(r, c, b, s.b, m, tol=1e-6)
    assert done1 and done2 and threads >= 1
    assert abs(k2 - st1["iterations"]) <= 1
    assert np.linalg.norm(x2 - x1) <= 1e-6 * np.linalg.norm(x1)
    assert rel <= 1e-6


def test_block_jacobi_cg_baseline_converges():
    """The CPU block-Jacobi CG baseline (threaded) reaches the tolerance and agrees with a
    direct solve."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    from conftest import cube_system
    from oracle import oracle as orc
    s = cube_system(6)
    r, c, bl = orc.convert(s.rows, s.cols, s.blocks)
    x, k, _, _, done, threads, rel = orc.cg_bj_timed_mt(r, c, bl, s.b, tol=1e-8)
    assert done and rel <= 1e-8 and threads >= 1
    n = s.b.size
    I, J, V = [], [], []
    for kk in range(r.size):
        B = bl[kk].reshape(3, 3).T
        for a in range(3):
            for bb in range(3):
                I.append(3 * r[kk] + a); J.append(3 * c[kk] + bb); V.append(B[a, bb])
                if r[kk] != c[kk]:
                    I.append(3 * c[kk] + bb); J.append(3 * r[kk] + a); V.append(B[a, bb])
    A = sp.csr_matrix((V, (I, J)), shape=(n, n))
    xe = spl.spsolve(A.tocsc(), s.b)
    assert np.linalg.norm(x - xe) <= 1e-6 * np.linalg.norm(xe)
