"""GPU parity: libstgipc (sm_100a) against the CPU oracle, through the C ABI.

Tolerances:
  * integer work (convert indices, MAS masks / coarse ids / tables): bit-exact;
  * convert block sums: bit-exact (both sum duplicates in input order);
  * FP64 SpMV: 1e-13 relative (different summation order);
  * MAS Galerkin matrices, FP32 inverses and apply: bit-exact.  The reference sums these
    with atomics, in no defined order; the oracle (ORC_ORDER_FIXED) fixes the order the
    kernels use, and tests/test_oracle.py checks that order against the literal walk of the
    reference's loops (ORC_ORDER_WALK);
  * PCG, FP64 (block Jacobi or MAS): the same iteration count and x within 1e-8 relative of
    the oracle (only the FP64 SpMV and dot-product orders differ);
  * FP32 storage path: against the FP64 oracle, with its FP64 true residual <= 1.5e-4.
"""
import numpy as np
import pytest

from conftest import cube_system, fixture_system, random_contacts

pytestmark = pytest.mark.gpu


def _t(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def _solver(**kw):
    from stgipc import PCGSolverConfig, Solver
    return Solver(PCGSolverConfig(**kw))


def _converted(sysm):
    from oracle import oracle as orc
    return orc.convert(sysm.rows, sysm.cols, sysm.blocks)


# ------------------------------------------------------------------------------------------
def test_convert_bit_exact(dev):
    from oracle import oracle as orc
    s = cube_system(16)
    rng = np.random.default_rng(7)
    perm = rng.permutation(s.rows.size)
    extra = rng.integers(0, s.rows.size, size=5000)   # duplicate some triplets
    rows = np.concatenate([s.rows[perm], s.rows[extra]])
    cols = np.concatenate([s.cols[perm], s.cols[extra]])
    blocks = np.concatenate([s.blocks[perm], s.blocks[extra] * 0.5])
    er, ec, eb = orc.convert(rows, cols, blocks)
    R, Cc, Bk = _t(rows, dev), _t(cols, dev), _t(blocks.reshape(-1), dev)
    u = _solver().convert(R, Cc, Bk)
    assert u == er.size
    assert np.array_equal(R[:u].cpu().numpy(), er)
    assert np.array_equal(Cc[:u].cpu().numpy(), ec)
    assert np.array_equal(Bk[:9 * u].cpu().numpy().reshape(-1, 9), eb)


def test_convert_edge_cases(dev):
    from oracle import oracle as orc
    solver = _solver()
    # single triplet
    R, Cc, Bk = _t(np.array([3], np.int32), dev), _t(np.array([5], np.int32), dev), _t(np.arange(9.0), dev)
    assert solver.convert(R, Cc, Bk) == 1
    # all duplicates of one key, and a row with no entries in between
    rows = np.array([0, 0, 0, 2, 2], np.int32)
    cols = np.array([1, 1, 1, 2, 2], np.int32)
    blocks = np.random.default_rng(1).standard_normal((5, 9))
    er, ec, eb = orc.convert(rows, cols, blocks)
    R, Cc, Bk = _t(rows, dev), _t(cols, dev), _t(blocks.reshape(-1), dev)
    u = solver.convert(R, Cc, Bk)
    assert u == 2 and np.array_equal(R[:u].cpu().numpy(), er) and np.array_equal(Cc[:u].cpu().numpy(), ec)
    assert np.array_equal(Bk[:9 * u].cpu().numpy().reshape(-1, 9), eb)


def test_convert_long_rows_bit_exact(dev):
    """Rows far longer than the warp sort's 128 entries (sorted by a CTA each) and runs of
    more than a thousand duplicates of one block (summed warp-cooperatively in input order):
    a 1,500-entry row with a 1,200-entry run, a 5,000-entry row (beyond the CTA's
    shared-memory sort, ranked), and rows of exactly 129 entries, mixed with short rows."""
    from oracle import oracle as orc
    rng = np.random.default_rng(23)
    rows, cols = [], []
    rows += [7] * 1500
    cols += [7] * 1200 + list(rng.integers(7, 200, size=300))
    rows += [11] * 5000
    cols += list(rng.integers(11, 400, size=5000))
    rows += [13] * 129
    cols += list(rng.integers(13, 60, size=129))
    for r in range(400):
        k = int(rng.integers(1, 20))
        rows += [r] * k
        cols += list(rng.integers(r, 400, size=k))
    rows, cols = np.array(rows, np.int32), np.array(cols, np.int32)
    perm = rng.permutation(rows.size)
    rows, cols = rows[perm], cols[perm]
    blocks = rng.standard_normal((rows.size, 9))
    er, ec, eb = orc.convert(rows, cols, blocks)
    R, Cc, Bk = _t(rows, dev), _t(cols, dev), _t(blocks.reshape(-1), dev)
    u = _solver().convert(R, Cc, Bk)
    assert u == er.size
    assert np.array_equal(R[:u].cpu().numpy(), er) and np.array_equal(Cc[:u].cpu().numpy(), ec)
    assert np.array_equal(Bk[:9 * u].cpu().numpy().reshape(-1, 9), eb)


# ------------------------------------------------------------------------------------------
@pytest.mark.parametrize("a,b", [(1.0, 0.0), (-0.5, 2.0)])
def test_spmv(dev, a, b):
    from oracle import oracle as orc
    s = cube_system(16)
    r, c, bl = _converted(s)
    rng = np.random.default_rng(3)
    x = rng.standard_normal(s.n)
    y0 = rng.standard_normal(s.n)
    ye = orc.spmv(r, c, bl, x, a=a, b=b, y=y0)
    Y = _t(y0, dev)
    _solver().spmv(a, _t(bl.reshape(-1), dev), _t(r, dev), _t(c, dev), r.size, _t(x, dev), b, Y)
    yg = Y.cpu().numpy()
    assert np.max(np.abs(yg - ye)) <= 1e-13 * np.max(np.abs(ye))


def test_spmv_deterministic(dev):
    s = cube_system(16)
    r, c, bl = _converted(s)
    x = np.random.default_rng(4).standard_normal(s.n)
    solver = _solver()
    outs = []
    for _ in range(3):
        Y = _t(np.zeros(s.n), dev)
        solver.spmv(1.0, _t(bl.reshape(-1), dev), _t(r, dev), _t(c, dev), r.size, _t(x, dev), 0.0, Y)
        outs.append(Y.cpu().numpy())
    assert all(np.array_equal(outs[0], o) for o in outs[1:])


# ------------------------------------------------------------------------------------------
def _mas_pair(sysm, bank, part=None, contacts=None, dev=None):
    from stgipc import scenes
    from oracle import oracle as orc
    if part is None:
        pm, rm = sysm.slot_maps(bank)
    else:
        pm, rm = scenes.slot_maps_from_parts(part, bank)
    om = orc.Mas(bank, sysm.num_verts, sysm.neighbor_start, sysm.neighbor_num, sysm.neighbor_list, pm, rm)
    om.build(contacts)
    solver = _solver(bank_size=bank)
    solver.mas_init(sysm.num_verts, sysm.neighbor_start, sysm.neighbor_num, sysm.neighbor_list, pm, rm)
    r, c, bl = _converted(sysm)
    om.assemble(r, c, bl)
    C = None if contacts is None else _t(contacts, dev)
    solver.mas_assemble(_t(bl.reshape(-1), dev), _t(r, dev), _t(c, dev), r.size, 0, C)
    return om, solver, pm, (r, c, bl)


def _compare_hierarchy(om, solver, pm):
    e = om.hierarchy()
    g = solver.export_hierarchy(pm.size)
    L, T, ls = solver.mas_info()
    assert L == om.L and T == om.total
    assert np.array_equal(ls, e["level_size"])
    assert np.array_equal(g["fine_mask"], e["fine_mask"])
    assert np.array_equal(g["prefix_orig"], e["prefix_orig"])
    assert np.array_equal(g["coarse_tables"], e["coarse_tables"])
    V = om.V
    assert np.array_equal(g["going_next"][:V], e["going_next"][:V])
    assert np.array_equal(g["going_next"][om.M:T], e["going_next"][om.M:T])
    if L > 1:
        assert np.array_equal(g["coarse_table"], e["coarse_table"])


@pytest.mark.parametrize("bank", [16, 32])
@pytest.mark.parametrize("with_contacts", [False, True])
def test_mas_hierarchy_bit_exact_morton(dev, bank, with_contacts):
    s = cube_system(16)
    cp = random_contacts(s.num_verts, 600, seed=11) if with_contacts else None
    om, solver, pm, _ = _mas_pair(s, bank, contacts=cp, dev=dev)
    _compare_hierarchy(om, solver, pm)


@pytest.mark.parametrize("name", ["bunny2", "high_mat"])
@pytest.mark.parametrize("with_contacts", [False, True])
def test_mas_hierarchy_bit_exact_metis_fixture(dev, name, with_contacts):
    """The reference's METIS-sorted meshes as it ships them: 16-vertex partitions (bunny2:
    19,193 vertices in 1,280 parts; high_mat: 45,000 in 3,000), partition-sorted.  The
    hierarchy, and the bank matrices and inverses assembled on it, are bit-exact."""
    s, part = fixture_system(name)
    cp = random_contacts(s.num_verts, 2000, seed=12) if with_contacts else None
    om, solver, pm, _ = _mas_pair(s, 16, part=part, contacts=cp, dev=dev)
    _compare_hierarchy(om, solver, pm)
    em, ei = om.matrices()
    gm, gi = solver.export_matrices()
    assert np.array_equal(gm, em) and np.array_equal(gi, ei)


@pytest.mark.parametrize("bank", [16, 32])
def test_mas_matrices_and_inverse(dev, bank):
    s = cube_system(16)
    om, solver, pm, _ = _mas_pair(s, bank, dev=dev)
    em, ei = om.matrices()
    gm, gi = solver.export_matrices()
    assert gm.shape == em.shape
    assert np.array_equal(gm, em)
    assert np.array_equal(gi, ei)


@pytest.mark.parametrize("bank", [16, 32])
def test_mas_apply(dev, bank):
    s = cube_system(16)
    om, solver, pm, _ = _mas_pair(s, bank, dev=dev)
    rvec = np.random.default_rng(5).standard_normal(s.n)
    ze = om.apply(rvec)
    Z = _t(np.zeros(s.n), dev)
    solver.mas_apply(_t(rvec, dev), Z)
    assert np.array_equal(Z.cpu().numpy(), ze)


def test_mas_apply_metis_fixture_with_contacts(dev):
    s, part = fixture_system("bunny2")
    cp = random_contacts(s.num_verts, 2000, seed=13)
    om, solver, pm, _ = _mas_pair(s, 16, part=part, contacts=cp, dev=dev)
    rvec = np.random.default_rng(6).standard_normal(s.n)
    ze = om.apply(rvec)
    Z = _t(np.zeros(s.n), dev)
    solver.mas_apply(_t(rvec, dev), Z)
    assert np.array_equal(Z.cpu().numpy(), ze)
    em, ei = om.matrices()
    gm, gi = solver.export_matrices()
    assert np.array_equal(gm, em) and np.array_equal(gi, ei)


# ------------------------------------------------------------------------------------------
@pytest.mark.parametrize("loop", ["host", "graph", "persistent"])
def test_pcg_block_jacobi_fp64(dev, loop):
    """All-FP64 path (global 3x3 block-Jacobi = DiagPreconditioner): x within 1e-8."""
    from oracle import oracle as orc
    s = cube_system(16)
    r, c, bl = _converted(s)
    xe, st_e = orc.pcg(r, c, bl, s.b, use_diag=True)
    solver = _solver(preconditioner="diag", loop=loop)
    X = _t(np.zeros(s.n), dev)
    st = solver.pcg_solve(_t(bl.reshape(-1), dev), _t(r, dev), _t(c, dev), r.size, _t(s.b, dev), X)
    assert st["iterations"] == st_e["iterations"]
    xg = X.cpu().numpy()
    assert np.linalg.norm(xg - xe) <= 1e-8 * np.linalg.norm(xe)
    assert abs(st["rel_residual"] - st_e["rel_residual"]) <= 1e-6 * max(st_e["rel_residual"], 1e-30)


@pytest.mark.parametrize("bank", [16, 32])
@pytest.mark.parametrize("loop", ["host", "graph", "persistent"])
def test_pcg_mas_vs_oracle(dev, bank, loop):
    from oracle import oracle as orc
    s = cube_system(16)
    om, _, pm, (r, c, bl) = _mas_pair(s, bank, dev=dev)
    xe, st_e = orc.pcg(r, c, bl, s.b, mas=om)
    G = _t(bl.reshape(-1), dev), _t(r, dev), _t(c, dev)
    solver = _solver(bank_size=bank, loop=loop)
    solver.mas_init(s.num_verts, s.neighbor_start, s.neighbor_num, s.neighbor_list, *s.slot_maps(bank))
    solver.mas_assemble(G[0], G[1], G[2], r.size, 0, None)
    X = _t(np.zeros(s.n), dev)
    st = solver.pcg_solve(G[0], G[1], G[2], r.size, _t(s.b, dev), X)
    assert st["iterations"] == st_e["iterations"]
    xg = X.cpu().numpy()
    assert np.linalg.norm(xg - xe) <= 1e-8 * np.linalg.norm(xe)


@pytest.mark.parametrize("precond,precision", [("diag", "fp64"), ("mas", "fp64"), ("mas", "fp32")])
def test_loop_modes_agree(dev, precond, precision):
    """host and graph drivers launch the same kernels with the same grids: bitwise equal.
    The persistent kernel partitions the FP64 reductions differently and uses the untiled
    SpMV: same iterations (+-1), solution within 1e-8 (FP64) / 1e-5 (FP32 storage) relative."""
    from stgipc import GlobalLinearSystem, PCGSolverConfig
    s = cube_system(16)
    res = {}
    for loop in ("host", "graph", "persistent"):
        cfg = PCGSolverConfig(loop=loop, preconditioner=precond, precision=precision, refine_interval=8,
                              stop_rule="relative_residual")
        gls = GlobalLinearSystem(s, cfg, device=dev)
        st = gls.solve_linear_system()
        assert st["status"] == 0, (loop, st)
        res[loop] = (st["iterations"], gls.x.cpu().numpy(), st["replacements"])
    assert res["host"][0] == res["graph"][0] and np.array_equal(res["host"][1], res["graph"][1])
    assert res["host"][2] == res["graph"][2]
    assert abs(res["persistent"][0] - res["host"][0]) <= 1
    # FP64: only the FP64 dot-product and SpMV orders differ (the MAS bank solves of all
    # drivers share one order); FP32 storage: the SpMV sums FP32 products in another order
    tol = 1e-8 if precision == "fp64" else 1e-5
    assert np.linalg.norm(res["persistent"][1] - res["host"][1]) <= tol * np.linalg.norm(res["host"][1])


def test_dot_products_deterministic(dev):
    """Two solves of the same system give bitwise identical x (no atomics in any sum)."""
    from stgipc import GlobalLinearSystem, PCGSolverConfig
    s = cube_system(16)
    xs = []
    for _ in range(2):
        gls = GlobalLinearSystem(s, PCGSolverConfig(precision="fp32", stop_rule="relative_residual"), device=dev)
        gls.solve_linear_system()
        xs.append(gls.x.cpu().numpy())
    assert np.array_equal(xs[0], xs[1])


@pytest.mark.parametrize("bank", [16, 32])
def test_solve_linear_system_end_to_end(dev, bank):
    """Triplets -> convert -> MAS build/assemble -> PCG, against the oracle pipeline."""
    from oracle import oracle as orc
    from stgipc import GlobalLinearSystem, PCGSolverConfig
    s = cube_system(16)
    r, c, bl = _converted(s)
    om = orc.Mas(bank, s.num_verts, s.neighbor_start, s.neighbor_num, s.neighbor_list, *s.slot_maps(bank))
    om.build()
    om.assemble(r, c, bl)
    xe, st_e = orc.pcg(r, c, bl, s.b, mas=om)
    gls = GlobalLinearSystem(s, PCGSolverConfig(bank_size=bank), device=dev)
    st = gls.solve_linear_system()
    assert st["nnzb"] == r.size == 35937
    assert st["iterations"] == st_e["iterations"]
    assert np.linalg.norm(gls.x.cpu().numpy() - xe) <= 1e-8 * np.linalg.norm(xe)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_solve_with_contacts_end_to_end(dev, precision):
    """The whole solve with sign-encoded contact pairs of all seven encodings: they join the
    MAS in-bank connectivity (collision_connection) and so change the preconditioner; the
    GPU hierarchy and solve follow the oracle's."""
    from oracle import oracle as orc
    from stgipc import PCGSolverConfig, Solver
    s = cube_system(16)
    cp = random_contacts(s.num_verts, 400, seed=17)
    r, c, bl = _converted(s)
    om = orc.Mas(16, s.num_verts, s.neighbor_start, s.neighbor_num, s.neighbor_list, *s.slot_maps(16))
    om.build(cp)
    om.assemble(r, c, bl)
    xe, st_e = orc.pcg(r, c, bl, s.b, mas=om)
    om0 = orc.Mas(16, s.num_verts, s.neighbor_start, s.neighbor_num, s.neighbor_list, *s.slot_maps(16))
    om0.build()
    assert om.total != om0.total  # the contacts do change the hierarchy
    solver = Solver(PCGSolverConfig(precision=precision))
    solver.mas_init(s.num_verts, s.neighbor_start, s.neighbor_num, s.neighbor_list, *s.slot_maps(16))
    X = _t(np.zeros(s.n), dev)
    st = solver.solve_linear_system(_t(s.rows, dev), _t(s.cols, dev), _t(s.blocks.reshape(-1), dev), _t(s.b, dev), X,
                                    contacts=_t(cp, dev))
    assert st["total_clusters"] == om.total
    xg = X.cpu().numpy()
    if precision == "fp64":
        assert st["iterations"] == st_e["iterations"]
        assert np.linalg.norm(xg - xe) <= 1e-8 * np.linalg.norm(xe)
    else:
        assert abs(st["iterations"] - st_e["iterations"]) <= 4
        assert np.linalg.norm(xg - xe) <= 1e-3 * np.linalg.norm(xe)


@pytest.mark.parametrize("bank", [16, 32])
def test_fused_level0_pass_bit_exact(dev, bank):
    """stg_solve_linear_system builds the hierarchy first and lets the fine convert store the
    level-0 bank blocks and emit the level-1 Galerkin triplets in its emit pass; the bank
    matrices and inverses it leaves are bit-identical to the oracle's (and so to the
    standalone stg_mas_assemble path's), here with contacts."""
    from oracle import oracle as orc
    from stgipc import PCGSolverConfig, Solver
    s = cube_system(16)
    cp = random_contacts(s.num_verts, 400, seed=29)
    r, c, bl = _converted(s)
    om = orc.Mas(bank, s.num_verts, s.neighbor_start, s.neighbor_num, s.neighbor_list, *s.slot_maps(bank))
    om.build(cp)
    om.assemble(r, c, bl)
    em, ei = om.matrices()
    solver = Solver(PCGSolverConfig(bank_size=bank))
    solver.mas_init(s.num_verts, s.neighbor_start, s.neighbor_num, s.neighbor_list, *s.slot_maps(bank))
    X = _t(np.zeros(s.n), dev)
    st = solver.solve_linear_system(_t(s.rows, dev), _t(s.cols, dev), _t(s.blocks.reshape(-1), dev), _t(s.b, dev), X,
                                    contacts=_t(cp, dev))
    assert st["status"] == 0
    gm, gi = solver.export_matrices()
    assert np.array_equal(gm, em) and np.array_equal(gi, ei)


def test_fp32_mode_relative_residual(dev):
    """FP32 SpMV/MAS storage, FP64 dots + residual replacement: FP64 residual <= 1e-4."""
    from oracle import oracle as orc
    from stgipc import GlobalLinearSystem, PCGSolverConfig
    s = cube_system(16)
    r, c, bl = _converted(s)
    om = orc.Mas(16, s.num_verts, s.neighbor_start, s.neighbor_num, s.neighbor_list, *s.slot_maps(16))
    om.build()
    om.assemble(r, c, bl)
    xe, _ = orc.pcg(r, c, bl, s.b, mas=om, tol=1e-10)
    gls = GlobalLinearSystem(s, PCGSolverConfig(precision="fp32", stop_rule="relative_residual", refine_interval=8),
                             device=dev)
    st = gls.solve_linear_system()
    assert st["status"] == 0
    assert st["rel_residual"] <= 1.5e-4
    err = np.linalg.norm(gls.x.cpu().numpy() - xe) / np.linalg.norm(xe)
    assert err <= 1e-2


def test_invalid_arguments_raise(dev):
    from stgipc import StgError
    solver = _solver()
    import torch
    x = torch.zeros(5, dtype=torch.float64, device=dev)
    with pytest.raises(StgError):
        solver.spmv(1.0, x, x.int(), x.int(), 1, x, 0.0, x)   # n = 5 not a multiple of 3
    with pytest.raises(StgError):
        solver.mas_apply(x, x)                                 # MAS not initialised
    with pytest.raises(StgError):
        bad = np.array([0, 1, 99], np.int32)                  # part map entry out of range
        solver.mas_init(2, np.zeros(2), np.zeros(2), np.zeros(0), bad, np.array([0, 1]))
