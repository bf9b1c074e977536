"""GPU: the contact barrier producer (stg_contact_barrier) against the oracle, and a Newton
solve that includes its triplets.

Bars: rows / cols and the skipped count bit-exact; blocks and gradients within 1e-10 of the
largest entry of their pair (the GPU differentiates the distance in forward mode, the oracle
in closed form, both FP64); the solve of elastic + contact triplets (contacts also in the MAS
connectivity) at the oracle's FP64 iteration count and within 1e-8 of its x.
"""
import numpy as np
import pytest

from conftest import random_contacts

pytestmark = pytest.mark.gpu


def _t(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def _compare(pairs, x, dhat, kappa, dev, offset=0):
    from oracle import oracle as orc
    from stgipc.contact import barrier
    er, ec, eb, eg, esk = orc.contact_barrier(pairs, x, dhat, kappa, block_offset=offset)
    r, c, b, g, sk = barrier(_t(pairs.astype(np.int32), dev), _t(x, dev), dhat, kappa, block_offset=offset)
    assert np.array_equal(r.cpu().numpy(), er) and np.array_equal(c.cpu().numpy(), ec)
    assert int(sk.item()) == esk
    b, g = b.cpu().numpy().reshape(-1, 90), g.cpu().numpy()
    eb = eb.reshape(-1, 90)
    sb = np.maximum(np.abs(eb).max(axis=1, keepdims=True), 1e-300)
    sg = np.maximum(np.abs(eg).max(axis=1, keepdims=True), 1e-300)
    assert np.all(np.abs(b - eb) <= 1e-10 * sb)
    assert np.all(np.abs(g - eg) <= 1e-10 * sg)
    assert np.array_equal(eb == 0, b == 0)
    return b, g


def test_random_pairs_all_encodings(dev):
    """A jittered point cloud with pairs of every encoding (the mollified ones are skipped)."""
    rng = np.random.default_rng(21)
    V = 3000
    x = rng.uniform(0, 1, size=(V, 3))
    pairs = random_contacts(V, 7000, seed=22, local=8)
    # pull the pairs' vertices close together so that many are inside the barrier
    for q in pairs[:4000]:
        ids = [(-i - 1) if i < 0 else i for i in q]
        x[ids[1:]] = x[ids[0]] + rng.normal(scale=0.01, size=(3, 3))
    b, _ = _compare(pairs, x, 4e-4, 1e5, dev, offset=12)
    assert (np.abs(b).sum(axis=1) > 0).sum() > 1000  # many active pairs


def test_empty_and_edge_cases(dev):
    import torch
    from stgipc.contact import barrier
    from stgipc import StgError
    x = _t(np.zeros((4, 3)), dev)
    r, c, b, g, sk = barrier(torch.zeros((0, 4), dtype=torch.int32, device=dev), x, 1e-6, 1.0)
    assert r.numel() == 0 and int(sk.item()) == 0
    with pytest.raises(StgError):
        barrier(torch.zeros((1, 4), dtype=torch.int32, device=dev), x, 0.0, 1.0)  # dhat must be > 0
    # s >= 1 (outside the barrier) and coincident points (s = 0) give zero terms, not skips
    pts = np.array([[0, 0, 0], [1, 0, 0], [0, 0, 0], [0, 0, 0]], np.float64)
    pairs = np.array([[-1, 1, -1, -1], [-3, 3, -1, -1]], np.int32)
    bb, gg = _compare(pairs, pts, 0.25, 1.0, dev)
    assert np.all(bb == 0) and np.all(gg == 0)


def test_stacked_cubes_solve_with_contacts(dev):
    """Two cubes in contact: elastic + inertia + ground triplets plus the producer's contact
    triplets; the contacts also enter the MAS connectivity.  The GPU solve follows the oracle's
    FP64 PCG on the same triplets."""
    from oracle import oracle as orc
    from stgipc import PCGSolverConfig, Solver, scenes
    from stgipc.contact import barrier, scatter_gradient
    s, pairs, _ = scenes.make_stacked_cubes(8)
    dhat, kappa = 1e-6, 1e5
    P = _t(pairs, dev)
    cr, cc, cb, cg, sk = barrier(P, _t(s.pos, dev), dhat, kappa)
    assert int(sk.item()) == 0
    rows = np.concatenate([cr.cpu().numpy(), s.rows])
    cols = np.concatenate([cc.cpu().numpy(), s.cols])
    blocks = np.concatenate([cb.cpu().numpy(), s.blocks])
    b = s.b + scatter_gradient(P, cg, s.num_verts).cpu().numpy().reshape(-1)
    r, c, bl = orc.convert(rows, cols, blocks)
    om = orc.Mas(16, s.num_verts, s.neighbor_start, s.neighbor_num, s.neighbor_list, *s.slot_maps(16))
    om.build(pairs)
    om.assemble(r, c, bl)
    xe, st_e = orc.pcg(r, c, bl, b, mas=om)
    solver = Solver(PCGSolverConfig(precision="fp64"))
    solver.mas_init(s.num_verts, s.neighbor_start, s.neighbor_num, s.neighbor_list, *s.slot_maps(16))
    X = _t(np.zeros(s.n), dev)
    st = solver.solve_linear_system(_t(rows, dev), _t(cols, dev), _t(blocks.reshape(-1), dev), _t(b, dev), X,
                                    contacts=P)
    assert st["status"] == 0
    assert st["total_clusters"] == om.total
    assert st["iterations"] == st_e["iterations"]
    assert np.linalg.norm(X.cpu().numpy() - xe) <= 1e-8 * np.linalg.norm(xe)


def test_energy_matches_oracle(dev):
    """Per-pair barrier energies (stg_contact_energy) against the oracle, within 1e-12 of the
    largest."""
    from oracle import oracle as orc
    from stgipc.contact import energy
    rng = np.random.default_rng(31)
    V = 2000
    x = rng.uniform(0, 1, size=(V, 3))
    pairs = random_contacts(V, 5000, seed=32, local=8)
    for q in pairs[:3000]:
        ids = [(-i - 1) if i < 0 else i for i in q]
        x[ids[1:]] = x[ids[0]] + rng.normal(scale=0.01, size=(3, 3))
    want = orc.contact_energy(pairs, x, 4e-4, 1e5)
    got = energy(_t(pairs, dev), _t(x, dev), 4e-4, 1e5).cpu().numpy()
    assert (want > 0).sum() > 500
    assert np.array_equal(want == 0, got == 0)
    # near s = 1 the energy goes as (1 - s^2)^4, so a pair's relative error grows there: the
    # bound is relative to the largest energy of the set
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
