"""GPU: batched solves of uneven scenes over several streams give, scene by scene, bitwise
the results of solving each scene alone; the single-rank distributed path gathers them."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _t(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def _scenes():
    from stgipc import scenes
    return scenes.make_batched_cubes(count=10, seed=78, n_lo=3, n_hi=8)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_batch_matches_single_solves(dev, precision):
    import torch
    from stgipc import PCGSolverConfig, Solver
    from stgipc.batch import BatchSolver
    sysl = _scenes()
    cfg = PCGSolverConfig(precision=precision, stop_rule="relative_residual")
    bs = BatchSolver(sysl, cfg, streams=4)
    try:
        stats = bs.solve()
        for k, s in enumerate(sysl):
            single = Solver(cfg)
            pm, rm = s.slot_maps(cfg.bank_size)
            single.mas_init(s.num_verts, s.neighbor_start, s.neighbor_num, s.neighbor_list, pm, rm)
            rows, cols = torch.from_numpy(s.rows).to(dev), torch.from_numpy(s.cols).to(dev)
            blocks, b = torch.from_numpy(s.blocks.reshape(-1)).to(dev), torch.from_numpy(s.b).to(dev)
            contacts = torch.from_numpy(s.contacts).to(dev) if s.contacts.size else None
            x = torch.zeros_like(b)
            st = single.solve_linear_system(rows, cols, blocks, b, x, fem_block_offset=s.fem_block_offset,
                                            contacts=contacts)
            single.close()
            assert stats[k]["iterations"] == st["iterations"], k
            assert np.array_equal(bs.solution(k), x.cpu().numpy()), k
            assert stats[k]["rel_residual"] <= 1.5e-4, (k, stats[k]["rel_residual"])
    finally:
        bs.close()


def test_solve_distributed_one_rank_on_gpu(dev):
    from stgipc import PCGSolverConfig
    from stgipc.batch import solve_distributed
    sysl = _scenes()
    out = solve_distributed(sysl, rank=0, world=1, config=PCGSolverConfig(stop_rule="relative_residual"),
                            streams=3)
    assert len(out) == len(sysl)
    assert all(o["rel_residual"] <= 1.5e-4 for o in out)


@pytest.mark.parametrize("per_scene,prec,loop", [(True, "fp32", "graph"), (True, "fp64", "host"),
                                                  (False, "fp32", "graph")])
def test_concatenated_batch_meets_every_scene_tolerance(dev, per_scene, prec, loop):
    """The whole batch as one block-diagonal system (one handle): every scene's own FP64
    relative residual meets the tolerance, checked with the oracle's convert and SpMV.  With
    per-scene recurrences each scene stops on its own test and the loop ends with the last
    one.  (Iteration counts are not those of the scenes solved alone: coarse MAS banks group
    the concatenated nodes differently, so the preconditioner differs.)"""
    from oracle import oracle as orc
    from stgipc import PCGSolverConfig, scenes
    from stgipc.batch import ConcatenatedBatch
    sysl = scenes.make_batched_cubes(count=12, seed=1004, n_lo=3, n_hi=9)
    cfg = PCGSolverConfig(precision=prec, stop_rule="relative_residual", global_tol_rate=1e-4, loop=loop)
    cb = ConcatenatedBatch(sysl, cfg, device=dev, per_scene=per_scene)
    st = cb.solve()
    assert st["status"] == 0
    res_gpu = cb.scene_residuals()
    for k, s in enumerate(sysl):
        r, c, bl = orc.convert(s.rows, s.cols, s.blocks)
        x = cb.solution(k)
        y = orc.spmv(r, c, bl, x)
        rel = np.linalg.norm(s.b - y) / np.linalg.norm(s.b)
        assert rel <= 1.1e-4, (k, rel)
        assert abs(rel - res_gpu[k]) <= 1e-6 + 1e-3 * rel
    if per_scene:
        its, rels = cb.scene_stats()
        assert np.all(rels <= 1e-4) and np.all(its > 0)
        assert st["iterations"] == its.max()
    cb.close()


def test_per_scene_recurrences_match_each_scene_alone(dev):
    """With FP64 block-Jacobi (no coarse levels, so each scene's preconditioner is exactly its
    own) every scene's recurrence inside the concatenated solve is the scene's own PCG: the
    same iteration count as the oracle solving the scene alone (+-1 for summation order) and
    the same solution."""
    from oracle import oracle as orc
    from stgipc import PCGSolverConfig, scenes
    from stgipc.batch import ConcatenatedBatch
    sysl = scenes.make_batched_cubes(count=8, seed=1007, n_lo=3, n_hi=8)
    cfg = PCGSolverConfig(precision="fp64", preconditioner="diag", stop_rule="relative_residual",
                          global_tol_rate=1e-6)
    cb = ConcatenatedBatch(sysl, cfg, device=dev, per_scene=True)
    st = cb.solve()
    its, rels = cb.scene_stats()
    assert st["iterations"] == its.max()
    for k, s in enumerate(sysl):
        r, c, bl = orc.convert(s.rows, s.cols, s.blocks)
        # uncapped: the batch's iteration cap is 0.3 n of the whole batch, not of the scene
        xe, se, _, done = orc.pcg_timed(r, c, bl, s.b, use_diag=True, tol=1e-6, stop_rule="relative",
                                        max_iter_ratio=100.0)
        assert done and se["rel_residual"] <= 1.1e-6
        assert abs(int(its[k]) - se["iterations"]) <= 1, (k, its[k], se["iterations"])
        x = cb.solution(k)
        # equal counts: the same iterates up to FP64 summation order
        tol = 1e-7 if int(its[k]) == se["iterations"] else 1e-5
        assert np.linalg.norm(x - xe) <= tol * np.linalg.norm(xe), (k, np.linalg.norm(x - xe) / np.linalg.norm(xe))
    cb.close()
