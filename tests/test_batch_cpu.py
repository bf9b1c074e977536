"""CPU: sharding of scene batches over ranks, and the distributed solve's gather, on gloo
with two ranks (the per-scene solve is the CPU oracle here, so no GPU is involved)."""
import os
import socket

import numpy as np
import pytest

from conftest import ROOT


def _scenes(count=7):
    from stgipc import scenes
    return scenes.make_batched_cubes(count=count, seed=77, n_lo=2, n_hi=5)


def _oracle_shard(systems):
    """Per-scene block-Jacobi PCG of the oracle, standing in for the GPU batch solver."""
    from oracle import oracle as orc
    out = []
    for s in systems:
        r, c, b = orc.convert(s.rows, s.cols, s.blocks)
        x, st = orc.pcg(r, c, b, s.b, use_diag=True, tol=1e-4)
        out.append({"iterations": int(st["iterations"]), "rel_residual": float(st["rel_residual"]),
                    "x_norm": float(np.linalg.norm(x)), "n": int(s.n)})
    return out


def test_shard_by_dof_partitions_and_balances():
    from stgipc.batch import shard_by_dof
    rng = np.random.default_rng(5)
    for world in (1, 2, 3, 8):
        dofs = rng.integers(375, 47000, size=256).tolist()
        shards = shard_by_dof(dofs, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(dofs)))
        loads = [sum(dofs[i] for i in s) for s in shards]
        # greedy largest-first: no rank exceeds another by more than the largest scene
        assert max(loads) - min(loads) <= max(dofs)
        assert shards == shard_by_dof(dofs, world)  # deterministic on every rank
    assert shard_by_dof([10, 10, 10], 5)[3:] == [[], []]
    with pytest.raises(ValueError):
        shard_by_dof([1], 0)


def test_solve_distributed_single_rank():
    from stgipc.batch import solve_distributed
    sysl = _scenes(4)
    out = solve_distributed(sysl, rank=0, world=1, solve_shard=_oracle_shard)
    assert [o["n"] for o in out] == [s.n for s in sysl]
    assert all(o["iterations"] > 0 and np.isfinite(o["x_norm"]) for o in out)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import sys
    sys.path.insert(0, os.path.join(ROOT, "stiff-gipc_b200"))
    sys.path.insert(0, ROOT)
    import datetime
    import pickle
    import torch.distributed as dist
    from stgipc.batch import shard_by_dof, solve_distributed
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        sysl = _scenes(7)
        mine = shard_by_dof([s.n for s in sysl], world)[rank]
        out = solve_distributed(sysl, rank=rank, world=world, solve_shard=_oracle_shard)
        with open(os.path.join(out_dir, f"rank{rank}.pkl"), "wb") as f:
            pickle.dump({"mine": mine, "out": out}, f)
    finally:
        dist.destroy_process_group()


def test_solve_distributed_gloo_two_ranks(tmp_path):
    import pickle
    import torch.multiprocessing as mp
    port = _free_port()
    mp.spawn(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    r0 = pickle.load(open(tmp_path / "rank0.pkl", "rb"))
    r1 = pickle.load(open(tmp_path / "rank1.pkl", "rb"))
    # disjoint shards covering every scene; identical gathered results on both ranks
    assert sorted(r0["mine"] + r1["mine"]) == list(range(7))
    assert not set(r0["mine"]) & set(r1["mine"])
    assert r0["out"] == r1["out"]
    # the same as solving everything on one rank
    ref = _oracle_shard(_scenes(7))
    assert r0["out"] == ref


def test_concatenated_inputs():
    """The block-diagonal batch's host arrays: triplets and neighbours shifted per scene,
    every partition inside one scene, part_map / real_map inverse to each other and equal
    to each scene's own slot maps shifted by its partitions."""
    from stgipc import scenes
    from stgipc.batch import concat_inputs
    sysl = scenes.make_batched_cubes(count=5, seed=1004, n_lo=2, n_hi=5)
    cat = concat_inputs(sysl, 16)
    voff = cat["voff"]
    V = cat["V"]
    assert V == sum(s.num_verts for s in sysl)
    pm, rm = cat["part_map"], cat["real_map"]
    assert np.all(pm[rm] == np.arange(V))
    assert np.count_nonzero(pm >= 0) == V
    scene_of = np.repeat(np.arange(len(sysl)), np.diff(voff))
    for bank in range(pm.size // 16):
        members = pm[16 * bank:16 * bank + 16]
        members = members[members >= 0]
        assert np.unique(scene_of[members]).size <= 1
    soff = 0
    for k, s in enumerate(sysl):
        pm_s, rm_s = s.slot_maps(16)
        np.testing.assert_array_equal(rm[voff[k]:voff[k + 1]], rm_s + soff)
        soff += pm_s.size
        a, e = 3 * voff[k], 3 * voff[k + 1]
        np.testing.assert_array_equal(cat["b"][a:e], s.b)
    r = cat["rows"]
    assert np.all(scene_of[r] == scene_of[cat["cols"]])  # no coupling block between scenes
    nl = cat["neighbor_list"].astype(np.int64)
    ns = cat["neighbor_start"].astype(np.int64)
    nn = cat["neighbor_num"].astype(np.int64)
    for v in range(0, V, 7):
        nb = nl[ns[v]:ns[v] + nn[v]]
        assert np.all(scene_of[nb] == scene_of[v])
