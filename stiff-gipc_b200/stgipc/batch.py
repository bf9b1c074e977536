"""Batches of independent Newton systems of uneven size, and their sharding over ranks.

A batch (e.g. 256 cubes of 375 to 47k DOFs, each with its own Hessian, contacts and MAS
partition) is solved scene by scene through the same C ABI as a single system
(``stg_solve_linear_system``).  On one GPU the scenes are spread over ``streams`` CUDA
streams, one host thread and one handle per scene.  The ctypes calls release the GIL, so
the solves overlap on the device: every scene runs its own graph-captured PCG, and small
scenes fill the SMs that a single small solve leaves idle.  Results are bitwise those of
a solve of the scene alone (the kernels are deterministic and per-handle).

Over several ranks the scenes are the units: ``shard_by_dof`` assigns whole scenes to
ranks by greedy DOF-balanced bin packing (largest first, onto the least-loaded rank).
Each rank solves its shard with no exchange during the solves.  The only collective is the
final gather of the per-scene statistics (``solve_distributed``).
"""
from __future__ import annotations

import concurrent.futures as cf
from typing import Callable, List, Optional, Sequence

import numpy as np

from .linear_system import PCGSolverConfig, Solver


def shard_by_dof(dofs: Sequence[int], world: int) -> List[List[int]]:
    """Scene indices per rank: largest scene first onto the least-loaded rank (ties go to
    the lower rank); each shard sorted.  Deterministic, so every rank computes the same
    assignment without communicating."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(dofs)), key=lambda i: (-int(dofs[i]), i))
    loads = [0] * world
    shards: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        shards[r].append(i)
        loads[r] += int(dofs[i])
    return [sorted(s) for s in shards]


class BatchSolver:
    """Solves a list of ``scenes.NewtonSystem`` on one GPU over ``streams`` CUDA streams."""

    def __init__(self, systems, config: Optional[PCGSolverConfig] = None, device="cuda", streams: int = 8):
        import torch
        self.config = config or PCGSolverConfig()
        self.device = torch.device(device)
        if self.device.index is None:
            self.device = torch.device(self.device.type, torch.cuda.current_device())
        self.systems = list(systems)
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(max(1, min(streams, len(self.systems))))]
        self.items = []
        for k, s in enumerate(self.systems):
            st = self.streams[k % len(self.streams)]
            solver = Solver(self.config, stream=st)
            if self.config.preconditioner == "mas":
                pm, rm = s.slot_maps(self.config.bank_size)
                solver.mas_init(s.num_verts, s.neighbor_start, s.neighbor_num, s.neighbor_list, pm, rm,
                                collision_node_offset=0)
            with torch.cuda.stream(st):
                t = dict(rows=torch.from_numpy(s.rows).to(self.device), cols=torch.from_numpy(s.cols).to(self.device),
                         blocks=torch.from_numpy(s.blocks.reshape(-1)).to(self.device),
                         b=torch.from_numpy(s.b).to(self.device),
                         contacts=(torch.from_numpy(s.contacts).to(self.device) if s.contacts.size else None))
                t["x"] = torch.zeros_like(t["b"])
            self.items.append((solver, st, t, s))
        torch.cuda.synchronize(self.device)

    def _solve_lane(self, lane: int) -> list:
        import torch
        torch.cuda.set_device(self.device)
        out = []
        for k in range(lane, len(self.items), len(self.streams)):
            solver, st, t, s = self.items[k]
            stats = solver.solve_linear_system(t["rows"], t["cols"], t["blocks"], t["b"], t["x"],
                                               fem_block_offset=s.fem_block_offset, contacts=t["contacts"])
            out.append((k, stats))
        return out

    def solve(self) -> List[dict]:
        """One Newton solve of every scene; per-scene statistics in scene order."""
        res: List[Optional[dict]] = [None] * len(self.items)
        with cf.ThreadPoolExecutor(max_workers=len(self.streams)) as ex:
            for part in ex.map(self._solve_lane, range(len(self.streams))):
                for k, stats in part:
                    res[k] = stats
        return res  # type: ignore[return-value]

    def upload_from_host(self):
        """Copies every scene's triplets, b (and contacts) again from pinned host memory on
        the scene's stream (the host-to-device part of an end-to-end step)."""
        import torch
        if not hasattr(self, "_host"):
            self._host = []
            for _, _, t, _ in self.items:
                self._host.append({k: v.cpu().pin_memory() for k, v in t.items() if v is not None and k != "x"})
        for (solver, st, t, s), h in zip(self.items, self._host):
            with torch.cuda.stream(st):
                for k, v in h.items():
                    t[k].copy_(v, non_blocking=True)

    def host_bytes(self):
        """(host-to-device, device-to-host) bytes of one end-to-end step."""
        h2d = sum(v.numel() * v.element_size() for _, _, t, _ in self.items for k, v in t.items()
                  if v is not None and k != "x")
        d2h = sum(t["x"].numel() * t["x"].element_size() for _, _, t, _ in self.items)
        return h2d, d2h

    def scene_stats(self):
        """(iterations, recurrence relative residual) per scene of the last solve
        (per-scene mode)."""
        return self.solver.segment_stats()

    def solution(self, k: int) -> np.ndarray:
        return self.items[k][2]["x"].cpu().numpy()

    def close(self):
        for solver, _, _, _ in self.items:
            solver.close()
        self.items = []


def solve_distributed(systems, rank: int, world: int, solve_shard: Optional[Callable] = None,
                      config: Optional[PCGSolverConfig] = None, streams: int = 8, group=None) -> List[dict]:
    """Solves ``systems`` sharded over ``world`` ranks (whole scenes per rank, see
    shard_by_dof) and returns every scene's statistics, in scene order, on every rank.

    ``solve_shard(list_of_systems) -> list_of_stats`` solves one rank's scenes (default: a
    BatchSolver on this rank's current GPU).  The statistics are gathered with
    ``torch.distributed.all_gather_object`` when ``world > 1``.
    """
    shards = shard_by_dof([s.n for s in systems], world)
    mine = shards[rank]
    if solve_shard is None:
        def solve_shard(local):
            bs = BatchSolver(local, config=config, streams=streams)
            try:
                return bs.solve()
            finally:
                bs.close()
    local_stats = solve_shard([systems[i] for i in mine]) if mine else []
    pairs = list(zip(mine, local_stats))
    if world > 1:
        import torch.distributed as dist
        gathered: list = [None] * world
        dist.all_gather_object(gathered, pairs, group=group)
    else:
        gathered = [pairs]
    out: List[Optional[dict]] = [None] * len(systems)
    for part in gathered:
        for i, st in part:
            if out[i] is not None:
                raise RuntimeError(f"scene {i} solved on two ranks")
            out[i] = st
    missing = [i for i, st in enumerate(out) if st is None]
    if missing:
        raise RuntimeError(f"scenes {missing[:8]} were not solved")
    return out  # type: ignore[return-value]


# ----------------------------------------------------------------------------------------
# one system for the whole batch
# ----------------------------------------------------------------------------------------
def concat_inputs(systems, bank: int = 16) -> dict:
    """The host arrays of the block-diagonal system of `systems`: triplets with block rows
    shifted by the vertices of the scenes before, concatenated gradients, CSR neighbour
    lists shifted the same way, and Morton partitions of `bank` vertices that never cross a
    scene (part_map with -1 padding, real_map = slot of each vertex, as set_mas_partition
    lays them out).  voff[s] is the first vertex (block row) of scene s."""
    nv = [s.num_verts for s in systems]
    voff = np.concatenate([[0], np.cumsum(nv)]).astype(np.int64)
    V = int(voff[-1])
    rows = np.concatenate([s.rows.astype(np.int64) + o for s, o in zip(systems, voff)]).astype(np.int32)
    cols = np.concatenate([s.cols.astype(np.int64) + o for s, o in zip(systems, voff)]).astype(np.int32)
    blocks = np.concatenate([s.blocks.reshape(-1, 9) for s in systems])
    b = np.concatenate([s.b for s in systems])
    starts, nums, lists, loff = [], [], [], 0
    for s, o in zip(systems, voff):
        starts.append(s.neighbor_start.astype(np.int64) + loff)
        nums.append(s.neighbor_num.astype(np.int64))
        lists.append(s.neighbor_list.astype(np.int64) + o)
        loff += int(s.neighbor_list.size)
    part = np.concatenate([np.arange(n) // bank for n in nv])
    pcount = np.concatenate([[0], np.cumsum([(n + bank - 1) // bank for n in nv])])
    part = part + np.repeat(pcount[:-1], nv)
    first = np.searchsorted(part, part)  # first vertex of each vertex's partition
    part_map = np.full(int(pcount[-1]) * bank, -1, np.int32)
    slot = part * bank + (np.arange(V) - first)
    part_map[slot] = np.arange(V, dtype=np.int32)
    return dict(voff=voff, V=V, rows=rows, cols=cols, blocks=blocks, b=b, part_map=part_map,
                real_map=slot.astype(np.int32), neighbor_start=np.concatenate(starts).astype(np.uint32),
                neighbor_num=np.concatenate(nums).astype(np.uint32), neighbor_list=np.concatenate(lists).astype(np.uint32))


class ConcatenatedBatch:
    """The scenes of a batch as one block-diagonal system, solved by one handle: one
    convert, one MAS hierarchy, one assembly and one graph-captured PCG for every scene.

    Vertices, triplets, neighbour lists and MAS partitions of scene s are shifted by the
    vertex count of the scenes before it, and every partition stays inside its scene, so
    no bank mixes scenes at level 0; at coarser levels nodes of different scenes may share
    a bank, but with no edges between them they are never merged and their bank matrix is
    block-diagonal, so the preconditioner never couples scenes.

    spmv_tiles: the SpMV kernel (Solver.spmv_tiles); 0, the default, lets the autotuner time
    the candidates on the batch's first solve and keep the choice for its shape class.

    per_scene=True (stg_set_segments): every scene runs its own recurrence (alpha, beta,
    stop test ||r_s|| <= tol ||b_s||) inside the one loop.  per_scene=False: one recurrence
    with global scalars and the stop test tightened to tol min_s ||b_s|| / ||b||, so that
    ||r_s|| <= ||r|| <= tol min_s ||b_s|| <= tol ||b_s|| for every scene s."""

    def __init__(self, systems, config: Optional[PCGSolverConfig] = None, device="cuda", bank: int = 16,
                 per_scene: bool = True, spmv_tiles: int = 0):
        import torch
        self.systems = list(systems)
        self.device = torch.device(device)
        cat = concat_inputs(self.systems, bank)
        self.voff = cat["voff"]
        V = cat["V"]
        rows, cols, blocks, b = cat["rows"], cat["cols"], cat["blocks"], cat["b"]
        part_map, real_map = cat["part_map"], cat["real_map"]
        starts, nums, lists = [cat["neighbor_start"]], [cat["neighbor_num"]], [cat["neighbor_list"]]
        bb = np.array([float(s.b @ s.b) for s in self.systems])
        self.tol = (config.global_tol_rate if config else 1e-4)
        self.per_scene = per_scene
        tol_eff = self.tol if per_scene else (self.tol * float(np.sqrt(bb.min() / bb.sum())) if bb.sum() > 0 else self.tol)
        cfg = dataclasses_replace(config or PCGSolverConfig(), bank_size=bank, stop_rule="relative_residual",
                                  global_tol_rate=tol_eff)
        self.config = cfg
        self.solver = Solver(cfg)
        self.solver.mas_init(V, np.concatenate(starts).astype(np.uint32), np.concatenate(nums).astype(np.uint32),
                             np.concatenate(lists).astype(np.uint32), part_map, real_map)
        if per_scene:
            self.solver.set_segments(self.voff.astype(np.int32))
        # the SpMV kernel of this batch's shape class: autotuned once per process by default
        # (stg_spmv_tiles: 0), or fixed
        self.solver.spmv_tiles(spmv_tiles)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(self.device)
        self.rows, self.cols, self.blocks, self.b = t(rows), t(cols), t(blocks.reshape(-1)), t(b)
        self.x = torch.zeros_like(self.b)
        self.V = V

    def solve(self, stats: bool = True) -> dict:
        self.x.zero_()
        return self.solver.solve_linear_system(self.rows, self.cols, self.blocks, self.b, self.x, stats=stats)

    def scene_stats(self):
        """(iterations, recurrence relative residual) per scene of the last solve
        (per-scene mode)."""
        return self.solver.segment_stats()

    def solution(self, k: int) -> np.ndarray:
        a, e = 3 * int(self.voff[k]), 3 * int(self.voff[k + 1])
        return self.x[a:e].cpu().numpy()

    def scene_residuals(self) -> np.ndarray:
        """||b_s - A_s x_s|| / ||b_s|| of every scene, from the triplets in FP64 (a check
        outside the solve: every triplet block and its transpose applied with gathers and
        scatter-adds)."""
        import torch
        B = self.blocks.view(-1, 3, 3).transpose(1, 2)  # row-major blocks
        r = self.rows.long()
        c = self.cols.long()
        X = self.x.view(-1, 3)
        y = torch.zeros_like(X)
        y.index_add_(0, r, torch.bmm(B, X[c].unsqueeze(2)).squeeze(2))
        off = r != c
        y.index_add_(0, c[off], torch.bmm(B[off].transpose(1, 2), X[r[off]].unsqueeze(2)).squeeze(2))
        d = (self.b.view(-1, 3) - y).pow(2).sum(1)
        bb = self.b.view(-1, 3).pow(2).sum(1)
        seg = torch.from_numpy(np.repeat(np.arange(len(self.systems)), np.diff(self.voff))).to(self.device)
        num = torch.zeros(len(self.systems), dtype=torch.float64, device=self.device).index_add_(0, seg, d)
        den = torch.zeros(len(self.systems), dtype=torch.float64, device=self.device).index_add_(0, seg, bb)
        return torch.sqrt(num / den).cpu().numpy()

    def close(self):
        self.solver.close()


def dataclasses_replace(cfg, **kw):
    import dataclasses
    return dataclasses.replace(cfg, **kw)
