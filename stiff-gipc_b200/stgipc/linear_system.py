"""Python mirror of the reference's linear-system plugin API over the C ABI.

Names and argument meaning follow StiffGIPC/linear_system:
  * ``PCGSolverConfig`` -- linear_system/solver/pcg_solver.h:6-16
  * ``GlobalLinearSystem.solve_linear_system`` -- global_linear_system.cu:136-148
  * ``MASPreconditioner.assemble / apply`` -- preconditioner/fem_mas_preconditioner.cu:18-37
  * ``Spmv.srbk_spmv`` -- utils/spmv.cu:188-313, ``Converter.srbk_convert`` -- utils/converter.cu:32-51

Device memory is PyTorch CUDA tensors (plumbing only); every compute step runs in
libstgipc.so.  Errors raise ``StgError`` with the library's message.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Optional

import numpy as np

from . import _lib as _L
from ._lib import StgError, check

__all__ = ["PCGSolverConfig", "Solver", "GlobalLinearSystem", "StgError"]


@dataclasses.dataclass
class PCGSolverConfig:
    """PCGSolverConfig (pcg_solver.h:6-16) plus the B200 build's knobs."""
    max_iter_ratio: float = 0.3
    global_tol_rate: float = 1e-4
    bank_size: int = 16
    precision: str = "fp64"            # "fp64" (reference numerics) | "fp32"
    preconditioner: str = "mas"        # "mas" (P_type == 1) | "diag" | "none"
    stop_rule: str = "reference"       # "reference": |r.z| <= tol r0.z0 | "relative_residual"
    refine_interval: int = 32
    loop: str = "graph"                # "host" | "graph" | "persistent"
    graph_batch: int = 8
    learned: bool = False

    def to_c(self, stream_ptr: int = 0) -> _L.Config:
        c = _L.Config()
        _L.lib().stg_config_default(C.byref(c))
        c.bank_size = self.bank_size
        c.precision = _L.PREC[self.precision]
        c.preconditioner = _L.PRECOND[self.preconditioner]
        c.stop_rule = _L.STOP[self.stop_rule]
        c.tol = self.global_tol_rate
        c.max_iter_ratio = self.max_iter_ratio
        c.refine_interval = self.refine_interval
        c.loop_mode = _L.LOOP[self.loop]
        c.graph_batch = self.graph_batch
        c.learned = 1 if self.learned else 0
        c.stream = stream_ptr or None
        return c


def _ptr(t) -> Optional[int]:
    if t is None:
        return None
    if isinstance(t, np.ndarray):
        return t.ctypes.data
    if not t.is_contiguous():
        raise ValueError("tensor must be contiguous")
    return t.data_ptr()


def _require_cuda(*ts):
    for t in ts:
        if t is not None and not t.is_cuda:
            raise ValueError("device arrays must be CUDA tensors")


def spmv_noalloc(a, blocks, rows, cols, nnzb, x, b, y, stream=None):
    """y = a A x + b y without a handle and without device allocation (stg_spmv_noalloc).

    For callers that cannot allocate device memory; sizes up to STG_NOALLOC_MAX_ROWS block
    rows and STG_NOALLOC_MAX_BLOCKS blocks.  Calls share one fixed device scratch array, so
    calls that overlap on the GPU race.  `stream` is a torch.cuda.Stream or None (legacy
    default stream).  The call is synchronous and cannot be captured in a CUDA graph."""
    import torch
    _require_cuda(blocks, rows, cols, x, y)
    if len({t.device for t in (blocks, rows, cols, x, y)}) != 1:
        raise ValueError("spmv_noalloc: all tensors must be on one device")
    if blocks.dtype != torch.float64 or x.dtype != torch.float64 or y.dtype != torch.float64:
        raise ValueError("spmv_noalloc: blocks, x and y must be float64")
    if rows.dtype != torch.int32 or cols.dtype != torch.int32:
        raise ValueError("spmv_noalloc: rows and cols must be int32")
    nnzb = int(nnzb)
    if x.numel() != y.numel() or blocks.numel() < 9 * nnzb or rows.numel() < nnzb or cols.numel() < nnzb:
        raise ValueError("spmv_noalloc: x and y must have the same size, blocks 9 nnzb and rows/cols nnzb entries")
    if stream is not None and stream.device != y.device:
        raise ValueError("spmv_noalloc: stream is on another device")
    s = None if stream is None else stream.cuda_stream
    with torch.cuda.device(y.device):
        check(_L.lib().stg_spmv_noalloc(float(a), _ptr(blocks), _ptr(rows), _ptr(cols), nnzb, _ptr(x), float(b),
                                        _ptr(y), int(y.numel()), s), "stg_spmv_noalloc")


def morton_keys(pos, stream=None):
    """Per-vertex 64-bit Morton keys (code << 32) | index of device positions (stg_morton_keys,
    _calcVertMChash at GIPC.cu:453-502); pos: CUDA float64 tensor [V, 3] or [3V].  Returns an
    int64 tensor [V] on the same device holding the keys' uint64 bit patterns (view it as
    uint64 on the host: keys.cpu().numpy().view(np.uint64))."""
    import torch
    _require_cuda(pos)
    if pos.dtype != torch.float64 or pos.numel() % 3 != 0:
        raise ValueError("morton_keys: pos must be float64 with 3 values per vertex")
    pos = pos.contiguous()
    n = pos.numel() // 3
    keys = torch.empty(n, dtype=torch.int64, device=pos.device)
    s = None if stream is None else stream.cuda_stream
    with torch.cuda.device(pos.device):
        check(_L.lib().stg_morton_keys(n, _ptr(pos), _ptr(keys), s), "stg_morton_keys")
    return keys


class Solver:
    """One handle: GlobalLinearSystem + PCGSolver + MAS preconditioner on one stream."""

    def __init__(self, config: Optional[PCGSolverConfig] = None, stream=None):
        self.config = config or PCGSolverConfig()
        sp = 0 if stream is None else int(stream.cuda_stream)
        self._cfg = self.config.to_c(sp)
        h = C.c_void_p()
        check(_L.lib().stg_create(C.byref(self._cfg), C.byref(h)), "stg_create")
        self.h = h
        self.num_verts = 0

    def close(self):
        if getattr(self, "h", None):
            _L.lib().stg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- MAS set-up (host arrays) -------------------------------------------------------
    def mas_init(self, num_verts, neighbor_start, neighbor_num, neighbor_list, part_map, real_map,
                 collision_node_offset=0):
        """initPreconditioner_Neighbor + initPreconditioner_Matrix (MASPreconditioner.cu:2291-2358)."""
        ns = np.ascontiguousarray(neighbor_start, np.uint32)
        nn = np.ascontiguousarray(neighbor_num, np.uint32)
        nl = np.ascontiguousarray(neighbor_list, np.uint32)
        pm = np.ascontiguousarray(part_map, np.int32)
        rm = np.ascontiguousarray(real_map, np.int32)
        check(_L.lib().stg_mas_init(self.h, int(num_verts), int(collision_node_offset), ns.ctypes.data, nn.ctypes.data,
                                    nl.ctypes.data if nl.size else None, int(nl.size), pm.ctypes.data, int(pm.size),
                                    rm.ctypes.data), "stg_mas_init")
        self.num_verts = int(num_verts)

    # -- stages ---------------------------------------------------------------------------
    def convert(self, rows, cols, blocks) -> int:
        """srbk_convert in place on device tensors; returns the unique block count."""
        _require_cuda(rows, cols, blocks)
        u = C.c_int(0)
        check(_L.lib().stg_convert(self.h, int(rows.numel()), _ptr(rows), _ptr(cols), _ptr(blocks), C.byref(u)),
              "stg_convert")
        return u.value

    def spmv(self, a, blocks, rows, cols, nnzb, x, b, y):
        """y = a A x + b y (srbk_spmv)."""
        _require_cuda(blocks, rows, cols, x, y)
        check(_L.lib().stg_spmv(self.h, float(a), _ptr(blocks), _ptr(rows), _ptr(cols), int(nnzb), _ptr(x), float(b),
                                _ptr(y), int(y.numel())), "stg_spmv")

    def mas_assemble(self, blocks, rows, cols, nnzb, fem_block_offset=0, contacts=None):
        _require_cuda(blocks, rows, cols, contacts)
        ncp = 0 if contacts is None else int(contacts.shape[0])
        check(_L.lib().stg_mas_assemble(self.h, _ptr(blocks), _ptr(rows), _ptr(cols), int(nnzb), int(fem_block_offset),
                                        _ptr(contacts) if ncp else None, ncp), "stg_mas_assemble")

    def mas_apply(self, r, z):
        _require_cuda(r, z)
        check(_L.lib().stg_mas_apply(self.h, _ptr(r), _ptr(z)), "stg_mas_apply")

    def pcg_solve(self, blocks, rows, cols, nnzb, b, x) -> dict:
        _require_cuda(blocks, rows, cols, b, x)
        st = _L.Stats()
        check(_L.lib().stg_pcg_solve(self.h, _ptr(blocks), _ptr(rows), _ptr(cols), int(nnzb), _ptr(b), _ptr(x),
                                     int(b.numel()), C.byref(st)), "stg_pcg_solve", ok=(_L.STG_OK, _L.STG_MAX_ITER))
        return st.as_dict()

    def solve_linear_system(self, rows, cols, blocks, b, x, fem_block_offset=0, contacts=None, abd_inv=None,
                            abd_bodies=0, stats=True) -> dict:
        """GlobalLinearSystem::solve_linear_system on device triplets (pre-convert)."""
        _require_cuda(rows, cols, blocks, b, x, contacts, abd_inv)
        sysc = _L.System()
        sysc.triplet_count = int(rows.numel())
        sysc.rows, sysc.cols, sysc.blocks = _ptr(rows), _ptr(cols), _ptr(blocks)
        sysc.n = int(b.numel())
        sysc.b = _ptr(b)
        sysc.fem_block_offset = int(fem_block_offset)
        sysc.contacts = _ptr(contacts) if contacts is not None and contacts.numel() else None
        sysc.ncp = 0 if sysc.contacts is None else int(contacts.shape[0])
        sysc.abd_bodies = int(abd_bodies)
        sysc.abd_inv = _ptr(abd_inv)
        st = _L.Stats()
        check(_L.lib().stg_solve_linear_system(self.h, C.byref(sysc), _ptr(x), C.byref(st) if stats else None),
              "stg_solve_linear_system", ok=(_L.STG_OK, _L.STG_MAX_ITER))
        return st.as_dict()

    # -- introspection ----------------------------------------------------------------------
    def mas_info(self):
        L, T = C.c_int(), C.c_int()
        ls = np.zeros(2 * 7, np.int32)
        check(_L.lib().stg_mas_info(self.h, C.byref(L), C.byref(T), ls.ctypes.data), "stg_mas_info")
        return L.value, T.value, ls[:2 * (L.value + 1)].reshape(-1, 2)

    def export_hierarchy(self, num_part_slots: int):
        L, T, ls = self.mas_info()
        V = self.num_verts
        bank = self.config.bank_size
        fine = np.zeros(V, np.uint32)
        pref = np.zeros(num_part_slots // bank, np.int32)
        ct = np.zeros(L * V, np.int32)
        gn = np.zeros(max(T, V), np.int32)
        tab = np.zeros(V * max(L - 1, 1), np.int32)
        check(_L.lib().stg_mas_export_hierarchy(self.h, fine.ctypes.data, pref.ctypes.data, ct.ctypes.data,
                                                gn.ctypes.data, tab.ctypes.data), "stg_mas_export_hierarchy")
        return dict(fine_mask=fine, prefix_orig=pref, coarse_tables=ct.reshape(L, V), going_next=gn,
                    coarse_table=tab.reshape(V, max(L - 1, 1)), level_size=ls)

    # -- independent scenes in one solve (stg_set_segments) --------------------------------------
    def set_segments(self, row_offsets):
        """Block-row offsets of the scenes of a block-diagonal batch (nseg + 1 entries);
        None or empty: one system."""
        if row_offsets is None or len(row_offsets) == 0:
            check(_L.lib().stg_set_segments(self.h, None, 0), "stg_set_segments")
            self._nseg = 0
            return
        off = np.ascontiguousarray(row_offsets, np.int32)
        check(_L.lib().stg_set_segments(self.h, off.ctypes.data, int(off.size - 1)), "stg_set_segments")
        self._nseg = int(off.size - 1)

    def segment_stats(self):
        """(iterations, relative residual of the recurrence) per scene of the last solve."""
        it = np.zeros(self._nseg, np.int32)
        rel = np.zeros(self._nseg, np.float64)
        check(_L.lib().stg_segment_stats(self.h, it.ctypes.data, rel.ctypes.data), "stg_segment_stats")
        return it, rel

    # -- BCOO tile autotuner -------------------------------------------------------------------
    def spmv_tiles(self, rows_per_tile: int):
        """0: autotune at the next solve of a new shape class; -1: default; -2: the halo
        kernel; -3: the upper kernel; else a fixed tile shape of the full-copy kernel."""
        check(_L.lib().stg_spmv_tiles(self.h, int(rows_per_tile)), "stg_spmv_tiles")

    def spmv_tiles_info(self):
        """(rows per tile of the last solve (-2: halo kernel, -3: upper kernel), tuner us per
        launch: default shape, alternative shape, halo kernel, upper kernel)."""
        rt, a, b, h, u = C.c_int(), C.c_float(), C.c_float(), C.c_float(), C.c_float()
        check(_L.lib().stg_spmv_tiles_info(self.h, C.byref(rt), C.byref(a), C.byref(b), C.byref(h), C.byref(u)),
              "stg_spmv_tiles_info")
        return rt.value, a.value, b.value, h.value, u.value

    # -- learned coarse correction (stg_net_*) ---------------------------------------------
    def net_configure(self, level: int):
        """Coarse level of the network; the next MAS assembly builds its graph."""
        check(_L.lib().stg_net_configure(self.h, int(level)), "stg_net_configure")

    def net_graph(self, device="cuda"):
        """The level's graph (learned.NetGraph) exported to new device tensors."""
        import torch
        from .learned import NetGraph
        n, e = C.c_int(), C.c_int()
        check(_L.lib().stg_net_graph_info(self.h, C.byref(n), C.byref(e)), "stg_net_graph_info")
        n, e = n.value, e.value
        dev = torch.device(device)
        row = torch.zeros(n + 1, dtype=torch.int32, device=dev)
        col = torch.zeros(max(e, 1), dtype=torch.int32, device=dev)
        w = torch.zeros(max(e, 1), dtype=torch.float32, device=dev)
        oblk = torch.zeros(max(e, 1) * 9, dtype=torch.float32, device=dev)
        dblk = torch.zeros(n * 9, dtype=torch.float32, device=dev)
        feat = torch.zeros(n, dtype=torch.float32, device=dev)
        check(_L.lib().stg_net_export_graph(self.h, _ptr(row), _ptr(col), _ptr(w), _ptr(oblk), _ptr(dblk), _ptr(feat)),
              "stg_net_export_graph")
        torch.cuda.synchronize(dev)
        return NetGraph(n, e, row, col, w, oblk, dblk, feat)

    def net_record(self, rc, zc, capacity: int, every: int):
        """Record (r_c, z_c) of the level every `every` iterations of the following solves."""
        _require_cuda(rc, zc)
        check(_L.lib().stg_net_record(self.h, _ptr(rc), _ptr(zc), int(capacity), int(every)), "stg_net_record")
        self._rec = (rc, zc)

    def net_recorded(self) -> int:
        c = C.c_int()
        check(_L.lib().stg_net_recorded(self.h, C.byref(c)), "stg_net_recorded")
        return c.value

    def net_set_params(self, params):
        _require_cuda(params)
        check(_L.lib().stg_net_set_params(self.h, _ptr(params)), "stg_net_set_params")

    def profile_spmv(self, reps: int = 50):
        """(mean ms per PCG SpMV launch, algorithmic bytes per launch) on the last solve."""
        ms, by = C.c_float(), C.c_double()
        check(_L.lib().stg_profile_spmv(self.h, int(reps), C.byref(ms), C.byref(by)), "stg_profile_spmv")
        return ms.value, by.value

    def export_matrices(self):
        nb = C.c_int()
        check(_L.lib().stg_mas_export_matrices(self.h, None, None, C.byref(nb)), "stg_mas_export_matrices")
        ns = self.config.bank_size * (self.config.bank_size + 1) // 2
        mat = np.zeros(nb.value * ns * 9, np.float64)
        inv = np.zeros(nb.value * ns * 9, np.float32)
        check(_L.lib().stg_mas_export_matrices(self.h, mat.ctypes.data, inv.ctypes.data, C.byref(nb)),
              "stg_mas_export_matrices")
        return mat.reshape(nb.value, ns, 9), inv.reshape(nb.value, ns, 9)


class GlobalLinearSystem:
    """Convenience owner of a Solver + the device copy of one NewtonSystem (scenes.py)."""

    def __init__(self, system, config: Optional[PCGSolverConfig] = None, device="cuda", stream=None):
        import torch
        self.sys = system
        self.config = config or PCGSolverConfig()
        self.solver = Solver(self.config, stream=stream)
        if self.config.preconditioner == "mas":
            pm, rm = system.slot_maps(self.config.bank_size)
            self.solver.mas_init(system.num_verts, system.neighbor_start, system.neighbor_num, system.neighbor_list, pm,
                                 rm, collision_node_offset=0)
        self.rows = torch.from_numpy(system.rows).to(device)
        self.cols = torch.from_numpy(system.cols).to(device)
        self.blocks = torch.from_numpy(system.blocks.reshape(-1)).to(device)
        self.b = torch.from_numpy(system.b).to(device)
        self.x = torch.zeros_like(self.b)
        self.contacts = (torch.from_numpy(system.contacts).to(device) if system.contacts.size else None)

    def solve_linear_system(self) -> dict:
        return self.solver.solve_linear_system(self.rows, self.cols, self.blocks, self.b, self.x,
                                               fem_block_offset=self.sys.fem_block_offset, contacts=self.contacts)
