"""ctypes binding of libstgipc.so (include/stgipc.h).

The library is built in-tree by ``stiff-gipc_b200/build.py``.  There is no fallback: if the
shared library is missing or cannot be loaded, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "libstgipc.so")
HEADER = os.path.join(os.path.dirname(PKG), "include", "stgipc.h")

STG_OK, STG_ERR_INVALID, STG_ERR_CUDA, STG_ERR_NOT_READY, STG_MAX_ITER, STG_BREAKDOWN, STG_ERR_TIMEOUT, \
    STG_ERR_NO_DEVICE = range(8)
STATUS_NAMES = {0: "OK", 1: "ERR_INVALID", 2: "ERR_CUDA", 3: "ERR_NOT_READY", 4: "MAX_ITER", 5: "BREAKDOWN",
                6: "ERR_TIMEOUT", 7: "ERR_NO_DEVICE"}
PREC = {"fp64": 0, "fp32": 1}
PRECOND = {"diag": 0, "mas": 1, "none": 2}
STOP = {"reference": 0, "relative_residual": 1}
LOOP = {"host": 0, "graph": 1, "persistent": 2}


class Config(C.Structure):
    _fields_ = [("bank_size", C.c_int), ("precision", C.c_int), ("preconditioner", C.c_int),
                ("stop_rule", C.c_int), ("tol", C.c_double), ("max_iter_ratio", C.c_double),
                ("refine_interval", C.c_int), ("loop_mode", C.c_int), ("graph_batch", C.c_int),
                ("learned", C.c_int), ("stream", C.c_void_p)]


class Stats(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int), ("rz0", C.c_double), ("rz_final", C.c_double),
                ("rel_residual", C.c_double), ("rel_residual_recursive", C.c_double), ("nnzb", C.c_int),
                ("levels", C.c_int), ("total_clusters", C.c_int), ("replacements", C.c_int),
                ("learned_accepted", C.c_int), ("learned_rejected", C.c_int), ("ms_convert", C.c_float),
                ("ms_mas_build", C.c_float), ("ms_mas_assemble", C.c_float), ("ms_pcg", C.c_float),
                ("ms_total", C.c_float), ("kernel_launches", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class System(C.Structure):
    _fields_ = [("triplet_count", C.c_int), ("rows", C.c_void_p), ("cols", C.c_void_p), ("blocks", C.c_void_p),
                ("n", C.c_int), ("b", C.c_void_p), ("fem_block_offset", C.c_int), ("contacts", C.c_void_p),
                ("ncp", C.c_int), ("abd_bodies", C.c_int), ("abd_inv", C.c_void_p)]


class NetGraphC(C.Structure):
    _fields_ = [("nodes", C.c_int), ("entries", C.c_int), ("row", C.c_void_p), ("col", C.c_void_p), ("w", C.c_void_p),
                ("oblk", C.c_void_p), ("dblk", C.c_void_p), ("feat", C.c_void_p)]


NET_PARAMS = 26376


class StgError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_lib = None
vp, ci, cd = C.c_void_p, C.c_int, C.c_double


def header_symbols() -> list[str]:
    """Every function the public header declares."""
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ ]*\*?\s+\**(stg_[a-z_0-9]+)\s*\(", txt, re.M)))


def lib():
    """Load libstgipc.so (raises if it is missing: the CUDA path has no substitute)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libstgipc.so not built ({LIB_PATH}); run stiff-gipc_b200/build.py")
    L = C.CDLL(LIB_PATH)
    L.stg_last_error.restype = C.c_char_p
    L.stg_config_default.argtypes = [C.POINTER(Config)]
    L.stg_config_default.restype = None
    L.stg_create.argtypes = [C.POINTER(Config), C.POINTER(vp)]
    L.stg_destroy.argtypes = [vp]
    L.stg_mas_init.argtypes = [vp, ci, ci, vp, vp, vp, ci, vp, ci, vp]
    L.stg_convert.argtypes = [vp, ci, vp, vp, vp, C.POINTER(ci)]
    L.stg_spmv.argtypes = [vp, cd, vp, vp, vp, ci, vp, cd, vp, ci]
    L.stg_mas_assemble.argtypes = [vp, vp, vp, vp, ci, ci, vp, ci]
    L.stg_mas_apply.argtypes = [vp, vp, vp]
    L.stg_pcg_solve.argtypes = [vp, vp, vp, vp, ci, vp, vp, ci, C.POINTER(Stats)]
    L.stg_solve_linear_system.argtypes = [vp, C.POINTER(System), vp, C.POINTER(Stats)]
    L.stg_mas_info.argtypes = [vp, C.POINTER(ci), C.POINTER(ci), vp]
    L.stg_mas_export_hierarchy.argtypes = [vp, vp, vp, vp, vp, vp]
    L.stg_mas_export_matrices.argtypes = [vp, vp, vp, C.POINTER(ci)]
    L.stg_profile_spmv.argtypes = [vp, ci, C.POINTER(C.c_float), C.POINTER(cd)]
    L.stg_spmv_noalloc.argtypes = [cd, vp, vp, vp, ci, vp, cd, vp, ci, vp]
    L.stg_morton_keys.argtypes = [ci, vp, vp, vp]
    L.stg_selftest_wait_timeout.argtypes = [C.POINTER(ci), C.POINTER(cd)]
    L.stg_spmv_tiles.argtypes = [vp, ci]
    L.stg_set_segments.argtypes = [vp, vp, ci]
    L.stg_segment_stats.argtypes = [vp, vp, vp]
    L.stg_fem_scratch_bytes.argtypes = [ci, ci]
    L.stg_fem_newton_system.argtypes = [ci, vp, vp, vp, vp, ci, vp, vp, cd, cd, cd, cd, ci, vp, vp, vp, vp, vp, vp,
                                        C.c_size_t, vp]
    L.stg_fem_energy.argtypes = [ci, vp, vp, vp, ci, vp, vp, cd, cd, cd, ci, vp, vp, C.c_size_t, C.POINTER(cd),
                                 C.POINTER(ci), vp]
    L.stg_abd_body_system.argtypes = [ci, vp, vp, vp, vp, vp, cd, cd, vp, vp, vp, vp, vp]
    L.stg_abd_map_triplets.argtypes = [ci, vp, vp, vp, ci, vp, vp, ci, vp, vp, vp, vp, vp]
    L.stg_abd_points.argtypes = [ci, vp, vp, vp, vp, vp]
    L.stg_abd_gather_gradient.argtypes = [ci, vp, vp, vp, vp, vp]
    L.stg_ccd_step_size.argtypes = [ci, vp, vp, vp, ci, cd, cd, vp, vp, vp, vp, vp]
    L.stg_contact_energy.argtypes = [ci, vp, vp, ci, cd, cd, vp, vp]
    L.stg_cloth_membrane.argtypes = [ci, vp, vp, vp, vp, ci, cd, cd, cd, cd, ci, vp, vp, vp, vp, vp, vp]
    L.stg_cloth_bending.argtypes = [ci, vp, vp, vp, vp, ci, cd, cd, ci, vp, vp, vp, vp, vp, vp]
    L.stg_contact_barrier.argtypes = [ci, vp, vp, ci, ci, cd, cd, vp, vp, vp, vp, vp, vp]
    L.stg_spmv_tiles_info.argtypes = [vp, C.POINTER(ci), C.POINTER(C.c_float), C.POINTER(C.c_float),
                                      C.POINTER(C.c_float), C.POINTER(C.c_float)]
    L.stg_net_configure.argtypes = [vp, ci]
    L.stg_net_graph_info.argtypes = [vp, C.POINTER(ci), C.POINTER(ci)]
    L.stg_net_export_graph.argtypes = [vp, vp, vp, vp, vp, vp, vp]
    L.stg_net_record.argtypes = [vp, vp, vp, ci, ci]
    L.stg_net_recorded.argtypes = [vp, C.POINTER(ci)]
    L.stg_net_set_params.argtypes = [vp, vp]
    L.stg_net_scratch_bytes.argtypes = [ci, ci]
    L.stg_net_forward.argtypes = [C.POINTER(NetGraphC), vp, vp, ci, vp, vp, vp, C.c_size_t, vp]
    L.stg_net_apply.argtypes = [C.POINTER(NetGraphC), vp, vp, vp, vp, C.c_size_t, C.POINTER(ci), vp]
    L.stg_net_train_step.argtypes = [C.POINTER(NetGraphC), vp, vp, ci, vp, vp, vp, vp, ci, C.c_float, vp, vp,
                                     C.c_size_t, vp]
    for name in header_symbols():
        if name not in ("stg_last_error", "stg_config_default", "stg_net_scratch_bytes", "stg_fem_scratch_bytes"):
            getattr(L, name).restype = ci
    L.stg_net_scratch_bytes.restype = C.c_size_t
    L.stg_fem_scratch_bytes.restype = C.c_size_t
    _lib = L
    return L


def check(status: int, where: str, ok=(STG_OK,)) -> int:
    if status not in ok:
        raise StgError(status, where, lib().stg_last_error().decode())
    return status
