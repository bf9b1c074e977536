"""ctypes front-end of the CPU oracle (oracle/stg_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg as the checker.  The product library never routes through it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libstg_oracle.so")
_lib = None

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")


class PcgStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("rz0", C.c_double), ("rz_final", C.c_double),
                ("rel_residual", C.c_double)]


def build() -> str:
    """Compile the oracle with gcc (make -C oracle)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.orc_convert.argtypes = [C.c_int, _i32p, _i32p, _f64p, _i32p, _i32p, _f64p]
        L.orc_convert.restype = C.c_int
        L.orc_spmv.argtypes = [C.c_double, C.c_int, _i32p, _i32p, _f64p, _f64p, C.c_double, _f64p, C.c_int]
        L.orc_spmv.restype = None
        L.orc_mas_num_levels.argtypes = [C.c_int, C.c_int]
        L.orc_mas_num_levels.restype = C.c_int
        L.orc_mas_create.argtypes = [C.c_int, C.c_int, _u32p, _u32p, _u32p, C.c_int, _i32p, C.c_int, _i32p, C.c_int]
        L.orc_mas_create.restype = C.c_void_p
        L.orc_mas_destroy.argtypes = [C.c_void_p]
        L.orc_mas_set_order.argtypes = [C.c_void_p, C.c_int]
        L.orc_mas_set_order.restype = None
        L.orc_mas_levels.argtypes = [C.c_void_p]
        L.orc_mas_levels.restype = C.c_int
        L.orc_mas_total_clusters.argtypes = [C.c_void_p]
        L.orc_mas_total_clusters.restype = C.c_int
        L.orc_mas_build.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        L.orc_mas_build.restype = C.c_int
        L.orc_mas_export.argtypes = [C.c_void_p] + [C.c_void_p] * 8
        L.orc_mas_export.restype = None
        L.orc_select_range.argtypes = [C.c_int, _i32p, _i32p, C.c_int, C.c_int, _i32p]
        L.orc_select_range.restype = C.c_int
        L.orc_mas_assemble.argtypes = [C.c_void_p, _i32p, _i32p, _f64p, _i32p, C.c_int, C.c_int]
        L.orc_mas_assemble.restype = None
        L.orc_mas_nbanks.argtypes = [C.c_void_p]
        L.orc_mas_nbanks.restype = C.c_int
        L.orc_mas_export_matrices.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_mas_apply.argtypes = [C.c_void_p, _f64p, _f64p]
        L.orc_mas_apply.restype = None
        L.orc_pcg.argtypes = [_i32p, _i32p, _f64p, C.c_int, C.c_int, _f64p, _f64p, C.c_void_p, C.c_int, C.c_int,
                              C.c_int, C.c_void_p, C.c_double, C.c_double, C.POINTER(PcgStats)]
        L.orc_pcg.restype = C.c_int
        L.orc_contact_barrier.argtypes = [C.c_int, _i32p, _f64p, C.c_int, C.c_int, C.c_double, C.c_double, _i32p,
                                          _i32p, _f64p, _f64p]
        L.orc_contact_barrier.restype = C.c_int
        L.orc_accd.argtypes = [C.c_int, _f64p, _f64p, C.c_double, C.c_double]
        L.orc_accd.restype = C.c_double
        L.orc_ccd_step_size.argtypes = [C.c_int, _i32p, _f64p, _f64p, C.c_double]
        L.orc_ccd_step_size.restype = C.c_double
        L.orc_contact_energy.argtypes = [C.c_int, _i32p, _f64p, C.c_int, C.c_double, C.c_double, _f64p]
        L.orc_contact_energy.restype = None
        L.orc_contact_d2.argtypes = [C.c_int, _f64p, _f64p]
        L.orc_contact_d2.restype = C.c_double
        L.orc_pcg_ex.argtypes = [_i32p, _i32p, _f64p, C.c_int, C.c_int, _f64p, _f64p, C.c_void_p, C.c_int, C.c_int,
                                 C.c_int, C.c_void_p, C.c_double, C.c_double, C.c_int, C.c_double,
                                 C.POINTER(PcgStats), C.POINTER(C.c_double), C.POINTER(C.c_int)]
        L.orc_pcg_ex.restype = C.c_int
        L.orc_pcg_mt.argtypes = [_i32p, _i32p, _f64p, C.c_int, C.c_int, _f64p, _f64p, C.c_void_p, C.c_double,
                                 C.c_double, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                 C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.orc_pcg_mt.restype = C.c_int
        L.orc_cg_bj_mt.argtypes = [_i32p, _i32p, _f64p, C.c_int, C.c_int, _f64p, _f64p, C.c_double, C.c_double,
                                   C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int),
                                   C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.orc_cg_bj_mt.restype = C.c_int
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def convert(rows, cols, blocks):
    """Triplets -> sorted unique BCOO (srbk_convert)."""
    rows = np.ascontiguousarray(rows, np.int32)
    cols = np.ascontiguousarray(cols, np.int32)
    blocks = np.ascontiguousarray(blocks, np.float64).reshape(-1, 9)
    t = rows.size
    orow = np.empty(max(t, 1), np.int32)
    ocol = np.empty(max(t, 1), np.int32)
    oblk = np.empty((max(t, 1), 9), np.float64)
    u = lib().orc_convert(t, rows, cols, blocks.reshape(-1), orow, ocol, oblk.reshape(-1))
    return orow[:u].copy(), ocol[:u].copy(), oblk[:u].copy()


def spmv(rows, cols, blocks, x, a=1.0, b=0.0, y=None):
    n = x.size
    y = np.zeros(n) if y is None else np.ascontiguousarray(y, np.float64).copy()
    lib().orc_spmv(a, rows.size, np.ascontiguousarray(rows, np.int32), np.ascontiguousarray(cols, np.int32),
                   np.ascontiguousarray(blocks, np.float64).reshape(-1), np.ascontiguousarray(x, np.float64), b, y, n)
    return y


ORDER_WALK, ORDER_FIXED = 0, 1


class Mas:
    """Oracle MAS preconditioner (one instance per mesh).

    order: ORDER_FIXED (default) sums the coarse bank matrices, the multilevel residual and
    the bank-solve rows in one fixed order, the one the GPU kernels use; ORDER_WALK follows
    the reference's loops literally (its atomics taken in loop order).  The reference itself
    leaves these orders undefined (atomics); see stg_oracle.c."""

    def __init__(self, bank, num_verts, nstart, nnum, nlist, part_map, real_map, node_offset=0, order=ORDER_FIXED):
        self.bank = bank
        self.V = num_verts
        self.M = part_map.size
        self._keep = [np.ascontiguousarray(a, np.uint32) for a in (nstart, nnum, nlist)]
        self._keep += [np.ascontiguousarray(part_map, np.int32), np.ascontiguousarray(real_map, np.int32)]
        s, n_, l_, pm, rm = self._keep
        self.h = lib().orc_mas_create(bank, num_verts, s, n_, l_, l_.size, pm, pm.size, rm, node_offset)
        lib().orc_mas_set_order(self.h, order)
        self.L = lib().orc_mas_levels(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_mas_destroy(self.h)
            self.h = None

    def build(self, contacts=None):
        c = None if contacts is None or len(contacts) == 0 else np.ascontiguousarray(contacts, np.int32)
        self.total = lib().orc_mas_build(self.h, _p(c), 0 if c is None else c.shape[0])
        return self.total

    def hierarchy(self):
        V, L = self.V, self.L
        fine = np.zeros(V, np.uint32)
        pref = np.zeros(self.M // self.bank, np.int32)
        ct = np.zeros(L * V, np.int32)
        gn = np.zeros(max(self.total, V), np.int32)
        tab = np.zeros(V * max(L - 1, 1), np.int32)
        ls = np.zeros(2 * (L + 1), np.int32)
        nl = np.zeros(max(self._keep[2].size, 1), np.uint32)
        nn = np.zeros(V, np.uint32)
        lib().orc_mas_export(self.h, _p(fine), _p(pref), _p(ct), _p(gn), _p(tab), _p(ls), _p(nl), _p(nn))
        return dict(fine_mask=fine, prefix_orig=pref, coarse_tables=ct.reshape(L, V), going_next=gn,
                    coarse_table=tab.reshape(V, max(L - 1, 1)), level_size=ls.reshape(L + 1, 2),
                    neighbor_list=nl[:self._keep[2].size], neighbor_num=nn)

    def assemble(self, rows, cols, blocks, fem_offset=0):
        rows = np.ascontiguousarray(rows, np.int32)
        cols = np.ascontiguousarray(cols, np.int32)
        blocks = np.ascontiguousarray(blocks, np.float64).reshape(-1)
        sel = np.empty(max(rows.size, 1), np.int32)
        ns = lib().orc_select_range(rows.size, rows, cols, fem_offset, fem_offset + self.V, sel)
        lib().orc_mas_assemble(self.h, rows, cols, blocks, sel, ns, fem_offset)
        self.nbanks = lib().orc_mas_nbanks(self.h)

    def matrices(self):
        ns = self.bank * (self.bank + 1) // 2
        mat = np.zeros(self.nbanks * ns * 9, np.float64)
        inv = np.zeros(self.nbanks * ns * 9, np.float32)
        lib().orc_mas_export_matrices(self.h, _p(mat), _p(inv))
        return mat.reshape(self.nbanks, ns, 9), inv.reshape(self.nbanks, ns, 9)

    def apply(self, r):
        z = np.zeros(3 * self.V)
        lib().orc_mas_apply(self.h, np.ascontiguousarray(r, np.float64), z)
        return z


def pcg(rows, cols, blocks, b, mas: Mas | None = None, fem_offset=0, use_diag=False, tol=1e-4,
        max_iter_ratio=0.3, abd_bodies=0, abd_inv=None):
    """PCGSolver::pcg with the composed preconditioner; returns (x, stats dict)."""
    n = b.size
    x = np.zeros(n)
    st = PcgStats()
    ai = None if abd_inv is None else np.ascontiguousarray(abd_inv, np.float64)
    lib().orc_pcg(np.ascontiguousarray(rows, np.int32), np.ascontiguousarray(cols, np.int32),
                  np.ascontiguousarray(blocks, np.float64).reshape(-1), rows.size, n,
                  np.ascontiguousarray(b, np.float64), x, mas.h if mas is not None else None, fem_offset,
                  1 if use_diag else 0, abd_bodies, _p(ai), tol, max_iter_ratio, C.byref(st))
    return x, dict(iterations=st.iterations, rz0=st.rz0, rz_final=st.rz_final, rel_residual=st.rel_residual)


def pcg_timed(rows, cols, blocks, b, mas: Mas | None = None, fem_offset=0, use_diag=False, tol=1e-4,
              max_iter_ratio=0.3, stop_rule="reference", budget_s=0.0, abd_bodies=0, abd_inv=None):
    """PCG with a wall-time budget (CPU baseline sampling).  Returns (x, stats, seconds per
    iteration, finished)."""
    n = b.size
    x = np.zeros(n)
    st = PcgStats()
    ai = None if abd_inv is None else np.ascontiguousarray(abd_inv, np.float64).reshape(-1)
    t_iter = C.c_double()
    done = C.c_int()
    L = lib()
    L.orc_pcg_ex(np.ascontiguousarray(rows, np.int32), np.ascontiguousarray(cols, np.int32),
                 np.ascontiguousarray(blocks, np.float64).reshape(-1), rows.size, n, np.ascontiguousarray(b, np.float64),
                 x, mas.h if mas is not None else None, fem_offset, 1 if use_diag else 0, abd_bodies, _p(ai), tol,
                 max_iter_ratio,
                 0 if stop_rule == "reference" else 1, float(budget_s), C.byref(st), C.byref(t_iter), C.byref(done))
    stats = dict(iterations=st.iterations, rz0=st.rz0, rz_final=st.rz_final, rel_residual=st.rel_residual)
    return x, stats, t_iter.value, bool(done.value)


def pcg_timed_mt(rows, cols, blocks, b, mas: Mas, tol=1e-4, max_iter_ratio=0.3, budget_s=0.0):
    """The MAS-PCG recurrence on all host threads (OpenMP; stop rule ||r|| <= tol ||b||),
    for timing only.  Returns (x, iterations, seconds of set-up, seconds per iteration,
    finished, threads, last relative residual)."""
    n = b.size
    x = np.zeros(n)
    t_setup, t_iter, rel = C.c_double(), C.c_double(), C.c_double()
    done, threads = C.c_int(), C.c_int()
    k = lib().orc_pcg_mt(np.ascontiguousarray(rows, np.int32), np.ascontiguousarray(cols, np.int32),
                         np.ascontiguousarray(blocks, np.float64).reshape(-1), rows.size, n,
                         np.ascontiguousarray(b, np.float64), x, mas.h, tol, max_iter_ratio, float(budget_s),
                         C.byref(t_setup), C.byref(t_iter), C.byref(done), C.byref(threads), C.byref(rel))
    return x, int(k), t_setup.value, t_iter.value, bool(done.value), threads.value, rel.value


def cg_bj_timed_mt(rows, cols, blocks, b, tol=1e-4, max_iter_ratio=0.3, budget_s=0.0):
    """Block-Jacobi CG on all host threads (the Eigen ConjugateGradient + block-Jacobi
    baseline, restated; stop rule ||r|| <= tol ||b||), for timing.  Returns (x, iterations,
    seconds of set-up, seconds per iteration, finished, threads, last relative residual)."""
    n = b.size
    x = np.zeros(n)
    t_setup, t_iter, rel = C.c_double(), C.c_double(), C.c_double()
    done, threads = C.c_int(), C.c_int()
    k = lib().orc_cg_bj_mt(np.ascontiguousarray(rows, np.int32), np.ascontiguousarray(cols, np.int32),
                           np.ascontiguousarray(blocks, np.float64).reshape(-1), rows.size, n,
                           np.ascontiguousarray(b, np.float64), x, tol, max_iter_ratio, float(budget_s),
                           C.byref(t_setup), C.byref(t_iter), C.byref(done), C.byref(threads), C.byref(rel))
    return x, int(k), t_setup.value, t_iter.value, bool(done.value), threads.value, rel.value


def extrapolated_iterations(stats, target=1e-4):
    """Iterations a time-bounded run would need to reach `target` relative residual,
    assuming its observed geometric rate continues."""
    it, rel = stats["iterations"], stats["rel_residual"]
    if rel <= target or it <= 0 or not (0 < rel < 1):
        return it
    rate = rel ** (1.0 / it)
    return int(np.ceil(np.log(target) / np.log(rate)))


def contact_barrier(pairs, x, dhat, kappa, block_offset=0):
    """(rows, cols, blocks [10 P, 9] column-major, grad [P, 12], skipped) of the contact
    barrier of the sign-encoded pairs [P, 4] at positions x [V, 3] (the restatement of
    GIPC.cu:3149-4988 in stg_oracle.c)."""
    pairs = np.ascontiguousarray(pairs, np.int32).reshape(-1, 4)
    x = np.ascontiguousarray(x, np.float64).reshape(-1, 3)
    P = pairs.shape[0]
    rows, cols = np.empty(10 * P, np.int32), np.empty(10 * P, np.int32)
    blocks, grad = np.empty((10 * P, 9)), np.empty((P, 12))
    sk = lib().orc_contact_barrier(P, pairs.reshape(-1), x.reshape(-1), x.shape[0], block_offset, float(dhat),
                                   float(kappa), rows, cols, blocks.reshape(-1), grad.reshape(-1))
    return rows, cols, blocks, grad, int(sk)


def contact_d2(kind, v):
    """(d^2, d(d^2)/dx [12]) of one pair of kind 0 PP, 1 PE, 2 PT, 3 EE; v: [k, 3] vertices."""
    w = np.zeros(12)
    v = np.asarray(v, np.float64).reshape(-1)
    w[:v.size] = v
    g = np.zeros(12)
    return float(lib().orc_contact_d2(int(kind), w, g)), g


def accd(kind, x, dx, eta, thickness=0.0):
    """Time of impact of one pair (kind 0 point-triangle, 1 edge-edge); x, dx: [4, 3]."""
    return float(lib().orc_accd(int(kind), np.ascontiguousarray(x, np.float64).reshape(-1),
                                np.ascontiguousarray(dx, np.float64).reshape(-1), float(eta), float(thickness)))


def ccd_step_size(pairs, x, dx, slackness=0.8):
    """The line search's step bound over CCD pairs (GIPC::self_largestFeasibleStepSize)."""
    pairs = np.ascontiguousarray(pairs, np.int32).reshape(-1, 4)
    return float(lib().orc_ccd_step_size(pairs.shape[0], pairs.reshape(-1), np.ascontiguousarray(x, np.float64).reshape(-1),
                                         np.ascontiguousarray(dx, np.float64).reshape(-1), float(slackness)))


def contact_energy(pairs, x, dhat, kappa):
    """Per-pair barrier energies of the sign-encoded pairs at positions x [V, 3]."""
    pairs = np.ascontiguousarray(pairs, np.int32).reshape(-1, 4)
    x = np.ascontiguousarray(x, np.float64).reshape(-1, 3)
    e = np.zeros(pairs.shape[0])
    lib().orc_contact_energy(pairs.shape[0], pairs.reshape(-1), x.reshape(-1), x.shape[0], float(dhat), float(kappa), e)
    return e
