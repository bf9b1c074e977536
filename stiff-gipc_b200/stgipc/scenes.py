"""Seeded synthetic Newton systems in the layout StiffGIPC hands to its linear solver.

The reference assembles, every Newton iteration, a triplet buffer (``GIPCTripletMatrix``,
StiffGIPC/linear_system/linear_system/global_matrix.h:52-253) in this order
(StiffGIPC/GIPC.cu:10258-10493):

1. contact / ground barrier blocks, one 3x3 ``n n^T`` block per active vertex
   (``_computeGroundGradientAndHessian``, GIPC.cu:6506-6557);
2. FEM tetrahedra, 10 upper blocks per tet in (ii <= jj) order with the row <= col swap
   (``_calculate_fem_gradient_hessian``, femEnergy.cu:1832-1854);
3. one mass block ``m_i I`` per FEM vertex (GIPC.cu:10466-10482).

Blocks are 3x3 FP64 stored column-major (Eigen ``Matrix3d``), rows/cols are int32 block
indices (vertex id + 4 * abd_body_num).  The right-hand side is the gradient
(fem_linear_subsystem.cu:56-84).

This module only produces inputs for the solver (the Hessian producer sits upstream of the
hot path); it is plain numpy, deterministic for a given seed.

Meshes: an n x n x n hex grid split into 6 tets per hex along the main diagonal
(Kuhn/Freudenthal), vertices renumbered by the reference's 30-bit Morton code
(``hash_code(type=-1)`` / ``_calcVertMChash``, GIPC.cu:183-241, 453-502) so that
consecutive vertices form the MAS partitions ("GPU MAS, Morton ordered").
"""
from __future__ import annotations

import dataclasses
import os
from typing import Optional

import numpy as np

# ----------------------------------------------------------------------------------------
# Morton code (GIPC.cu:183-241)
# ----------------------------------------------------------------------------------------


def expand_bits(v: np.ndarray) -> np.ndarray:
    """Spread the low 10 bits of ``v`` three apart (GIPC.cu:183-190), uint32 arithmetic."""
    v = v.astype(np.uint64)
    m = np.uint64(0xFFFFFFFF)
    v = ((v * np.uint64(0x00010001)) & m) & np.uint64(0xFF0000FF)
    v = ((v * np.uint64(0x00000101)) & m) & np.uint64(0x0F00F00F)
    v = ((v * np.uint64(0x00000011)) & m) & np.uint64(0xC30C30C3)
    v = ((v * np.uint64(0x00000005)) & m) & np.uint64(0x49249249)
    return v.astype(np.uint32)


def morton_hash(pos: np.ndarray, resolution: float = 1024.0) -> np.ndarray:
    """Per-vertex 64-bit key ``(mc32 << 32) | idx`` of ``_calcVertMChash`` (GIPC.cu:453-502).

    Positions are normalised per axis to the scene AABB, scaled to ``resolution`` cells,
    clamped to ``[0, resolution-1]`` and truncated (``hash_code`` type -1, GIPC.cu:192-208).
    """
    lower = pos.min(axis=0)
    upper = pos.max(axis=0)
    size = upper - lower
    off = (pos - lower) / size
    q = np.clip(off * resolution, 0.0, resolution - 1.0).astype(np.uint32)
    xx, yy, zz = expand_bits(q[:, 0]), expand_bits(q[:, 1]), expand_bits(q[:, 2])
    mc32 = ((xx.astype(np.uint64) << np.uint64(2)) + (yy.astype(np.uint64) << np.uint64(1))
            + zz.astype(np.uint64)) & np.uint64(0xFFFFFFFF)
    idx = np.arange(pos.shape[0], dtype=np.uint64)
    return (mc32 << np.uint64(32)) | idx


# ----------------------------------------------------------------------------------------
# Mesh
# ----------------------------------------------------------------------------------------


def cube_mesh(n: int, size: float = 1.0, origin=(0.0, 0.0, 0.0)):
    """(n+1)^3 grid vertices and 6 n^3 Kuhn tets (all sharing each hex's main diagonal)."""
    return box_mesh(n, n, n, size / n, origin)


def box_mesh(nx: int, ny: int, nz: int, h: float, origin=(0.0, 0.0, 0.0)):
    """(nx+1)(ny+1)(nz+1) grid vertices of spacing h (x fastest) and 6 nx ny nz Kuhn tets."""
    mx, my, mz = nx + 1, ny + 1, nz + 1
    z, y, x = np.meshgrid(np.arange(mz) * h, np.arange(my) * h, np.arange(mx) * h, indexing="ij")
    pos = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1) + np.asarray(origin, dtype=np.float64)

    def vid(i, j, k):
        return i + mx * (j + my * k)

    ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ii, jj, kk = ii.ravel(), jj.ravel(), kk.ravel()
    e = [(1, 0, 0), (0, 1, 0), (0, 0, 1)]
    perms = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]
    tets = []
    for p in perms:
        a = e[p[0]]
        b = tuple(e[p[0]][t] + e[p[1]][t] for t in range(3))
        v0 = vid(ii, jj, kk)
        v1 = vid(ii + a[0], jj + a[1], kk + a[2])
        v2 = vid(ii + b[0], jj + b[1], kk + b[2])
        v3 = vid(ii + 1, jj + 1, kk + 1)
        tets.append(np.stack([v0, v1, v2, v3], axis=1))
    # hex-major order: the 6 tets of a hex are consecutive
    tets = np.stack(tets, axis=1).reshape(-1, 4).astype(np.int64)
    # positive orientation
    d = pos[tets[:, 1:]] - pos[tets[:, :1]]
    det = np.linalg.det(np.transpose(d, (0, 2, 1)))
    neg = det < 0
    tets[neg, 1], tets[neg, 2] = tets[neg, 2].copy(), tets[neg, 1].copy()
    return pos, tets


def morton_renumber(pos: np.ndarray, tets: np.ndarray):
    """Renumber vertices by ascending Morton key; returns (pos', tets', old_of_new)."""
    key = morton_hash(pos)
    order = np.argsort(key, kind="stable")
    new_of_old = np.empty_like(order)
    new_of_old[order] = np.arange(order.size)
    return pos[order], new_of_old[tets], order


def edge_neighbors(num_verts: int, pairs: np.ndarray):
    """CSR vertex neighbour lists from oriented vertex pairs, with the ordering rule of
    vert_neighbors (first orientation met kept, set walked in lexicographic order)."""
    pairs = np.asarray(pairs, dtype=np.int64).reshape(-1, 2)
    lo = np.minimum(pairs[:, 0], pairs[:, 1])
    hi = np.maximum(pairs[:, 0], pairs[:, 1])
    ukey = lo * num_verts + hi
    _, first = np.unique(ukey, return_index=True)
    edges = pairs[np.sort(first)]
    order = np.lexsort((edges[:, 1], edges[:, 0]))
    edges = edges[order]
    a, b = edges[:, 0], edges[:, 1]
    src = np.empty(2 * a.size, dtype=np.int64)
    dst = np.empty(2 * a.size, dtype=np.int64)
    src[0::2], dst[0::2] = a, b
    src[1::2], dst[1::2] = b, a
    order = np.argsort(src, kind="stable")
    nlist = dst[order].astype(np.uint32)
    num = np.bincount(src, minlength=num_verts).astype(np.uint32)
    start = np.zeros(num_verts, dtype=np.uint32)
    start[1:] = np.cumsum(num[:-1], dtype=np.int64).astype(np.uint32)
    return start, num, nlist


def vert_neighbors(num_verts: int, tets: np.ndarray):
    """CSR vertex neighbour lists with the ordering of ``getVertNeighbors``.

    load_mesh.cpp:934-1040: every tet edge is inserted into a ``std::set<pair>`` in the
    orientation it is first met (tet order, edge order 01,02,03,12,13,23), the set is walked
    in lexicographic order and each edge (a, b) appends b to a's list and a to b's list.
    Returns (start, num, list) as uint32 arrays.
    """
    pairs = np.stack([tets[:, [0, 0, 0, 1, 1, 2]], tets[:, [1, 2, 3, 2, 3, 3]]], axis=2).reshape(-1, 2)
    lo = np.minimum(pairs[:, 0], pairs[:, 1])
    hi = np.maximum(pairs[:, 0], pairs[:, 1])
    ukey = lo.astype(np.int64) * num_verts + hi
    # first occurrence of each undirected edge keeps its orientation
    _, first = np.unique(ukey, return_index=True)
    edges = pairs[np.sort(first)]
    # std::set order: lexicographic on (first, second)
    order = np.lexsort((edges[:, 1], edges[:, 0]))
    edges = edges[order]
    a, b = edges[:, 0], edges[:, 1]
    # append order: walk edges; for edge e, a gets b, then b gets a
    src = np.empty(2 * a.size, dtype=np.int64)
    dst = np.empty(2 * a.size, dtype=np.int64)
    src[0::2], dst[0::2] = a, b
    src[1::2], dst[1::2] = b, a
    order = np.argsort(src, kind="stable")
    nlist = dst[order].astype(np.uint32)
    num = np.bincount(src, minlength=num_verts).astype(np.uint32)
    start = np.zeros(num_verts, dtype=np.uint32)
    start[1:] = np.cumsum(num[:-1], dtype=np.int64).astype(np.uint32)
    return start, num, nlist


def mas_partition_morton(num_verts: int, bank: int):
    """Slot maps of ``set_mas_partition`` (app/common/sim_bootstrap.cpp:90-113) for a
    Morton-ordered mesh where partition p = vertices [p*bank, (p+1)*bank)."""
    part_id = np.arange(num_verts) // bank
    return slot_maps_from_parts(part_id, bank)


def slot_maps_from_parts(part_id: np.ndarray, bank: int):
    """``set_mas_partition`` (sim_bootstrap.cpp:90-113): partId_map_real (size
    part_offset*bank, -1 padding) and real_map_partId, for vertices grouped by part id."""
    part_id = np.asarray(part_id, dtype=np.int64)
    nparts = int(part_id[-1]) + 1
    part_map = np.full(nparts * bank, -1, dtype=np.int32)
    index = 0
    for i in range(part_id.size):
        part_map[bank * part_id[i] + index] = i
        index += 1
        if i <= part_id.size - 2 and part_id[i + 1] != part_id[i]:
            index = 0
    inv = np.zeros(part_id.size, dtype=np.int32)
    index = 0
    for i in range(part_map.size):
        if part_map[i] == index:
            inv[index] = i
            index += 1
    return part_map, inv


# ----------------------------------------------------------------------------------------
# Energies (FP64, PSD projected)
# ----------------------------------------------------------------------------------------

_EPS = np.zeros((3, 3, 3))
_EPS[0, 1, 2] = _EPS[1, 2, 0] = _EPS[2, 0, 1] = 1.0
_EPS[0, 2, 1] = _EPS[2, 1, 0] = _EPS[1, 0, 2] = -1.0
# _HJ_OP[(m,n), (i,j,k,l)] = eps_ikm eps_jln (row-major vec indices)
_HJ_OP = np.einsum("ikm,jln->mnijkl", _EPS, _EPS).reshape(9, 81)


def _dFdx(dm_inv: np.ndarray) -> np.ndarray:
    """(T, 9, 12) Jacobian of vec_rowmajor(F) w.r.t. the 4 vertex positions."""
    t = dm_inv.shape[0]
    d = np.empty((t, 4, 3))
    d[:, 1:, :] = dm_inv
    d[:, 0, :] = -dm_inv.sum(axis=1)
    P = np.zeros((t, 9, 12))
    for i in range(3):
        for j in range(3):
            for a in range(4):
                P[:, 3 * i + j, 3 * a + i] = d[:, a, j]
    return P


def snh_gradient_hessian(F, mu, lam):
    """Stable Neo-Hookean (Smith et al. 2018, no log term):
    psi = mu/2 (|F|^2 - 3) + lam/2 (J - alpha)^2, alpha = 1 + mu/lam.
    Returns (dpsi/dF as (T,9) row-major, PSD-projected d2psi/dF2 (T,9,9))."""
    t = F.shape[0]
    J = np.linalg.det(F)
    alpha = 1.0 + mu / lam
    # d2J/dF_ij dF_kl = eps_ikm eps_jln F_mn: a linear map of vec(F) (one matmul)
    HJ = (F.reshape(t, 9) @ _HJ_OP).reshape(t, 9, 9)
    # cof(F) = dJ/dF = 1/2 HJ : F
    g = 0.5 * np.matmul(HJ, F.reshape(t, 9, 1)).reshape(t, 9)
    P = mu[:, None] * F.reshape(t, 9) + (lam * (J - alpha))[:, None] * g
    H = (mu[:, None, None] * np.eye(9)[None] + lam[:, None, None] * g[:, :, None] * g[:, None, :]
         + (lam * (J - alpha))[:, None, None] * HJ)
    H = 0.5 * (H + np.transpose(H, (0, 2, 1)))
    w, V = np.linalg.eigh(H)
    if (w < 0).any():
        w = np.maximum(w, 0.0)
        H = np.matmul(V * w[:, None, :], np.transpose(V, (0, 2, 1)))
    return P, H


def ground_barrier(dist, dhat, kappa):
    """IPC plane barrier on squared distance (GIPC.cu:6524-6551).

    Returns (dE/dd along the normal, scalar s such that the 3x3 Hessian is s * n n^T)."""
    dist2 = dist * dist
    dh2 = dhat * dhat
    t = dist2 - dh2
    g_b = t * np.log(dist2 / dh2) * -2.0 - (t * t) / dist2
    H_b = (np.log(dist2 / dh2) * -2.0 - t * 4.0 / dist2) + 1.0 / (dist2 * dist2) * (t * t)
    grad = kappa * g_b * 2.0 * dist
    param = 4.0 * H_b * dist2 + 2.0 * g_b
    return grad, kappa * param


# ----------------------------------------------------------------------------------------
# System container
# ----------------------------------------------------------------------------------------


@dataclasses.dataclass
class NewtonSystem:
    """One Newton linear system: triplets (pre-convert), RHS and MAS inputs."""
    name: str
    num_verts: int
    rows: np.ndarray          # int32 [T]
    cols: np.ndarray          # int32 [T]
    blocks: np.ndarray        # float64 [T, 9] column-major 3x3
    b: np.ndarray             # float64 [3V]
    pos: np.ndarray           # float64 [V, 3]
    tets: np.ndarray          # int64 [Tet, 4]
    neighbor_start: np.ndarray
    neighbor_num: np.ndarray
    neighbor_list: np.ndarray
    contacts: np.ndarray      # int32 [C, 4] (sign-encoded collision pairs, may be empty)
    fem_block_offset: int = 0
    abd_bodies: int = 0

    @property
    def n(self) -> int:
        return 3 * self.num_verts

    def slot_maps(self, bank: int):
        return mas_partition_morton(self.num_verts, bank)


def _assemble(name, pos_rest, pos, tets, E, nu, rho, dt, vel, barriers, rng_contacts=None):
    """Build triplets + gradient of one implicit-Euler Newton iteration at ``pos``."""
    V = pos.shape[0]
    T = tets.shape[0]
    mu_all = E / (2.0 * (1.0 + nu))
    lam_all = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))

    grad = np.zeros((V, 3))
    mass = np.zeros(V)
    tet_blocks = np.empty((T, 10, 9))
    tet_rows = np.empty((T, 10), dtype=np.int32)
    tet_cols = np.empty((T, 10), dtype=np.int32)
    chunk = 1 << 15
    pairs = [(ii, jj) for ii in range(4) for jj in range(ii, 4)]
    for s in range(0, T, chunk):
        tt = tets[s:s + chunk]
        nt = tt.shape[0]
        Dm = np.transpose(pos_rest[tt[:, 1:]] - pos_rest[tt[:, :1]], (0, 2, 1))
        vol = np.abs(np.linalg.det(Dm)) / 6.0
        Dminv = np.linalg.inv(Dm)
        Ds = np.transpose(pos[tt[:, 1:]] - pos[tt[:, :1]], (0, 2, 1))
        F = Ds @ Dminv
        Pf, H9 = snh_gradient_hessian(F, mu_all[s:s + chunk], lam_all[s:s + chunk])
        Jx = _dFdx(Dminv)
        w = vol * dt * dt
        JxT = np.transpose(Jx, (0, 2, 1))
        f12 = w[:, None] * np.matmul(JxT, Pf[:, :, None])[:, :, 0]
        H12 = w[:, None, None] * np.matmul(np.matmul(JxT, H9), Jx)
        for a in range(4):
            np.add.at(grad, tt[:, a], f12[:, 3 * a:3 * a + 3])
            np.add.at(mass, tt[:, a], rho * vol / 4.0)
        for kk, (ii, jj) in enumerate(pairs):
            r = tt[:, ii]
            c = tt[:, jj]
            blk = H12[:, 3 * ii:3 * ii + 3, 3 * jj:3 * jj + 3]
            swap = r > c
            blk = np.where(swap[:, None, None], np.transpose(blk, (0, 2, 1)), blk)
            tet_rows[s:s + nt, kk] = np.where(swap, c, r)
            tet_cols[s:s + nt, kk] = np.where(swap, r, c)
            # column-major 3x3 (Eigen Matrix3d)
            tet_blocks[s:s + nt, kk] = np.transpose(blk, (0, 2, 1)).reshape(nt, 9)

    # kinetic gradient: M (x - x_tilde), x_tilde = x_n + dt v + dt^2 g with x_n = pos_rest path
    x_tilde = pos + dt * vel + dt * dt * np.array([0.0, -9.8, 0.0])
    grad += mass[:, None] * (pos - x_tilde)

    bar_rows, bar_blocks = [], []
    for (normal, offset, dhat, kappa) in barriers:
        normal = np.asarray(normal, dtype=np.float64)
        dist = pos @ normal - offset
        act = np.nonzero(dist < dhat)[0]
        if act.size == 0:
            continue
        g, s_ = ground_barrier(dist[act], dhat, kappa)
        grad[act] += g[:, None] * normal[None, :]
        nn = np.outer(normal, normal).T.reshape(9)  # symmetric: layout irrelevant
        bar_rows.append(act.astype(np.int32))
        bar_blocks.append(s_[:, None] * nn[None, :])
    if bar_rows:
        bar_rows = np.concatenate(bar_rows)
        bar_blocks = np.concatenate(bar_blocks)
    else:
        bar_rows = np.zeros(0, dtype=np.int32)
        bar_blocks = np.zeros((0, 9))

    mass_blocks = np.zeros((V, 9))
    mass_blocks[:, 0] = mass_blocks[:, 4] = mass_blocks[:, 8] = mass
    vids = np.arange(V, dtype=np.int32)

    rows = np.concatenate([bar_rows, tet_rows.reshape(-1), vids])
    cols = np.concatenate([bar_rows, tet_cols.reshape(-1), vids])
    blocks = np.concatenate([bar_blocks, tet_blocks.reshape(-1, 9), mass_blocks])
    start, num, nlist = vert_neighbors(V, tets)
    return NewtonSystem(name=name, num_verts=V, rows=rows.astype(np.int32), cols=cols.astype(np.int32),
                        blocks=np.ascontiguousarray(blocks), b=grad.reshape(-1).copy(), pos=pos, tets=tets,
                        neighbor_start=start, neighbor_num=num, neighbor_list=nlist,
                        contacts=np.zeros((0, 4), dtype=np.int32))


def make_cube_drop(n: int = 16, seed: int = 1001, E: float = 1e5, nu: float = 0.45,
                   rho: float = 1000.0, dt: float = 1.0 / 60.0, v0: float = -2.0,
                   jitter: float = 1e-3, gap: float = 5e-4, dhat: float = 1e-3,
                   kappa: float = 1e5, state_only: bool = False) -> NewtonSystem:
    """Plain FP64 MAS-PCG workload, one Newton step: a 1 m cube of n^3 hexes (6 tets each),
    vertices jittered U(+-jitter) from ``seed``, falling at ``v0`` m/s in y, resting ``gap``
    above a ground plane with an IPC barrier (d_hat, kappa).  n=16: 4,913 vertices,
    24,576 tets, 14,739 DOF.  state_only: the mesh state and material instead (the inputs of
    _assemble, or of stgipc.newton for a trajectory)."""
    rng = np.random.default_rng(seed)
    pos, tets = cube_mesh(n, 1.0, origin=(0.0, gap, 0.0))
    pos = pos + rng.uniform(-jitter, jitter, size=pos.shape)
    bottom = np.isclose(pos[:, 1], gap, atol=2 * jitter)
    pos[bottom, 1] = gap  # the resting face sits exactly gap above the ground
    pos, tets, _ = morton_renumber(pos, tets)
    E_t = np.full(tets.shape[0], E)
    vel = np.zeros_like(pos)
    vel[:, 1] = v0
    state = dict(name=f"cube{n}_drop", pos_rest=pos, pos=pos, tets=tets, E=E_t, nu=nu, rho=rho, dt=dt, vel=vel,
                 barriers=[((0.0, 1.0, 0.0), 0.0, dhat, kappa)])
    if state_only:
        return state
    return _assemble(**state)


def make_heterogeneous_cube(n: int = 48, seed: int = 1005, nu: float = 0.45, rho: float = 1000.0,
                            dt: float = 1.0 / 60.0, e_lo: float = 1e4, e_hi: float = 1e8,
                            regions: int = 8, squash: float = 0.08, jitter: float = 1e-3,
                            dhat: float = 1e-3, kappa: float = 1e5, slab_speed: float = 1.0,
                            state_only: bool = False) -> NewtonSystem:
    """Heterogeneous cube under a rigid slab: n^3 hexes (6 tets each), per-tet Young's modulus
    log-uniform in [e_lo, e_hi] from ``regions`` seeded Voronoi sites, nu=0.45; one Newton
    iteration of a step where the slab (moving down at ``slab_speed``) has squashed the top by
    ``squash`` m.  The slab and the ground act through IPC plane barriers.  n=48: 117,649
    vertices, 663,552 tets, 352,947 DOF.  state_only: return the mesh state and material
    instead (the inputs of _assemble, or of the GPU Hessian producer stgipc.fem)."""
    rng = np.random.default_rng(seed)
    rest, tets = cube_mesh(n, 1.0, origin=(0.0, 0.0, 0.0))
    rest = rest + rng.uniform(-jitter, jitter, size=rest.shape)
    sites = rng.uniform(0.0, 1.0, size=(regions, 3))
    site_E = np.exp(rng.uniform(np.log(e_lo), np.log(e_hi), size=regions))
    rest, tets, _ = morton_renumber(rest, tets)
    cent = rest[tets].mean(axis=1)
    d2 = ((cent[:, None, :] - sites[None, :, :]) ** 2).sum(axis=2)
    E_t = site_E[np.argmin(d2, axis=1)]
    # deformed state: top squashed down non-uniformly, bottom resting just above the ground
    pos = rest.copy()
    y = rest[:, 1]
    bulge = 1.0 + 0.3 * np.sin(np.pi * rest[:, 0]) * np.sin(np.pi * rest[:, 2])
    pos[:, 1] = y - squash * y * y * bulge
    pos[:, 0] += 0.02 * squash * (rest[:, 0] - 0.5) * y
    pos[:, 2] += 0.02 * squash * (rest[:, 2] - 0.5) * y
    pos += rng.uniform(-0.05 * jitter, 0.05 * jitter, size=pos.shape)
    pos[:, 1] += 4e-4 - pos[:, 1].min()
    top = pos[:, 1].max() + 4e-4
    vel = np.zeros_like(pos)
    vel[:, 1] = -slab_speed * (rest[:, 1])
    state = dict(name=f"hetcube{n}", pos_rest=rest, pos=pos, tets=tets, E=E_t, nu=nu, rho=rho, dt=dt, vel=vel,
                 barriers=[((0.0, 1.0, 0.0), 0.0, dhat, kappa), ((0.0, -1.0, 0.0), -top, dhat, kappa)])
    if state_only:
        return state
    return _assemble(**state)


def make_batched_cubes(count: int = 256, seed: int = 1004, n_lo: int = 4, n_hi: int = 24,
                       e_lo: float = 1e4, e_hi: float = 1e7, nu: float = 0.45, rho: float = 1000.0,
                       dt: float = 1.0 / 60.0, press: float = 5e-4, dhat: float = 1e-3,
                       kappa: float = 1e5, max_dof: Optional[int] = None):
    """Independent Neo-Hookean cubes, n x n x n hexes with n log-uniform in [n_lo, n_hi]
    and E log-uniform in [e_lo, e_hi], each pressed ``press`` into a ground barrier."""
    rng = np.random.default_rng(seed)
    out = []
    for c in range(count):
        n = int(round(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi)))))
        E = float(np.exp(rng.uniform(np.log(e_lo), np.log(e_hi))))
        sub = int(rng.integers(0, 2**31 - 1))
        r2 = np.random.default_rng(sub)
        rest, tets = cube_mesh(n, 0.1 * n / n_hi + 0.02, origin=(0.0, 0.0, 0.0))
        rest = rest + r2.uniform(-1e-5, 1e-5, size=rest.shape)
        rest, tets, _ = morton_renumber(rest, tets)
        pos = rest.copy()
        # pressed into the ground: bottom at dhat - press (inside the barrier zone)
        pos[:, 1] += (dhat - press) - pos[:, 1].min() + 1e-6
        pos[:, 1] *= 1.0
        E_t = np.full(tets.shape[0], E)
        vel = np.zeros_like(pos)
        sysm = _assemble(f"batch{c}_n{n}", rest, pos, tets, E_t, nu, rho, dt, vel,
                         barriers=[((0.0, 1.0, 0.0), 0.0, dhat, kappa)])
        out.append(sysm)
        if max_dof is not None and sum(s.n for s in out) >= max_dof:
            break
    return out


_CACHE_ENV = "STGIPC_SCENE_CACHE"


def cached(builder, key: str, **kw) -> NewtonSystem:
    """Build a system, memoised as an .npz under $STGIPC_SCENE_CACHE (if set)."""
    root = os.environ.get(_CACHE_ENV)
    if not root:
        return builder(**kw)
    os.makedirs(root, exist_ok=True)
    path = os.path.join(root, key + ".npz")
    if os.path.exists(path):
        z = np.load(path)
        return NewtonSystem(name=str(z["name"]), num_verts=int(z["num_verts"]), rows=z["rows"], cols=z["cols"],
                            blocks=z["blocks"], b=z["b"], pos=z["pos"], tets=z["tets"],
                            neighbor_start=z["neighbor_start"], neighbor_num=z["neighbor_num"],
                            neighbor_list=z["neighbor_list"], contacts=z["contacts"])
    s = builder(**kw)
    np.savez(path, name=s.name, num_verts=s.num_verts, rows=s.rows, cols=s.cols, blocks=s.blocks, b=s.b,
             pos=s.pos, tets=s.tets, neighbor_start=s.neighbor_start, neighbor_num=s.neighbor_num,
             neighbor_list=s.neighbor_list, contacts=s.contacts)
    return s


# ----------------------------------------------------------------------------------------
# Contact pairs between bodies (the input of stgipc.contact.barrier)
# ----------------------------------------------------------------------------------------


def boundary_faces(tets: np.ndarray) -> np.ndarray:
    """The triangles of a tet mesh that belong to exactly one tet."""
    f = np.concatenate([tets[:, [0, 1, 2]], tets[:, [0, 1, 3]], tets[:, [0, 2, 3]], tets[:, [1, 2, 3]]])
    key = np.sort(f, axis=1)
    _, idx, cnt = np.unique(key, axis=0, return_index=True, return_counts=True)
    return f[idx[cnt == 1]].astype(np.int64)


def face_edges(tris: np.ndarray) -> np.ndarray:
    e = np.concatenate([tris[:, [0, 1]], tris[:, [1, 2]], tris[:, [2, 0]]])
    return np.unique(np.sort(e, axis=1), axis=0)


def _pt_type(p, t0, t1, t2):
    """Closest feature of triangle (t0, t1, t2) to p, per pair (the regions of _dType_PT,
    mlbvh.cu:288-446): 0..2 vertex t_k, 3..5 edge (t0 t1), (t1 t2), (t2 t0), 6 interior."""
    n = np.cross(t1 - t0, t2 - t0)
    out = np.full(p.shape[0], 6, np.int64)
    pars = []
    for (a, b) in ((t0, t1), (t1, t2), (t2, t0)):
        e = b - a
        side = np.cross(e, n)                       # in-plane, pointing out of the triangle
        w = p - a
        s = np.einsum("ij,ij->i", w, e) / np.einsum("ij,ij->i", e, e)
        h = np.einsum("ij,ij->i", w, side)
        pars.append((s, h))
    done = np.zeros(p.shape[0], bool)
    for k, (s, h) in enumerate(pars):
        m = ~done & (s > 0) & (s < 1) & (h >= 0)
        out[m], done = 3 + k, done | m
    for k in range(3):   # vertex t_k: beyond the start of edge k and the end of edge k-1
        s_out, s_in = pars[k][0], pars[k - 1][0]
        m = ~done & (s_out <= 0) & (s_in >= 1)
        out[m], done = k, done | m
    return out


def contact_pairs(pos: np.ndarray, tris: np.ndarray, body: np.ndarray, dhat: float, mollify_eps: float = 1e-3,
                  return_d2: bool = False):
    """Sign-encoded int4 pairs (GIPC.cuh:49-66) between the surfaces of different bodies
    within distance sqrt(dhat): every (surface vertex, triangle) pair classified by its
    closest feature into PT, PE or PP, and every (edge, edge) pair whose closest points are
    interior to both edges as EE.  Near-parallel edge pairs (|ea x eb|^2 < mollify_eps
    |ea|^2 |eb|^2, the reference's mollifier zone, mlbvh.cu:278-285) and edge pairs whose closest
    points sit at an endpoint are left out.  Duplicates are merged.  Brute force over a
    uniform grid of cell size max(longest edge, sqrt(dhat)); meant for scene synthesis and the
    host side of the Newton driver.  return_d2: also the squared distance of every pair."""
    r = np.sqrt(dhat)
    dout = []
    edges = face_edges(tris)
    verts = np.unique(tris)
    h = max(float(np.linalg.norm(pos[edges[:, 0]] - pos[edges[:, 1]], axis=1).max()), r) * 1.0001

    def cand(prim_a, prim_b):
        """Pairs (i, j) of primitives (vertex lists) whose cells are within one of each other."""
        ca = np.floor(pos[prim_a].min(axis=1) / h).astype(np.int64)
        cb_lo = np.floor((pos[prim_b].min(axis=1) - r) / h).astype(np.int64)
        cb_hi = np.floor((pos[prim_b].max(axis=1) + r) / h).astype(np.int64)
        ka = (ca + (1 << 20)) @ np.array([1 << 42, 1 << 21, 1])
        order = np.argsort(ka, kind="stable")
        ks = ka[order]
        out_i, out_j = [], []
        span = cb_hi - cb_lo
        for dx in range(int(span[:, 0].max()) + 3):
            for dy in range(int(span[:, 1].max()) + 3):
                for dz in range(int(span[:, 2].max()) + 3):
                    c = cb_lo + np.array([dx, dy, dz]) - 1
                    ok = np.all(c <= cb_hi + 1, axis=1)
                    kb = (c + (1 << 20)) @ np.array([1 << 42, 1 << 21, 1])
                    lo = np.searchsorted(ks, kb, "left")
                    hi = np.searchsorted(ks, kb, "right")
                    cnt = np.where(ok, hi - lo, 0)
                    tot = int(cnt.sum())
                    if tot == 0:
                        continue
                    first = np.cumsum(cnt) - cnt
                    out_i.append(order[np.repeat(lo, cnt) + np.arange(tot) - np.repeat(first, cnt)])
                    out_j.append(np.repeat(np.arange(cnt.size), cnt))
        if not out_i:
            return np.zeros(0, np.int64), np.zeros(0, np.int64)
        pi, pj = np.concatenate(out_i), np.concatenate(out_j)
        key = np.unique(pi * (prim_b.shape[0] + 1) + pj)
        return key // (prim_b.shape[0] + 1), key % (prim_b.shape[0] + 1)

    out = []
    # point - triangle
    i, j = cand(verts[:, None], tris)
    p = verts[i]
    t = tris[j]
    keep = body[p] != body[t[:, 0]]
    p, t = p[keep], t[keep]
    if p.size:
        P, T0, T1, T2 = pos[p], pos[t[:, 0]], pos[t[:, 1]], pos[t[:, 2]]
        ty = _pt_type(P, T0, T1, T2)
        n = np.cross(T1 - T0, T2 - T0)
        d2 = np.full(p.size, np.inf)
        m = ty == 6
        d2[m] = np.einsum("ij,ij->i", P[m] - T0[m], n[m]) ** 2 / np.einsum("ij,ij->i", n[m], n[m])
        ea = [(0, 1), (1, 2), (2, 0)]
        tv = [T0, T1, T2]
        enc = np.zeros((p.size, 4), np.int64)
        enc[m] = np.stack([-p[m] - 1, t[m, 0], t[m, 1], t[m, 2]], 1)
        for k, (a, b) in enumerate(ea):
            mk = ty == 3 + k
            e = tv[b][mk] - tv[a][mk]
            c = np.cross(tv[a][mk] - P[mk], tv[b][mk] - P[mk])
            d2[mk] = np.einsum("ij,ij->i", c, c) / np.einsum("ij,ij->i", e, e)
            enc[mk] = np.stack([-p[mk] - 1, t[mk, a], t[mk, b], -np.ones(mk.sum(), np.int64)], 1)
        for k in range(3):
            mk = ty == k
            dv = P[mk] - tv[k][mk]
            d2[mk] = np.einsum("ij,ij->i", dv, dv)
            enc[mk] = np.stack([-p[mk] - 1, t[mk, k], -np.ones(mk.sum(), np.int64), -np.ones(mk.sum(), np.int64)], 1)
        out.append(enc[d2 < dhat])
        dout.append(d2[d2 < dhat])
    # edge - edge
    i, j = cand(edges, edges)
    keep = (i < j) & (body[edges[i, 0]] != body[edges[j, 0]])
    ea_, eb_ = edges[i[keep]], edges[j[keep]]
    if ea_.size:
        A0, A1, B0, B1 = pos[ea_[:, 0]], pos[ea_[:, 1]], pos[eb_[:, 0]], pos[eb_[:, 1]]
        u, v, w = A1 - A0, B1 - B0, A0 - B0
        a = np.einsum("ij,ij->i", u, u)
        b = np.einsum("ij,ij->i", u, v)
        c = np.einsum("ij,ij->i", v, v)
        d = np.einsum("ij,ij->i", u, w)
        e = np.einsum("ij,ij->i", v, w)
        D = a * c - b * b
        cr = np.cross(u, v)
        cr2 = np.einsum("ij,ij->i", cr, cr)
        ok = cr2 >= mollify_eps * a * c
        Ds = np.where(ok, D, 1.0)
        s = (b * e - c * d) / Ds
        tt = (a * e - b * d) / Ds
        ok &= (s > 0) & (s < 1) & (tt > 0) & (tt < 1)
        d2 = np.einsum("ij,ij->i", w, cr) ** 2 / np.where(ok, cr2, 1.0)
        ok &= d2 < dhat
        out.append(np.stack([ea_[ok, 0], ea_[ok, 1], eb_[ok, 0], eb_[ok, 1]], 1))
        dout.append(d2[ok])
    if not out:
        return (np.zeros((0, 4), np.int32), np.zeros(0)) if return_d2 else np.zeros((0, 4), np.int32)
    allp, idx = np.unique(np.concatenate(out), axis=0, return_index=True)
    if return_d2:
        return allp.astype(np.int32), np.concatenate(dout)[idx]
    return allp.astype(np.int32)


def make_stacked_cubes(n: int = 8, seed: int = 1006, E: float = 1e5, nu: float = 0.45, rho: float = 1000.0,
                       dt: float = 1.0 / 60.0, size: float = 0.5, gap: float = 4e-4, dhat: float = 1e-6,
                       kappa: float = 1e5, jitter: float = 1e-5, v0: float = -0.5, v_top: Optional[float] = None,
                       state_only: bool = False):
    """Two soft cubes, one resting on the other, with the upper one shifted by half a cell in
    x and z so its bottom vertices lie over the lower one's top triangles, ``gap`` m apart
    (inside the barrier's sqrt(dhat)); the lower cube rests ``gap`` above a ground barrier.
    Returns (NewtonSystem of the elastic + inertia + ground terms, contact pairs [C, 4],
    body id per vertex); the contact barrier terms come from stgipc.contact.barrier.  Both
    cubes move at v0 in y (the upper one at v_top when given).  state_only: (scene state for stgipc.newton, surface triangles,
    body id per vertex) instead."""
    rng = np.random.default_rng(seed)
    pa, ta = cube_mesh(n, size, origin=(0.0, gap, 0.0))
    h = size / n
    pb, tb = cube_mesh(n, size, origin=(0.5 * h, gap + size + gap, 0.5 * h))
    pos = np.concatenate([pa, pb])
    tets = np.concatenate([ta, tb + pa.shape[0]])
    body = np.concatenate([np.zeros(pa.shape[0], np.int64), np.ones(pb.shape[0], np.int64)])
    pos = pos + rng.uniform(-jitter, jitter, size=pos.shape)
    pos, tets, old_of_new = morton_renumber(pos, tets)
    body = body[old_of_new]
    E_t = np.full(tets.shape[0], E)
    vel = np.zeros_like(pos)
    vel[:, 1] = v0
    if v_top is not None:
        vel[body == 1, 1] = v_top
    barriers = [((0.0, 1.0, 0.0), 0.0, np.sqrt(dhat), kappa)]
    if state_only:
        state = dict(name=f"stacked{n}", pos_rest=pos, pos=pos.copy(), tets=tets, E=E_t, nu=nu, rho=rho, dt=dt,
                     vel=vel, barriers=barriers)
        return state, boundary_faces(tets), body
    sysm = _assemble(f"stacked{n}", pos, pos, tets, E_t, nu, rho, dt, vel, barriers=barriers)
    pairs = contact_pairs(pos, boundary_faces(tets), body, dhat)
    sysm.contacts = pairs
    return sysm, pairs, body


def random_rotation(rng) -> np.ndarray:
    """A uniformly random rotation (QR of a Gaussian matrix with the sign fixed)."""
    Q, R = np.linalg.qr(rng.normal(size=(3, 3)))
    Q = Q * np.sign(np.diag(R))
    if np.linalg.det(Q) < 0:
        Q[:, 0] = -Q[:, 0]
    return Q


@dataclasses.dataclass
class AbdScene:
    """Affine bodies over a FEM mesh at one Newton iteration: bodies own block rows
    [0, 4 N), FEM vertex v block row 4 N + v.  Points [0, P) are the bodies' mesh points
    (point_body, rest coordinates xbar), FEM vertices follow as points P + v."""
    name: str
    q: np.ndarray             # [N, 12] current (t, a1, a2, a3)
    q_tilde: np.ndarray       # [N, 12] inertial target
    mass: np.ndarray          # [N, 13] dyadic mass (m, m xbar, m xbar xbar^T)
    volume: np.ndarray        # [N]
    kappa: float
    dt: float
    point_body: np.ndarray    # int32 [P]
    xbar: np.ndarray          # [P, 3]
    body_point_start: np.ndarray  # int32 [N + 1]
    fem: NewtonSystem         # FEM elastic + inertia + ground terms (vertex numbering)
    contacts: np.ndarray      # int32 [C, 4] pairs over the point numbering
    dhat: float               # squared activation distance of the contacts
    kappa_contact: float

    @property
    def bodies(self) -> int:
        return self.q.shape[0]

    @property
    def abd_points(self) -> int:
        return self.point_body.shape[0]

    @property
    def n(self) -> int:
        return 3 * (4 * self.bodies + self.fem.num_verts)


def make_abd_slab(lattice: int = 8, body_size: float = 0.1, body_n: int = 2, kappa_abd: float = 1e8,
                  rho: float = 1000.0, slab_n: int = 64, slab_layers: int = 8, slab_size: float = 1.5,
                  E: float = 1e5, nu: float = 0.45, dt: float = 1.0 / 100.0, body_gap: float = 2e-3,
                  dhat: float = 1e-6, kappa: float = 1e5, seed: int = 1003, warp: float = 1e-3) -> AbdScene:
    """lattice^3 affine cubes (body_n^3 hexes, 6 tets each, uniform-random rotations baked
    into their rest shape) on a lattice of pitch (diagonal + body_gap), falling onto a slab of
    slab_n x slab_n x slab_layers hexes; the Newton iteration of the step at which the lowest
    corner of every bottom-layer body sits 2e-4 .. 8e-4 m above the slab (inside sqrt(dhat)).
    A is I plus a U(+-warp) perturbation, so the orthogonality terms are active; q_tilde is
    q minus the step's gravity drop.  The slab rests 5e-4 m above a ground barrier.  Defaults:
    512 bodies, 65 x 65 x 9 = 38,025 slab vertices, 196,608 tets; 6,144 + 114,075 DOF."""
    rng = np.random.default_rng(seed)
    h = slab_size / slab_n
    srest, stets = box_mesh(slab_n, slab_layers, slab_n, h, origin=(0.0, 5e-4, 0.0))
    srest, stets, _ = morton_renumber(srest, stets)
    top = float(srest[:, 1].max())
    bpos, btets = cube_mesh(body_n, body_size, origin=(-0.5 * body_size,) * 3)
    nb = lattice ** 3
    pitch = body_size * np.sqrt(3.0) + body_gap
    x0 = 0.5 * slab_size - 0.5 * pitch * (lattice - 1)
    xbar, point_body, tris, start, q, masses_all, vols = [], [], [], [0], [], [], []
    tet_vol = np.abs(np.linalg.det(np.transpose(bpos[btets[:, 1:]] - bpos[btets[:, :1]], (0, 2, 1)))) / 6.0
    btris = boundary_faces(btets)
    P = 0
    for b in range(nb):
        i, j, k = b % lattice, (b // lattice) % lattice, b // (lattice * lattice)
        Rm = random_rotation(rng)
        rest = bpos @ Rm.T
        c = np.array([x0 + pitch * i, 0.0, x0 + pitch * k])
        c[1] = top + rng.uniform(2e-4, 8e-4) - rest[:, 1].min() + pitch * j
        rest = rest + c  # rest shape in world coordinates (x = A xbar + t, q = (0, I) at rest)
        m = np.zeros(rest.shape[0])
        np.add.at(m, btets.reshape(-1), np.repeat(rho * tet_vol / 4.0, 4))
        A = np.eye(3) + rng.uniform(-warp, warp, size=(3, 3))
        low = rest[np.argmin(rest[:, 1])]
        t = low - A @ low  # the lowest point stays where it is
        xbar.append(rest)
        point_body.append(np.full(rest.shape[0], b, np.int32))
        tris.append(btris + P)
        masses_all.append(m)
        vols.append(float(tet_vol.sum()))
        q.append(np.concatenate([t, A.reshape(-1)]))
        P += rest.shape[0]
        start.append(P)
    xbar = np.concatenate(xbar)
    point_body = np.concatenate(point_body)
    q = np.stack(q)
    mass = np.zeros((nb, 13))
    for b in range(nb):
        xb, m = xbar[start[b]:start[b + 1]], masses_all[b]
        mass[b, 0] = m.sum()
        mass[b, 1:4] = (m[:, None] * xb).sum(0)
        mass[b, 4:] = (m[:, None, None] * xb[:, :, None] * xb[:, None, :]).sum(0).reshape(-1)
    q_tilde = q.copy()
    q_tilde[:, 1] += -9.8 * dt * dt
    fem = _assemble(f"slab{slab_n}x{slab_layers}", srest, srest.copy(), stets, np.full(stets.shape[0], E), nu, rho,
                    dt, np.zeros_like(srest), barriers=[((0.0, 1.0, 0.0), 0.0, np.sqrt(dhat), kappa)])
    # contacts between the bodies and the slab's top, over the point numbering
    xa = np.einsum("pij,pj->pi", q[point_body, 3:].reshape(-1, 3, 3), xbar) + q[point_body, :3]
    allpos = np.concatenate([xa, srest])
    body_of = np.concatenate([point_body.astype(np.int64), np.full(srest.shape[0], nb, np.int64)])
    alltris = np.concatenate([np.concatenate(tris), boundary_faces(stets) + P])
    band = allpos[alltris].min(axis=1)[:, 1] < top + 0.02
    pairs = contact_pairs(allpos, alltris[band], body_of, dhat)
    return AbdScene(name=f"abd{nb}_slab{slab_n}", q=q, q_tilde=q_tilde, mass=mass, volume=np.array(vols),
                    kappa=kappa_abd, dt=dt, point_body=point_body, xbar=xbar,
                    body_point_start=np.array(start, np.int32), fem=fem, contacts=pairs, dhat=dhat,
                    kappa_contact=kappa)


def _box_pairs(lo_a, hi_a, lo_b, hi_b, pad):
    """Index pairs (i, j) whose boxes [lo_a, hi_a] and [lo_b - pad, hi_b + pad] overlap, found
    on a uniform grid whose cell is at least every box's extent."""
    if lo_a.shape[0] == 0 or lo_b.shape[0] == 0:
        return np.zeros(0, np.int64), np.zeros(0, np.int64)
    h = max(float((hi_a - lo_a).max()), float((hi_b - lo_b).max()) + 2 * pad, 1e-12) * 1.0001
    w = np.array([1 << 42, 1 << 21, 1])
    ka = (np.floor(lo_a / h).astype(np.int64) + (1 << 20)) @ w
    order = np.argsort(ka, kind="stable")
    ks = ka[order]
    clo = np.floor((lo_b - pad) / h).astype(np.int64) - 1
    out_i, out_j = [], []
    for dx in range(3):
        for dy in range(3):
            for dz in range(3):
                kb = (clo + np.array([dx, dy, dz]) + (1 << 20)) @ w
                lo = np.searchsorted(ks, kb, "left")
                cnt = np.searchsorted(ks, kb, "right") - lo
                tot = int(cnt.sum())
                if tot == 0:
                    continue
                first = np.cumsum(cnt) - cnt
                out_i.append(order[np.repeat(lo, cnt) + np.arange(tot) - np.repeat(first, cnt)])
                out_j.append(np.repeat(np.arange(cnt.size), cnt))
    if not out_i:
        return np.zeros(0, np.int64), np.zeros(0, np.int64)
    i, j = np.concatenate(out_i), np.concatenate(out_j)
    ok = np.all(lo_a[i] <= hi_b[j] + pad, axis=1) & np.all(hi_a[i] >= lo_b[j] - pad, axis=1)
    return i[ok], j[ok]


def ccd_candidates(pos: np.ndarray, disp: np.ndarray, tris: np.ndarray, body: Optional[np.ndarray] = None,
                   pad: float = 0.0) -> np.ndarray:
    """The CCD pairs of a step (the reference's _ccd_collisonPairs): every (surface vertex,
    triangle) and (edge, edge) pair whose boxes swept over pos -> pos + disp overlap (within
    pad), sharing no vertex and, with `body`, of different bodies; point-triangle encoded
    (-p-1, t0, t1, t2), edge-edge (a0, a1, b0, b1)."""
    end = pos + disp
    lo_v, hi_v = np.minimum(pos, end), np.maximum(pos, end)
    verts = np.unique(tris)
    edges = face_edges(tris)
    out = []
    i, j = _box_pairs(lo_v[verts], hi_v[verts], lo_v[tris].min(axis=1), hi_v[tris].max(axis=1), pad)
    p, t = verts[i], tris[j]
    keep = (p != t[:, 0]) & (p != t[:, 1]) & (p != t[:, 2])
    if body is not None:
        keep &= body[p] != body[t[:, 0]]
    out.append(np.stack([-p[keep] - 1, t[keep, 0], t[keep, 1], t[keep, 2]], 1))
    i, j = _box_pairs(lo_v[edges].min(axis=1), hi_v[edges].max(axis=1), lo_v[edges].min(axis=1),
                      hi_v[edges].max(axis=1), pad)
    a, b = edges[i], edges[j]
    keep = (i < j) & (a[:, 0] != b[:, 0]) & (a[:, 0] != b[:, 1]) & (a[:, 1] != b[:, 0]) & (a[:, 1] != b[:, 1])
    if body is not None:
        keep &= body[a[:, 0]] != body[b[:, 0]]
    out.append(np.concatenate([a[keep], b[keep]], axis=1))
    return np.concatenate(out).astype(np.int32)


# ----------------------------------------------------------------------------------------
# Cloth on a soft ball (the cloth-on-solid configuration)
# ----------------------------------------------------------------------------------------


def cloth_rest_frame(rest: np.ndarray, tris: np.ndarray):
    """(Dm^-1 [T, 4] row-major 2x2, rest area [T]) of each triangle in the reference's 2D frame
    (__calculateDm2D_double, femEnergy.cu:256-303: the triangle rotated so that its normal is
    +z, then its x, y coordinates)."""
    x0, x1, x2 = rest[tris[:, 0]], rest[tris[:, 1]], rest[tris[:, 2]]
    n = np.cross(x1 - x0, x2 - x0)
    area = 0.5 * np.linalg.norm(n, axis=1)
    n = n / np.linalg.norm(n, axis=1, keepdims=True)
    z = np.array([0.0, 0.0, 1.0])
    vec = np.cross(n, z)
    cos = n @ z
    T = tris.shape[0]
    R = np.tile(np.eye(3), (T, 1, 1))
    flip = cos + 1 == 0
    R[flip, 0, 0] = R[flip, 1, 1] = -1
    k = ~flip
    C = np.zeros((T, 3, 3))
    C[:, 0, 1], C[:, 0, 2] = -vec[:, 2], vec[:, 1]
    C[:, 1, 0], C[:, 1, 2] = vec[:, 2], -vec[:, 0]
    C[:, 2, 0], C[:, 2, 1] = -vec[:, 1], vec[:, 0]
    R[k] = R[k] + C[k] + (C[k] @ C[k]) / (1 + cos[k])[:, None, None]
    u0 = np.einsum("tij,tj->ti", R, x1)[:, :2] - np.einsum("tij,tj->ti", R, x0)[:, :2]
    u1 = np.einsum("tij,tj->ti", R, x2)[:, :2] - np.einsum("tij,tj->ti", R, x0)[:, :2]
    Dm = np.stack([u0, u1], axis=2)  # columns u0, u1
    return np.linalg.inv(Dm).reshape(T, 4), area


def bending_stencils(rest: np.ndarray, tris: np.ndarray):
    """Interior edges (v0, v1, opposite of the first triangle, opposite of the second), their
    rest lengths and the quadratic bending matrices Q (PrepareQuadBendingQ,
    femEnergy.cu:2490-2618: Q = 3 / (A0 + A1) K K^T from the cotangent weights K)."""
    e = np.concatenate([tris[:, [0, 1, 2]], tris[:, [1, 2, 0]], tris[:, [2, 0, 1]]])  # edge a b, opposite c
    key = np.minimum(e[:, 0], e[:, 1]) * (rest.shape[0] + 1) + np.maximum(e[:, 0], e[:, 1])
    order = np.argsort(key, kind="stable")
    ks = key[order]
    pair = np.nonzero(ks[1:] == ks[:-1])[0]
    a, b = e[order[pair]], e[order[pair + 1]]
    st = np.stack([a[:, 0], a[:, 1], a[:, 2], b[:, 2]], axis=1)
    v0, v1, v2, v3 = (rest[st[:, i]] for i in range(4))
    e0, e1, e2, e3, e4 = v1 - v0, v2 - v0, v3 - v0, v2 - v1, v3 - v1

    def cot(p, q):
        cr = np.linalg.norm(np.cross(p, q), axis=1)
        return np.where(cr < 1e-12, 0.0, np.einsum("ij,ij->i", p, q) / np.where(cr < 1e-12, 1.0, cr))

    c01, c02, c03, c04 = cot(e0, e1), cot(e0, e2), cot(-e0, e3), cot(-e0, e4)
    K = np.stack([c03 + c04, c01 + c02, -c01 - c03, -c02 - c04], axis=1)
    a0 = 0.5 * np.linalg.norm(np.cross(e0, e1), axis=1)
    a1 = 0.5 * np.linalg.norm(np.cross(e0, e2), axis=1)
    Q = 3.0 / (a0 + a1)[:, None, None] * K[:, :, None] * K[:, None, :]
    return st.astype(np.int32), np.linalg.norm(e0, axis=1), Q.reshape(-1, 16)


def ball_mesh(n: int, radius: float, center):
    """A tet ball: the n^3-hex cube grid over [-1, 1]^3 mapped onto the ball (each point of the
    cube moved along the map x' = x sqrt(1 - y^2/2 - z^2/2 + y^2 z^2/3), cyclically)."""
    p, tets = box_mesh(n, n, n, 2.0 / n, origin=(-1.0, -1.0, -1.0))
    x, y, z = p[:, 0], p[:, 1], p[:, 2]
    q = np.stack([x * np.sqrt(1 - y * y / 2 - z * z / 2 + y * y * z * z / 3),
                  y * np.sqrt(1 - z * z / 2 - x * x / 2 + z * z * x * x / 3),
                  z * np.sqrt(1 - x * x / 2 - y * y / 2 + x * x * y * y / 3)], axis=1)
    return q * radius + np.asarray(center, np.float64), tets


@dataclasses.dataclass
class ClothScene:
    """Cloth (vertices with cloth triangles) and a tet ball in one vertex numbering (Morton
    ordered), at one Newton iteration.  base: the ball's elastic + inertia terms and a
    diagonal mass block per vertex (cloth vertices: their lumped cloth mass), with the
    inertia gradient of all vertices; the cloth membrane and bending terms and the contacts
    are added by stgipc.cloth.cloth_system."""
    name: str
    base: NewtonSystem
    tris: np.ndarray          # int32 [T, 3] cloth triangles
    dminv: np.ndarray         # [T, 4]
    area: np.ndarray          # [T] rest area x thickness
    stencil: np.ndarray       # int32 [E, 4]
    elen: np.ndarray          # [E]
    Q: np.ndarray             # [E, 16]
    stretch: float
    shear: float
    strain_rate: float
    bend: float
    dt: float
    contacts: np.ndarray      # int32 [C, 4]
    dhat: float
    kappa: float
    cloth_verts: int


def make_cloth_sphere(n: int = 256, size: float = 1.0, thickness: float = 1e-3, E_cloth: float = 1e4,
                      nu: float = 0.45, density_cloth: float = 200.0, strain_rate: float = 1.0,
                      bend: float = 1e-4, radius: float = 0.3, ball_n: int = 19, E_ball: float = 1e6,
                      rho_ball: float = 1000.0, dt: float = 1.0 / 60.0, drop_speed: float = 1.0, dhat: float = 1e-6,
                      kappa: float = 1e4, jitter: float = 1e-4, seed: int = 1002) -> ClothScene:
    """n x n cloth vertices over size x size m (2 (n-1)^2 triangles), Baraff-Witkin membrane
    with stretch stiffness E / (2 (1 + nu)) and shear 0.03 x stretch x strain rate, quadratic
    bending k = bend, thickness and density as given; draped over a tet ball of radius 0.3 m
    (ball_n^3 hexes, 6 tets each, Neo-Hookean E_ball): its middle follows the ball's cap 0.2 to
    0.8 mm above the surface out to 0.6 r, then continues along the cap's tangent cone; it
    moves down at drop_speed (the speed after a 5 cm drop); vertices jittered U(+-jitter) in
    the plane.  The Newton iteration of the step at which it lands.  kappa is sized to the
    cloth's weight (0.2 kg/m^2 over some 10^4 pairs: about 1e-5 N per pair, and a pair's barrier
    force at half the activation distance is about 9e-9 kappa N at dhat = 1e-6); a much stiffer
    barrier only makes the system worse conditioned."""
    rng = np.random.default_rng(seed)
    h = size / (n - 1)
    g = np.arange(n) * h
    X, Z = np.meshgrid(g, g, indexing="xy")
    cloth = np.stack([X.ravel(), np.zeros(n * n), Z.ravel()], axis=1)
    cloth[:, [0, 2]] += rng.uniform(-jitter, jitter, size=(n * n, 2))
    ii, jj = np.meshgrid(np.arange(n - 1), np.arange(n - 1), indexing="xy")
    a = (jj * n + ii).ravel()
    tris = np.concatenate([np.stack([a, a + 1, a + n + 1], 1), np.stack([a, a + n + 1, a + n], 1)])
    center = np.array([0.5 * size, radius, 0.5 * size])
    bpos, btets = ball_mesh(ball_n, radius, center)
    rest_cloth = cloth.copy()
    rest_cloth[:, 1] = 2 * radius + 0.05
    # draped shape
    r = np.hypot(cloth[:, 0] - center[0], cloth[:, 2] - center[2])
    r0 = 0.6 * radius
    cap = lambda rr: center[1] + np.sqrt(radius * radius - rr * rr)
    slope = r0 / np.sqrt(radius * radius - r0 * r0)
    gap = rng.uniform(2e-4, 8e-4, size=n * n)
    cloth[:, 1] = np.where(r < r0, cap(np.minimum(r, r0)) + gap, cap(r0) + gap - (r - r0) * slope)
    Vc = n * n
    pos = np.concatenate([cloth, bpos])
    rest = np.concatenate([rest_cloth, bpos])
    tets = btets + Vc
    # one Morton order for all vertices (the MAS banks are runs of consecutive vertices)
    key = morton_hash(pos)
    order = np.argsort(key, kind="stable")
    new_of_old = np.empty_like(order)
    new_of_old[order] = np.arange(order.size)
    pos, rest = pos[order], rest[order]
    tets = new_of_old[tets]
    tris = new_of_old[tris].astype(np.int64)
    body = (order >= Vc).astype(np.int64)   # 0 cloth, 1 ball
    V = pos.shape[0]
    vel = np.zeros_like(pos)
    vel[body == 0, 1] = -drop_speed
    base = _assemble(f"cloth{n}_ball", rest, pos, tets, np.full(tets.shape[0], E_ball), nu, rho_ball, dt, vel,
                     barriers=[])
    dminv, area0 = cloth_rest_frame(rest, tris)
    area = area0 * thickness
    mass = np.zeros(V)
    np.add.at(mass, tris.reshape(-1), np.repeat(density_cloth * area / 3.0, 3))
    # the cloth's lumped mass on its diagonal blocks and its inertia gradient M (x - xtilde)
    diag = np.arange(base.rows.size - V, base.rows.size)  # _assemble appends one mass block per vertex
    assert np.array_equal(base.rows[diag], np.arange(V)) and np.array_equal(base.cols[diag], np.arange(V))
    mb = base.blocks.copy()
    cm = mass[base.rows[diag]]
    mb[diag, 0] += cm
    mb[diag, 4] += cm
    mb[diag, 8] += cm
    x_tilde = pos + dt * vel + dt * dt * np.array([0.0, -9.8, 0.0])
    b = base.b.reshape(V, 3) + mass[:, None] * (pos - x_tilde)
    pairs_edges = np.concatenate([tris[:, [0, 1]], tris[:, [1, 2]], tris[:, [0, 2]],
                                  tets[:, [0, 1]], tets[:, [0, 2]], tets[:, [0, 3]], tets[:, [1, 2]], tets[:, [1, 3]],
                                  tets[:, [2, 3]]])
    start, num, nlist = edge_neighbors(V, pairs_edges)
    base = dataclasses.replace(base, blocks=mb, b=b.reshape(-1), neighbor_start=start, neighbor_num=num,
                               neighbor_list=nlist)
    st, elen, Q = bending_stencils(rest, tris)
    # contacts between the cloth and the ball's surface near it
    faces = np.concatenate([tris, boundary_faces(tets)])
    near = np.linalg.norm(pos[faces].mean(axis=1) - center, axis=1) < radius + 0.02
    contacts = contact_pairs(pos, faces[near], body, dhat)
    stretch = E_cloth / (2 * (1 + nu))
    return ClothScene(name=f"cloth{n}_ball", base=base, tris=tris.astype(np.int32), dminv=dminv, area=area,
                      stencil=st, elen=elen, Q=Q, stretch=stretch, shear=0.03 * stretch * strain_rate,
                      strain_rate=strain_rate, bend=bend, dt=dt, contacts=contacts, dhat=dhat, kappa=kappa,
                      cloth_verts=Vc)
