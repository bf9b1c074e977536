"""CPU oracle of the affine-body (ABD) part of the Newton system (numpy, FP64).

TEST INFRASTRUCTURE ONLY: imported by tests/ and bench.py's CPU legs as the checker of
libstgipc's stg_abd_* entry points.  Restates, with explicit matrices rather than the device
code's entry formulas:
  - body Hessian / gradient: ABDSystem::_cal_abd_body_gradient_and_hessian
    (abd_system/abd_system_function/setup_abd_system_gradient_and_hessian.cu:200-262), the
    orthogonality potential of abd_system/details/abd_energy.inl:9-140 and the dyadic mass of
    abd_jacobi_matrix.inl:95-150, with make_pd (:186-198) as an eigen-decomposition clamp;
  - J = [I3 | xbar^T (x) I3 rows] (ABDJacobi::to_mat, abd_jacobi_matrix.inl:24-35) and the
    point-to-body mapping of write_barrier_hessian / the ABD-FEM kernel (:89-126, 510-551);
  - the ABD block-Jacobi of _cal_abd_system_preconditioner (:612-655).
"""
from __future__ import annotations

import numpy as np

SLOTS = [(i, j) for i in range(4) for j in range(i, 4)]


def jacobian(xbar) -> np.ndarray:
    """The 3x12 ABDJacobi of a rest point: x = J q."""
    J = np.zeros((3, 12))
    J[:, :3] = np.eye(3)
    for r in range(3):
        J[r, 3 + 3 * r:6 + 3 * r] = xbar
    return J


def dyadic_mass_matrix(m13) -> np.ndarray:
    """12x12 M from (m, m xbar, m xbar xbar^T) = sum_i m_i J_i^T J_i."""
    M = np.zeros((12, 12))
    m, mx, D = m13[0], np.asarray(m13[1:4]), np.asarray(m13[4:13]).reshape(3, 3)
    M[:3, :3] = m * np.eye(3)
    for r in range(3):
        M[r, 3 + 3 * r:6 + 3 * r] = mx
        M[3 + 3 * r:6 + 3 * r, r] = mx
        M[3 + 3 * r:6 + 3 * r, 3 + 3 * r:6 + 3 * r] = D
    return M


def dyadic_mass(masses, xbars) -> np.ndarray:
    """(m, m xbar, m xbar xbar^T) of a body from its points' masses and rest positions."""
    m = float(np.sum(masses))
    mx = (masses[:, None] * xbars).sum(0)
    D = (masses[:, None, None] * xbars[:, :, None] * xbars[:, None, :]).sum(0)
    return np.concatenate([[m], mx, D.reshape(-1)])


def shape_gradient_hessian(q):
    """dS/da (9) and d2S/da2 (9x9) of S = ||A A^T - I||_F^2, a = (a1, a2, a3) the rows of A."""
    a = np.asarray(q[3:12]).reshape(3, 3)
    G = a @ a.T
    g = np.zeros(9)
    H = np.zeros((9, 9))
    for i in range(3):
        g[3 * i:3 * i + 3] = 4 * (G[i, i] - 1) * a[i] + sum(4 * G[j, i] * a[j] for j in range(3) if j != i)
        for j in range(3):
            if i == j:
                blk = 8 * np.outer(a[i], a[i]) + 4 * (G[i, i] - 1) * np.eye(3)
                blk += sum(4 * np.outer(a[k], a[k]) for k in range(3) if k != i)
            else:
                blk = 4 * np.outer(a[j], a[i]) + 4 * G[i, j] * np.eye(3)
            H[3 * i:3 * i + 3, 3 * j:3 * j + 3] = blk
    return g, H


def psd(H):
    w, V = np.linalg.eigh(H)
    if np.all(w >= 0):
        return H
    return (V * np.maximum(w, 0)) @ V.T


def body_system(q, q_tilde, mass13, volume, kappa, dt, fixed=None):
    """(rows, cols, blocks [10 N, 9] column-major, grad [N, 12]) of the bodies' inertia +
    orthogonality terms."""
    q, q_tilde = np.asarray(q).reshape(-1, 12), np.asarray(q_tilde).reshape(-1, 12)
    N = q.shape[0]
    rows, cols = np.zeros(10 * N, np.int32), np.zeros(10 * N, np.int32)
    blocks, grad = np.zeros((10 * N, 9)), np.zeros((N, 12))
    for b in range(N):
        M = dyadic_mass_matrix(mass13[b])
        H = M.copy()
        if fixed is not None and fixed[b]:
            g = np.zeros(12)
        else:
            g = M @ (q[b] - q_tilde[b])
            k = kappa * volume[b] * dt * dt
            sg, sh = shape_gradient_hessian(q[b])
            g[3:] += k * sg
            H[3:, 3:] += psd(k * sh)
        grad[b] = g
        for s, (i, j) in enumerate(SLOTS):
            rows[10 * b + s], cols[10 * b + s] = 4 * b + i, 4 * b + j
            blocks[10 * b + s] = H[3 * i:3 * i + 3, 3 * j:3 * j + 3].T.reshape(9)
    return rows, cols, blocks, grad


def map_triplets(rows, cols, blocks, P, point_body, xbar, N):
    """16 output triplets per input, as stg_abd_map_triplets documents."""
    cnt = len(rows)
    orow, ocol = np.zeros(16 * cnt, np.int32), np.zeros(16 * cnt, np.int32)
    oblk = np.zeros((16 * cnt, 9))
    for t in range(cnt):
        i, j = int(rows[t]), int(cols[t])
        B = np.asarray(blocks[t]).reshape(3, 3).T  # column-major -> matrix
        if i > j:
            i, j, B = j, i, B.T
        out = []
        if i >= P:
            out.append((4 * N + i - P, 4 * N + j - P, B))
        elif j >= P:
            X = jacobian(xbar[i]).T @ B  # 12x3
            for k in range(4):
                out.append((4 * point_body[i] + k, 4 * N + j - P, X[3 * k:3 * k + 3]))
        else:
            bi, bj = int(point_body[i]), int(point_body[j])
            X = jacobian(xbar[i]).T @ B @ jacobian(xbar[j])
            if bi < bj:
                for ii in range(4):
                    for jj in range(4):
                        out.append((4 * bi + ii, 4 * bj + jj, X[3 * ii:3 * ii + 3, 3 * jj:3 * jj + 3]))
            elif bi > bj:
                XT = X.T
                for ii in range(4):
                    for jj in range(4):
                        out.append((4 * bj + jj, 4 * bi + ii, XT[3 * jj:3 * jj + 3, 3 * ii:3 * ii + 3]))
            else:
                Y = X if i == j else X + X.T
                for (ii, jj) in SLOTS:
                    out.append((4 * bi + ii, 4 * bi + jj, Y[3 * ii:3 * ii + 3, 3 * jj:3 * jj + 3]))
        r0 = out[0][0]
        for s in range(16):
            o = 16 * t + s
            if s < len(out):
                orow[o], ocol[o] = out[s][0], out[s][1]
                oblk[o] = out[s][2].T.reshape(9)
            else:
                orow[o] = ocol[o] = r0
    return orow, ocol, oblk


def points(point_body, xbar, q):
    q = np.asarray(q).reshape(-1, 12)
    return np.stack([jacobian(xbar[i]) @ q[point_body[i]] for i in range(len(point_body))])


def gather_gradient(start, xbar, point_grad, body_grad):
    out = np.array(body_grad, dtype=np.float64).copy()
    for b in range(len(start) - 1):
        for i in range(start[b], start[b + 1]):
            out[b] += jacobian(xbar[i]).T @ point_grad[i]
    return out


def block_jacobi(rows, cols, blocks, N):
    """Row-major inverses of the bodies' diagonal 12x12 tiles of a sorted unique upper BCOO."""
    P = np.zeros((N, 12, 12))
    for r, c, b in zip(rows, cols, blocks):
        if r < 4 * N and r // 4 == c // 4:
            B = np.asarray(b).reshape(3, 3).T
            R, C = 3 * (r % 4), 3 * (c % 4)
            P[r // 4, R:R + 3, C:C + 3] = B
            if r != c:
                P[r // 4, C:C + 3, R:R + 3] = B.T
    return np.linalg.inv(P)


def coupled_system(sc):
    """The triplets and b of an AbdScene's Newton iteration, built on the host from these
    restatements and the contact oracle (the CPU counterpart of stgipc.abd.coupled_system)."""
    from oracle import oracle as orc
    N, P, V = sc.bodies, sc.abd_points, sc.fem.num_verts
    br, bc, bb, bg = body_system(sc.q, sc.q_tilde, sc.mass, sc.volume, sc.kappa, sc.dt)
    allpos = np.concatenate([points(sc.point_body, sc.xbar, sc.q), sc.fem.pos])
    cr, cc, cb, cg, _ = orc.contact_barrier(sc.contacts, allpos, sc.dhat, sc.kappa_contact)
    mr, mc, mb = map_triplets(cr, cc, cb, P, sc.point_body, sc.xbar, N)
    pg = np.zeros((P + V, 3))
    for p, q in enumerate(sc.contacts):
        vid = [(-q[0] - 1) if q[0] < 0 else q[0], q[1], q[2], q[3]]
        for k in range(4):
            if vid[k] >= 0:
                pg[vid[k]] += cg[p, 3 * k:3 * k + 3]
    bgrad = gather_gradient(sc.body_point_start, sc.xbar, pg[:P], bg)
    b = np.concatenate([bgrad.reshape(-1), sc.fem.b + pg[P:].reshape(-1)])
    rows = np.concatenate([br, mr, sc.fem.rows + 4 * N]).astype(np.int32)
    cols = np.concatenate([bc, mc, sc.fem.cols + 4 * N]).astype(np.int32)
    return rows, cols, np.concatenate([bb, mb, sc.fem.blocks]), b
