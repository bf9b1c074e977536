"""CPU oracle of the cloth terms of the Newton system (numpy, FP64).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of libstgipc's
stg_cloth_membrane / stg_cloth_bending.  Restates, per element and with explicit matrices:
  - the Baraff-Witkin membrane of _calculate_triangle_fem_gradient_hessian
    (StiffGIPC/femEnergy.cu:2146-2216): __computePEPF_BaraffWitkinStretch_double (:351-396) for
    the gradient, __project_BaraffWitkinStretch_H (:535-629) and the reference's analytic
    eigen-projection __project_BaraffWitkinShear_H (:631-706) for the Hessian, mapped by the
    6x9 dF/dx of __computePFDsPX3D_6x9_double (:1171-1220);
  - the quadratic bending of _calculate_quad_bending_gradient_hessian (:2620-2755).
Outputs use the device layout: per triangle 6 upper 3x3 blocks (column-major, row <= col) and
9 gradient entries; per edge stencil 10 upper blocks and 12 gradient entries.
"""
from __future__ import annotations

import numpy as np

TRI_SLOTS = [(a, b) for a in range(3) for b in range(a, 3)]
EDGE_SLOTS = [(a, b) for a in range(4) for b in range(a, 4)]


def dfdx(dminv):
    """The 6x9 map from the triangle's vertex coordinates to vec(F) (column u, then v)."""
    D = np.asarray(dminv, np.float64).reshape(2, 2)
    M = np.zeros((6, 9))
    for c in range(2):
        w = [-(D[0, c] + D[1, c]), D[0, c], D[1, c]]
        for a in range(3):
            for d in range(3):
                M[3 * c + d, 3 * a + d] = w[a]
    return M


def _shear_projected(F):
    """__project_BaraffWitkinShear_H, restated (femEnergy.cu:631-706)."""
    S = np.zeros((6, 6))
    for i in range(3):
        S[3 + i, i] = S[i, 3 + i] = 1.0
    fu, fv = F[:, 0], F[:, 1]
    I6 = float(fu @ fv)
    sign = 1.0 if I6 >= 0 else -1.0
    g = np.concatenate([fv, fu])
    I2 = float((F * F).sum())
    lam0 = 0.5 * (I2 + np.sqrt(I2 * I2 + 12 * I6 * I6))
    q0 = I6 * (S @ g) + lam0 * g
    q0 = q0 / np.linalg.norm(q0)
    T = 0.5 * (np.eye(6) + sign * S)
    Tq = T @ q0
    tmp = (T - np.outer(Tq, Tq) / float(Tq @ Tq)) * abs(I6)
    tmp = tmp + lam0 * np.outer(q0, q0)
    return 2 * tmp


def _stretch_projected(F, sr):
    """__project_BaraffWitkinStretch_H, restated (femEnergy.cu:535-629)."""
    H = np.zeros((6, 6))
    for c in range(2):
        f = F[:, c]
        I5 = float(f @ f)
        s = np.sqrt(I5)
        iso = 2 * (((s - 1) * (3 * s * sr - 3 * sr + 2)) / (2 * s)) if s > 1 else 0.0
        along = (3 * I5 * sr - 3 * sr + 2) / s if s > 1 else 2.0
        fh = f / s
        H[3 * c:3 * c + 3, 3 * c:3 * c + 3] = iso * np.eye(3) + along * np.outer(fh, fh)
    return H


def membrane_energy_F(F, kst, ksh, sr):
    """The Baraff-Witkin energy density the gradient differentiates (without area dt^2)."""
    su, sv = np.linalg.norm(F[:, 0]), np.linalg.norm(F[:, 1])
    e = (su - 1) ** 2 + (sv - 1) ** 2
    e += sr * (max(su - 1, 0.0) ** 3 + max(sv - 1, 0.0) ** 3)
    return kst * e + ksh * float(F[:, 0] @ F[:, 1]) ** 2


def membrane(tris, dminv, area, x, kst, ksh, sr, dt, off=0):
    """(rows, cols, blocks [6 T, 9], grad [T, 9]) of the triangles' membrane terms."""
    tris = np.asarray(tris).reshape(-1, 3)
    T = tris.shape[0]
    rows, cols = np.zeros(6 * T, np.int32), np.zeros(6 * T, np.int32)
    blocks, grad = np.zeros((6 * T, 9)), np.zeros((T, 9))
    for t in range(T):
        v = tris[t]
        X = x[v]
        D = np.asarray(dminv[t]).reshape(2, 2)
        Ds = np.stack([X[1] - X[0], X[2] - X[0]], axis=1)
        F = Ds @ D
        fu, fv = F[:, 0], F[:, 1]
        su, sv = np.linalg.norm(fu), np.linalg.norm(fv)
        cu, cv = 1 - 1 / su, 1 - 1 / sv
        if su * su > 1:
            cu += 1.5 * sr * (su + 1 / su - 2)
        if sv * sv > 1:
            cv += 1.5 * sr * (sv + 1 / sv - 2)
        I6 = float(fu @ fv)
        P = np.concatenate([kst * 2 * cu * fu + ksh * 2 * I6 * fv, kst * 2 * cv * fv + ksh * 2 * I6 * fu])
        M = dfdx(D)
        k = area[t] * dt * dt
        grad[t] = k * (M.T @ P)
        Hq = kst * _stretch_projected(F, sr) + ksh * _shear_projected(F)
        H = k * (M.T @ Hq @ M)
        for s, (a, b) in enumerate(TRI_SLOTS):
            gi, gj = off + v[a], off + v[b]
            B = H[3 * a:3 * a + 3, 3 * b:3 * b + 3]
            if gi > gj:
                gi, gj, B = gj, gi, B.T
            rows[6 * t + s], cols[6 * t + s] = gi, gj
            blocks[6 * t + s] = B.T.reshape(9)
    return rows, cols, blocks, grad


def bending(stencil, Q, length, x, kb, dt, off=0):
    """(rows, cols, blocks [10 E, 9], grad [E, 12]) of the quadratic bending stencils."""
    stencil = np.asarray(stencil).reshape(-1, 4)
    E = stencil.shape[0]
    rows, cols = np.zeros(10 * E, np.int32), np.zeros(10 * E, np.int32)
    blocks, grad = np.zeros((10 * E, 9)), np.zeros((E, 12))
    for e in range(E):
        v = stencil[e]
        if v[3] < 0:
            rows[10 * e:10 * e + 10] = cols[10 * e:10 * e + 10] = off + v[0]
            continue
        Qe = np.asarray(Q[e]).reshape(4, 4)
        c = length[e] * kb * dt * dt
        grad[e] = c * (Qe @ x[v]).reshape(-1)
        for s, (a, b) in enumerate(EDGE_SLOTS):
            gi, gj = off + v[a], off + v[b]
            if gi > gj:
                gi, gj = gj, gi
            rows[10 * e + s], cols[10 * e + s] = gi, gj
            blocks[10 * e + s] = (c * Qe[a, b] * np.eye(3)).reshape(9)
    return rows, cols, blocks, grad
