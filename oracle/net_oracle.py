"""CPU oracle of the learned coarse correction (test infrastructure only).

The reference has no learned part, so this is a restatement of this project's own network
(include/stgipc.h, stg_net_*): the coarse level's graph, the forward pass with the same
BF16 rounding points as the CUDA kernels, the energy loss, its exact gradient (float64
backward) and Adam.  It checks the CUDA forward, gradients and optimiser step, and is
itself checked against central finite differences (tests/test_net_oracle.py).  Only the
tests may import it.
"""
from __future__ import annotations

import numpy as np

IN, H, OUT, LAYERS = 16, 64, 8, 3
P = dict(W0=(0, (H, IN)), b0=(1024, (H,)), W1=(1088, (LAYERS, H, 2 * H)), b1=(25664, (LAYERS, H)),
         Wo=(25856, (OUT, H)), bo=(26368, (OUT,)))
COUNT = 26376


def unpack(p):
    out = {}
    for k, (o, shp) in P.items():
        out[k] = p[o:o + int(np.prod(shp))].reshape(shp)
    return out


def pack(d):
    p = np.zeros(COUNT, np.float64)
    for k, (o, shp) in P.items():
        p[o:o + int(np.prod(shp))] = np.asarray(d[k], np.float64).reshape(-1)
    return p


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(np.asarray(x, np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32).reshape(a.shape)


def build_graph(n, urow, ucol, ublk):
    """The level's graph from its sorted unique upper BCOO (level-local ids; blocks [k][9]
    column-major): full symmetric neighbour lists sorted by column, A_(i,col) row-major,
    diagonal blocks, coupling weights |A_ij|_F / sqrt(|A_ii|_F |A_jj|_F) and the centred log
    trace of the diagonal blocks.  learned.cu: k_ng_count / k_ng_fill / k_ng_finish /
    k_ng_feat."""
    H9 = np.asarray(ublk, np.float64).reshape(-1, 3, 3).transpose(0, 2, 1)  # row-major A_(r,c)
    dblk = np.zeros((n, 3, 3), np.float32)
    nbr = [[] for _ in range(n)]
    for k, (r, c) in enumerate(zip(urow, ucol)):
        if r == c:
            dblk[r] = H9[k]
        else:
            nbr[r].append((c, k, 0))
            nbr[c].append((r, k, 1))
    row = np.zeros(n + 1, np.int32)
    col, w, oblk = [], [], []
    dn = np.sqrt((dblk.astype(np.float32) ** 2).sum(axis=(1, 2)))
    for i in range(n):
        lst = sorted(nbr[i])
        row[i + 1] = row[i] + len(lst)
        for c, k, t in lst:
            A = H9[k].T if t else H9[k]
            col.append(c)
            oblk.append(A.astype(np.float32))
            fro = np.sqrt((H9[k].astype(np.float32) ** 2).sum())
            den = np.sqrt(dn[i] * dn[c])
            w.append(fro / den if den > 0 else 0.0)
    tr = np.log(np.maximum(dblk[:, 0, 0].astype(np.float64) + dblk[:, 1, 1] + dblk[:, 2, 2], 1e-30))
    feat = (tr - tr.mean()).astype(np.float32)
    return dict(n=n, row=row, col=np.array(col, np.int32), w=np.array(w, np.float32),
                oblk=np.array(oblk, np.float32).reshape(-1, 3, 3), dblk=dblk, feat=feat)


def level_matvec(g, v):
    """y = A_c v, v [n][3] (float64)."""
    y = np.einsum("nab,nb->na", g["dblk"].astype(np.float64), v)
    for i in range(g["n"]):
        for e in range(g["row"][i], g["row"][i + 1]):
            y[i] += g["oblk"][e].astype(np.float64) @ v[g["col"][e]]
    return y


def aggregate(g, h):
    """m_i = sum_j w_ij h_j over neighbours (float64)."""
    m = np.zeros_like(h, dtype=np.float64)
    for i in range(g["n"]):
        for e in range(g["row"][i], g["row"][i + 1]):
            m[i] += float(g["w"][e]) * h[g["col"][e]]
    return m


def forward(g, rc, zc, params, rounding=True):
    """One sample (rc, zc: [n][3]).  Returns d [n][3] and the cache for backward."""
    R = bf16 if rounding else (lambda x: np.asarray(x, np.float64))
    q = unpack(params)
    n = g["n"]
    rc = np.asarray(rc, np.float32)
    zc = np.asarray(zc, np.float32)
    sr = np.float32(np.sqrt((rc.astype(np.float64) ** 2).sum() / n))
    sz = np.float32(np.sqrt((zc.astype(np.float64) ** 2).sum() / n))
    sr = sr if sr > 0 else np.float32(1)
    sz = sz if sz > 0 else np.float32(1)
    x = np.zeros((n, IN), np.float64)
    if rounding:
        x[:, 0:3] = R(rc * (np.float32(1) / sr))
        x[:, 3:6] = R(zc * (np.float32(1) / sz))
        x[:, 6] = R(g["feat"])
    else:
        x[:, 0:3] = rc / float(sr)
        x[:, 3:6] = zc / float(sz)
        x[:, 6] = g["feat"]
    x[:, 7] = 1.0
    W0, W1, Wo = R(q["W0"]), R(q["W1"]), R(q["Wo"])
    W0, W1, Wo = (np.asarray(a, np.float64) for a in (W0, W1, Wo))

    def act(u):
        return np.asarray(R(np.maximum(u, 0.0).astype(np.float32) if rounding else np.maximum(u, 0.0)), np.float64)

    hs = [act((x @ W0.T).astype(np.float32 if rounding else np.float64) + q["b0"])]
    ms = []
    for k in range(LAYERS):
        m = np.asarray(R(aggregate(g, hs[-1]).astype(np.float32) if rounding else aggregate(g, hs[-1])), np.float64)
        ms.append(m)
        u = np.concatenate([hs[-1], m], axis=1) @ W1[k].T
        hs.append(act(u.astype(np.float32 if rounding else np.float64) + q["b1"][k]))
    d = (hs[-1] @ Wo.T)[:, :3]
    d = d.astype(np.float32 if rounding else np.float64) + q["bo"][:3]
    cache = dict(x=x, hs=hs, ms=ms, W0=W0, W1=W1, Wo=Wo, sz=float(sz), sr=float(sr))
    return np.asarray(d, np.float64), cache


def loss_grad(g, rc, zc, d, sz):
    """J(z + s_z d) / |J(z)| and its gradient in d (float64), J(v) = v.A v / 2 - v.r."""
    rc = np.asarray(rc, np.float64)
    zc = np.asarray(zc, np.float64)
    gv = zc + sz * d
    y = level_matvec(g, gv)
    y0 = level_matvec(g, zc)
    J = 0.5 * (gv * y).sum() - (gv * rc).sum()
    J0 = 0.5 * (zc * y0).sum() - (zc * rc).sum()
    inv = 1.0 / abs(J0) if J0 != 0 else 0.0
    return J * inv, sz * inv * (y - rc)


def backward(g, cache, dd):
    """Gradient of the loss in the flat parameter vector, given dL/dd [n][3]."""
    hs, ms, x = cache["hs"], cache["ms"], cache["x"]
    W1, Wo = cache["W1"], cache["Wo"]
    grads = {k: np.zeros(shp) for k, (_, shp) in P.items()}
    ddo = np.zeros((dd.shape[0], OUT))
    ddo[:, :3] = dd
    grads["Wo"] = ddo.T @ hs[-1]
    grads["bo"] = ddo.sum(0)
    dh = ddo @ Wo
    for k in range(LAYERS - 1, -1, -1):
        du = dh * (hs[k + 1] > 0)
        X = np.concatenate([hs[k], ms[k]], axis=1)
        grads["W1"][k] = du.T @ X
        grads["b1"][k] = du.sum(0)
        dX = du @ W1[k]
        dh = dX[:, :H] + aggregate(g, dX[:, H:])
    du = dh * (hs[0] > 0)
    grads["W0"] = du.T @ x
    grads["b0"] = du.sum(0)
    return pack(grads)


def batch_loss_grad(g, rcs, zcs, params, rounding=True):
    """Mean loss over samples and its parameter gradient (the CUDA training step's loss /
    grad outputs)."""
    S = len(rcs)
    losses, grad = [], np.zeros(COUNT)
    for rc, zc in zip(rcs, zcs):
        d, cache = forward(g, rc, zc, params, rounding)
        L, dd = loss_grad(g, rc, zc, d, cache["sz"])
        losses.append(L)
        grad += backward(g, cache, dd / S)
    return np.array(losses), grad


def adam(p, grad, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (learned.cu: k_net_adam)."""
    m = b1 * m + (1 - b1) * grad
    v = b2 * v + (1 - b2) * grad * grad
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return p - lr * mh / (np.sqrt(vh) + eps), m, v


def random_level(n=40, seed=0):
    """A random SPD 3x3-block operator on a ring-with-chords graph, as a sorted unique upper
    BCOO (level-local ids, column-major blocks), with samples r_c and z_c = D^-1 r_c."""
    rng = np.random.default_rng(seed)
    edges = set()
    for i in range(n):
        edges.add((i, (i + 1) % n))
        edges.add((i, int(rng.integers(0, n))))
    up = sorted({(min(a, b), max(a, b)) for a, b in edges if a != b})
    blocks = {}
    diag = np.zeros((n, 3, 3))
    for (a, b) in up:
        B = rng.standard_normal((3, 3)) * 0.3
        blocks[(a, b)] = B
        s = np.abs(B).sum()
        diag[a] += s * np.eye(3)
        diag[b] += s * np.eye(3)
    for i in range(n):
        Q = rng.standard_normal((3, 3))
        diag[i] += Q @ Q.T + np.eye(3) * (1 + 10 ** rng.uniform(0, 2))
    keys = sorted([(i, i) for i in range(n)] + up)
    urow = np.array([k[0] for k in keys], np.int32)
    ucol = np.array([k[1] for k in keys], np.int32)
    ublk = np.array([(diag[i] if i == j else blocks[(i, j)]).T.reshape(9) for i, j in keys])
    return urow, ucol, ublk
