"""The learned coarse correction: data, training and inference helpers over the C ABI.

The network (stgipc.h, ``stg_net_*``) reads one coarse MAS level: its restricted residual
r_c and bank solve z_c = D^-1 r_c, and predicts g = z_c + s_z d(r_c, z_c) in place of z_c.
Training minimises the energy loss J(g) / |J(z_c)| with J(g) = g.A_c g / 2 - g.r_c over
(residual, error) samples that the plain FP64 solver records (``record_samples``); all
forward, backward and Adam work runs in the library's kernels on the GPU.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os
from typing import List, Optional

import numpy as np

from . import _lib as _L
from ._lib import check

NET_PARAMS = _L.NET_PARAMS
IN, H, OUT, LAYERS = 16, 64, 8, 3
OFF = dict(W0=0, b0=1024, W1=1088, b1=25664, Wo=25856, bo=26368)


def _ptr(t):
    return None if t is None else t.data_ptr()


@dataclasses.dataclass
class NetGraph:
    """One coarse level as a graph (device tensors, layout of stg_net_export_graph)."""
    nodes: int
    entries: int
    row: object
    col: object
    w: object
    oblk: object
    dblk: object
    feat: object

    def c(self) -> _L.NetGraphC:
        g = _L.NetGraphC()
        g.nodes, g.entries = self.nodes, self.entries
        g.row, g.col, g.w = _ptr(self.row), _ptr(self.col), _ptr(self.w)
        g.oblk, g.dblk, g.feat = _ptr(self.oblk), _ptr(self.dblk), _ptr(self.feat)
        return g

    def numpy(self) -> dict:
        e = max(self.entries, 1)
        return dict(n=self.nodes, row=self.row.cpu().numpy(), col=self.col.cpu().numpy()[:self.entries],
                    w=self.w.cpu().numpy()[:self.entries], oblk=self.oblk.cpu().numpy()[:9 * e].reshape(e, 3, 3)[:self.entries],
                    dblk=self.dblk.cpu().numpy().reshape(-1, 3, 3), feat=self.feat.cpu().numpy())


def init_params(seed: int = 0, head_scale: float = 1e-3) -> np.ndarray:
    """He-initialised weights, zero biases, a small head (the untrained network is close to
    plain MAS: d ~ 0)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NET_PARAMS, np.float32)
    p[OFF["W0"]:OFF["b0"]] = rng.standard_normal(H * IN) * np.sqrt(2.0 / 8)  # 8 live inputs
    for k in range(LAYERS):
        a = OFF["W1"] + k * H * 2 * H
        p[a:a + H * 2 * H] = rng.standard_normal(H * 2 * H) * np.sqrt(2.0 / (2 * H))
    p[OFF["Wo"]:OFF["Wo"] + 3 * H] = rng.standard_normal(3 * H) * head_scale
    return p


def scratch(nodes: int, samples: int, device="cuda"):
    import torch
    nb = int(_L.lib().stg_net_scratch_bytes(int(nodes), int(samples)))
    return torch.empty(nb, dtype=torch.uint8, device=device)


def forward(graph: NetGraph, rc, zc, params, samples: int, stream=None, buf=None):
    """d [samples][nodes][4] for samples rc / zc ([samples][nodes][4] FP32)."""
    import torch
    buf = buf if buf is not None else scratch(graph.nodes, samples, rc.device)
    delta = torch.empty(samples * graph.nodes * 4, dtype=torch.float32, device=rc.device)
    s = None if stream is None else stream.cuda_stream
    g = graph.c()
    check(_L.lib().stg_net_forward(C.byref(g), _ptr(rc), _ptr(zc), int(samples), _ptr(params), _ptr(delta), _ptr(buf),
                                   buf.numel(), s), "stg_net_forward")
    return delta.view(samples, graph.nodes, 4)


def apply(graph: NetGraph, rc, z, params, stream=None, buf=None) -> int:
    """In place z += theta s_z d(rc, z) for one sample (rc, z: [nodes][4] FP32), as inside the
    PCG loop.  Returns the cluster size of the fused kernel used (0: layered kernels)."""
    buf = buf if buf is not None else scratch(graph.nodes, 1, rc.device)
    fused = C.c_int()
    s = None if stream is None else stream.cuda_stream
    g = graph.c()
    check(_L.lib().stg_net_apply(C.byref(g), _ptr(rc), _ptr(z), _ptr(params), _ptr(buf), buf.numel(),
                                 C.byref(fused), s), "stg_net_apply")
    return fused.value


class Trainer:
    """Adam on the library's kernels; params / moments / gradient are FP32 device tensors."""

    def __init__(self, params: np.ndarray, device="cuda"):
        import torch
        self.device = torch.device(device)
        self.params = torch.from_numpy(np.ascontiguousarray(params, np.float32)).to(self.device)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.grad = torch.zeros_like(self.params)
        self.t = 0
        self._buf = {}

    def _scratch(self, nodes, samples):
        key = (nodes, samples)
        if key not in self._buf:
            self._buf[key] = scratch(nodes, samples, self.device)
        return self._buf[key]

    def step(self, graph: NetGraph, rc, zc, samples: int, lr: float):
        """One Adam step on `samples` samples (lr 0: gradient only).  Returns the per-sample
        losses (device tensor)."""
        import torch
        buf = self._scratch(graph.nodes, samples)
        loss = torch.empty(samples, dtype=torch.float32, device=self.device)
        if lr > 0:
            self.t += 1
        g = graph.c()
        check(_L.lib().stg_net_train_step(C.byref(g), _ptr(rc), _ptr(zc), int(samples), _ptr(self.params),
                                          _ptr(self.grad), _ptr(self.m), _ptr(self.v), max(self.t, 1), float(lr),
                                          _ptr(loss), _ptr(buf), buf.numel(), None), "stg_net_train_step")
        return loss

    def evaluate(self, graph: NetGraph, rc, zc, samples: int) -> float:
        """Mean loss without an update."""
        return float(self.step(graph, rc, zc, samples, 0.0).mean())


@dataclasses.dataclass
class Dataset:
    graph: NetGraph
    rc: object       # [samples][nodes][4]
    zc: object
    samples: int


def record_samples(solver, sysm, capacity: int = 256, every: int = 1, device="cuda") -> Dataset:
    """Run the plain solver of `solver` (MAS, learned off, level configured) on the scene
    `sysm` (stgipc.scenes system) with the recorder armed; returns the level's graph and
    the recorded (r_c, z_c) samples."""
    import torch
    dev = torch.device(device)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    rows, cols, blocks, b = t(sysm.rows), t(sysm.cols), t(sysm.blocks.reshape(-1)), t(sysm.b)
    x = torch.zeros_like(b)
    # the first assembly (inside the solve) builds the graph; its size sizes the buffers
    solver.solve_linear_system(rows, cols, blocks, b, x)
    g = solver.net_graph(device)
    rc = torch.zeros(capacity * g.nodes * 4, dtype=torch.float32, device=dev)
    zc = torch.zeros_like(rc)
    solver.net_record(rc, zc, capacity, every)
    x.zero_()
    st = solver.solve_linear_system(rows, cols, blocks, b, x)
    n = solver.net_recorded()
    solver.net_record(rc, zc, 0, 1)
    return Dataset(g, rc.view(capacity, g.nodes, 4)[:n].contiguous(), zc.view(capacity, g.nodes, 4)[:n].contiguous(), n), st


def train(trainer: Trainer, data: List[Dataset], steps: int, batch: int = 16, lr: float = 1e-3, seed: int = 0,
          log_every: int = 0, lr_final: Optional[float] = None) -> list:
    """Minibatch Adam over the datasets (one dataset per step, round robin; random samples);
    the step size decays from lr to lr_final on a cosine when lr_final is given."""
    import torch
    rng = np.random.default_rng(seed)
    hist = []
    for it in range(steps):
        d = data[it % len(data)]
        k = min(batch, d.samples)
        idx = torch.from_numpy(rng.choice(d.samples, size=k, replace=False)).to(d.rc.device)
        a = lr if lr_final is None else lr_final + 0.5 * (lr - lr_final) * (1 + np.cos(np.pi * it / max(steps - 1, 1)))
        loss = trainer.step(d.graph, d.rc[idx].contiguous(), d.zc[idx].contiguous(), k, a)
        if log_every and (it % log_every == 0 or it == steps - 1):
            hist.append((it, float(loss.mean())))
    return hist


WEIGHTS = os.path.join(os.path.dirname(__file__), "weights")


def default_weights(level: int = 2, n: int = 48) -> str:
    return os.path.join(WEIGHTS, f"net_hetcube{n}_L{level}.npz")


def load_weights(path: str):
    """(params FP32 [STG_NET_PARAMS], level, metadata dict) from a file ``train`` wrote."""
    z = np.load(path, allow_pickle=False)
    meta = {k: z[k].item() if z[k].ndim == 0 else z[k].tolist() for k in z.files if k != "params"}
    return z["params"].astype(np.float32), int(z["level"]), meta


def train_hetcube(n: int = 48, seeds=range(2000, 2008), level: int = 2, steps: int = 12000, batch: int = 16,
                  lr: float = 1e-3, lr_final: float = 5e-5, capacity: int = 600, every: int = 1, device="cuda",
                  log=print):
    """The shipped network's recipe: (residual, error) samples from the plain FP64 solver on
    heterogeneous cubes with seed-distinct materials (seeds 2000.. ; the benchmark scene uses
    1005), then Adam on the library's kernels.  Returns (params, metadata)."""
    import time
    from . import scenes
    from .linear_system import PCGSolverConfig, Solver
    data, t0 = [], time.time()
    for sd in seeds:
        sysm = scenes.make_heterogeneous_cube(n=n, seed=int(sd))
        s = Solver(PCGSolverConfig(precision="fp64", stop_rule="relative_residual", global_tol_rate=1e-4))
        pm, rm = sysm.slot_maps(16)
        s.mas_init(sysm.num_verts, sysm.neighbor_start, sysm.neighbor_num, sysm.neighbor_list, pm, rm)
        s.net_configure(level)
        d, st = record_samples(s, sysm, capacity=capacity, every=every, device=device)
        data.append(d)
        s.close()
        log(f"seed {sd}: level {level} nodes {d.graph.nodes}, {d.samples} samples ({st['iterations']} iterations)")
    samples = sum(d.samples for d in data)
    tr = Trainer(init_params(0), device)
    loss0 = float(np.mean([tr.evaluate(d.graph, d.rc[:64].contiguous(), d.zc[:64].contiguous(), min(64, d.samples))
                           for d in data]))
    hist = train(tr, data, steps, batch=batch, lr=lr, lr_final=lr_final, log_every=max(1, steps // 10))
    loss1 = float(np.mean([tr.evaluate(d.graph, d.rc[:64].contiguous(), d.zc[:64].contiguous(), min(64, d.samples))
                           for d in data]))
    log(f"{samples} samples, {steps} steps in {time.time() - t0:.1f} s: loss {loss0:.4f} -> {loss1:.4f}")
    meta = dict(level=level, n=n, seeds=[int(s) for s in seeds], steps=steps, batch=batch, lr=lr, lr_final=lr_final,
                samples=samples, loss_initial=loss0, loss_final=loss1, history=[h[1] for h in hist])
    return tr.params.cpu().numpy(), meta


def solve_hetcube(n: int = 48, seed: int = 1005, precision: str = "fp32", loop: str = "graph", weights=None,
                  plain: bool = True, device="cuda", log=print):
    """One heterogeneous-cube Newton system solved with the shipped network (and, with
    plain=True, without it): iterations, relative residual, solve wall time."""
    import time
    import torch
    from . import scenes
    from .linear_system import PCGSolverConfig, Solver
    params, level, _ = load_weights(weights or default_weights())
    sysm = scenes.make_heterogeneous_cube(n=n, seed=seed)
    dev = torch.device(device)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    rows, cols, blocks, b = t(sysm.rows), t(sysm.cols), t(sysm.blocks.reshape(-1)), t(sysm.b)
    pm, rm = sysm.slot_maps(16)
    out = {}
    for on in ([False] if plain else []) + [True]:
        s = Solver(PCGSolverConfig(precision=precision, stop_rule="relative_residual", global_tol_rate=1e-4, loop=loop,
                                   learned=on))
        s.mas_init(sysm.num_verts, sysm.neighbor_start, sysm.neighbor_num, sysm.neighbor_list, pm, rm)
        s.net_configure(level)
        if on:
            s.net_set_params(t(params))
        x = torch.zeros_like(b)
        s.solve_linear_system(rows, cols, blocks, b, x)
        torch.cuda.synchronize(dev)
        t0 = time.time()
        st = s.solve_linear_system(rows, cols, blocks, b, x)
        torch.cuda.synchronize(dev)
        key = "learned" if on else "plain"
        out[key] = dict(iterations=st["iterations"], rel_residual=st["rel_residual"], ms=(time.time() - t0) * 1e3,
                        accepted=st["learned_accepted"], rejected=st["learned_rejected"])
        log(f"{key}: {out[key]}")
        s.close()
    return out


def _main(argv=None):
    import argparse
    ap = argparse.ArgumentParser(description="train or run the learned coarse correction on heterogeneous cubes")
    ap.add_argument("cmd", choices=["train", "solve"])
    ap.add_argument("--n", type=int, default=48)
    ap.add_argument("--seeds", default="2000-2007", help="train: scene seeds")
    ap.add_argument("--seed", type=int, default=1005, help="solve: scene seed")
    ap.add_argument("--level", type=int, default=2)
    ap.add_argument("--steps", type=int, default=12000)
    ap.add_argument("--precision", default="fp32")
    ap.add_argument("--loop", default="graph")
    ap.add_argument("--learned-only", action="store_true")
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    if a.cmd == "solve":
        solve_hetcube(a.n, a.seed, a.precision, a.loop, plain=not a.learned_only)
        return
    lo, _, hi = a.seeds.partition("-")
    seeds = range(int(lo), int(hi or lo) + 1)
    params, meta = train_hetcube(n=a.n, seeds=seeds, level=a.level, steps=a.steps)
    out = a.out or default_weights(a.level, a.n)
    os.makedirs(os.path.dirname(out), exist_ok=True)
    np.savez(out, params=params, **{k: np.asarray(v) for k, v in meta.items()})
    print("wrote", out)


if __name__ == "__main__":
    _main()
