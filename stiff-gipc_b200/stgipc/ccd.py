"""The line search's step bound from continuous collision detection on the GPU
(stg_ccd_step_size): the reference's additive CCD over point-triangle and edge-edge pairs
(ACCD.cu, GIPC::self_largestFeasibleStepSize)."""
from __future__ import annotations

from . import _lib as _L
from ._lib import check


def step_size(pairs, x, dx, slackness=0.8, thickness=0.0, per_pair=False, stream=None):
    """alpha (a device scalar tensor), and the per-pair times of impact if per_pair.
    pairs: CUDA int32 [P, 4] (point-triangle (-p-1, t0, t1, t2), edge-edge (a0, a1, b0, b1));
    x, dx: CUDA float64 [V, 3] positions and displacement."""
    import torch
    if pairs.dtype != torch.int32 or x.dtype != torch.float64 or dx.dtype != torch.float64:
        raise ValueError("pairs must be int32, x and dx float64 CUDA tensors")
    pairs, x, dx = pairs.contiguous().view(-1, 4), x.contiguous(), dx.contiguous()
    dev = x.device
    alpha = torch.empty(1, dtype=torch.float64, device=dev)
    scratch = torch.empty(1, dtype=torch.int64, device=dev)
    toc = torch.empty(pairs.shape[0], dtype=torch.float64, device=dev) if per_pair else None
    bad = torch.zeros(1, dtype=torch.int32, device=dev)
    s = None if stream is None else stream.cuda_stream
    check(_L.lib().stg_ccd_step_size(pairs.shape[0], pairs.data_ptr(), x.data_ptr(), dx.data_ptr(), x.numel() // 3,
                                     float(slackness), float(thickness), alpha.data_ptr(),
                                     None if toc is None else toc.data_ptr(), bad.data_ptr(), scratch.data_ptr(), s),
          "stg_ccd_step_size")
    if int(bad.item()):
        raise ValueError(f"stg_ccd_step_size: {int(bad.item())} pairs with a vertex out of range")
    return (alpha, toc) if per_pair else alpha
