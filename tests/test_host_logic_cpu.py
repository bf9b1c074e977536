"""CPU: host logic of the Newton driver (vertex-plane step bound) and of the learned
correction (parameter layout, the shipped weights file)."""
import types

import numpy as np
import torch


def _scene(planes):
    pl = torch.tensor(planes, dtype=torch.float64).reshape(-1, 6)
    return types.SimpleNamespace(planes=pl, nplanes=pl.shape[0])


def test_plane_step_bound():
    from stgipc import newton
    sc = _scene([[0.0, 1.0, 0.0, 0.0, 1e-3, 1e5]])
    x = torch.tensor([[0.0, 1e-3, 0.0], [0.0, 0.5, 0.0]], dtype=torch.float64)
    # vertex 0 approaches at 1e-2 per unit step: impact at alpha = 0.1, bound 0.8 of it
    p = torch.tensor([[0.0, -1e-2, 0.0], [0.0, 1.0, 0.0]], dtype=torch.float64)
    assert abs(newton.plane_step_bound(sc, x, p) - 0.08) < 1e-12
    # moving away from every plane: the full step
    away = torch.tensor([[0.0, 1e-2, 0.0], [0.0, 1.0, 0.0]], dtype=torch.float64)
    assert newton.plane_step_bound(sc, x, away) == 1.0
    # the reversed direction brings vertex 1 down from 0.5 at rate 1: impact at 0.5
    assert abs(newton.plane_step_bound(sc, x, -p) - 0.4) < 1e-12
    # two planes: the nearer impact wins
    sc2 = _scene([[0.0, 1.0, 0.0, 0.0, 1e-3, 1e5], [0.0, -1.0, 0.0, -0.6, 1e-3, 1e5]])
    p2 = torch.tensor([[0.0, 0.0, 0.0], [0.0, 0.2, 0.0]], dtype=torch.float64)
    assert abs(newton.plane_step_bound(sc2, x, p2) - 0.8 * 0.5) < 1e-12
    assert abs(newton.min_plane_distance(sc2, x) - 1e-3) < 1e-15


def test_parameter_layout_matches_header():
    from oracle import net_oracle as no
    from stgipc import _lib, learned
    assert learned.NET_PARAMS == _lib.NET_PARAMS == no.COUNT == 26376
    for k, (o, shp) in no.P.items():
        assert learned.OFF[k] == o
    txt = open(_lib.HEADER).read()
    assert "#define STG_NET_PARAMS 26376" in txt
    p = learned.init_params(0)
    assert p.dtype == np.float32 and p.shape == (26376,)
    assert np.all(p[learned.OFF["b0"]:learned.OFF["W1"]] == 0)


def test_shipped_weights_file():
    from stgipc import learned
    params, level, meta = learned.load_weights(learned.default_weights())
    assert params.shape == (learned.NET_PARAMS,) and np.isfinite(params).all()
    assert level == 2 and 1005 not in meta["seeds"] and meta["samples"] >= 2000
    assert meta["loss_final"] < meta["loss_initial"] - 0.3
