"""GPU: implicit-Euler steps with surface contact between two soft cubes, the upper one
coming down at 3 m/s onto the resting lower one (5 cm per step against a 5 mm gap and a 1 mm
barrier zone, so the first Newton steps see no contact and only the CCD stops the cube):
contact barrier triplets in every Newton system, the additive CCD bounding every line search.

Bars: every step converges; after every step every contact pair is apart and no surface
vertex sits on the wrong side of the other cube's facing surface (a signed test, so a vertex
that tunnelled through would fail it); the CCD bound was active (< 1) when the cubes met;
the FP32-storage and FP64 solves give the same trajectory within 5x the Newton tolerance (the
reference's rule: largest step entry below 1e-2 x bbox diagonal x dt, about 2e-4 m here).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _signed_ok(pos, tris, body):
    """Every vertex of either cube lies on its own side of the facing surface of the other:
    for vertices within 5 mm of a triangle of the other body, whose projection falls inside
    it, the signed distance along the triangle's upward normal is positive for the upper cube's
    vertices over the lower cube's top, negative for the lower cube's vertices under the upper
    cube's bottom."""
    from stgipc import scenes
    p, _ = scenes.contact_pairs(pos, tris, body, (5e-3) ** 2, return_d2=True)
    pt = p[(p[:, 0] < 0) & (p[:, 2] >= 0) & (p[:, 3] >= 0)]
    n_checked = 0
    for q in pt:
        v = -q[0] - 1
        t0, t1, t2 = pos[q[1]], pos[q[2]], pos[q[3]]
        n = np.cross(t1 - t0, t2 - t0)
        if abs(n[1]) < 0.9 * np.linalg.norm(n):
            continue  # a side face: not between the cubes
        n = n * np.sign(n[1])
        s = np.dot(pos[v] - t0, n)
        want = 1.0 if body[v] == 1 else -1.0
        assert s * want > 0, (v, s)
        n_checked += 1
    return n_checked


@pytest.mark.parametrize("steps", [6])
def test_stacked_cubes_fall_without_interpenetration(dev, steps):
    from stgipc import PCGSolverConfig, newton, scenes
    # kappa sized to carry the cubes (about 1.2 kN over some 50 pairs, 2.5 kN on the ground): the
    # barrier force of one pair at half the activation distance is about 9e-9 kappa N at
    # dhat = 1e-6; the ground plane gets the same stiffness
    state, tris, body = scenes.make_stacked_cubes(6, kappa=1e10, gap=5e-3, v0=0.0, v_top=-3.0, state_only=True)
    contact = newton.ContactModel(tris=tris, body=body, dhat=1e-6, kappa=1e10)
    # the reference's Newton stop: the largest step entry below 1e-2 x bbox diagonal x dt
    # (GIPC.cu:11082, Newton_solver_threshold = 1e-2 at gl_main.cu:669).  With the rank-one
    # (Gauss-Newton) barrier Hessian the iteration converges linearly along the cubes' sliding
    # mode, so a much tighter stop only adds iterations.
    diag = float(np.linalg.norm(state["pos"].max(axis=0) - state["pos"].min(axis=0)))
    tol = 1e-2 * diag
    runs = {}
    for prec in ("fp64", "fp32"):
        cfg = PCGSolverConfig(precision=prec, stop_rule="relative_residual", global_tol_rate=1e-6,
                              refine_interval=8)
        pos, stats = newton.trajectory(state, steps, config=cfg, contact=contact, device=dev, tol=tol)
        runs[prec] = (pos, stats)
        for k, (p, st) in enumerate(zip(pos, stats)):
            assert st.newton_iterations < 30, (prec, k, st)
            assert np.all(np.isfinite(p))
            assert st.min_contact_distance > 0, (prec, k, st)
            assert st.min_plane_distance > 0
            _signed_ok(p, tris, body)
        assert min(st.ccd_alpha for st in stats) < 1.0
        assert max(st.contacts for st in stats) > 50
        assert _signed_ok(pos[-1], tris, body) > 20
    # the two runs stop their Newton loops within tol x dt (2e-4 m) of the same optimum
    d = max(np.abs(a - b).max() for a, b in zip(runs["fp64"][0], runs["fp32"][0]))
    assert d <= 5 * tol * state["dt"], d
