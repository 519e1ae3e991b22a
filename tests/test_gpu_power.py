"""Gradient of the two-body mechanical power (paper/Power.jl:13-83) with
respect to the sphere radius r1, the gap dx1 and the frequency, against
central finite differences with h = 1e-6 (the reference's check of the same
objective, paper/meshGradients_pair.jl:38-39, uses finite differences too)
(GPU).  Two hemispheres, heave on both, Rankine + reflected Rankine + Wu;
direct and indirect formulations; FP64 and mixed precision."""
from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu

RES = (8, 12)


@pytest.mark.parametrize("direct", [True, False])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_power_gradient_matches_finite_differences(mh, gpu, direct, precision):
    r1, dx1, w = 1.0, 4.0, 1.03
    J, g = mh.two_body_power(r1, dx1, w, resolution=RES, direct=direct, precision=precision,
                             tol=1e-13, grad=True, ctx=gpu)
    J64 = mh.two_body_power(r1, dx1, w, resolution=RES, direct=direct, precision="fp64", ctx=gpu)
    assert abs(J - J64) <= 1e-9 * abs(J64)
    h = 1e-6
    f = lambda a, b, c: mh.two_body_power(a, b, c, resolution=RES, direct=direct, precision="fp64", ctx=gpu)
    fd = {"r1": (f(r1 + h, dx1, w) - f(r1 - h, dx1, w)) / (2 * h),
          "dx1": (f(r1, dx1 + h, w) - f(r1, dx1 - h, w)) / (2 * h),
          "omega": (f(r1, dx1, w + h) - f(r1, dx1, w - h)) / (2 * h)}
    for k in ("r1", "dx1", "omega"):
        assert abs(g[k] - fd[k]) <= 1e-5 * max(abs(fd[k]), 1e-3 * abs(J)), (k, g[k], fd[k])


def test_power_direct_and_indirect_agree(mh, gpu):
    a = mh.two_body_power(1.0, 4.0, 1.03, resolution=RES, direct=True, precision="fp64", ctx=gpu)
    b = mh.two_body_power(1.0, 4.0, 1.03, resolution=RES, direct=False, precision="fp64", ctx=gpu)
    assert abs(a - b) <= 0.05 * abs(a)


def test_power_optimisation_in_a_box(mh, gpu):
    """The design loop of paper/optimization.jl (start (2, 3), bounds [1, 4]^2,
    gradient tolerance 1e-3) on a coarse mesh: the accepted iterates raise
    the power monotonically, stay in the box, and end where the projected
    gradient vanishes (each coordinate interior with dJ/dx ~ 0, or on a bound
    with dJ/dx pointing out of the box)."""
    lo, hi = (1.0, 1.0), (4.0, 4.0)
    out = mh.optimize_two_body_power(2.0, 3.0, lo, hi, resolution=RES, precision="mixed", tol=1e-12,
                                     iterations=40, ctx=gpu)
    pw = [h[2] for h in out["history"]]
    assert all(b >= a - 1e-12 * abs(a) for a, b in zip(pw, pw[1:])), pw
    assert out["power"] >= pw[0] and out["evaluations"] >= 2
    x = out["x"]
    assert all(l <= v <= u for v, l, u in zip(x, lo, hi))
    _, g0 = mh.two_body_power(2.0, 3.0, 1.03, resolution=RES, precision="mixed", tol=1e-12, grad=True, ctx=gpu)
    _, g = mh.two_body_power(x[0], x[1], 1.03, resolution=RES, precision="mixed", tol=1e-12, grad=True, ctx=gpu)
    scale = max(abs(g0["r1"]), abs(g0["dx1"]))
    for v, l, u, d in zip(x, lo, hi, (g["r1"], g["dx1"])):
        viol = max(d, 0.0) if v <= l else (max(-d, 0.0) if v >= u else abs(d))
        assert viol <= 1e-3 + 1e-2 * scale, (x, g, out["message"])
