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
