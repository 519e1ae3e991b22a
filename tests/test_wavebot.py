"""WaveBot meshes (src/meshes.jl:247-479): the profile, the revolved
connectivity, the polygon-mesh geometry conventions and the exact tangents
with respect to (r1, r2, d1, d2).  Host only; the GPU gradient through these
tangents is in test_gpu_wavebot.py."""
import math

import numpy as np
import pytest


def test_profile_points(mh):
    p = mh.wavebot_profile(0.16, 0.37, 0.88, 0.35, (5, 10, 5))
    assert p.shape == (5 + 9 + 4, 2)
    assert np.allclose(p[0], (0.88, 0.0)) and np.allclose(p[4], (0.88, -0.16))
    assert np.allclose(p[13], (0.35, -0.53)) and np.allclose(p[-1], (0.0, -0.53))
    # the frustum narrows linearly from the top to the bottom radius
    assert np.allclose(np.diff(p[4:14, 0]), (0.35 - 0.88) / 9)


def test_default_mesh_structure(mh):
    m = mh.wavebot_mesh(0.88, 0.35, 0.16, 0.37)
    assert (m.nfaces, m.nvertices) == (17 * 72, 17 * 72 + 1)
    tri = m.faces[:, 2] == m.faces[:, 3]
    assert tri.sum() == 72 and np.all(tri[-72:])          # the bottom ring, apex second
    assert np.all(m.faces[-72:, 1] == m.nvertices - 1)
    # quads (upper i, lower i, lower i + 1, upper i + 1)
    assert tuple(m.faces[0]) == (0, 72, 73, 1) and tuple(m.faces[71]) == (71, 143, 72, 0)
    # outward normals: radial on the cylinder, down on the bottom
    th = 2 * math.pi * (np.arange(72) + 0.5) / 72
    assert np.allclose(m.normals[:72], np.stack([np.cos(th), np.sin(th), 0 * th], 1), atol=1e-12)
    assert np.allclose(m.normals[-72:], (0.0, 0.0, -1.0))
    # radius: distance from the centre to the first vertex
    assert np.allclose(m.radii, np.linalg.norm(m.vertices[m.faces[:, 0]] - m.centers, axis=1))


def test_polygon_areas_match_trapezoids(mh):
    """Every revolved band is n_theta planar isosceles trapezoids with parallel
    sides 2 r sin(pi/n) and height sqrt(((r1 - r2) cos(pi/n))^2 + dz^2)."""
    n = 40
    m = mh.wavebot_mesh(1.1, 0.5, 0.3, 0.6, (4, 6, 3), n)
    prof = mh.wavebot_profile(0.3, 0.6, 1.1, 0.5, (4, 6, 3))
    s, c = math.sin(math.pi / n), math.cos(math.pi / n)
    total = 0.0
    for (ra, za), (rb, zb) in zip(prof[:-1], prof[1:]):
        h = math.hypot((ra - rb) * c, za - zb)
        total += n * (ra + rb) * s * h
    assert abs(m.areas.sum() - total) <= 1e-13 * total
    # centres on the bands, inside the hull in z
    assert np.all(m.centers[:, 2] <= 0.0) and np.all(m.centers[:, 2] >= -0.9 - 1e-12)


def test_argument_checks(mh):
    with pytest.raises(ValueError):
        mh.axisymmetric_mesh([(1.0, 0.0), (0.5, -1.0)], 2)
    with pytest.raises(ValueError):
        mh.axisymmetric_mesh([(0.0, 0.0), (0.0, -1.0)], 8)
    with pytest.raises(ValueError):
        mh.axisymmetric_mesh([(-1.0, 0.0), (0.5, -1.0)], 8)
    with pytest.raises(ValueError):
        mh.wavebot_profile(0.1, 0.2, 1.0, 0.5, (1, 4, 4))


@pytest.mark.parametrize("name", ["r1", "r2", "d1", "d2"])
def test_tangents_match_central_differences(mh, name):
    p = dict(r1=0.88, r2=0.35, d1=0.16, d2=0.37)
    kw = dict(n_points=(4, 5, 3), n_theta=16)
    t = mh.wavebot_tangents(**p, **kw)[name]
    h = 1e-6
    hi = mh.wavebot_mesh(**{**p, name: p[name] + h}, **kw)
    lo = mh.wavebot_mesh(**{**p, name: p[name] - h}, **kw)
    for f in ("vertices", "centers", "normals", "areas", "radii"):
        fd = (getattr(hi, f) - getattr(lo, f)) / (2 * h)
        ex = getattr(t, f)
        assert np.max(np.abs(fd - ex)) <= 1e-7 * max(1.0, np.max(np.abs(ex))), (name, f)
