"""Meshes generated on the device and their parameter derivatives (GPU).

The device generators against the host ones (``mesh_hemisphere``,
``mesh_two_hemispheres``, ``wavebot_mesh``: the same faces, fields within a
few ulps -- the device's sine and cosine may differ from the C library's in
the last bit), their tangents against the host's exact tangents
(``hemisphere_tangents``, ``two_hemispheres_tangents``,
``wavebot_tangents``), the reverse-mode pull-back of the adjoint's mesh
cotangent against the host contraction and against central differences of
the forward batch on regenerated meshes, and the batch on a generated mesh
against the same batch on the host mesh."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _same_mesh(a, b, tol=1e-13):
    assert a.nfaces == b.nfaces and a.nvertices == b.nvertices
    assert np.array_equal(a.faces, b.faces)
    for f in ("vertices", "centers", "normals", "areas", "radii"):
        x, y = getattr(a, f), getattr(b, f)
        assert np.max(np.abs(x - y)) <= tol * max(1.0, np.max(np.abs(y))), f


def _same_tangent(a, b, tol=1e-12):
    for f in ("vertices", "centers", "normals", "areas", "radii"):
        x, y = np.asarray(getattr(a, f)), np.asarray(getattr(b, f))
        assert np.max(np.abs(x - y)) <= tol * max(1.0, np.max(np.abs(y))), f


@pytest.mark.parametrize("radius,center,res", [(1.0, (0.0, 0.0, 0.0), (10, 10)), (1.7, (0.3, -2.0, 0.1), (7, 9)),
                                               (1.0, (0.0, 0.0, 0.0), (64, 64))])
def test_hemisphere_matches_host(mh, gpu, radius, center, res):
    g = mh.generate_hemisphere(radius, center, res, ctx=gpu)
    _same_mesh(g, mh.mesh_hemisphere(radius, center, res))
    host = mh.hemisphere_tangents(radius, center, res)
    dev = mh.generated_tangents(g)
    assert set(dev) == set(host)
    for k in host:
        _same_tangent(dev[k], host[k])


@pytest.mark.parametrize("args", [(0.88, 0.35, 0.16, 0.37, (5, 10, 5), 72), (1.2, 0.5, 0.3, 0.6, (3, 4, 2), 16)])
def test_wavebot_matches_host(mh, gpu, args):
    r1, r2, d1, d2, npts, nth = args
    g = mh.generate_wavebot(r1, r2, d1, d2, npts, nth, ctx=gpu)
    _same_mesh(g, mh.wavebot_mesh(r1, r2, d1, d2, npts, nth))
    host = mh.wavebot_tangents(r1, r2, d1, d2, npts, nth)
    dev = mh.generated_tangents(g)
    for k in host:
        _same_tangent(dev[k], host[k])


def test_two_hemispheres_match_host(mh, gpu):
    g = mh.generate_two_hemispheres(1.3, 4.0, (8, 12), ctx=gpu)
    _same_mesh(g, mh.mesh_two_hemispheres(1.3, 4.0, (8, 12)))
    host = mh.two_hemispheres_tangents(1.3, 4.0, (8, 12))
    dev = mh.generated_tangents(g)
    _same_tangent(dev["radius0"] + dev["radius1"], host["radius"])
    _same_tangent(dev["cx1"], host["separation"])


def test_combined_with_an_uploaded_mesh(mh, gpu):
    up = mh.mesh_hemisphere(1.0, (0.0, 0.0, 0.0), (6, 8))
    g = mh.generate_hemisphere(0.8, (3.0, 0.0, 0.0), (6, 8), ctx=gpu)
    c = mh.generate_combined([up, g], ctx=gpu)
    _same_mesh(c, up + g, tol=0.0)
    dev = mh.generated_tangents(c)
    assert set(dev) == {"radius1", "cx1", "cy1", "cz1"}
    t = dev["radius1"]
    assert not np.any(t.vertices[:up.nvertices]) and not np.any(t.centers[:up.nfaces])
    _same_tangent(mh.MeshTangent(t.vertices[up.nvertices:], t.centers[up.nfaces:], t.normals[up.nfaces:],
                                 t.areas[up.nfaces:], t.radii[up.nfaces:]), mh.generated_tangents(g)["radius"],
                  tol=0.0)


def test_batch_on_generated_mesh_matches_host_mesh(mh, gpu):
    res = (12, 16)
    g = mh.generate_hemisphere(1.0, (0.0, 0.0, 0.0), res, ctx=gpu)
    h = mh.mesh_hemisphere(1.0, (0.0, 0.0, 0.0), res)
    om = [0.7, 1.4]
    kw = dict(precision="fp64", ctx=gpu)
    A1, B1, _, _, _ = mh.hydro_batch(g, om, [mh.translational_dofs(g, "Heave")], **kw)
    A2, B2, _, _, _ = mh.hydro_batch(h, om, [mh.translational_dofs(h, "Heave")], **kw)
    assert np.max(np.abs(A1 - A2)) <= 1e-11 * np.max(np.abs(A2))
    assert np.max(np.abs(B1 - B2)) <= 1e-11 * np.max(np.abs(B2))


def test_param_vjp_matches_contraction_and_differences(mh, gpu):
    """dB33/dR and dA33/dR of a generated hemisphere: the adjoint's mesh
    cotangent pulled back on the device equals its host contraction with the
    device tangents, and central differences (h = 1e-5) of the forward batch
    on regenerated meshes."""
    res, R, om = (10, 12), 1.1, [0.9]
    g = mh.generate_hemisphere(R, (0.0, 0.0, 0.0), res, ctx=gpu)
    dof = [mh.translational_dofs(g, "Heave")]
    r = mh.hydro_batch_vjp(g, om, dof, bar_damping=np.ones((1, 1, 1)), precision="fp64", ctx=gpu)
    grad = mh.generated_param_grad(g, r.mesh)
    tang = mh.generated_tangents(g)
    for k in tang:
        assert abs(grad[k] - r.mesh.dot(tang[k])) <= 1e-12 * max(1.0, abs(grad[k]))

    def b33(rad):
        m = mh.generate_hemisphere(rad, (0.0, 0.0, 0.0), res, ctx=gpu)
        _, B, _, _, _ = mh.hydro_batch(m, om, [mh.translational_dofs(m, "Heave")], precision="fp64", ctx=gpu)
        return float(B[0, 0, 0])

    h = 1e-5
    fd = (b33(R + h) - b33(R - h)) / (2 * h)
    assert abs(grad["radius"] - fd) <= 1e-5 * max(abs(fd), 1e-3)


def test_generator_arguments_are_checked(mh, gpu):
    with pytest.raises(mh.ArgumentError):
        mh.generate_hemisphere(-1.0, (0.0, 0.0, 0.0), (10, 10), ctx=gpu)
    with pytest.raises(mh.ArgumentError):
        mh.generate_hemisphere(1.0, (0.0, 0.0, 0.0), (1, 10), ctx=gpu)
    with pytest.raises(mh.ArgumentError):
        mh.generate_wavebot(0.88, 0.0, 0.16, 0.37, ctx=gpu)
    with pytest.raises(ValueError):
        mh.generated_tangents(mh.mesh_hemisphere(1.0, (0.0, 0.0, 0.0), (4, 4)))
