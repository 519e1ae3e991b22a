"""Forward-mode derivatives (mh_hydro_batch_jvp), the counterpart of the
reference's ForwardDiff path (test/outputs_differentiation.jl:133-151) (GPU).

* dot-product identity with the reverse mode: for a random input direction
  t and output cotangent c, <c, JVP(t)> = <VJP(c), t> (both exact
  derivatives of the same discrete function): 1e-10 relative;
* central differences of the FP64 forward along t, h = 1e-6: 1e-6;
* mixed vs FP64 tangents: 1e-8; frequency-batched vs one frequency per
  call: 1e-9.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WU = (1 | 2 | 8)
DELH = (1 | 2 | 16)


def _gfs(mh, mask):
    t = []
    if mask & 1:
        t.append(mh.Rankine())
    if mask & 2:
        t.append(mh.RankineReflected())
    if mask & 4:
        t.append(mh.RankineReflectedNegative())
    if mask & 8:
        t.append(mh.GFWu())
    if mask & 16:
        t.append(mh.ExactGuevelDelhommeau())
    return tuple(t)


def _direction(mh, mesh, nw, nd, seed=7):
    rng = np.random.default_rng(seed)
    t = mh.MeshTangent(rng.uniform(-1, 1, mesh.vertices.shape), rng.uniform(-1, 1, mesh.centers.shape),
                       rng.uniform(-1, 1, mesh.normals.shape), rng.uniform(-1, 1, mesh.areas.shape) * mesh.areas,
                       np.zeros_like(mesh.radii))
    tw = rng.uniform(-1, 1, nw)
    td = [rng.uniform(-1, 1, (mesh.nfaces, 3)) for _ in range(nd)]
    return t, tw, td


def _perturb(mh, mesh, t, h):
    return mh.Mesh(mesh.vertices + h * t.vertices, mesh.faces, mesh.centers + h * t.centers,
                   mesh.normals + h * t.normals, mesh.areas + h * t.areas, mesh.radii)


@pytest.fixture(scope="module")
def setup(mh):
    mesh = mh.mesh_hemisphere(1.0, (0, 0, -0.05), (8, 10))
    body = mh.FloatingBody.rigid(mesh, ["Heave", "Surge"])
    return mesh, list(body.dofs.values()), np.array([0.7, 1.4]), [0.3]


def _inner(c, r):
    cA, cB, cF, cK = c
    return float(np.sum(cA * r.d_added_mass) + np.sum(cB * r.d_damping)
                 + np.real(np.sum(np.conj(cF) * r.d_diffraction)) + np.real(np.sum(np.conj(cK) * r.d_froude_krylov)))


@pytest.mark.parametrize("mask", [WU, DELH, 1 | 4 | 8])
@pytest.mark.parametrize("direct", [True, False])
def test_jvp_vjp_dot_product(mh, gpu, setup, mask, direct):
    mesh, dofs, om, betas = setup
    nd, nw, nb = len(dofs), len(om), len(betas)
    t, tw, td = _direction(mh, mesh, nw, nd)
    rng = np.random.default_rng(3)
    c = (rng.normal(size=(nd, nd, nw)), rng.normal(size=(nd, nd, nw)),
         rng.normal(size=(nd, nw, nb)) + 1j * rng.normal(size=(nd, nw, nb)),
         rng.normal(size=(nd, nw, nb)) + 1j * rng.normal(size=(nd, nw, nb)))
    kw = dict(green_functions=_gfs(mh, mask), direct=direct, precision="fp64", ctx=gpu)
    j = mh.hydro_batch_jvp(mesh, om, dofs, betas, t, tw, td, **kw)
    v = mh.hydro_batch_vjp(mesh, om, dofs, betas, *c, **kw)
    lhs = _inner(c, j)
    rhs = v.mesh.dot(t) + float(np.sum(v.omegas * tw)) + sum(float(np.sum(a * b)) for a, b in zip(v.dofs, td))
    assert abs(lhs - rhs) <= 1e-10 * max(abs(lhs), abs(rhs)), (lhs, rhs)


@pytest.mark.parametrize("mask", [WU, DELH])
@pytest.mark.parametrize("direct", [True, False])
def test_jvp_matches_finite_differences(mh, gpu, setup, mask, direct):
    mesh, dofs, om, betas = setup
    t, tw, td = _direction(mh, mesh, len(om), len(dofs), seed=11)
    kw = dict(green_functions=_gfs(mh, mask), direct=direct, precision="fp64", ctx=gpu)
    j = mh.hydro_batch_jvp(mesh, om, dofs, betas, t, tw, td, **kw)
    h = 1e-6
    p = mh.hydro_batch(_perturb(mh, mesh, t, h), om + h * tw, [d + h * e for d, e in zip(dofs, td)], betas, **kw)
    m = mh.hydro_batch(_perturb(mh, mesh, t, -h), om - h * tw, [d - h * e for d, e in zip(dofs, td)], betas, **kw)
    for got, a, b in ((j.d_added_mass, p[0], m[0]), (j.d_damping, p[1], m[1]),
                      (j.d_diffraction, p[2], m[2]), (j.d_froude_krylov, p[3], m[3])):
        fd = (a - b) / (2 * h)
        assert np.max(np.abs(got - fd)) <= 1e-6 * np.max(np.abs(fd)), np.max(np.abs(got - fd)) / np.max(np.abs(fd))


@pytest.mark.parametrize("direct", [True, False])
def test_jvp_mixed_and_batched(mh, gpu, direct, series_fp64):
    """Mixed (frequency-batched Delhommeau tangent for >= 4 frequencies) vs
    FP64 one frequency per call."""
    mesh = mh.mesh_hemisphere(1.3, (0, 0, 0), (10, 14))
    body = mh.FloatingBody.rigid(mesh, ["Heave", "Surge"])
    dofs = list(body.dofs.values())
    om = np.linspace(0.3, 4.0, 7)
    tan = mh.hemisphere_tangents(1.3, (0, 0, 0), (10, 14))["radius"]
    tw = np.linspace(0.1, 0.2, 7)
    kw = dict(green_functions=_gfs(mh, DELH), direct=direct, ctx=gpu)
    b = mh.hydro_batch_jvp(mesh, om, dofs, [0.2], tan, tw, None, precision="mixed", tol=1e-13, **kw)
    for z in range(len(om)):
        s = mh.hydro_batch_jvp(mesh, om[z:z + 1], dofs, [0.2], tan, tw[z:z + 1], None, precision="fp64", **kw)
        for x, y in ((b.d_added_mass[:, :, z], s.d_added_mass[:, :, 0]), (b.d_damping[:, :, z], s.d_damping[:, :, 0]),
                     (b.d_diffraction[:, z], s.d_diffraction[:, 0])):
            assert np.max(np.abs(x - y)) <= 1e-8 * np.max(np.abs(y)), z
