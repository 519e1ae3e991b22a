"""Adjoint gradients (mh_hydro_batch_vjp) against central finite differences
of the forward batch, as the reference checks its Zygote gradients
(test/outputs_differentiation.jl:59-68: dA/domega vs finite differences with
h = 1e-6; :21-35: cotangents of the mesh fields) (GPU).

Objective: J = sum(wA A) + sum(wB B) + Re sum(conj(wF) Fd) + Re sum(conj(wK) Fk)
with seeded weights.  Directional derivatives along random perturbations of
each mesh field (vertices, centres, normals, areas), of the frequencies, and
of the generator parameters (radius, separation) are compared with central
differences of the FP64 forward path, h = 1e-6 relative: agreement to 1e-6
relative to the largest term of the objective's sensitivity.  The mixed path's
gradients must agree with the FP64 path's to 1e-8.
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


def _weights(nd, nw, nb, seed=3):
    rng = np.random.default_rng(seed)
    wA = rng.normal(size=(nd, nd, nw))
    wB = rng.normal(size=(nd, nd, nw))
    wF = rng.normal(size=(nd, nw, nb)) + 1j * rng.normal(size=(nd, nw, nb))
    wK = rng.normal(size=(nd, nw, nb)) + 1j * rng.normal(size=(nd, nw, nb))
    return wA, wB, wF, wK


def _J(mh, gpu, mesh, om, dofs, betas, w, mask, direct):
    A, B, Fd, Fk, _ = mh.hydro_batch(mesh, om, dofs, betas, green_functions=_gfs(mh, mask),
                                     direct=direct, precision="fp64", ctx=gpu)
    wA, wB, wF, wK = w
    return float(np.sum(wA * A) + np.sum(wB * B) + np.real(np.sum(np.conj(wF) * Fd))
                 + np.real(np.sum(np.conj(wK) * Fk)))


def _vjp(mh, gpu, mesh, om, dofs, betas, w, mask, direct, precision="fp64"):
    wA, wB, wF, wK = w
    return mh.hydro_batch_vjp(mesh, om, dofs, betas, wA, wB, wF, wK,
                              green_functions=_gfs(mh, mask), direct=direct,
                              precision=precision, tol=1e-13, ctx=gpu)


def _perturbed(mh, mesh, field, delta, h):
    f = dict(vertices=mesh.vertices, faces=mesh.faces, centers=mesh.centers,
             normals=mesh.normals, areas=mesh.areas, radii=mesh.radii)
    f[field] = f[field] + h * delta
    return mh.Mesh(**f)


def _close(a, b, scale, tol):
    assert abs(a - b) <= tol * scale, (a, b, abs(a - b) / scale)


@pytest.fixture(scope="module")
def setup(mh):
    mesh = mh.mesh_hemisphere(1.0, (0, 0, -0.05), (8, 10))
    body = mh.FloatingBody.rigid(mesh, ["Heave", "Surge"])
    dofs = list(body.dofs.values())
    om = np.array([0.7, 1.4])
    betas = [0.3]
    w = _weights(len(dofs), len(om), len(betas))
    return mesh, dofs, om, betas, w


@pytest.mark.parametrize("mask", [WU, DELH, 1 | 4 | 8])
@pytest.mark.parametrize("direct", [True, False])
def test_vjp_mesh_fields_match_finite_differences(mh, gpu, setup, mask, direct):
    mesh, dofs, om, betas, w = setup
    r = _vjp(mh, gpu, mesh, om, dofs, betas, w, mask, direct)
    rng = np.random.default_rng(11)
    h = 1e-6
    grads = dict(vertices=r.mesh.vertices, centers=r.mesh.centers, normals=r.mesh.normals,
                 areas=r.mesh.areas)
    scale = max(float(np.abs(g).sum()) for g in grads.values())
    for field, g in grads.items():
        delta = rng.uniform(-1.0, 1.0, size=g.shape)
        if field == "areas":
            delta = delta * mesh.areas
        jp = _J(mh, gpu, _perturbed(mh, mesh, field, delta, h), om, dofs, betas, w, mask, direct)
        jm = _J(mh, gpu, _perturbed(mh, mesh, field, delta, -h), om, dofs, betas, w, mask, direct)
        fd = (jp - jm) / (2 * h)
        _close(float(np.sum(g * delta)), fd, scale, 1e-6)
    assert np.all(r.mesh.radii == 0.0)


@pytest.mark.parametrize("mask", [WU, DELH])
@pytest.mark.parametrize("direct", [True, False])
def test_vjp_omega_matches_finite_differences(mh, gpu, setup, mask, direct):
    mesh, dofs, om, betas, w = setup
    r = _vjp(mh, gpu, mesh, om, dofs, betas, w, mask, direct)
    h = 1e-6
    for z in range(len(om)):
        e = np.zeros_like(om)
        e[z] = h
        fd = (_J(mh, gpu, mesh, om + e, dofs, betas, w, mask, direct)
              - _J(mh, gpu, mesh, om - e, dofs, betas, w, mask, direct)) / (2 * h)
        _close(r.omegas[z], fd, np.abs(r.omegas).max(), 1e-6)


def test_vjp_dofs_match_finite_differences(mh, gpu, setup):
    mesh, dofs, om, betas, w = setup
    r = _vjp(mh, gpu, mesh, om, dofs, betas, w, WU, True)
    rng = np.random.default_rng(5)
    h = 1e-6
    scale = sum(float(np.abs(d).sum()) for d in r.dofs)
    for q in range(len(dofs)):
        delta = rng.uniform(-1, 1, size=dofs[q].shape)
        dp = [d.copy() for d in dofs]
        dm = [d.copy() for d in dofs]
        dp[q] = dp[q] + h * delta
        dm[q] = dm[q] - h * delta
        fd = (_J(mh, gpu, mesh, om, dp, betas, w, WU, True)
              - _J(mh, gpu, mesh, om, dm, betas, w, WU, True)) / (2 * h)
        _close(float(np.sum(r.dofs[q] * delta)), fd, scale, 1e-6)


@pytest.mark.parametrize("mask", [WU, DELH])
@pytest.mark.parametrize("direct", [True, False])
def test_vjp_mixed_matches_fp64(mh, gpu, setup, mask, direct):
    mesh, dofs, om, betas, w = setup
    a = _vjp(mh, gpu, mesh, om, dofs, betas, w, mask, direct, "fp64")
    b = _vjp(mh, gpu, mesh, om, dofs, betas, w, mask, direct, "mixed")
    for x, y in ((a.mesh.vertices, b.mesh.vertices), (a.mesh.centers, b.mesh.centers),
                 (a.mesh.normals, b.mesh.normals), (a.mesh.areas, b.mesh.areas),
                 (a.omegas, b.omegas)):
        assert np.max(np.abs(x - y)) <= 1e-8 * np.max(np.abs(x))
    assert np.max(np.abs(a.added_mass - b.added_mass)) <= 1e-9 * np.max(np.abs(a.added_mass))


def test_vjp_radius_and_separation(mh, gpu):
    """Two hemispheres, heave on both, Wu, indirect (the two-body design
    study): dJ/dR and dJ/dd through the exact mesh tangents vs central
    differences of the regenerated meshes."""
    R, d, res = 1.0, 5.0, (6, 8)
    mesh = mh.mesh_two_hemispheres(R, d, res)
    b1 = mh.FloatingBody.rigid(mh.mesh_hemisphere(R, (0, 0, 0), res), ["Heave"])
    b2 = mh.FloatingBody.rigid(mh.mesh_hemisphere(R, (d, 0, 0), res), ["Heave"])
    both = b1 + b2
    dofs = list(both.dofs.values())
    om = np.array([1.03])
    w = _weights(2, 1, 0, seed=9)
    r = _vjp(mh, gpu, mesh, om, dofs, (), w, WU, False, "mixed")
    tan = mh.two_hemispheres_tangents(R, d, res)
    h = 1e-6
    for name in ("radius", "separation"):
        g = r.mesh.dot(tan[name])
        Rp, dp = (R + h, d) if name == "radius" else (R, d + h)
        Rm, dm_ = (R - h, d) if name == "radius" else (R, d - h)
        jp = _J(mh, gpu, mh.mesh_two_hemispheres(Rp, dp, res), om, dofs, (), w, WU, False)
        jm = _J(mh, gpu, mh.mesh_two_hemispheres(Rm, dm_, res), om, dofs, (), w, WU, False)
        fd = (jp - jm) / (2 * h)
        _close(g, fd, max(abs(fd), abs(g)), 1e-5)


def test_vjp_exact_delhommeau(mh, gpu):
    """Quadrature path: second derivatives from dG/dr, dG/dz = G + 2/R and
    the harmonic identity."""
    mesh = mh.mesh_hemisphere(1.0, (0, 0, -0.1), (6, 8))
    dofs = [mh.translational_dofs(mesh, "Heave")]
    om = np.array([1.1])
    w = _weights(1, 1, 0, seed=2)
    gpu.set_delhommeau_method("exact")
    try:
        r = _vjp(mh, gpu, mesh, om, dofs, (), w, DELH, True)
        h = 1e-6
        rng = np.random.default_rng(1)
        delta = rng.uniform(-1, 1, size=mesh.centers.shape)
        fd = (_J(mh, gpu, _perturbed(mh, mesh, "centers", delta, h), om, dofs, (), w, DELH, True)
              - _J(mh, gpu, _perturbed(mh, mesh, "centers", delta, -h), om, dofs, (), w, DELH, True)) / (2 * h)
        _close(float(np.sum(r.mesh.centers * delta)), fd, float(np.abs(r.mesh.centers).sum()), 1e-6)
        e = 1e-6
        fdw = (_J(mh, gpu, mesh, om + e, dofs, (), w, DELH, True)
               - _J(mh, gpu, mesh, om - e, dofs, (), w, DELH, True)) / (2 * e)
        _close(r.omegas[0], fdw, abs(r.omegas[0]), 1e-6)
    finally:
        gpu.set_delhommeau_method("table")


def test_rrule_pullback(mh, gpu, setup):
    mesh, dofs, om, betas, w = setup
    (A, B, Fd, Fk), pb = mh.hydro_batch_rrule(mesh, om, dofs, betas, precision="fp64", ctx=gpu)
    wA, wB, wF, wK = w
    mt, wbar, dbar = pb(wA, wB, wF, wK)
    r = _vjp(mh, gpu, mesh, om, dofs, betas, w, WU, True)
    assert np.allclose(mt.centers, r.mesh.centers, rtol=1e-12, atol=0)
    assert np.allclose(wbar, r.omegas, rtol=1e-12, atol=0)
    assert np.allclose(A, r.added_mass, rtol=1e-12, atol=0)


@pytest.mark.parametrize("direct", [True, False])
def test_vjp_frequency_batched_delhommeau(mh, gpu, direct, series_fp64):
    """Chunks of >= 4 frequencies take the frequency-batched Delhommeau
    adjoint (alpha contraction once per pair); over [0.3, 4.0] rad/s pairs
    leave the polar patch, so the per-point path runs too.  Checked against
    the per-frequency path (one frequency per call) and, for omega, against
    central differences."""
    mesh = mh.mesh_hemisphere(1.3, (0, 0, 0), (10, 14))
    body = mh.FloatingBody.rigid(mesh, ["Heave", "Surge"])
    dofs = list(body.dofs.values())
    om = np.linspace(0.3, 4.0, 7)
    w = _weights(2, len(om), 1, seed=4)
    batched = _vjp(mh, gpu, mesh, om, dofs, [0.2], w, DELH, direct, "mixed")
    wA, wB, wF, wK = w
    acc = None
    for z in range(len(om)):
        r = mh.hydro_batch_vjp(mesh, om[z:z + 1], dofs, [0.2], wA[:, :, z:z + 1], wB[:, :, z:z + 1],
                               wF[:, z:z + 1], wK[:, z:z + 1], green_functions=_gfs(mh, DELH),
                               direct=direct, precision="fp64", ctx=gpu)
        acc = r.mesh if acc is None else acc + r.mesh
        assert abs(r.omegas[0] - batched.omegas[z]) <= 1e-8 * np.max(np.abs(batched.omegas))
    for f in ("vertices", "centers", "normals", "areas"):
        x, y = getattr(batched.mesh, f), getattr(acc, f)
        assert np.max(np.abs(x - y)) <= 1e-8 * np.max(np.abs(y)), f


def test_vjp_frequency_batched_many_slices(mh, gpu, series_fp64):
    """A chunk of 150 frequencies: the forward writes the (G, G_r) tape in
    slices of 128 frequencies, which the adjoint reads back at the same
    offsets; mixed against FP64."""
    mesh = mh.mesh_hemisphere(1.0, (0, 0, 0), (6, 8))
    dofs = [mh.translational_dofs(mesh, "Heave"), mh.translational_dofs(mesh, "Surge")]
    om = np.linspace(0.3, 4.0, 150)
    w = _weights(2, len(om), 1, seed=9)
    a = _vjp(mh, gpu, mesh, om, dofs, [0.1], w, DELH, True, "mixed")
    b = _vjp(mh, gpu, mesh, om, dofs, [0.1], w, DELH, True, "fp64")
    assert np.max(np.abs(a.omegas - b.omegas)) <= 1e-8 * np.max(np.abs(b.omegas))
    for f in ("vertices", "centers", "normals", "areas"):
        x, y = getattr(a.mesh, f), getattr(b.mesh, f)
        assert np.max(np.abs(x - y)) <= 1e-8 * np.max(np.abs(y)), f


@pytest.mark.parametrize("names,betas", [
    (["Heave"], []),
    (["Heave"], [0.2]),
    (["Surge", "Heave", "Pitch"], [0.2]),
    (["Surge", "Sway", "Heave", "Roll", "Pitch", "Yaw"], [0.2]),
])
def test_vjp_tape_right_hand_side_counts(mh, gpu, names, betas, series_fp64):
    """The tape adjoint loads the row vectors of all right-hand sides of a
    frequency together for 1 to 4 of them and one at a time beyond (here 7,
    six rigid modes and a wave); the column vectors pass through shared
    memory in chunks whose length depends on the count.  Mixed (tape) against
    FP64 (no tape) on the same frequencies."""
    mesh = mh.mesh_hemisphere(1.1, (0, 0, 0), (10, 14))
    body = mh.FloatingBody.rigid(mesh, names, rotation_center=(0.0, 0.0, -0.2))
    dofs = list(body.dofs.values())
    om = np.linspace(0.3, 4.0, 9)
    w = _weights(len(dofs), len(om), len(betas), seed=11)
    a = _vjp(mh, gpu, mesh, om, dofs, betas, w, DELH, True, "mixed")
    b = _vjp(mh, gpu, mesh, om, dofs, betas, w, DELH, True, "fp64")
    assert np.max(np.abs(a.omegas - b.omegas)) <= 1e-8 * np.max(np.abs(b.omegas))
    for f in ("vertices", "centers", "normals", "areas"):
        x, y = getattr(a.mesh, f), getattr(b.mesh, f)
        assert np.max(np.abs(x - y)) <= 1e-8 * np.max(np.abs(y)), f


@pytest.mark.parametrize("mask", [WU, DELH])
@pytest.mark.parametrize("direct", [True, False])
def test_batched_fp64_vjp_matches_per_frequency_fp64(mh, gpu, mask, direct):
    """MH_PRECISION_FP64_BATCHED in the adjoint (the frequency-batched FP64
    forward, its pivoted factors reused conjugate-transposed, the shared
    contraction tail) against the one-frequency-at-a-time FP64 adjoint: 1e-9.
    Eight frequencies take the frequency-batched Delhommeau pass and its tape."""
    mesh = mh.mesh_hemisphere(1.0, (0, 0, -0.05), (10, 12))
    dofs = list(mh.FloatingBody.rigid(mesh, ["Heave", "Surge"]).dofs.values())
    om = np.linspace(0.5, 2.0, 8)
    w = _weights(len(dofs), len(om), 1)
    a = _vjp(mh, gpu, mesh, om, dofs, [0.4], w, mask, direct, precision="fp64_batched")
    b = _vjp(mh, gpu, mesh, om, dofs, [0.4], w, mask, direct, precision="fp64")
    for x, y in ((a.added_mass, b.added_mass), (a.damping, b.damping), (a.diffraction, b.diffraction)):
        assert np.max(np.abs(x - y)) <= 1e-10 * np.max(np.abs(y))
    assert np.max(np.abs(a.omegas - b.omegas)) <= 1e-9 * np.max(np.abs(b.omegas))
    for f in ("vertices", "centers", "normals", "areas"):
        x, y = getattr(a.mesh, f), getattr(b.mesh, f)
        assert np.max(np.abs(x - y)) <= 1e-9 * np.max(np.abs(y)), f
