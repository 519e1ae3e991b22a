"""Batched hydrodynamic coefficients (mh_hydro_batch) against the oracle's
per-problem restatement of compute_hydrodynamic_coefficients (GPU).

FP64 path: 1e-10 relative to the largest entry of each output.
Mixed path (FP32 LU + FP64 refinement to tol 1e-12): 1e-9, i.e. well inside
the 1e-6 accuracy target for A, B and F.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WU = (1 | 2 | 8)
DELH = (1 | 2 | 16)


def _gfs(mh, mask):
    t = [mh.Rankine(), mh.RankineReflected()]
    if mask & 8:
        t.append(mh.GFWu())
    if mask & 16:
        t.append(mh.ExactGuevelDelhommeau())
    return tuple(t)


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def body(mh):
    mesh = mh.mesh_hemisphere(1.0, (0, 0, 0), (10, 12))
    return mh.FloatingBody.rigid(mesh, ["Heave", "Surge", "Pitch"], (0.0, 0.0, -0.2), "hemi")


@pytest.mark.parametrize("mask", [WU, DELH])
@pytest.mark.parametrize("direct", [True, False])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_matches_oracle(mh, oracle, gpu, body, mask, direct, precision):
    omegas = [0.4, 1.03, 2.2]
    betas = [0.0, 0.6]
    dofs = list(body.dofs.values())
    A, B, Fd, Fk, info = mh.hydro_batch(body.mesh, omegas, dofs, betas,
                                        green_functions=_gfs(mh, mask), direct=direct,
                                        precision=precision, tol=1e-12, ctx=gpu)
    Ao, Bo, Fdo, Fko = oracle.hydro_coefficients(body.mesh, omegas, dofs, betas, gf_mask=mask,
                                                 direct=direct)
    tol = 1e-10 if precision == "fp64" else 1e-9
    assert _rel(A, Ao) < tol
    assert _rel(B, Bo) < tol
    assert _rel(Fd, Fdo) < tol
    assert _rel(Fk, Fko) < 1e-12
    if precision == "mixed":
        assert info.n_fallback == 0
        assert 1 <= info.refine_iterations <= 10
        assert info.max_rel_residual <= 1e-12


def test_batch_two_bodies_indirect(mh, oracle, gpu):
    m1 = mh.mesh_hemisphere(1.0, (0, 0, 0), (8, 12))
    b1 = mh.FloatingBody.rigid(m1, ["Heave"], body_name="sphere")
    b2 = mh.FloatingBody.rigid(m1.translated((5.0, 0, 0)), ["Heave"], body_name="sphere")
    both = b1 + b2
    assert list(both.dofs) == ["sphere__Heave", "sphere_2__Heave"]
    dofs = list(both.dofs.values())
    A, B, Fd, _, info = mh.hydro_batch(both.mesh, [1.03], dofs, [0.0], direct=False,
                                       precision="mixed", tol=1e-12, ctx=gpu)
    Ao, Bo, Fdo, _ = oracle.hydro_coefficients(both.mesh, [1.03], dofs, [0.0], direct=False)
    assert _rel(A, Ao) < 1e-9 and _rel(B, Bo) < 1e-9 and _rel(Fd, Fdo) < 1e-9
    # symmetric bodies: A11 == A22, A12 == A21 (the reference's Power.jl assumes it)
    assert abs(A[0, 0, 0] - A[1, 1, 0]) < 1e-8 * abs(A[0, 0, 0])
    assert abs(A[0, 1, 0] - A[1, 0, 0]) < 1e-6 * abs(A[0, 0, 0])


def test_compute_hydrodynamic_coefficients_layout(mh, gpu, body):
    params = dict(wave_frequencies=[0.8, 1.5], radiating_dofs=["Heave"],
                  influenced_dofs=["Heave", "Pitch"], wave_directions=[0.0])
    out = mh.compute_hydrodynamic_coefficients(params, body, ctx=gpu)
    assert out["added_mass"].shape == (2, 1, 2)
    assert out["radiation_damping"].shape == (2, 1, 2)
    assert out["diffraction_force"].shape == (2, 2, 1)
    assert np.allclose(out["excitation_force"],
                       out["diffraction_force"] + out["Froude_Krylov_force"])
    # the single-problem front door agrees with the batch (heave, FP64)
    AB = mh.calculate_radiation_forces(body.mesh, [0, 0, 1.0], 0.8, ctx=gpu)
    assert abs(out["added_mass"][0, 0, 0] - AB[0]) < 1e-8 * abs(AB[0])
    assert abs(out["radiation_damping"][0, 0, 0] - AB[1]) < 1e-8 * abs(AB[1])


def test_batch_many_frequencies_chunk(mh, oracle, gpu):
    mesh = mh.mesh_hemisphere(1.0, (0, 0, 0), (8, 10))
    dofs = [mh.translational_dofs(mesh, "Heave")]
    om = np.linspace(0.3, 3.0, 17)
    A, B, _, _, info = mh.hydro_batch(mesh, om, dofs, precision="mixed", tol=1e-12, ctx=gpu)
    Ao, Bo, _, _ = oracle.hydro_coefficients(mesh, om, dofs)
    assert _rel(A, Ao) < 1e-9 and _rel(B, Bo) < 1e-9


def test_batch_argument_errors(mh, gpu, body):
    dofs = list(body.dofs.values())
    with pytest.raises(mh.ArgumentError):
        mh.hydro_batch(body.mesh, [-1.0], dofs, ctx=gpu)
    with pytest.raises(mh.ArgumentError):
        mh.hydro_batch(body.mesh, [1.0], dofs * 6, ctx=gpu)  # 18 right-hand sides > 16
    with pytest.raises(mh.ArgumentError):
        mh.hydro_batch(body.mesh, [1.0], dofs, precision="mixed", tol=0.0, ctx=gpu)
    with pytest.raises(mh.ArgumentError):
        mh.hydro_batch(body.mesh, [1.0], dofs, precision="mixed",
                       green_functions=(mh.Rankine(), mh.GFWu(), mh.ExactGuevelDelhommeau()),
                       ctx=gpu)


@pytest.mark.parametrize("direct", [True, False])
def test_frequency_batched_delhommeau(mh, oracle, gpu, direct, series_fp64):
    """Chunks of >= 6 frequencies take the frequency-batched Delhommeau pass
    (alpha contraction once per pair); across [0.3, 4.0] rad/s pairs move from
    the polar patch into the Cartesian cells, so both branches run."""
    mesh = mh.mesh_hemisphere(1.3, (0, 0, 0), (10, 14))
    body = mh.FloatingBody.rigid(mesh, ["Heave", "Surge"])
    dofs = list(body.dofs.values())
    om = np.linspace(0.3, 4.0, 9)
    gfs = (mh.Rankine(), mh.RankineReflected(), mh.ExactGuevelDelhommeau())
    A, B, Fd, _, info = mh.hydro_batch(mesh, om, dofs, [0.3], green_functions=gfs, direct=direct,
                                       precision="mixed", tol=1e-12, ctx=gpu)
    Ao, Bo, Fdo, _ = oracle.hydro_coefficients(mesh, om, dofs, [0.3], gf_mask=DELH, direct=direct)
    assert _rel(A, Ao) < 1e-9 and _rel(B, Bo) < 1e-9 and _rel(Fd, Fdo) < 1e-9
    A64, B64, _, _, _ = mh.hydro_batch(mesh, om, dofs, [0.3], green_functions=gfs, direct=direct,
                                       precision="fp64", ctx=gpu)
    assert _rel(A, A64) < 1e-10 and _rel(B, B64) < 1e-10


def test_frequency_batched_delhommeau_many_slices(mh, oracle, gpu, series_fp64):
    """More frequencies in one chunk than one launch of the batched pass
    takes (128): the chunk runs in frequency slices whose outputs and tape
    land at their own offsets."""
    mesh = mh.mesh_hemisphere(1.0, (0, 0, 0), (6, 8))
    dofs = [mh.translational_dofs(mesh, "Heave")]
    om = np.linspace(0.3, 4.0, 150)
    gfs = (mh.Rankine(), mh.RankineReflected(), mh.ExactGuevelDelhommeau())
    A, B, Fd, _, _ = mh.hydro_batch(mesh, om, dofs, [0.0], green_functions=gfs, precision="mixed",
                                    tol=1e-12, ctx=gpu)
    A64, B64, Fd64, _, _ = mh.hydro_batch(mesh, om, dofs, [0.0], green_functions=gfs, precision="fp64",
                                          ctx=gpu)
    assert _rel(A, A64) < 1e-10 and _rel(B, B64) < 1e-10 and _rel(Fd, Fd64) < 1e-10
    sel = [0, 127, 128, 149]
    Ao, Bo, _, _ = oracle.hydro_coefficients(mesh, om[sel], dofs, [0.0], gf_mask=DELH)
    assert _rel(A[..., sel], Ao) < 1e-9 and _rel(B[..., sel], Bo) < 1e-9


@pytest.mark.parametrize("mask", [WU, DELH])
@pytest.mark.parametrize("direct", [True, False])
@pytest.mark.parametrize("nw", [3, 8])
def test_batched_fp64_matches_oracle(mh, oracle, gpu, body, mask, direct, nw):
    """MH_PRECISION_FP64_BATCHED (the Rankine part once, the frequency-batched
    wave pass, cuSOLVER per frequency on several streams): the FP64 bound.
    Eight frequencies take the frequency-batched Delhommeau pass, three the
    per-frequency one."""
    omegas = list(np.linspace(0.4, 2.2, nw))
    betas = [0.0, 0.6]
    dofs = list(body.dofs.values())
    A, B, Fd, Fk, _ = mh.hydro_batch(body.mesh, omegas, dofs, betas, green_functions=_gfs(mh, mask),
                                     direct=direct, precision="fp64_batched", ctx=gpu)
    Ao, Bo, Fdo, Fko = oracle.hydro_coefficients(body.mesh, omegas, dofs, betas, gf_mask=mask, direct=direct)
    assert _rel(A, Ao) < 1e-10 and _rel(B, Bo) < 1e-10 and _rel(Fd, Fdo) < 1e-10 and _rel(Fk, Fko) < 1e-12


@pytest.mark.parametrize("level", [1, 2])
def test_wave_series_fp32_levels(mh, oracle, gpu, body, level):
    """The reduced-precision levels of the mixed path's wave pass (1: the
    Horner series in FP32; 2: also the alpha contraction; logs, S and D in
    FP64), bounded against the oracle at 1e-6, the metric's bound."""
    omegas = list(np.linspace(0.4, 2.2, 8))
    dofs = list(body.dofs.values())
    old = gpu.wave_series_level()
    gpu.set_wave_series_fp32(level)
    try:
        A, B, _, _, _ = mh.hydro_batch(body.mesh, omegas, dofs, green_functions=_gfs(mh, DELH),
                                       precision="mixed", tol=1e-12, ctx=gpu)
    finally:
        gpu.set_wave_series_fp32(old)
    Ao, Bo, _, _ = oracle.hydro_coefficients(body.mesh, omegas, dofs, gf_mask=DELH)
    assert _rel(A, Ao) < 1e-6 and _rel(B, Bo) < 1e-6
