"""The CUDA path at the benchmark's own sizes against the FP64 oracle
(GPU).

The fixtures in ``tests/golden/*.npz`` were written by
``tests/golden/make_fixtures.py`` from the CPU oracle: exact adaptive
quadrature for the Guevel-Delhommeau term (the reference's method,
src/green_functions/exact_Guevel_Delhommeau.jl:8-13), LAPACK for the solve.
The device uses its Delhommeau table, so these tests bound the table's error
where the metric is quoted, not only point-wise.

* 1024-panel hemisphere, omega = 1.03, heave, Delhommeau, direct (FP64 and
  mixed precision): A, B, F, FK and 512 sampled entries of S and D;
* 2048-panel hemisphere, the bench's 64 frequencies in [0.3, 3.0], heave and
  surge, Delhommeau, direct: A, B, F, FK at every frequency, S and D sampled
  at three frequencies;
* two 1024-panel hemispheres 5 m apart, Wu, indirect, omega = 1.03: A, B, F,
  FK and sampled S, K; the two-body power J(r1, dx1, omega) and its gradient
  against central differences (h = 1e-6) of the oracle.

Tolerances, relative to the largest entry of each output: FP64 path 1e-9;
mixed path 1e-6 at refinement tolerance 1e-8 (the benchmark's setting and
the metric's bound), 1e-8 at 1e-12 with the default FP32 Horner series of
the wave pass and 1e-9 with its FP64 form; matrix entries 1e-9 of the
largest sampled entry; gradients 1e-5.
"""
from __future__ import annotations

import pathlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = pathlib.Path(__file__).parent / "golden"


def _load(name):
    return dict(np.load(GOLDEN / f"{name}.npz"))


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _gfs(mh, mask):
    t = [mh.Rankine(), mh.RankineReflected()]
    if mask & 8:
        t.append(mh.GFWu())
    if mask & 16:
        t.append(mh.ExactGuevelDelhommeau())
    return tuple(t)


def _fingerprint(mesh):
    return np.array([mesh.nfaces, np.sum(mesh.centers), np.sum(mesh.normals), np.sum(mesh.areas),
                     np.sum(mesh.radii), np.sum(mesh.vertices)])


def _hemisphere_case(mh, res, dof_names):
    mesh = mh.mesh_hemisphere(1.0, (0.0, 0.0, 0.0), res)
    body = mh.FloatingBody.rigid(mesh, dof_names)
    return mesh, [body.dofs[n] for n in dof_names]


def _two_body_case(mh):
    m1 = mh.mesh_hemisphere(1.0, (0.0, 0.0, 0.0), (32, 64))
    m2 = mh.mesh_hemisphere(1.0, (5.0, 0.0, 0.0), (32, 64))
    body = mh.FloatingBody.rigid(m1, ["Heave"], body_name="sphere") + \
        mh.FloatingBody.rigid(m2, ["Heave"], body_name="sphere")
    return body.mesh, list(body.dofs.values())


CASES = {
    "hemisphere_1024p_delhommeau": lambda mh: _hemisphere_case(mh, (32, 64), ["Heave"]),
    "hemisphere_2048p_delhommeau": lambda mh: _hemisphere_case(mh, (64, 64), ["Heave", "Surge"]),
    "two_hemispheres_2048p_wu": _two_body_case,
}


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("precision,tol,bound,level", [("fp64", 1e-12, 1e-9, 1), ("mixed", 1e-8, 1e-6, 1),
                                                       ("mixed", 1e-12, 1e-8, 1), ("mixed", 1e-12, 1e-9, 0),
                                                       ("mixed", 1e-8, 1e-6, 2)])
def test_coefficients_match_oracle_at_size(mh, gpu, name, precision, tol, bound, level):
    """level: the precision level of the mixed path's wave series (0 FP64,
    1 the default FP32 Horner series, 2 also the FP32 alpha contraction)."""
    fx = _load(name)
    gpu.set_wave_series_fp32(level)
    try:
        _check_at_size(mh, gpu, name, fx, precision, tol, bound)
    finally:
        gpu.set_wave_series_fp32(1)


def _check_at_size(mh, gpu, name, fx, precision, tol, bound):
    mesh, dofs = CASES[name](mh)
    assert np.allclose(_fingerprint(mesh), fx["fingerprint"], rtol=1e-13, atol=1e-10)
    mask = int(fx["gf_mask"])
    A, B, Fd, Fk, info = mh.hydro_batch(mesh, fx["omegas"], dofs, fx["betas"], green_functions=_gfs(mh, mask),
                                        direct=bool(fx["direct"]), precision=precision, tol=tol,
                                        rho=float(fx["rho"]), g=float(fx["g"]), ctx=gpu)
    errs = {"A": _rel(A, fx["added_mass"]), "B": _rel(B, fx["damping"]),
            "F": _rel(Fd, fx["diffraction"]), "FK": _rel(Fk, fx["froude_krylov"])}
    assert max(errs.values()) <= bound, errs
    # per frequency too: no frequency is allowed to hide behind a larger one
    for w in range(len(fx["omegas"])):
        assert _rel(B[:, :, w], fx["damping"][:, :, w]) <= 10 * bound or \
            np.max(np.abs(fx["damping"][:, :, w])) < 1e-3 * np.max(np.abs(fx["damping"])), w
    if precision == "mixed":
        assert info.n_fallback == 0


@pytest.mark.parametrize("name", list(CASES))
def test_sampled_matrix_entries_match_oracle(mh, gpu, name):
    fx = _load(name)
    mesh, _ = CASES[name](mh)
    mask = int(fx["gf_mask"])
    rows, cols = fx["sample_rows"], fx["sample_cols"]
    for s, w_i in enumerate(fx["sample_omega_index"]):
        w = float(fx["omegas"][w_i])
        S, D = mh.assemble_matrices(_gfs(mh, mask), mesh, w * w / float(fx["g"]),
                                    direct=bool(fx["direct"]), ctx=gpu)
        assert _rel(S[rows, cols], fx["S_samples"][s]) <= 1e-9
        assert _rel(D[rows, cols], fx["D_samples"][s]) <= 1e-9


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_two_body_power_gradient_matches_oracle_differences(mh, gpu, precision):
    """Config of paper/Power.jl at size: two 1024-panel hemispheres, Wu,
    indirect; dJ/d(r1, dx1, omega) from one adjoint call against central
    differences of the oracle's forward."""
    fx = _load("two_hemispheres_2048p_wu")
    J, g = mh.two_body_power(float(fx["r1"]), float(fx["dx1"]), 1.03, resolution=(32, 64), direct=False,
                             precision=precision, tol=1e-10, grad=True, ctx=gpu)
    assert abs(J - float(fx["power"])) <= 1e-8 * abs(float(fx["power"]))
    for k in ("r1", "dx1", "omega"):
        ref = float(fx[f"fd_{k}"])
        assert abs(g[k] - ref) <= 1e-5 * max(abs(ref), 1e-3 * abs(J)), (k, g[k], ref)
