"""FP64 CUDA path against the FP64 CPU oracle (GPU).

Tolerances (max abs difference relative to the matrix's max abs entry):
Rankine / reflected / Wu terms 1e-12 (the same arithmetic, differing only in
the last bits of CUDA's and the C library's transcendental functions);
Delhommeau 1e-10 (the adaptive quadrature's acceptance decisions may differ
at the tolerance boundary, 1e-13 relative per integral).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

GF = dict(R=1, RR=2, RN=4, WU=8, DE=16)
MASKS = [GF["R"], GF["R"] | GF["RR"], GF["R"] | GF["RN"], GF["R"] | GF["RR"] | GF["WU"],
         GF["WU"], GF["R"] | GF["RR"] | GF["DE"], GF["DE"]]


def _gfs(mh, mask):
    out = []
    for bit, cls in ((1, mh.Rankine), (2, mh.RankineReflected), (4, mh.RankineReflectedNegative),
                     (8, mh.GFWu), (16, mh.ExactGuevelDelhommeau)):
        if mask & bit:
            out.append(cls())
    return tuple(out)


@pytest.fixture(scope="module")
def meshes(mh):
    one = mh.mesh_hemisphere(1.0, (0, 0, 0), (10, 10))
    two = one + mh.mesh_hemisphere(1.0, (5.0, 0, 0), (10, 10))
    return {"sphere": one, "two_spheres": two}


@pytest.mark.parametrize("mask", MASKS)
@pytest.mark.parametrize("direct", [True, False])
@pytest.mark.parametrize("which", ["sphere", "two_spheres"])
def test_assembly_matches_oracle(mh, oracle, gpu, meshes, mask, direct, which):
    mesh = meshes[which]
    k = 1.0 if which == "sphere" else 2.0
    S, D = mh.assemble_matrices(_gfs(mh, mask), mesh, k, direct=direct, ctx=gpu)
    So, Do = oracle.assemble(mesh, k, mask, direct)
    tol = 1e-10 if mask & GF["DE"] else 1e-12
    assert rel_err(S, So) < tol
    assert rel_err(D, Do) < tol


@pytest.mark.parametrize("k", [0.01, 0.3, 3.0])
def test_assembly_wavenumbers(mh, oracle, gpu, meshes, k):
    mesh = meshes["sphere"]
    for mask in (GF["R"] | GF["RR"] | GF["WU"], GF["R"] | GF["RR"] | GF["DE"]):
        S, D = mh.assemble_matrices(_gfs(mh, mask), mesh, k, ctx=gpu)
        So, Do = oracle.assemble(mesh, k, mask, True)
        tol = 1e-10 if mask & GF["DE"] else 1e-12
        assert rel_err(S, So) < tol and rel_err(D, Do) < tol


@pytest.mark.parametrize("direct", [True, False])
def test_solve_matches_lapack(mh, oracle, gpu, meshes, direct):
    mesh = meshes["two_spheres"]
    mask = GF["R"] | GF["RR"] | GF["WU"]
    So, Do = oracle.assemble(mesh, 0.5, mask, direct)
    rng = np.random.default_rng(3)
    bc = rng.standard_normal((mesh.nfaces, 3)) + 1j * rng.standard_normal((mesh.nfaces, 3))
    phi = mh.solve(Do, So, bc, direct=direct, ctx=gpu)
    ref = oracle.solve(Do, So, bc, direct)
    assert rel_err(phi, ref) < 1e-12
    phi1 = mh.solve(Do, So, bc[:, 0], direct=direct, ctx=gpu)
    assert phi1.shape == (mesh.nfaces,)
    assert rel_err(phi1, ref[:, 0]) < 1e-12


@pytest.mark.parametrize("gf", ["wu", "delhommeau"])
@pytest.mark.parametrize("direct", [True, False])
def test_radiation_forces_match_oracle(mh, oracle, gpu, meshes, gf, direct):
    mesh = meshes["sphere"]
    mask = GF["R"] | GF["RR"] | (GF["WU"] if gf == "wu" else GF["DE"])
    for dof in ([0, 0, 1.0], [1.0, 0, 0]):
        for w in (0.5, 1.03, 2.0):
            got = mh.calculate_radiation_forces(mesh, dof, w, green_functions=_gfs(mh, mask),
                                                direct=direct, ctx=gpu)
            ref = oracle.calculate_radiation_forces(mesh, dof, w, gf_mask=mask, direct=direct)
            assert np.allclose(got, ref, rtol=1e-10, atol=1e-9 * np.max(np.abs(ref)))


def test_diffraction_force_matches_oracle(mh, oracle, gpu, meshes):
    mesh = meshes["two_spheres"]
    for beta in (0.0, 0.7):
        got = mh.DiffractionForce(mesh, 1.03, [0, 0, 1.0], beta=beta, ctx=gpu)
        ref = oracle.diffraction_force(mesh, 1.03, [0, 0, 1.0], beta=beta)
        assert abs(got - ref) <= 1e-10 * abs(ref)


def test_dof_matrix_form(mh, oracle, gpu, meshes):
    mesh = meshes["two_spheres"]
    dof = np.zeros((mesh.nfaces, 3))
    dof[: mesh.nfaces // 2, 2] = 1.0  # heave of body 1 only
    got = mh.calculate_radiation_forces(mesh, dof, 1.03, ctx=gpu)
    ref = oracle.calculate_radiation_forces(mesh, dof, 1.03)
    assert np.allclose(got, ref, rtol=1e-10)


def test_argument_errors(mh, gpu, meshes):
    mesh = meshes["sphere"]
    with pytest.raises(mh.ArgumentError):
        mh.calculate_radiation_forces(mesh, [0, 0, 1.0], -1.0, ctx=gpu)
    with pytest.raises(ValueError):
        mh.calculate_radiation_forces(mesh, np.zeros((3, 3)), 1.0, ctx=gpu)
    L = mh.native.lib()
    dm = mh.device_mesh(mesh, gpu)
    assert L.mh_assemble_matrices(gpu.handle, dm.handle, 1.0, 0, 1, None, None) == 1
    assert L.mh_assemble_matrices(gpu.handle, dm.handle, 1.0, 64, 1, None, None) == 1
    assert L.mh_assemble_matrices(gpu.handle, None, 1.0, 1, 1, None, None) == 1
    assert b"mesh" in L.mh_last_error(gpu.handle)


def test_singular_matrix_reported(mh, gpu):
    n = 4
    D = np.zeros((n, n), dtype=complex)
    S = np.eye(n, dtype=complex)
    with pytest.raises(mh.SingularMatrixError):
        mh.solve(D, S, np.ones(n, dtype=complex), ctx=gpu)


def test_kernel_launch_counter(mh, gpu, meshes):
    before = gpu.kernel_launches()
    mh.assemble_matrices(mh.DEFAULT_GREEN_FUNCTIONS, meshes["sphere"], 1.0, ctx=gpu)
    assert gpu.kernel_launches() == before + 1
