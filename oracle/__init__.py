"""FP64 CPU oracle for the MarineHydro.jl boundary-element hot path.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU legs import this package, and only as the checker or as the
timed CPU baseline.  The product library never imports, loads or calls it.

It is a restatement of the reference algorithm:

* ``oracle.c`` (built to ``_build/liboracle.so``): Green functions, panel
  integrals and influence-matrix assembly, FP64, OpenMP over columns;
* this module: the O(N) glue of ``src/waves.jl`` and the dense solve of
  ``src/matrix_assembly.jl:105-133`` through LAPACK (scipy's zgetrf/zgetrs,
  the same routines Julia's ``\\`` reaches).

Parity pins: the oracle is checked against every golden value the reference's
own tests hold for this path (``test/greens_function.jl:40-99``, the Hulme
table of ``test/consistency_with_analytical_solutions.jl:14-18``) and against
an independent scipy restatement.  The reference's Capytaine-anchored matrix
pins cannot be reproduced here (Capytaine is absent), so S/D-level parity is
pinned only through those per-pair goldens.
"""
from __future__ import annotations

import ctypes
import os
import pathlib
import subprocess

import numpy as np

_HERE = pathlib.Path(__file__).resolve().parent
_LIB_PATH = _HERE / "_build" / "liboracle.so"

GF_RANKINE = 1
GF_RANKINE_REFLECTED = 2
GF_RANKINE_REFL_NEG = 4
GF_WU = 8
GF_DELHOMMEAU = 16

_lib = None


def build() -> pathlib.Path:
    """Compile oracle.c with the committed Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not _LIB_PATH.exists():
        build()
    L = ctypes.CDLL(str(_LIB_PATH))
    dp = ctypes.POINTER(ctypes.c_double)
    i64p = ctypes.POINTER(ctypes.c_int64)
    L.orc_expint_e1.argtypes = [ctypes.c_double, ctypes.c_double, dp]
    L.orc_expint_e1.restype = None
    L.orc_rankine_integral.argtypes = [dp, dp, dp, dp, ctypes.c_double, ctypes.c_double]
    L.orc_rankine_integral.restype = ctypes.c_double
    L.orc_rankine_both.argtypes = [dp, dp, dp, dp, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_int, dp, dp]
    L.orc_rankine_both.restype = None
    L.orc_wu_dimless.argtypes = [ctypes.c_double, ctypes.c_double, dp]
    L.orc_wu_dimless.restype = None
    L.orc_delhommeau_dimless.argtypes = [ctypes.c_double, ctypes.c_double, dp]
    L.orc_delhommeau_dimless.restype = None
    L.orc_pair_integrals.argtypes = [dp, dp, dp, dp, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_uint32, ctypes.c_int, dp, dp]
    L.orc_pair_integrals.restype = None
    L.orc_assemble_columns.argtypes = [ctypes.c_int64, ctypes.c_int64, dp, dp, dp, dp, dp, i64p,
                                       ctypes.c_double, ctypes.c_uint32, ctypes.c_int,
                                       ctypes.c_int64, ctypes.c_int64, dp, dp, ctypes.c_int]
    L.orc_assemble_columns.restype = ctypes.c_int
    L.orc_max_threads.argtypes = []
    L.orc_max_threads.restype = ctypes.c_int
    _lib = L
    return L


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _v3(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(3))


def max_threads() -> int:
    return int(lib().orc_max_threads())


# --------------------------------------------------------------------------
# per-pair functions (src/green_functions/*.jl)
# --------------------------------------------------------------------------

def expint_e1(z: complex) -> complex:
    out = np.zeros(2)
    lib().orc_expint_e1(float(np.real(z)), float(np.imag(z)), _dp(out))
    return complex(out[0], out[1])


def _elem(e):
    verts = np.ascontiguousarray(np.asarray(e["vertices"], dtype=np.float64).reshape(4, 3))
    return (_v3(e["center"]), _v3(e["normal"]), verts, float(e["area"]), float(e["radius"]))


def rankine_integral(x, e) -> float:
    """``integral(Rankine(), e1, e2)`` (rankine.jl:24-63); ``e`` is a dict
    with center, normal, vertices (4x3), area, radius."""
    c, n, v, a, r = _elem(e)
    xx = _v3(x)
    return float(lib().orc_rankine_integral(_dp(xx), _dp(c), _dp(n), _dp(v), a, r))


def rankine_integral_gradient(x, e, with_respect_to_first_variable=False) -> np.ndarray:
    """``integral_gradient(Rankine(), ...)`` (rankine.jl:126-128)."""
    c, n, v, a, r = _elem(e)
    xx = _v3(x)
    out = np.zeros(1)
    g = np.zeros(3)
    lib().orc_rankine_both(_dp(xx), _dp(c), _dp(n), _dp(v), a, r,
                           int(bool(with_respect_to_first_variable)), _dp(out), _dp(g))
    return g


def wu_dimless(r: float, z: float):
    """(G, dG/dr, dG/dz) of the Wu et al. wave term (wu.jl:19-30)."""
    o = np.zeros(6)
    lib().orc_wu_dimless(float(r), float(z), _dp(o))
    return complex(o[0], o[1]), complex(o[2], o[3]), complex(o[4], o[5])


def delhommeau_dimless(r: float, z: float):
    """(G, dG/dr, dG/dz) of the exact Guevel-Delhommeau wave term
    (exact_Guevel_Delhommeau.jl:15-59)."""
    o = np.zeros(6)
    lib().orc_delhommeau_dimless(float(r), float(z), _dp(o))
    return complex(o[0], o[1]), complex(o[2], o[3]), complex(o[4], o[5])


def pair_integrals(x, e, k, gf_mask, with_respect_to_first_variable=False):
    """Sum over the GF tuple of ``integral`` and ``integral_gradient``
    (abstract_greens_function.jl:49,65)."""
    c, n, v, a, r = _elem(e)
    xx = _v3(x)
    s = np.zeros(2)
    g = np.zeros(6)
    lib().orc_pair_integrals(_dp(xx), _dp(c), _dp(n), _dp(v), a, r, float(k), int(gf_mask),
                             int(bool(with_respect_to_first_variable)), _dp(s), _dp(g))
    return complex(s[0], s[1]), g[0::2] + 1j * g[1::2]


# --------------------------------------------------------------------------
# assembly (src/matrix_assembly.jl:4-42)
# --------------------------------------------------------------------------

def _mesh_arrays(mesh):
    n = int(np.asarray(mesh.areas).shape[0])
    verts = np.asfortranarray(np.asarray(mesh.vertices, dtype=np.float64))
    faces = np.asfortranarray(np.asarray(mesh.faces, dtype=np.int64))
    centers = np.asfortranarray(np.asarray(mesh.centers, dtype=np.float64))
    normals = np.asfortranarray(np.asarray(mesh.normals, dtype=np.float64))
    areas = np.ascontiguousarray(np.asarray(mesh.areas, dtype=np.float64))
    radii = np.ascontiguousarray(np.asarray(mesh.radii, dtype=np.float64))
    return n, verts, faces, centers, normals, areas, radii


def assemble(mesh, k, gf_mask, direct=True, nthreads=0, columns=None, want_S=True, want_D=True):
    """S and D (or K) as N x N complex128, column-major, FP64.

    ``columns=(j0, j1)`` assembles only those source columns (the other
    columns are left zero); used to time a bounded sample."""
    n, verts, faces, centers, normals, areas, radii = _mesh_arrays(mesh)
    j0, j1 = (0, n) if columns is None else (int(columns[0]), int(columns[1]))
    S = np.zeros((n, n), dtype=np.complex128, order="F") if want_S else None
    D = np.zeros((n, n), dtype=np.complex128, order="F") if want_D else None
    rc = lib().orc_assemble_columns(
        n, verts.shape[0], _dp(centers), _dp(normals), _dp(areas), _dp(radii), _dp(verts),
        faces.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), float(k), int(gf_mask),
        int(bool(direct)), j0, j1,
        _dp(S) if S is not None else None, _dp(D) if D is not None else None, int(nthreads))
    if rc != 0:
        raise ValueError("oracle assembly rejected its arguments")
    return S, D


# --------------------------------------------------------------------------
# solve (src/matrix_assembly.jl:105-133)
# --------------------------------------------------------------------------

def solve(D, S, bc, direct=True):
    """direct: phi = D \\ (S bc);  indirect: sigma = K \\ bc, phi = S sigma."""
    import scipy.linalg as sla

    lu = sla.lu_factor(D, check_finite=False)
    if direct:
        return sla.lu_solve(lu, S @ bc, check_finite=False)
    return S @ sla.lu_solve(lu, bc, check_finite=False)


# --------------------------------------------------------------------------
# boundary conditions, pressure and forces (src/waves.jl)
# --------------------------------------------------------------------------

def _dof_matrix(normals, dof):
    dof = np.asarray(dof, dtype=np.float64)
    if dof.ndim == 1:
        return np.broadcast_to(dof.reshape(1, 3), normals.shape)
    return dof


def radiation_bc(normals, dof, omega):
    """waves.jl:4-18 / :89-101: -i omega (n . dof)."""
    normals = np.asarray(normals, dtype=np.float64)
    return -1j * omega * np.sum(normals * _dof_matrix(normals, dof), axis=1)


def airy_waves_potential(points, omega, beta=0.0, g=9.81):
    """waves.jl:112-119."""
    k = omega ** 2 / g
    p = np.asarray(points, dtype=np.float64)
    wbar = p[:, 0] * np.cos(beta) + p[:, 1] * np.sin(beta)
    return -1j * g / omega * np.exp(k * p[:, 2]) * np.exp(1j * k * wbar)


def airy_waves_velocity(points, omega, beta=0.0, g=9.81):
    """waves.jl:121-134."""
    k = omega ** 2 / g
    p = np.asarray(points, dtype=np.float64)
    wbar = p[:, 0] * np.cos(beta) + p[:, 1] * np.sin(beta)
    cih = np.exp(k * p[:, 2])
    f = g * k / omega * np.exp(1j * k * wbar)
    return np.stack([f * np.cos(beta) * cih, f * np.sin(beta) * cih, f * (-1j) * cih], axis=1)


def airy_waves_pressure(points, omega, beta=0.0, rho=1000.0, g=9.81):
    """waves.jl:150-154."""
    return 1j * omega * rho * airy_waves_potential(points, omega, beta, g)


def airy_bc(centers, normals, omega, beta=0.0, g=9.81):
    """waves.jl:138-142: -(v_inc . n)."""
    v = airy_waves_velocity(centers, omega, beta, g)
    return -np.sum(v * np.asarray(normals, dtype=np.float64), axis=1)


def integrate_pressure(normals, areas, pressure, dof):
    """waves.jl:21-25: sum(p * (-(n . dof)) * area)."""
    normals = np.asarray(normals, dtype=np.float64)
    amp = -np.sum(_dof_matrix(normals, dof) * normals, axis=1)
    return np.sum(pressure * amp * np.asarray(areas, dtype=np.float64))


def calculate_radiation_forces(mesh, dof, omega, rho=1000.0, g=9.81,
                               gf_mask=GF_RANKINE | GF_RANKINE_REFLECTED | GF_WU,
                               direct=True, nthreads=0):
    """waves.jl:29-37 (the reference hard-codes Wu + direct; both are
    parameters here, defaulting to the reference's choice)."""
    k = omega ** 2 / g
    S, D = assemble(mesh, k, gf_mask, direct, nthreads)
    bc = radiation_bc(mesh.normals, dof, omega)
    phi = solve(D, S, bc, direct)
    p = 1j * rho * omega * phi
    F = integrate_pressure(mesh.normals, mesh.areas, p, dof)
    return np.array([F.real / omega ** 2, F.imag / omega])


def diffraction_force(mesh, omega, dof, beta=0.0, rho=1000.0, g=9.81,
                      gf_mask=GF_RANKINE | GF_RANKINE_REFLECTED | GF_WU,
                      direct=True, nthreads=0):
    """waves.jl:40-59 (``DiffractionForce``)."""
    k = omega ** 2 / g
    S, D = assemble(mesh, k, gf_mask, direct, nthreads)
    bc = airy_bc(mesh.centers, mesh.normals, omega, beta, g)
    phi = solve(D, S, bc, direct)
    p = 1j * rho * phi * omega
    return integrate_pressure(mesh.normals, mesh.areas, p, dof)


def froude_krylov_force(mesh, omega, dof, beta=0.0, rho=1000.0, g=9.81):
    """waves.jl:62-66."""
    p = airy_waves_pressure(mesh.centers, omega, beta, rho, g)
    return integrate_pressure(mesh.normals, mesh.areas, p, dof)


def hydro_coefficients(mesh, omegas, dofs, betas=(), rho=1000.0, g=9.81,
                       gf_mask=GF_RANKINE | GF_RANKINE_REFLECTED | GF_WU, direct=True, nthreads=0):
    """Per-problem restatement of compute_hydrodynamic_coefficients
    (src/problems_and_results.jl:70-181, src/solve.jl:4-21): one radiation
    problem per (omega, dof), one diffraction problem per (omega, beta), all
    dofs influenced.  Returns added_mass[i, j, w], damping[i, j, w],
    diffraction[i, w, b], froude_krylov[i, w, b]."""
    omegas = np.atleast_1d(np.asarray(omegas, dtype=np.float64))
    nd, nw, nb = len(dofs), len(omegas), len(betas)
    A = np.zeros((nd, nd, nw))
    B = np.zeros((nd, nd, nw))
    Fd = np.zeros((nd, nw, nb), dtype=np.complex128)
    Fk = np.zeros((nd, nw, nb), dtype=np.complex128)
    for w_i, w in enumerate(omegas):
        S, D = assemble(mesh, w * w / g, gf_mask, direct, nthreads)
        A[:, :, w_i], B[:, :, w_i], Fd[:, w_i, :], Fk[:, w_i, :] = coefficients_from_matrices(
            mesh, S, D, w, dofs, betas, rho, g, direct)
    return A, B, Fd, Fk


def coefficients_from_matrices(mesh, S, D, omega, dofs, betas=(), rho=1000.0, g=9.81, direct=True):
    """The per-frequency part of ``hydro_coefficients`` on given S and D (or
    K): one LU, every radiation and diffraction problem at this frequency.
    Returns added_mass[i, j], damping[i, j], diffraction[i, b],
    froude_krylov[i, b] (src/problems_and_results.jl:105-181)."""
    import scipy.linalg as sla

    w = float(omega)
    nd, nb = len(dofs), len(betas)
    A = np.zeros((nd, nd))
    B = np.zeros((nd, nd))
    Fd = np.zeros((nd, nb), dtype=np.complex128)
    Fk = np.zeros((nd, nb), dtype=np.complex128)
    lu = sla.lu_factor(D, check_finite=False)
    for j, dj in enumerate(dofs):
        bc = radiation_bc(mesh.normals, dj, w)
        phi = sla.lu_solve(lu, S @ bc) if direct else S @ sla.lu_solve(lu, bc)
        p = 1j * rho * w * phi
        for i, di in enumerate(dofs):
            F = integrate_pressure(mesh.normals, mesh.areas, p, di)
            A[i, j] = F.real / w ** 2
            B[i, j] = F.imag / w
    for b_i, beta in enumerate(betas):
        bc = airy_bc(mesh.centers, mesh.normals, w, beta, g)
        phi = sla.lu_solve(lu, S @ bc) if direct else S @ sla.lu_solve(lu, bc)
        p = 1j * rho * phi * w
        pk = airy_waves_pressure(mesh.centers, w, beta, rho, g)
        for i, di in enumerate(dofs):
            Fd[i, b_i] = integrate_pressure(mesh.normals, mesh.areas, p, di)
            Fk[i, b_i] = integrate_pressure(mesh.normals, mesh.areas, pk, di)
    return A, B, Fd, Fk


def threads_env() -> int:
    v = os.environ.get("OMP_NUM_THREADS")
    return int(v) if v else 0
