"""Reference-named host API over the C ABI.

Mirrors MarineHydro.jl's public functions for the hot path, with the same
names, argument meaning and defaults:

  assemble_matrices(green_functions, mesh, wavenumber; direct=true)   src/matrix_assembly.jl:97
  assemble_matrix_wu(mesh, wavenumber; direct=true)                   src/matrix_assembly.jl:100-102
  solve(D, S, bc; direct=true)                                        src/matrix_assembly.jl:105-133
  calculate_radiation_forces(mesh, dof, omega)                        src/waves.jl:29-37
  DiffractionForce(mesh, omega, dof)                                  src/waves.jl:40-52

The matrix-level and output-level calls run on the GPU through
``libmarinehydro_b200.so``; there is no CPU fallback.  The O(N) helpers
(``radiation_bc``, ``AiryBC``, ``airy_waves_*``, ``integrate_pressure``,
``FroudeKrylovForce``) are host-side numpy glue with the reference's
semantics, provided for API completeness; the output-level calls evaluate
their device counterparts inside the library.
"""
from __future__ import annotations

import weakref
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .meshes import Mesh


# --------------------------------------------------------------------------
# settings (src/constants.jl:2-12)
# --------------------------------------------------------------------------

@dataclass
class _Settings:
    rho: float = 1000.0
    g: float = 9.81


SETTINGS = _Settings()


def set_g(val: float):
    SETTINGS.g = float(val)


def set_rho(val: float):
    SETTINGS.rho = float(val)


# --------------------------------------------------------------------------
# Green functions (src/green_functions/*.jl) -> C-ABI term bits
# --------------------------------------------------------------------------

class GreensFunction:
    mask = 0

    def __repr__(self):
        return f"{type(self).__name__}()"

    def __eq__(self, other):
        return type(self) is type(other)

    def __hash__(self):
        return hash(type(self))


class Rankine(GreensFunction):
    mask = 1


class RankineReflected(GreensFunction):
    mask = 2


class RankineReflectedNegative(GreensFunction):
    mask = 4


class GFWu(GreensFunction):
    mask = 8


class ExactGuevelDelhommeau(GreensFunction):
    mask = 16


def gf_mask(green_functions) -> int:
    """Term bitmask of a tuple of Green functions (summed as in
    abstract_greens_function.jl:49,65)."""
    if isinstance(green_functions, GreensFunction):
        green_functions = (green_functions,)
    m = 0
    for gf in green_functions:
        if not isinstance(gf, GreensFunction):
            raise TypeError(f"{gf!r} is not a GreensFunction")
        if m & gf.mask:
            raise ValueError(f"{gf!r} appears twice in the Green-function tuple")
        m |= gf.mask
    if m == 0:
        raise ValueError("empty Green-function tuple")
    return m


DEFAULT_GREEN_FUNCTIONS = (Rankine(), RankineReflected(), GFWu())


# --------------------------------------------------------------------------
# device meshes
# --------------------------------------------------------------------------

def _mesh_arrays(mesh: Mesh):
    return (mesh.vertices, mesh.faces, mesh.centers, mesh.normals, mesh.areas, mesh.radii)


def _mesh_snapshot(mesh: Mesh) -> tuple:
    """Copies of the mesh arrays, to see later whether they were changed in place."""
    return tuple(np.array(a, copy=True) for a in _mesh_arrays(mesh))


def _mesh_unchanged(snapshot: tuple, mesh: Mesh) -> bool:
    """Exact comparison with a snapshot (a few tens of microseconds at 2048
    panels, where hashing the arrays took most of a millisecond per call)."""
    return all(s.shape == np.shape(a) and np.array_equal(s, a) for s, a in zip(snapshot, _mesh_arrays(mesh)))


class DeviceMesh:
    """A mesh uploaded to one context (``mh_mesh``)."""

    def __init__(self, ctx: N.Context, mesh: Mesh):
        self.ctx = ctx
        self.nfaces = mesh.nfaces
        v = np.asfortranarray(mesh.vertices, dtype=np.float64)
        f = np.asfortranarray(mesh.faces, dtype=np.int64)
        c = np.asfortranarray(mesh.centers, dtype=np.float64)
        n = np.asfortranarray(mesh.normals, dtype=np.float64)
        a = np.ascontiguousarray(mesh.areas, dtype=np.float64)
        r = np.ascontiguousarray(mesh.radii, dtype=np.float64)
        self._h = N._P()
        N.check(N.lib().mh_mesh_create(ctx.handle, mesh.nfaces, mesh.nvertices, N.dptr(v),
                                       N.i64ptr(f), N.dptr(c), N.dptr(n), N.dptr(a), N.dptr(r),
                                       N.ctypes.byref(self._h)), ctx.handle)

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            N.lib().mh_mesh_destroy(self.ctx.handle, self._h)
            self._h = N._P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_mesh_cache: "weakref.WeakKeyDictionary[Mesh, tuple]" = weakref.WeakKeyDictionary()


def device_mesh(mesh: Mesh, ctx: N.Context | None = None) -> DeviceMesh:
    """Upload ``mesh`` (cached per mesh object while its arrays are unchanged)."""
    ctx = ctx or N.default_context()
    hit = _mesh_cache.get(mesh)
    if hit is not None and hit[0] is ctx and _mesh_unchanged(hit[1], mesh):
        return hit[2]
    dm = DeviceMesh(ctx, mesh)
    _mesh_cache[mesh] = (ctx, _mesh_snapshot(mesh), dm)
    return dm


def _precision_code(precision) -> int:
    if precision in ("fp64", N.MH_PRECISION_FP64):
        return N.MH_PRECISION_FP64
    if precision in ("mixed", N.MH_PRECISION_MIXED):
        return N.MH_PRECISION_MIXED
    if precision in ("fp64_batched", N.MH_PRECISION_FP64_BATCHED):
        return N.MH_PRECISION_FP64_BATCHED
    raise ValueError(f"unknown precision {precision!r}")


def _dof_array(dof, nfaces):
    d = np.asarray(dof, dtype=np.float64)
    if d.ndim == 1:
        if d.shape[0] != 3:
            raise ValueError("dof must be a 3-vector or an nfaces x 3 matrix")
        return np.ascontiguousarray(d), 1
    if d.shape != (nfaces, 3):
        raise ValueError("dof must be a 3-vector or an nfaces x 3 matrix")
    return np.asfortranarray(d), nfaces


# --------------------------------------------------------------------------
# matrix level
# --------------------------------------------------------------------------

def assemble_matrices(green_functions, mesh: Mesh, wavenumber: float, direct: bool = True,
                      ctx: N.Context | None = None):
    """(S, D) -- or (S, K) with ``direct=False`` -- as nfaces x nfaces
    complex128 arrays (src/matrix_assembly.jl:4-42)."""
    mask = gf_mask(green_functions)
    dm = device_mesh(mesh, ctx)
    n = mesh.nfaces
    S = np.empty((n, n), dtype=np.complex128, order="F")
    D = np.empty((n, n), dtype=np.complex128, order="F")
    N.check(N.lib().mh_assemble_matrices(dm.ctx.handle, dm.handle, float(wavenumber), mask,
                                         int(bool(direct)), N.dptr(S),
                                         N.dptr(D)), dm.ctx.handle)
    return S, D


def assemble_matrix_wu(mesh: Mesh, wavenumber: float, direct: bool = True, ctx=None):
    """src/matrix_assembly.jl:100-102."""
    return assemble_matrices(DEFAULT_GREEN_FUNCTIONS, mesh, wavenumber, direct=direct, ctx=ctx)


def solve(D, S, bc, direct: bool = True, ctx: N.Context | None = None):
    """direct: phi = D \\ (S bc); indirect: phi = S (K \\ bc)
    (src/matrix_assembly.jl:105-133).  FP64 LU on the device."""
    ctx = ctx or N.default_context()
    D = np.asfortranarray(D, dtype=np.complex128)
    S = np.asfortranarray(S, dtype=np.complex128)
    b = np.asarray(bc, dtype=np.complex128)
    vec = b.ndim == 1
    b2 = np.asfortranarray(b.reshape(b.shape[0], -1))
    n = D.shape[0]
    if D.shape != (n, n) or S.shape != (n, n) or b2.shape[0] != n:
        raise ValueError("solve: D and S must be n x n and bc must have n rows")
    phi = np.empty_like(b2, order="F")
    N.check(N.lib().mh_solve(ctx.handle, n, N.dptr(D), N.dptr(S),
                             N.dptr(b2), b2.shape[1], int(bool(direct)),
                             N.dptr(phi)), ctx.handle)
    return phi[:, 0].copy() if vec else phi


# --------------------------------------------------------------------------
# output level
# --------------------------------------------------------------------------

def calculate_radiation_forces(mesh: Mesh, dof, omega: float, *,
                               green_functions=DEFAULT_GREEN_FUNCTIONS, direct: bool = True,
                               precision="fp64", rho=None, g=None, ctx=None):
    """[added mass, radiation damping] (src/waves.jl:29-37).  The reference
    always uses Rankine + RankineReflected + GFWu with the direct method;
    those are the defaults here."""
    mask = gf_mask(green_functions)
    dm = device_mesh(mesh, ctx)
    d, rows = _dof_array(dof, mesh.nfaces)
    out = np.zeros(2)
    N.check(N.lib().mh_calculate_radiation_forces(
        dm.ctx.handle, dm.handle, N.dptr(d), rows, float(omega),
        float(SETTINGS.rho if rho is None else rho), float(SETTINGS.g if g is None else g),
        mask, int(bool(direct)), _precision_code(precision), N.dptr(out)), dm.ctx.handle)
    return out


def DiffractionForce(mesh: Mesh, omega: float, dof, *, beta: float = 0.0,
                     green_functions=DEFAULT_GREEN_FUNCTIONS, direct: bool = True,
                     precision="fp64", rho=None, g=None, ctx=None) -> complex:
    """Complex diffraction force (src/waves.jl:40-59)."""
    mask = gf_mask(green_functions)
    dm = device_mesh(mesh, ctx)
    d, rows = _dof_array(dof, mesh.nfaces)
    out = np.zeros(2)
    N.check(N.lib().mh_diffraction_force(
        dm.ctx.handle, dm.handle, float(omega), N.dptr(d), rows, float(beta),
        float(SETTINGS.rho if rho is None else rho), float(SETTINGS.g if g is None else g),
        mask, int(bool(direct)), _precision_code(precision), N.dptr(out)), dm.ctx.handle)
    return complex(out[0], out[1])


# --------------------------------------------------------------------------
# O(N) host helpers (src/waves.jl), reference semantics
# --------------------------------------------------------------------------

def radiation_bc(mesh: Mesh, dof, omega):
    """-i omega (n . dof) per panel (src/waves.jl:4-18, :89-101)."""
    d = np.asarray(dof, dtype=np.float64)
    d = np.broadcast_to(d.reshape(1, 3), mesh.normals.shape) if d.ndim == 1 else d
    return -1j * omega * np.sum(mesh.normals * d, axis=1)


def airy_waves_potential(points, omega, beta=0.0):
    """src/waves.jl:112-119."""
    g = SETTINGS.g
    k = omega ** 2 / g
    p = np.asarray(points, dtype=np.float64)
    wbar = p[:, 0] * np.cos(beta) + p[:, 1] * np.sin(beta)
    return -1j * g / omega * np.exp(k * p[:, 2]) * np.exp(1j * k * wbar)


def airy_waves_velocity(points, omega, beta=0.0, water_depth=np.inf):
    """src/waves.jl:121-134 (infinite depth)."""
    g = SETTINGS.g
    k = omega ** 2 / g
    p = np.asarray(points, dtype=np.float64)
    wbar = p[:, 0] * np.cos(beta) + p[:, 1] * np.sin(beta)
    cih = np.exp(k * p[:, 2])
    f = g * k / omega * np.exp(1j * k * wbar)
    return np.stack([f * np.cos(beta) * cih, f * np.sin(beta) * cih, -1j * f * cih], axis=1)


def airy_waves_pressure(points, omega, beta=0.0):
    """src/waves.jl:150-154."""
    return 1j * omega * SETTINGS.rho * airy_waves_potential(points, omega, beta)


def AiryBC(mesh: Mesh, omega, beta=0.0):
    """-(v_inc . n) per panel (src/waves.jl:138-142)."""
    return -np.sum(airy_waves_velocity(mesh.centers, omega, beta) * mesh.normals, axis=1)


def integrate_pressure(mesh: Mesh, pressure, dof):
    """sum(p * (-(n . dof)) * area) (src/waves.jl:21-25)."""
    d = np.asarray(dof, dtype=np.float64)
    d = np.broadcast_to(d.reshape(1, 3), mesh.normals.shape) if d.ndim == 1 else d
    amp = -np.sum(d * mesh.normals, axis=1)
    return np.sum(np.asarray(pressure) * amp * mesh.areas)


def FroudeKrylovForce(mesh: Mesh, omega, dof, beta=0.0):
    """src/waves.jl:62-66."""
    return integrate_pressure(mesh, airy_waves_pressure(mesh.centers, omega, beta), dof)
