"""Adjoint gradients of the batched coefficients (``mh_hydro_batch_vjp``).

The reference differentiates this path with Zygote (reverse mode through the
assembly, ImplicitAD's ``implicit_linear`` for the solve,
src/matrix_assembly.jl:105-133) and checks the result against finite
differences (test/outputs_differentiation.jl:21-35, :59-68).  Here one
library call runs the forward batch and its adjoint on the device and
returns the cotangents of every input: the mesh fields (a ``MeshTangent``,
the counterpart of the reference's ``Tangent{Mesh}``), the frequencies and
the dof motion fields.

``hydro_batch_jvp`` is the forward mode (the reference's ForwardDiff path):
the tangents of all outputs along one input direction, e.g. dA/dR for every
frequency at once.

``hydro_batch_rrule`` is the rrule / ``torch.autograd.Function`` shaped
entry point: it returns the outputs and a pullback; the pullback recomputes
the forward batch on the device (geometry and factors are recomputed rather
than stored).

``hemisphere_tangents`` / ``two_hemispheres_tangents`` give the exact
derivative of the generated meshes with respect to their parameters (radius,
centre, separation), so ``MeshTangent.dot`` turns mesh cotangents into
d/dR, d/dd: the reference gets these through finite-difference rrules of
its mesh generators (paper/MeshGradients_singlebody.jl:85-182,
paper/meshGradients_pair.jl:100-210).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from . import _native as N
from .api import DEFAULT_GREEN_FUNCTIONS, SETTINGS, _precision_code, device_mesh, gf_mask
from .bodies import BatchInfo, _Info
from .meshes import Mesh, mesh_hemisphere


@dataclass
class MeshTangent:
    """Cotangent (or tangent) of every field of a ``Mesh``: vertices (V x 3),
    centers, normals (N x 3), areas, radii (N)."""

    vertices: np.ndarray
    centers: np.ndarray
    normals: np.ndarray
    areas: np.ndarray
    radii: np.ndarray

    def dot(self, other: "MeshTangent") -> float:
        """Sum over all fields of the elementwise products."""
        return float(sum(np.sum(a * b) for a, b in
                         ((self.vertices, other.vertices), (self.centers, other.centers),
                          (self.normals, other.normals), (self.areas, other.areas),
                          (self.radii, other.radii))))

    def __add__(self, other: "MeshTangent") -> "MeshTangent":
        return MeshTangent(self.vertices + other.vertices, self.centers + other.centers,
                           self.normals + other.normals, self.areas + other.areas,
                           self.radii + other.radii)

    def scaled(self, s: float) -> "MeshTangent":
        return MeshTangent(s * self.vertices, s * self.centers, s * self.normals, s * self.areas,
                           s * self.radii)

    @classmethod
    def zeros_like(cls, mesh: Mesh) -> "MeshTangent":
        return cls(np.zeros_like(mesh.vertices), np.zeros_like(mesh.centers),
                   np.zeros_like(mesh.normals), np.zeros_like(mesh.areas),
                   np.zeros_like(mesh.radii))


@dataclass
class VjpResult:
    added_mass: np.ndarray
    damping: np.ndarray
    diffraction: np.ndarray
    froude_krylov: np.ndarray
    mesh: MeshTangent
    omegas: np.ndarray
    dofs: list
    info: BatchInfo


def _cotangent(a, shape, dtype):
    if a is None:
        return None
    arr = np.asarray(a, dtype=dtype)
    if arr.shape != shape:
        raise ValueError(f"cotangent shape {arr.shape} != output shape {shape}")
    return np.asfortranarray(arr)


def hydro_batch_vjp(mesh: Mesh, omegas, dofs, betas=(), bar_added_mass=None, bar_damping=None,
                    bar_diffraction=None, bar_froude_krylov=None, *,
                    green_functions=DEFAULT_GREEN_FUNCTIONS, direct: bool = True, precision="mixed",
                    tol: float = 1e-10, max_iter: int = 30, rho=None, g=None, ctx=None) -> VjpResult:
    """Forward batch (as ``hydro_batch``) plus the cotangents of its inputs for
    the given output cotangents (same shapes as the outputs; None = zero).
    For a scalar J of the outputs, pass dJ/dA, dJ/dB and, for complex F,
    dJ/dRe F + i dJ/dIm F."""
    mask = gf_mask(green_functions)
    dm = device_mesh(mesh, ctx)
    om = np.ascontiguousarray(np.asarray(omegas, dtype=np.float64).reshape(-1))
    d = [np.asarray(x, dtype=np.float64) for x in dofs]
    for x in d:
        if x.shape != (mesh.nfaces, 3):
            raise ValueError("each dof must be an nfaces x 3 motion field")
    nd = len(d)
    dof_arr = np.ascontiguousarray(
        np.concatenate([np.asfortranarray(x).reshape(-1, order="F") for x in d]) if nd else np.zeros(1))
    be = np.ascontiguousarray(np.asarray(betas, dtype=np.float64).reshape(-1))
    nw, nb = om.shape[0], be.shape[0]
    bA = _cotangent(bar_added_mass, (nd, nd, nw), np.float64)
    bB = _cotangent(bar_damping, (nd, nd, nw), np.float64)
    bF = _cotangent(bar_diffraction, (nd, nw, nb), np.complex128)
    bK = _cotangent(bar_froude_krylov, (nd, nw, nb), np.complex128)
    A = np.zeros((nd, nd, nw), order="F")
    B = np.zeros((nd, nd, nw), order="F")
    Fd = np.zeros((nd, nw, nb), dtype=np.complex128, order="F")
    Fk = np.zeros((nd, nw, nb), dtype=np.complex128, order="F")
    gv = np.zeros((mesh.nvertices, 3), order="F")
    gc = np.zeros((mesh.nfaces, 3), order="F")
    gn = np.zeros((mesh.nfaces, 3), order="F")
    ga = np.zeros(mesh.nfaces)
    gr = np.zeros(mesh.nfaces)
    gw = np.zeros(nw)
    gd = np.zeros(3 * mesh.nfaces * max(nd, 1))
    info = _Info()
    nbp = (lambda a: N.dptr(a) if (a is not None and nb) else None)
    N.check(N.lib().mh_hydro_batch_vjp(
        dm.ctx.handle, dm.handle, nw, N.dptr(om), nd, N.dptr(dof_arr), nb,
        N.dptr(be) if nb else None,
        float(SETTINGS.rho if rho is None else rho), float(SETTINGS.g if g is None else g), mask,
        int(bool(direct)), _precision_code(precision), float(tol), int(max_iter),
        N.dptr(bA), N.dptr(bB), nbp(bF), nbp(bK),
        N.dptr(A), N.dptr(B), nbp(Fd), nbp(Fk),
        N.dptr(gv), N.dptr(gc), N.dptr(gn), N.dptr(ga), N.dptr(gr), N.dptr(gw), N.dptr(gd),
        ctypes.byref(info)), dm.ctx.handle)
    ddofs = [gd[3 * mesh.nfaces * q:3 * mesh.nfaces * (q + 1)].reshape((mesh.nfaces, 3), order="F")
             for q in range(nd)]
    return VjpResult(A, B, Fd, Fk, MeshTangent(np.ascontiguousarray(gv), np.ascontiguousarray(gc),
                                               np.ascontiguousarray(gn), ga, gr), gw, ddofs,
                     BatchInfo(info.refine_iterations, info.n_fallback, info.max_rel_residual))


@dataclass
class JvpResult:
    added_mass: np.ndarray
    damping: np.ndarray
    diffraction: np.ndarray
    froude_krylov: np.ndarray
    d_added_mass: np.ndarray
    d_damping: np.ndarray
    d_diffraction: np.ndarray
    d_froude_krylov: np.ndarray
    info: BatchInfo


def hydro_batch_jvp(mesh: Mesh, omegas, dofs, betas=(), t_mesh: MeshTangent | None = None,
                    t_omegas=None, t_dofs=None, *, green_functions=DEFAULT_GREEN_FUNCTIONS,
                    direct: bool = True, precision="mixed", tol: float = 1e-10, max_iter: int = 30,
                    rho=None, g=None, ctx=None) -> JvpResult:
    """Forward batch (as ``hydro_batch``) plus the tangents of its outputs
    along one direction of the inputs (``mh_hydro_batch_jvp``): the tangent
    of the mesh fields (a ``MeshTangent``; radii have no effect), of the
    frequencies and of the dof fields (None = zero)."""
    mask = gf_mask(green_functions)
    dm = device_mesh(mesh, ctx)
    om = np.ascontiguousarray(np.asarray(omegas, dtype=np.float64).reshape(-1))
    d = [np.asarray(x, dtype=np.float64) for x in dofs]
    nd = len(d)
    dof_arr = np.ascontiguousarray(
        np.concatenate([np.asfortranarray(x).reshape(-1, order="F") for x in d]) if nd else np.zeros(1))
    be = np.ascontiguousarray(np.asarray(betas, dtype=np.float64).reshape(-1))
    nw, nb = om.shape[0], be.shape[0]
    f = lambda a: None if a is None else np.ascontiguousarray(np.asfortranarray(np.asarray(a, dtype=np.float64))
                                                                .reshape(-1, order="F"))
    tv = tc = tn = ta = None
    if t_mesh is not None:
        tv, tc, tn, ta = f(t_mesh.vertices), f(t_mesh.centers), f(t_mesh.normals), f(t_mesh.areas)
    tw = f(t_omegas)
    td = None
    if t_dofs is not None:
        td = np.ascontiguousarray(np.concatenate([np.asfortranarray(np.asarray(x, dtype=np.float64))
                                                  .reshape(-1, order="F") for x in t_dofs]))
    A = np.zeros((nd, nd, nw), order="F")
    B = np.zeros((nd, nd, nw), order="F")
    Fd = np.zeros((nd, nw, nb), dtype=np.complex128, order="F")
    Fk = np.zeros((nd, nw, nb), dtype=np.complex128, order="F")
    dA, dB, dFd, dFk = np.zeros_like(A), np.zeros_like(B), np.zeros_like(Fd), np.zeros_like(Fk)
    info = _Info()
    nbp = (lambda a: N.dptr(a) if nb else None)
    N.check(N.lib().mh_hydro_batch_jvp(
        dm.ctx.handle, dm.handle, nw, N.dptr(om), nd, N.dptr(dof_arr), nb,
        N.dptr(be) if nb else None,
        float(SETTINGS.rho if rho is None else rho), float(SETTINGS.g if g is None else g), mask,
        int(bool(direct)), _precision_code(precision), float(tol), int(max_iter),
        N.dptr(tv), N.dptr(tc), N.dptr(tn), N.dptr(ta), N.dptr(tw), N.dptr(td),
        N.dptr(A), N.dptr(B), nbp(Fd), nbp(Fk), N.dptr(dA), N.dptr(dB), nbp(dFd), nbp(dFk),
        ctypes.byref(info)), dm.ctx.handle)
    return JvpResult(A, B, Fd, Fk, dA, dB, dFd, dFk,
                     BatchInfo(info.refine_iterations, info.n_fallback, info.max_rel_residual))


def hydro_batch_rrule(mesh: Mesh, omegas, dofs, betas=(), **kw):
    """rrule-shaped entry: returns ((A, B, Fd, Fk), pullback) where
    pullback(bar_A, bar_B, bar_Fd, bar_Fk) -> (MeshTangent, omega-bar, dof-bars).
    The pullback reruns the forward batch with its adjoint on the device."""
    from .bodies import hydro_batch
    A, B, Fd, Fk, _ = hydro_batch(mesh, omegas, dofs, betas, **kw)

    def pullback(bar_A=None, bar_B=None, bar_Fd=None, bar_Fk=None):
        r = hydro_batch_vjp(mesh, omegas, dofs, betas, bar_A, bar_B, bar_Fd, bar_Fk, **kw)
        return r.mesh, r.omegas, r.dofs

    return (A, B, Fd, Fk), pullback


def hemisphere_tangents(radius: float = 1.0, center=(0.0, 0.0, 0.0), resolution=(10, 10), mesh=None) -> dict:
    """Exact derivatives of ``mesh_hemisphere(radius, center, resolution)``
    with respect to its parameters: {"radius", "cx", "cy", "cz"} ->
    MeshTangent.  Every field is homogeneous in the radius about the centre:
    vertices and centres are centre + R u, normals do not change, areas
    scale as R^2 and radii as R.  ``mesh``: that mesh when the caller has
    already generated it."""
    m = mesh if mesh is not None else mesh_hemisphere(radius, center, resolution)
    c = np.asarray(center, dtype=np.float64).reshape(1, 3)
    out = {"radius": MeshTangent((m.vertices - c) / radius, (m.centers - c) / radius,
                                 np.zeros_like(m.normals), 2.0 * m.areas / radius, m.radii / radius)}
    for k, name in enumerate(("cx", "cy", "cz")):
        e = np.zeros((1, 3))
        e[0, k] = 1.0
        out[name] = MeshTangent(np.repeat(e, m.nvertices, 0), np.repeat(e, m.nfaces, 0),
                                np.zeros_like(m.normals), np.zeros_like(m.areas),
                                np.zeros_like(m.radii))
    return out


def two_hemispheres_tangents(radius: float = 1.0, separation: float = 5.0,
                             resolution=(32, 64)) -> dict:
    """Exact derivatives of ``mesh_two_hemispheres`` with respect to
    {"radius", "separation"} (the second body moves along x)."""
    t1 = hemisphere_tangents(radius, (0.0, 0.0, 0.0), resolution)
    t2 = hemisphere_tangents(radius, (separation, 0.0, 0.0), resolution)

    def cat(a: MeshTangent, b: MeshTangent) -> MeshTangent:
        return MeshTangent(np.concatenate([a.vertices, b.vertices]),
                           np.concatenate([a.centers, b.centers]),
                           np.concatenate([a.normals, b.normals]),
                           np.concatenate([a.areas, b.areas]), np.concatenate([a.radii, b.radii]))

    zero = MeshTangent.zeros_like(mesh_hemisphere(radius, (0.0, 0.0, 0.0), resolution))
    return {"radius": cat(t1["radius"], t2["radius"]), "separation": cat(zero, t2["cx"])}


def polygon_geometry_jvp(vertices: np.ndarray, faces: np.ndarray, dvertices: np.ndarray) -> MeshTangent:
    """Tangent of every field of a mesh built by ``polygon_geometry`` (the
    reference's polygon-mesh conventions, src/meshes.jl:353-423) along a
    vertex tangent: the exact derivatives of the area-weighted centroid, the
    unit normal of (b - a) x (c - a), the area and the radius |a - centre|."""
    v, dv = vertices[faces], dvertices[faces]
    a, b, c, d = v[:, 0], v[:, 1], v[:, 2], v[:, 3]
    da, db, dc, dd = dv[:, 0], dv[:, 1], dv[:, 2], dv[:, 3]
    cr1, cr2 = np.cross(b - a, c - a), np.cross(c - a, d - a)
    dcr1 = np.cross(db - da, c - a) + np.cross(b - a, dc - da)
    dcr2 = np.cross(dc - da, d - a) + np.cross(c - a, dd - da)
    n1, n2 = np.linalg.norm(cr1, axis=1), np.linalg.norm(cr2, axis=1)
    area1, area2 = 0.5 * n1, 0.5 * n2
    # a degenerate second triangle (triangle panels) has no area and no tangent
    dn1 = np.einsum("ij,ij->i", cr1, dcr1) / n1
    dn2 = np.where(n2 > 0.0, np.einsum("ij,ij->i", cr2, dcr2) / np.where(n2 > 0.0, n2, 1.0), 0.0)
    darea1, darea2 = 0.5 * dn1, 0.5 * dn2
    areas, dareas = area1 + area2, darea1 + darea2
    c1, c2 = (a + b + c) / 3.0, (a + c + d) / 3.0
    dc1, dc2 = (da + db + dc) / 3.0, (da + dc + dd) / 3.0
    centers = (c1 * area1[:, None] + c2 * area2[:, None]) / areas[:, None]
    dcenters = (dc1 * area1[:, None] + c1 * darea1[:, None] + dc2 * area2[:, None] + c2 * darea2[:, None]
                - centers * dareas[:, None]) / areas[:, None]
    nrm = cr1 / n1[:, None]
    dnormals = dcr1 / n1[:, None] - nrm * (dn1 / n1)[:, None]
    ra = a - centers
    rr = np.linalg.norm(ra, axis=1)
    dradii = np.einsum("ij,ij->i", ra, da - dcenters) / rr
    return MeshTangent(np.asarray(dvertices, dtype=np.float64).copy(), dcenters, dnormals, dareas, dradii)


def wavebot_tangents(r1: float, r2: float, d1: float, d2: float, n_points=(5, 10, 5),
                     n_theta: int = 72) -> dict:
    """Exact derivatives of ``wavebot_mesh(r1, r2, d1, d2, n_points,
    n_theta)`` with respect to {"r1", "r2", "d1", "d2"} -> MeshTangent (the
    reference obtains them by automatic differentiation through
    src/meshes.jl:247-479).  The profile is linear in the four parameters,
    so its derivative along one of them is the profile with that parameter 1
    and the others 0; each ring's vertices (r cos theta, r sin theta, z)
    follow, and the face fields by ``polygon_geometry_jvp``.  Valid for
    r1, r2 > 0 (the ring structure does not change under the derivative)."""
    from .meshes import axisymmetric_mesh, wavebot_profile

    prof = wavebot_profile(d1, d2, r1, r2, n_points)
    verts, faces = axisymmetric_mesh(prof, n_theta)
    th = 2.0 * np.pi * np.arange(int(n_theta)) / int(n_theta)
    ct, st = np.cos(th), np.sin(th)
    unit = {"r1": (0.0, 0.0, 1.0, 0.0), "r2": (0.0, 0.0, 0.0, 1.0),
            "d1": (1.0, 0.0, 0.0, 0.0), "d2": (0.0, 1.0, 0.0, 0.0)}
    out = {}
    for name, (h1, h2, rt, rb) in unit.items():
        dprof = wavebot_profile(h1, h2, rt, rb, n_points)
        dv = []
        for (r, _), (dr, dz) in zip(prof, dprof):
            if r == 0.0:
                dv.append((0.0, 0.0, dz))
            else:
                dv.extend(zip(dr * ct, dr * st, np.full(th.shape, dz)))
        out[name] = polygon_geometry_jvp(verts, faces, np.asarray(dv, dtype=np.float64))
    return out
