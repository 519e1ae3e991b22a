"""Meshes generated on the device and their exact parameter derivatives
computed there: the immersed hemisphere, the pair of hemispheres of the
two-body power problem and the WaveBot buoy (the reference's generators,
src/meshes.jl:247-479, and the Capytaine hemispheres of its tests,
src/meshes.jl:122-127), through ``mh_mesh_hemisphere``,
``mh_mesh_wavebot``, ``mh_mesh_combine``, ``mh_mesh_tangent`` and
``mh_mesh_param_vjp``.

Each generator returns a host ``Mesh`` with the fields the device computed,
and registers the device geometry with the context, so ``hydro_batch``,
``hydro_batch_vjp`` and ``hydro_batch_jvp`` on that mesh use it without an
upload.  ``generated_tangents`` gives d(mesh fields)/d(parameter) for every
generator parameter (forward mode: the ``t_mesh`` of ``hydro_batch_jvp``);
``generated_param_grad`` contracts the mesh cotangent of ``hydro_batch_vjp``
into parameter cotangents (reverse mode), which replaces the
finite-difference rrules of the reference's paper scripts
(paper/MeshGradients_singlebody.jl:85-167, paper/meshGradients_pair.jl:100-210).
"""
from __future__ import annotations

import ctypes
import weakref

import numpy as np

from . import _native as N
from . import api
from .gradients import MeshTangent
from .meshes import Mesh

HEMISPHERE_PARAMS = ("radius", "cx", "cy", "cz")
WAVEBOT_PARAMS = ("r1", "r2", "d1", "d2")


class GeneratedMesh(api.DeviceMesh):
    """A mesh made on the device (``mh_mesh``), with the names of its
    generator parameters in the library's order."""

    def __init__(self, ctx: N.Context, handle: N._P, names):
        self.ctx = ctx
        self._h = handle
        n = ctypes.c_int64()
        N.check(N.lib().mh_mesh_nfaces(handle, ctypes.byref(n)), ctx.handle)
        self.nfaces = int(n.value)
        N.check(N.lib().mh_mesh_nvertices(handle, ctypes.byref(n)), ctx.handle)
        self.nvertices = int(n.value)
        k = ctypes.c_int()
        N.check(N.lib().mh_mesh_nparams(handle, ctypes.byref(k)), ctx.handle)
        if k.value != len(names):
            raise RuntimeError(f"{k.value} generator parameters, {len(names)} names")
        self.param_names = tuple(names)

    def host_mesh(self) -> Mesh:
        n, nv = self.nfaces, self.nvertices
        v = np.empty((nv, 3), order="F")
        f = np.empty((n, 4), dtype=np.int64, order="F")
        c = np.empty((n, 3), order="F")
        nr = np.empty((n, 3), order="F")
        a = np.empty(n)
        r = np.empty(n)
        N.check(N.lib().mh_mesh_fields(self.ctx.handle, self._h, N.dptr(v), N.i64ptr(f), N.dptr(c), N.dptr(nr),
                                       N.dptr(a), N.dptr(r)), self.ctx.handle)
        return Mesh(v, f, c, nr, a, r)

    def tangent(self, p: int) -> MeshTangent:
        n, nv = self.nfaces, self.nvertices
        tv = np.empty((nv, 3), order="F")
        tc = np.empty((n, 3), order="F")
        tn = np.empty((n, 3), order="F")
        ta = np.empty(n)
        tr = np.empty(n)
        N.check(N.lib().mh_mesh_tangent(self.ctx.handle, self._h, int(p), N.dptr(tv), N.dptr(tc), N.dptr(tn),
                                        N.dptr(ta), N.dptr(tr)), self.ctx.handle)
        return MeshTangent(tv, tc, tn, ta, tr)

    def param_vjp(self, bar: MeshTangent) -> np.ndarray:
        def f(x, shape):
            return None if x is None else np.asfortranarray(np.asarray(x, dtype=np.float64).reshape(shape))
        n, nv = self.nfaces, self.nvertices
        arrs = (f(bar.vertices, (nv, 3)), f(bar.centers, (n, 3)), f(bar.normals, (n, 3)), f(bar.areas, (n,)),
                f(bar.radii, (n,)))
        out = np.zeros(len(self.param_names))
        N.check(N.lib().mh_mesh_param_vjp(self.ctx.handle, self._h, *(N.dptr(x) for x in arrs), N.dptr(out)),
                self.ctx.handle)
        return out


_generated: "weakref.WeakKeyDictionary[Mesh, GeneratedMesh]" = weakref.WeakKeyDictionary()


def _register(ctx: N.Context, gm: GeneratedMesh) -> Mesh:
    mesh = gm.host_mesh()
    api._mesh_cache[mesh] = (ctx, api._mesh_snapshot(mesh), gm)
    _generated[mesh] = gm
    return mesh


def _new(fn, ctx, *args) -> N._P:
    h = N._P()
    N.check(fn(ctx.handle, *args, ctypes.byref(h)), ctx.handle)
    return h


def generate_hemisphere(radius: float = 1.0, center=(0.0, 0.0, 0.0), resolution=(10, 10),
                        ctx: N.Context | None = None) -> Mesh:
    """``mesh_hemisphere(radius, center, resolution)`` generated on the
    device (the same vertices, faces and fields, up to the last bits of the
    device's sine and cosine); parameters radius, cx, cy, cz."""
    ctx = ctx or N.default_context()
    cx, cy, cz = (float(c) for c in center)
    h = _new(N.lib().mh_mesh_hemisphere, ctx, float(radius), cx, cy, cz, int(resolution[0]), int(resolution[1]))
    return _register(ctx, GeneratedMesh(ctx, h, HEMISPHERE_PARAMS))


def generate_wavebot(r1: float, r2: float, d1: float, d2: float, n_points=(5, 10, 5), n_theta: int = 72,
                     ctx: N.Context | None = None) -> Mesh:
    """``wavebot_mesh(r1, r2, d1, d2, n_points, n_theta)`` generated on the
    device; parameters r1, r2, d1, d2 (r1, r2 > 0)."""
    ctx = ctx or N.default_context()
    nb, nf, nc = (int(x) for x in n_points)
    h = _new(N.lib().mh_mesh_wavebot, ctx, float(r1), float(r2), float(d1), float(d2), nb, nf, nc, int(n_theta))
    return _register(ctx, GeneratedMesh(ctx, h, WAVEBOT_PARAMS))


def generate_combined(meshes, ctx: N.Context | None = None) -> Mesh:
    """Concatenation on the device of meshes generated (or uploaded) on the
    same context (``combine_meshes``); the parameters of the k-th generated
    part carry the suffix k."""
    ctx = ctx or N.default_context()
    parts = [api.device_mesh(m, ctx) for m in meshes]
    names = []
    for k, dm in enumerate(parts):
        for nm in getattr(dm, "param_names", ()):
            names.append(f"{nm}{k}")
    arr = (N._P * len(parts))(*[dm.handle for dm in parts])
    h = _new(N.lib().mh_mesh_combine, ctx, len(parts), arr)
    return _register(ctx, GeneratedMesh(ctx, h, names))


def generate_two_hemispheres(radius: float = 1.0, separation: float = 5.0, resolution=(32, 64),
                             ctx: N.Context | None = None) -> Mesh:
    """``mesh_two_hemispheres`` generated on the device: centres (0, 0, 0)
    and (separation, 0, 0); parameters radius0, cx0, cy0, cz0, radius1,
    cx1, cy1, cz1 (d/d radius = radius0 + radius1, d/d separation = cx1)."""
    ctx = ctx or N.default_context()
    m1 = generate_hemisphere(radius, (0.0, 0.0, 0.0), resolution, ctx)
    m2 = generate_hemisphere(radius, (separation, 0.0, 0.0), resolution, ctx)
    return generate_combined([m1, m2], ctx)


def generated_mesh(mesh: Mesh) -> GeneratedMesh:
    gm = _generated.get(mesh)
    if gm is None or not api._mesh_unchanged(api._mesh_cache[mesh][1], mesh):
        raise ValueError("not a mesh made by a generate_* function (or changed since)")
    return gm


def generated_tangents(mesh: Mesh) -> dict:
    """{parameter name: MeshTangent}: the exact derivatives of every field
    of a generated mesh, computed on the device."""
    gm = generated_mesh(mesh)
    return {nm: gm.tangent(p) for p, nm in enumerate(gm.param_names)}


def generated_tangent(mesh: Mesh, name: str) -> MeshTangent:
    """The tangent of one generator parameter (see ``generated_tangents``)."""
    gm = generated_mesh(mesh)
    if name not in gm.param_names:
        raise ValueError(f"{name!r} is not a parameter of this mesh: {gm.param_names}")
    return gm.tangent(gm.param_names.index(name))


def generated_param_grad(mesh: Mesh, cotangent: MeshTangent) -> dict:
    """{parameter name: cotangent}: a mesh cotangent (``VjpResult.mesh`` of
    ``hydro_batch_vjp``) pulled back to the generator's parameters on the
    device."""
    gm = generated_mesh(mesh)
    return dict(zip(gm.param_names, (float(x) for x in gm.param_vjp(cotangent))))
