"""Floating bodies and the batched hydrodynamic-coefficient driver.

``FloatingBody`` mirrors src/bodies.jl: a mesh plus named rigid-body motion
fields (nfaces x 3 per dof).  ``compute_hydrodynamic_coefficients`` mirrors
src/problems_and_results.jl:231-236 and returns the same NamedTuple fields
(added_mass, radiation_damping, diffraction_force, Froude_Krylov_force,
excitation_force) with the same index order, computed by one
``mh_hydro_batch`` call per body.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

from . import _native as N
from .api import DEFAULT_GREEN_FUNCTIONS, SETTINGS, _precision_code, device_mesh, gf_mask
from .meshes import Mesh, combine_meshes

_TRANSLATIONS = {"Surge": 0, "Sway": 1, "Heave": 2}
_ROTATIONS = {"Roll": (1.0, 0.0, 0.0), "Pitch": (0.0, 1.0, 0.0), "Yaw": (0.0, 0.0, 1.0)}


def translational_dofs(mesh: Mesh, dof_name: str) -> np.ndarray:
    """src/bodies.jl:63-74."""
    d = np.zeros((mesh.nfaces, 3))
    if dof_name in _TRANSLATIONS:
        d[:, _TRANSLATIONS[dof_name]] = 1.0
    return d


def rotational_dofs(mesh: Mesh, dof_name: str, rotation_center) -> np.ndarray:
    """axis x (x - c) per panel centre (src/bodies.jl:76-89)."""
    axis = np.asarray(_ROTATIONS[dof_name])
    pos = mesh.centers - np.asarray(rotation_center, dtype=np.float64).reshape(1, 3)
    return np.cross(np.broadcast_to(axis, pos.shape), pos)


@dataclass(eq=False)
class FloatingBody:
    """src/bodies.jl:26-36: mesh, dofs (name -> nfaces x 3 motion), name."""

    mesh: Mesh
    dofs: dict = field(default_factory=dict)
    body_name: str = "body"

    @classmethod
    def rigid(cls, mesh: Mesh, rigid_dof_list: Sequence[str], rotation_center=(0.0, 0.0, 0.0),
              body_name: str = "body") -> "FloatingBody":
        """src/bodies.jl:40-53 / :92-100."""
        dofs = {}
        for name in rigid_dof_list:
            name = str(name)
            if name in _TRANSLATIONS:
                dofs[name] = translational_dofs(mesh, name)
            elif name in _ROTATIONS:
                dofs[name] = rotational_dofs(mesh, name, rotation_center)
            else:
                raise ValueError(f"unknown rigid dof {name!r}")
        return cls(mesh, dofs, body_name)

    def __add__(self, other):
        others = [other] if isinstance(other, FloatingBody) else list(other)
        return combine_floatingbodies([self, *others])


def make_body_name_list_unique(strings: Sequence[str]):
    """src/bodies.jl:102-125."""
    seen: dict = {}
    result = []
    for s in strings:
        if s not in seen:
            result.append(s)
            seen[s] = 2
        else:
            count = seen[s]
            new_s = f"{s}_{count}"
            while new_s in seen or new_s in strings:
                count += 1
                new_s = f"{s}_{count}"
            result.append(new_s)
            seen[s] = count + 1
            seen[new_s] = 1
    return result


def combine_floatingbodies(bodies: Sequence[FloatingBody], new_body_name: str | None = None):
    """src/bodies.jl:129-177: one mesh, dofs renamed body__dof and zero-padded."""
    names = make_body_name_list_unique([b.body_name.replace(" ", "_") for b in bodies])
    mesh = combine_meshes([b.mesh for b in bodies])
    dofs = {}
    offset = 0
    for b, name in zip(bodies, names):
        for dof_name, mat in b.dofs.items():
            full = np.zeros((mesh.nfaces, 3))
            full[offset:offset + b.mesh.nfaces] = mat
            dofs[f"{name}__{dof_name}"] = full
        offset += b.mesh.nfaces
    return FloatingBody(mesh, dofs, new_body_name or "+".join(names))


@dataclass
class BatchInfo:
    refine_iterations: int
    n_fallback: int
    max_rel_residual: float


class _Info(ctypes.Structure):
    _fields_ = [("refine_iterations", ctypes.c_int32), ("n_fallback", ctypes.c_int32),
                ("max_rel_residual", ctypes.c_double)]


def hydro_batch(mesh: Mesh, omegas, dofs, betas=(), *, green_functions=DEFAULT_GREEN_FUNCTIONS,
                direct: bool = True, precision="mixed", tol: float = 1e-10, max_iter: int = 30,
                rho=None, g=None, ctx=None):
    """All dofs radiating and influenced, all headings, all frequencies in
    one device call (``mh_hydro_batch``).  ``dofs``: sequence of nfaces x 3
    motion fields.  Returns (added_mass, damping, diffraction, froude_krylov,
    info) with shapes (d, d, w), (d, d, w), (d, w, b), (d, w, b)."""
    mask = gf_mask(green_functions)
    dm = device_mesh(mesh, ctx)
    om = np.ascontiguousarray(np.asarray(omegas, dtype=np.float64).reshape(-1))
    d = [np.asarray(x, dtype=np.float64) for x in dofs]
    for x in d:
        if x.shape != (mesh.nfaces, 3):
            raise ValueError("each dof must be an nfaces x 3 motion field")
    nd = len(d)
    dof_arr = np.concatenate([np.asfortranarray(x).reshape(-1, order="F") for x in d]) if nd else \
        np.zeros(1)
    dof_arr = np.ascontiguousarray(dof_arr)
    be = np.ascontiguousarray(np.asarray(betas, dtype=np.float64).reshape(-1))
    nw, nb = om.shape[0], be.shape[0]
    A = np.zeros((nd, nd, nw), order="F")
    B = np.zeros((nd, nd, nw), order="F")
    Fd = np.zeros((nd, nw, nb), dtype=np.complex128, order="F")
    Fk = np.zeros((nd, nw, nb), dtype=np.complex128, order="F")
    info = _Info()
    N.check(N.lib().mh_hydro_batch(
        dm.ctx.handle, dm.handle, nw, N.dptr(om), nd, N.dptr(dof_arr), nb,
        N.dptr(be) if nb else None,
        float(SETTINGS.rho if rho is None else rho), float(SETTINGS.g if g is None else g), mask,
        int(bool(direct)), _precision_code(precision), float(tol), int(max_iter), N.dptr(A),
        N.dptr(B), N.dptr(Fd) if nb else None, N.dptr(Fk) if nb else None, ctypes.byref(info)),
        dm.ctx.handle)
    return A, B, Fd, Fk, BatchInfo(info.refine_iterations, info.n_fallback, info.max_rel_residual)


def compute_hydrodynamic_coefficients(parameters: dict, floatingbody: FloatingBody, *,
                                      green_functions=DEFAULT_GREEN_FUNCTIONS, direct=True,
                                      precision="mixed", tol=1e-10, max_iter=30, ctx=None):
    """src/problems_and_results.jl:231-236 (with :105-181 for the layout).

    ``parameters`` keys: wave_frequencies, and optionally radiating_dofs,
    influenced_dofs (default: all dofs), wave_directions.  The reference
    solves with Wu + direct (src/solve.jl:6); those are the defaults."""
    omegas = np.atleast_1d(np.asarray(parameters["wave_frequencies"], dtype=np.float64))
    all_dofs = list(floatingbody.dofs.keys())
    inf = list(parameters.get("influenced_dofs", all_dofs))
    rad = list(parameters.get("radiating_dofs", []))
    betas = list(parameters.get("wave_directions", []))
    used = [n for n in all_dofs if n in set(inf) | set(rad)]
    for name in inf + rad:
        if name not in floatingbody.dofs:
            raise ValueError(f"{name!r} is not a dof of the body")
    A, B, Fd, Fk, info = hydro_batch(floatingbody.mesh, omegas,
                                     [floatingbody.dofs[n] for n in used], betas,
                                     green_functions=green_functions, direct=direct,
                                     precision=precision, tol=tol, max_iter=max_iter, ctx=ctx)
    ii = [used.index(n) for n in inf]
    jj = [used.index(n) for n in rad]
    out = dict(info=info)
    if rad:
        out["added_mass"] = A[np.ix_(ii, jj, range(len(omegas)))]
        out["radiation_damping"] = B[np.ix_(ii, jj, range(len(omegas)))]
    else:
        out["added_mass"] = out["radiation_damping"] = np.zeros(0)
    if betas:
        out["diffraction_force"] = Fd[ii]
        out["Froude_Krylov_force"] = Fk[ii]
        out["excitation_force"] = Fd[ii] + Fk[ii]
    else:
        out["diffraction_force"] = out["Froude_Krylov_force"] = out["excitation_force"] = np.zeros(0)
    return out
