"""Gradients anchored outside this library (GPU).

1. The reference's own gradients.  paper/Plots/11_heuristics_dx_DELhommeau.csv,
   11_heuristics_dr_DELhommeau.csv, added_mass_data_dimensionless.csv and
   damping_data_dimensionless.csv hold Zygote gradients that MarineHydro.jl
   computed for two heaving 6 x 6 hemispheres (paper/ArraySensitivities.jl,
   meshes from paper/meshGradients_pair.jl:7-15 with body 2 centred at
   x = r + dx, Rankine + reflected + Wu, direct, k = omega^2 / 9.81):
   dA11/d(dx), dB11/d(dx), dA11/dr, dB11/dr at omega = 1.03 for 14 gaps, and
   dA21/dr, dB21/dr on a 14 x 10 grid of (dx/r, kr).  The reference's mesh
   derivatives come from finite-difference rrules (h = 1e-2 in dx, 1e-5 in r)
   of Capytaine meshes; the meshes are linear in dx and r (areas quadratic),
   so those differences are exact up to rounding, and this package's
   hemisphere reproduces Capytaine's sphere at this resolution (the oracle
   matches all 308 values to 1e-7, tests/test_oracle.py).  Here the device's
   forward mode (one call per mesh gives every frequency) and adjoint must
   match them to 1e-6 of each column's scale.
2. Central differences of the oracle.  ``tests/golden/grad_fd_*.npz`` hold
   central differences (h = 1e-6) of the CPU oracle's forward (exact
   Delhommeau quadrature, LAPACK) for a seeded objective on a 100-panel
   hemisphere, along the radius, the frequencies and a seeded vertex
   direction; Wu and Delhommeau, direct and indirect.  The adjoint and the
   forward mode must match them to 1e-5 relative, FP64 and mixed precision.
"""
from __future__ import annotations

import json
import math
import pathlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = pathlib.Path(__file__).parent / "golden"
PINS = json.loads((GOLDEN / "reference_pins.json").read_text())


def _pair(mh, radius, dx, resolution=(6, 6)):
    m1 = mh.mesh_hemisphere(radius, (0.0, 0.0, 0.0), resolution)
    m2 = mh.mesh_hemisphere(radius, (radius + dx, 0.0, 0.0), resolution)
    mesh = m1 + m2
    h1 = np.zeros((mesh.nfaces, 3))
    h1[:m1.nfaces, 2] = 1.0
    h2 = np.zeros((mesh.nfaces, 3))
    h2[m1.nfaces:, 2] = 1.0
    t = mh.two_hemispheres_tangents(radius, radius + dx, resolution)
    # body 2's centre is r + dx: d/d(dx) moves it, d/dr also scales both bodies
    return mesh, [h1, h2], {"dx": t["separation"], "r": t["radius"] + t["separation"]}


WU_GFS = lambda mh: (mh.Rankine(), mh.RankineReflected(), mh.GFWu())


@pytest.mark.parametrize("table,which", [("pair_sensitivity_dx", "dx"), ("pair_sensitivity_dr", "r")])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_pair_gradients_match_reference_zygote(mh, gpu, table, which, precision):
    p = PINS[table]
    dA, dB, vA, vB = [], [], [], []
    for dx in p["dx"]:
        mesh, dofs, tan = _pair(mh, p["radius"], dx)
        kw = dict(green_functions=WU_GFS(mh), direct=True, precision=precision, tol=1e-12,
                  rho=p["rho"], g=p["g_wavenumber"], ctx=gpu)
        j = mh.hydro_batch_jvp(mesh, [p["omega"]], dofs, [], t_mesh=tan[which], **kw)
        dA.append(j.d_added_mass[0, 0, 0])
        dB.append(j.d_damping[0, 0, 0])
        e = np.zeros((2, 2, 1))
        e[0, 0, 0] = 1.0
        rA = mh.hydro_batch_vjp(mesh, [p["omega"]], dofs, [], e, None, **kw)
        rB = mh.hydro_batch_vjp(mesh, [p["omega"]], dofs, [], None, e, **kw)
        vA.append(rA.mesh.dot(tan[which]))
        vB.append(rB.mesh.dot(tan[which]))
    for got, ref in ((dA, p["dA11"]), (dB, p["dB11"]), (vA, p["dA11"]), (vB, p["dB11"])):
        ref = np.asarray(ref)
        err = np.max(np.abs(np.asarray(got) - ref)) / np.max(np.abs(ref))
        assert err <= 1e-6, (table, err)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_dimensionless_gradients_match_reference_zygote(mh, gpu, precision):
    p = PINS["pair_sensitivity_dimensionless"]
    r = p["radius"]
    dxr = np.asarray(p["dx_r_ratio"])
    kr = np.asarray(p["kr"])
    dA_ref, dB_ref = np.asarray(p["dA21_dr"]), np.asarray(p["dB21_dr"])
    dA, dB = np.zeros_like(dA_ref), np.zeros_like(dB_ref)
    for ratio in np.unique(dxr):
        rows = np.nonzero(dxr == ratio)[0]
        omegas = np.sqrt(kr[rows] * 9.8 / r)
        mesh, dofs, tan = _pair(mh, r, ratio * r)
        j = mh.hydro_batch_jvp(mesh, omegas, dofs, [], t_mesh=tan["r"], green_functions=WU_GFS(mh),
                               direct=True, precision=precision, tol=1e-12, rho=p["rho"],
                               g=p["g_wavenumber"], ctx=gpu)
        dA[rows] = j.d_added_mass[1, 0, :]
        dB[rows] = j.d_damping[1, 0, :]
    assert np.max(np.abs(dA - dA_ref)) <= 1e-6 * np.max(np.abs(dA_ref))
    assert np.max(np.abs(dB - dB_ref)) <= 1e-6 * np.max(np.abs(dB_ref))


# --------------------------------------------------------------------------
# central differences of the oracle
# --------------------------------------------------------------------------

def _gfs(mh, mask):
    t = [mh.Rankine(), mh.RankineReflected()]
    if mask & 8:
        t.append(mh.GFWu())
    if mask & 16:
        t.append(mh.ExactGuevelDelhommeau())
    return tuple(t)


@pytest.mark.parametrize("name", ["grad_fd_wu_direct", "grad_fd_wu_indirect", "grad_fd_delh_direct",
                                  "grad_fd_delh_indirect"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gradients_match_oracle_differences(mh, gpu, name, precision):
    fx = dict(np.load(GOLDEN / f"{name}.npz"))
    res = tuple(int(x) for x in fx["resolution"])
    mesh = mh.mesh_hemisphere(1.0, (0.0, 0.0, 0.0), res)
    dofs = [mh.translational_dofs(mesh, "Heave"), mh.translational_dofs(mesh, "Surge")]
    om = fx["omegas"]
    kw = dict(green_functions=_gfs(mh, int(fx["gf_mask"])), direct=bool(fx["direct"]), precision=precision,
              tol=1e-12, rho=1000.0, g=9.81, ctx=gpu)
    r = mh.hydro_batch_vjp(mesh, om, dofs, [0.0], fx["wA"], fx["wB"], fx["wF"], fx["wK"], **kw)
    t_rad = mh.hemisphere_tangents(1.0, (0.0, 0.0, 0.0), res)["radius"]
    t_ver = mh.polygon_geometry_jvp(mesh.vertices, mesh.faces, fx["vertex_direction"])
    adj = {"radius": r.mesh.dot(t_rad), "omega": float(np.sum(r.omegas)), "vertices": r.mesh.dot(t_ver)}

    def jvp(**t):
        j = mh.hydro_batch_jvp(mesh, om, dofs, [0.0], **t, **kw)
        return float(np.sum(fx["wA"] * j.d_added_mass) + np.sum(fx["wB"] * j.d_damping)
                     + np.real(np.sum(np.conj(fx["wF"]) * j.d_diffraction))
                     + np.real(np.sum(np.conj(fx["wK"]) * j.d_froude_krylov)))

    fwd = {"radius": jvp(t_mesh=t_rad), "omega": jvp(t_omegas=np.ones_like(om)), "vertices": jvp(t_mesh=t_ver)}
    J = float(np.sum(fx["wA"] * r.added_mass) + np.sum(fx["wB"] * r.damping)
              + np.real(np.sum(np.conj(fx["wF"]) * r.diffraction))
              + np.real(np.sum(np.conj(fx["wK"]) * r.froude_krylov)))
    assert abs(J - float(fx["J"])) <= 1e-9 * abs(float(fx["J"]))
    for k in ("radius", "omega", "vertices"):
        ref = float(fx[f"fd_{k}"])
        scale = max(abs(ref), 1e-3 * abs(float(fx["J"])))
        assert abs(adj[k] - ref) <= 1e-5 * scale, (k, "adjoint", adj[k], ref)
        assert abs(fwd[k] - ref) <= 1e-5 * scale, (k, "forward mode", fwd[k], ref)
