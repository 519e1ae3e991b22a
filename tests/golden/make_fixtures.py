#!/usr/bin/env python
"""Generate the oracle fixtures that pin the CUDA path at full size.

Every number here comes from the FP64 CPU oracle (``oracle/``: the C
restatement of the reference's Green functions and assembly, exact adaptive
quadrature for the Guevel-Delhommeau term, LAPACK for the solve); the GPU
tests and ``bench.py``'s accuracy block compare the device results against
these files.  The oracle is the checker; nothing here is product code.

Cases (all meshes from ``mesh_hemisphere``, the stand-in for Capytaine's
``mesh_sphere(...).immersed_part()``):

  hemisphere_1024p_delhommeau   R = 1, 32 x 64 (1024 panels), omega = 1.03,
                                heave, heading 0, Rankine + reflected +
                                exact Delhommeau, direct: A, B, F, FK
  hemisphere_2048p_delhommeau   R = 1, 64 x 64 (2048 panels), the 64
                                frequencies linspace(0.3, 3.0, 64), heave and
                                surge, heading 0, Rankine + reflected + exact
                                Delhommeau, direct: A, B, F, FK at every
                                frequency, S and D sampled at three of them
  two_hemispheres_2048p_wu      two hemispheres R = 1, centres 5 m apart
                                (2 x 1024 panels), omega = 1.03, heave of both
                                bodies, Rankine + reflected + Wu, indirect:
                                A, B, F, FK, S and K sampled, and the
                                two-body power J(r1, dx1, omega) of
                                paper/Power.jl:13-83 with its central
                                differences (h = 1e-6) in r1, dx1 and omega
  grad_fd_<wu|delh>_<direct|indirect>
                                a 100-panel hemisphere (10 x 20), omegas
                                (0.7, 1.4), heave and surge, heading 0, a
                                seeded objective J = sum(wA A) + sum(wB B)
                                + Re sum(conj(wF) F) + Re sum(conj(wK) FK):
                                central differences (h = 1e-6) of J along the
                                radius, the frequencies and a seeded vertex
                                direction (geometry recomputed from the moved
                                vertices) -- the independent anchor of the
                                adjoint and forward-mode gradients

    python tests/golden/make_fixtures.py [--case NAME ...] [--threads T]

Writes ``tests/golden/<case>.npz``.  Runtime on 8 cores: about 50 s per
2048-panel exact-Delhommeau frequency (the 64-frequency case dominates).
"""
from __future__ import annotations

import argparse
import importlib.util
import math
import pathlib
import sys
import time

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

import oracle as O  # noqa: E402

MASK_DELH = O.GF_RANKINE | O.GF_RANKINE_REFLECTED | O.GF_DELHOMMEAU
MASK_WU = O.GF_RANKINE | O.GF_RANKINE_REFLECTED | O.GF_WU
G = 9.81
RHO = 1000.0


def load_package():
    name = "marinehydro_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg_dir = ROOT / "marinehydro.jl_b200"
    spec = importlib.util.spec_from_file_location(
        name, pkg_dir / "__init__.py", submodule_search_locations=[str(pkg_dir)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def sample_indices(n: int, seed: int):
    """(rows, cols) of sampled matrix entries: 256 random pairs, 128 diagonal
    entries and 128 neighbours (i, i+1) -- the near field, where the panel
    integrals and the wave term's log singularity are hardest."""
    rng = np.random.default_rng(seed)
    r = rng.integers(0, n, 256)
    c = rng.integers(0, n, 256)
    d = rng.choice(n, 128, replace=False)
    e = rng.choice(n - 1, 128, replace=False)
    rows = np.concatenate([r, d, e])
    cols = np.concatenate([c, d, e + 1])
    return rows.astype(np.int64), cols.astype(np.int64)


def mesh_fingerprint(mesh):
    return np.array([mesh.nfaces, np.sum(mesh.centers), np.sum(mesh.normals), np.sum(mesh.areas),
                     np.sum(mesh.radii), np.sum(mesh.vertices)])


def run_case(mesh, omegas, dofs, betas, mask, direct, threads, sample_at=(), seed=0):
    nd, nw, nb = len(dofs), len(omegas), len(betas)
    A = np.zeros((nd, nd, nw))
    B = np.zeros((nd, nd, nw))
    Fd = np.zeros((nd, nw, nb), dtype=np.complex128)
    Fk = np.zeros((nd, nw, nb), dtype=np.complex128)
    rows, cols = sample_indices(mesh.nfaces, seed)
    S_s, D_s = [], []
    for w_i, w in enumerate(omegas):
        t0 = time.time()
        S, D = O.assemble(mesh, w * w / G, mask, direct, threads)
        A[:, :, w_i], B[:, :, w_i], Fd[:, w_i, :], Fk[:, w_i, :] = O.coefficients_from_matrices(
            mesh, S, D, w, dofs, betas, RHO, G, direct)
        if w_i in sample_at:
            S_s.append(S[rows, cols])
            D_s.append(D[rows, cols])
        print(f"  omega {w:.4f}: {time.time() - t0:.1f} s", flush=True)
    out = dict(omegas=np.asarray(omegas, dtype=np.float64), betas=np.asarray(betas, dtype=np.float64),
               added_mass=A, damping=B, diffraction=Fd, froude_krylov=Fk, gf_mask=np.int64(mask),
               direct=np.int64(bool(direct)), fingerprint=mesh_fingerprint(mesh), g=G, rho=RHO)
    if sample_at:
        out.update(sample_omega_index=np.asarray(sample_at, dtype=np.int64), sample_rows=rows,
                   sample_cols=cols, S_samples=np.asarray(S_s), D_samples=np.asarray(D_s))
    return out


# --------------------------------------------------------------------------
# the two-body power objective (paper/Power.jl:13-83), numpy form
# --------------------------------------------------------------------------

def power_objective(A, B, Fd, Fk, w, r1, rho=RHO, rho_diffraction=1023.0, g=G):
    """J from the boundary-element outputs of the two heaving hemispheres:
    A, B (2 x 2) with the radiation of sphere 1 in column 0, Fd, Fk (2,)."""
    C = rho * g * math.pi * r1 ** 2
    M = C
    A11, A12, B11, B12 = A[0, 0], A[1, 0], B[0, 0], B[1, 0]
    Am = np.array([[A11, A12], [A12, A11]])
    Bm = np.array([[B11, B12], [B12, B11]])
    pto = np.array([B11, B11])
    H = w ** 2 * (M * np.eye(2) + Am) - 1j * w * (Bm + np.diag(pto)) + C * np.eye(2)
    F = rho_diffraction / rho * Fd + Fk
    Xi = np.linalg.solve(H, F)
    P = 0.5 * pto * np.abs(1j * w * Xi) ** 2
    return float(np.sum(P) / ((2.0 / 3.0) * math.pi * r1 ** 3))


def two_body(mh, r1, dx1, resolution):
    m1 = mh.mesh_hemisphere(r1, (0.0, 0.0, 0.0), resolution)
    m2 = mh.mesh_hemisphere(r1, (r1 + dx1, 0.0, 0.0), resolution)
    body = mh.FloatingBody.rigid(m1, ["Heave"], body_name="sphere") + \
        mh.FloatingBody.rigid(m2, ["Heave"], body_name="sphere")
    return body.mesh, list(body.dofs.values())


def power_at(mh, r1, dx1, w, resolution, threads):
    mesh, dofs = two_body(mh, r1, dx1, resolution)
    S, K = O.assemble(mesh, w * w / G, MASK_WU, False, threads)
    A, B, Fd, Fk = O.coefficients_from_matrices(mesh, S, K, w, dofs, [0.0], RHO, G, False)
    return power_objective(A, B, Fd[:, 0], Fk[:, 0], w, r1)


# --------------------------------------------------------------------------
# gradient anchors on a small hemisphere
# --------------------------------------------------------------------------

GRAD_RES = (10, 20)
GRAD_OMEGAS = (0.7, 1.4)


def grad_weights(nd=2, nw=2, nb=1, seed=7):
    rng = np.random.default_rng(seed)
    wA = rng.standard_normal((nd, nd, nw))
    wB = rng.standard_normal((nd, nd, nw))
    wF = rng.standard_normal((nd, nw, nb)) + 1j * rng.standard_normal((nd, nw, nb))
    wK = rng.standard_normal((nd, nw, nb)) + 1j * rng.standard_normal((nd, nw, nb))
    return wA, wB, wF, wK


def grad_vertex_direction(nv, seed=11):
    return 0.1 * np.random.default_rng(seed).standard_normal((nv, 3))


def grad_objective(mh, mesh, omegas, mask, direct, threads):
    dofs = [np.tile([0.0, 0.0, 1.0], (mesh.nfaces, 1)), np.tile([1.0, 0.0, 0.0], (mesh.nfaces, 1))]
    A, B, Fd, Fk = O.hydro_coefficients(mesh, omegas, dofs, [0.0], RHO, G, mask, direct, threads)
    wA, wB, wF, wK = grad_weights()
    return float(np.sum(wA * A) + np.sum(wB * B) + np.real(np.sum(np.conj(wF) * Fd))
                 + np.real(np.sum(np.conj(wK) * Fk)))


def grad_case(mh, mask, direct, threads, h=1e-6):
    base = mh.mesh_hemisphere(1.0, (0.0, 0.0, 0.0), GRAD_RES)
    om = np.asarray(GRAD_OMEGAS)
    dv = grad_vertex_direction(base.nvertices)

    def moved(s):
        v = base.vertices + s * dv
        c, n, a, r = mh.panel_geometry(v, base.faces)
        return mh.Mesh(v, base.faces.copy(), c, n, a, r)

    J0 = grad_objective(mh, base, om, mask, direct, threads)
    fd = {}
    for name, f in (("radius", lambda s: grad_objective(mh, mh.mesh_hemisphere(1.0 + s, (0.0, 0.0, 0.0),
                                                                              GRAD_RES),
                                                         om, mask, direct, threads)),
                    ("omega", lambda s: grad_objective(mh, base, om + s, mask, direct, threads)),
                    ("vertices", lambda s: grad_objective(mh, moved(s), om, mask, direct, threads))):
        d1 = (f(h) - f(-h)) / (2 * h)
        d2 = (f(2 * h) - f(-2 * h)) / (4 * h)
        fd[name] = d1
        print(f"  dJ/d{name} = {d1:.12e} (2h: {d2:.12e})", flush=True)
    wA, wB, wF, wK = grad_weights()
    return dict(J=J0, fd_radius=fd["radius"], fd_omega=fd["omega"], fd_vertices=fd["vertices"],
                omegas=om, resolution=np.asarray(GRAD_RES), h=h, gf_mask=np.int64(mask),
                direct=np.int64(bool(direct)), fingerprint=mesh_fingerprint(base),
                wA=wA, wB=wB, wF=wF, wK=wK, vertex_direction=dv)


# --------------------------------------------------------------------------

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", action="append")
    ap.add_argument("--threads", type=int, default=0)
    args = ap.parse_args()
    mh = load_package()
    T = args.threads
    heave = np.array([0.0, 0.0, 1.0])
    surge = np.array([1.0, 0.0, 0.0])
    cases = {}

    def hemi1024():
        m = mh.mesh_hemisphere(1.0, (0.0, 0.0, 0.0), (32, 64))
        dofs = [np.tile(heave, (m.nfaces, 1))]
        return run_case(m, [1.03], dofs, [0.0], MASK_DELH, True, T, sample_at=(0,), seed=1)

    def hemi2048():
        m = mh.mesh_hemisphere(1.0, (0.0, 0.0, 0.0), (64, 64))
        dofs = [np.tile(heave, (m.nfaces, 1)), np.tile(surge, (m.nfaces, 1))]
        om = np.linspace(0.3, 3.0, 64)
        return run_case(m, om, dofs, [0.0], MASK_DELH, True, T, sample_at=(0, 32, 63), seed=2)

    def two2048():
        res = (32, 64)
        mesh, dofs = two_body(mh, 1.0, 4.0, res)
        out = run_case(mesh, [1.03], dofs, [0.0], MASK_WU, False, T, sample_at=(0,), seed=3)
        h = 1e-6
        J = power_objective(out["added_mass"][:, :, 0], out["damping"][:, :, 0],
                            out["diffraction"][:, 0, 0], out["froude_krylov"][:, 0, 0], 1.03, 1.0)
        fd = {}
        for name, (dr, dd, dw) in (("r1", (1, 0, 0)), ("dx1", (0, 1, 0)), ("omega", (0, 0, 1))):
            p = power_at(mh, 1.0 + h * dr, 4.0 + h * dd, 1.03 + h * dw, res, T)
            m_ = power_at(mh, 1.0 - h * dr, 4.0 - h * dd, 1.03 - h * dw, res, T)
            fd[name] = (p - m_) / (2 * h)
            print(f"  dJ/d{name} = {fd[name]:.12e}", flush=True)
        out.update(power=J, fd_r1=fd["r1"], fd_dx1=fd["dx1"], fd_omega=fd["omega"], fd_h=h,
                   r1=1.0, dx1=4.0)
        return out

    cases["hemisphere_1024p_delhommeau"] = hemi1024
    cases["hemisphere_2048p_delhommeau"] = hemi2048
    cases["two_hemispheres_2048p_wu"] = two2048
    for gname, mask in (("wu", MASK_WU), ("delh", MASK_DELH)):
        for dname, direct in (("direct", True), ("indirect", False)):
            cases[f"grad_fd_{gname}_{dname}"] = (lambda m=mask, d=direct: grad_case(mh, m, d, T))
    todo = args.case or list(cases)
    for name in todo:
        print(name, flush=True)
        t0 = time.time()
        out = cases[name]()
        np.savez_compressed(HERE / f"{name}.npz", **out)
        print(f"  wrote {name}.npz ({time.time() - t0:.0f} s)", flush=True)


if __name__ == "__main__":
    main()
