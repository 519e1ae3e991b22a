"""The CPU oracle against the reference's own golden values and an
independent scipy restatement (CPU only)."""
from __future__ import annotations

import json
import math
import pathlib

import numpy as np
import pytest

PINS = json.loads((pathlib.Path(__file__).parent / "golden" / "reference_pins.json").read_text())

E1 = dict(center=[0.0, 0.0, -1.0])
E2 = dict(center=[1.0, 1.0, -2.0],
          vertices=np.array([[-0.5, -0.5, 0.0], [0.5, -0.5, 0.0], [0.5, 0.5, 0.0],
                             [-0.5, 0.5, 0.0]]) + np.array([1.0, 1.0, -2.0]),
          normal=[0.0, 0.0, 1.0], area=1.0, radius=math.sqrt(2) / 2)


def _sym(e):
    """free_surface_symmetry of an element (src/meshes.jl:212-230)."""
    out = dict(e)
    c = np.array(e["center"], dtype=float)
    out["center"] = [c[0], c[1], -c[2]]
    if "normal" in e:
        n = np.array(e["normal"], dtype=float)
        out["normal"] = [n[0], n[1], -n[2]]
        v = np.array(e["vertices"], dtype=float)[::-1].copy()
        v[:, 2] *= -1
        out["vertices"] = v
    return out


def test_expint_e1_against_scipy(oracle):
    from scipy.special import exp1

    rng = np.random.default_rng(0)
    zs = list(rng.uniform(-12, 0.5, 300) + 1j * rng.uniform(0, 12, 300))
    zs += [complex(-x, 1e-17) for x in (0.01, 0.5, 3.0, 8.0, 20.0)]
    zs += [complex(x, y) for x in (-3.0, -0.5, 0.5, 3.0) for y in (0.01, 2.0, 5.0)]
    for z in zs:
        got = oracle.expint_e1(z)
        ref = exp1(z)
        assert abs(got - ref) <= 3e-13 * abs(ref), (z, got, ref)


def test_rankine_point_pins(oracle):
    """test/greens_function.jl:44-46 and :71-73: panel integral ~ one-point
    value (atol 1e-1), and the reflection identities :62-64."""
    x = E1["center"]
    one_point = 1 / math.sqrt(3) * E2["area"]
    assert abs(oracle.rankine_integral(x, E2) - one_point) < 1e-1
    g_first = oracle.rankine_integral_gradient(x, E2, True)
    expect = (np.array(E2["center"]) - np.array(x)) / math.sqrt(3) ** 3
    assert np.allclose(g_first, expect, atol=1e-1)
    xr = [x[0], x[1], -x[2]]
    assert abs(oracle.rankine_integral(xr, E2) - 1 / math.sqrt(11)) < 1e-1
    # integral(Rankine, sym(e1), e2) == integral(Rankine, e1, sym(e2))
    a = oracle.rankine_integral(xr, E2)
    b = oracle.rankine_integral(x, _sym(E2))
    assert abs(a - b) < 1e-12 * abs(a)
    for first in (True, False):
        ga = oracle.rankine_integral_gradient(xr, E2, first)
        gb = oracle.rankine_integral_gradient(x, _sym(E2), first)
        gb[2] = -gb[2]
        assert np.allclose(ga, gb, rtol=1e-12, atol=1e-14)


def test_delhommeau_dimless_golden(oracle):
    p = PINS["delhommeau_dimless_r1_zm1"]
    G, Gr, _ = oracle.delhommeau_dimless(1.0, -1.0)
    assert abs(G - complex(*p["G"])) < p["atol"]
    assert abs(Gr - complex(*p["dG_dr"])) < p["atol"]


def test_delhommeau_greens_golden(oracle):
    """k*G and the first-variable gradient for the reference's test
    elements at k = 1 (test/greens_function.jl:88-92); the oracle's
    one-point integral over a unit-area panel is k*G."""
    p = PINS["delhommeau_greens_k1"]
    s, g = oracle.pair_integrals(p["e1_center"], E2, p["wavenumber"], oracle.GF_DELHOMMEAU, True)
    assert abs(s - complex(*p["G"])) < p["atol"]
    for c in range(3):
        assert abs(g[c] - complex(*p["grad_first_variable"][c])) < p["atol"]


def _scipy_delhommeau(r, z):
    from scipy.integrate import quad
    from scipy.special import exp1

    def parts(t):
        c = math.cos(t)
        zeta = z + 1j * r * c
        ez = np.exp(zeta)
        j = ez * (exp1(zeta) / math.pi + 1j)
        return (j.real, ez.real, (1j * c * (j - 1 / (math.pi * zeta))).real, (1j * c * ez).real)

    vals = [quad(lambda t, q=q: parts(t)[q], 0, math.pi / 2, epsabs=1e-14, epsrel=1e-13,
                 limit=400)[0] for q in range(4)]
    return 4 * complex(vals[0], vals[1]), 4 * complex(vals[2], vals[3])


@pytest.mark.parametrize("r,z", [(0.0, -0.3), (0.1, -0.05), (1.0, -1.0), (2.5, -0.2),
                                 (0.02, -0.001), (4.0, -3.0), (8.0, -0.5)])
def test_delhommeau_against_scipy(oracle, r, z):
    G, Gr, Gz = oracle.delhommeau_dimless(r, z)
    Gs, Grs = _scipy_delhommeau(r, z)
    assert abs(G - Gs) <= 1e-10 * max(1.0, abs(Gs))
    assert abs(Gr - Grs) <= 1e-10 * max(1.0, abs(Grs))
    assert abs(Gz - (G + 2 / math.hypot(r, z))) < 1e-14 * max(1.0, abs(Gz))
    # Im G is 2 pi e^z J0(r) in closed form
    from scipy.special import j0

    assert abs(G.imag - 2 * math.pi * math.exp(z) * j0(r)) < 1e-11


@pytest.mark.parametrize("k", [0.1, 1.0, 10.0])
def test_wu_close_to_delhommeau(oracle, k):
    """test/greens_function.jl:96-99 (atol 2e-2)."""
    x = E1["center"]
    sd, gd = oracle.pair_integrals(x, E2, k, oracle.GF_DELHOMMEAU, False)
    sw, gw = oracle.pair_integrals(x, E2, k, oracle.GF_WU, False)
    assert abs(sd - sw) < 2e-2
    assert np.all(np.abs(gd - gw) < 2e-2)


def test_hulme_heave_table(mh, oracle):
    """test/consistency_with_analytical_solutions.jl:13-39 (Wu, rtol 1e-1,
    norm-wise as Julia's isapprox on arrays), on this package's 10 x 10
    hemisphere (Capytaine's mesh is not available)."""
    p = PINS["hulme_heave"]
    mesh = mh.mesh_hemisphere(1.0, (0, 0, 0), (10, 10))
    K = np.array(p["K"])
    w = np.sqrt(K * 9.8)
    for rho in (1000.0, 1025.0):
        AB = np.array([oracle.calculate_radiation_forces(mesh, [0, 0, 1.0], x, rho=rho, g=9.81)
                       for x in w])
        A = AB[:, 0] / ((2 / 3) * math.pi * rho)
        B = AB[:, 1] / ((2 / 3) * math.pi * rho) / w
        for got, ref in ((A, np.array(p["A"])), (B, np.array(p["B"]))):
            err = np.linalg.norm(got - ref) / max(np.linalg.norm(got), np.linalg.norm(ref))
            assert err <= p["rtol"]


def test_direct_vs_indirect_shapes(mh, oracle):
    """test/matrix_assembly.jl:9-23: S(direct) == S(indirect), D != K."""
    mesh = mh.mesh_hemisphere(1.0, (0, 0, 0), (6, 6))
    gfs = oracle.GF_RANKINE | oracle.GF_RANKINE_REFLECTED
    S, D = oracle.assemble(mesh, 1.0, gfs, True)
    S2, K = oracle.assemble(mesh, 1.0, gfs, False)
    assert S.shape == D.shape == S2.shape == K.shape == (mesh.nfaces, mesh.nfaces)
    assert np.array_equal(S, S2)
    assert not np.allclose(D, K)


def test_rankine_self_consistency(mh, oracle):
    """Gauss: for a closed Rankine surface the direct D rows sum to about 1
    (solid angle); on the open hemisphere the sum of D is bounded."""
    mesh = mh.mesh_hemisphere(1.0, (0, 0, 0), (12, 12))
    _, D = oracle.assemble(mesh, 1.0, oracle.GF_RANKINE, True)
    assert np.all(np.isfinite(D))
    assert np.all(np.abs(D.imag) == 0.0)
    assert np.allclose(np.diag(D).real, 0.5, atol=0.2)


def test_gk15_rule_exactness(oracle):
    """The adaptive rule integrates the r = 0 integrand (constant in theta)
    to machine precision: 4 * (pi/2) * Re(e^z (E1(z)/pi + i))."""
    z = -0.7
    G, _, _ = oracle.delhommeau_dimless(0.0, z)
    e1 = oracle.expint_e1(complex(z, 0.0))
    j = math.exp(z) * (e1 / math.pi + 1j)
    assert abs(G.real - 2 * math.pi * j.real) < 1e-13
    assert abs(G.imag - 2 * math.pi * math.exp(z)) < 1e-13


def _pair_coefficients(mh, oracle, radius, dx, omega, resolution=(6, 6)):
    """A, B (2 x 2) of two heaving hemispheres, body 2 centred at
    x = radius + dx; column j = radiation of body j (paper/ArraySensitivities.jl:16-50)."""
    m1 = mh.mesh_hemisphere(radius, (0.0, 0.0, 0.0), resolution)
    m2 = mh.mesh_hemisphere(radius, (radius + dx, 0.0, 0.0), resolution)
    mesh = m1 + m2
    h1 = np.zeros((mesh.nfaces, 3))
    h1[:m1.nfaces, 2] = 1.0
    h2 = np.zeros((mesh.nfaces, 3))
    h2[m1.nfaces:, 2] = 1.0
    A, B, _, _ = oracle.hydro_coefficients(mesh, [omega], [h1, h2], [], 1000.0, 9.81,
                                           oracle.GF_RANKINE | oracle.GF_RANKINE_REFLECTED | oracle.GF_WU,
                                           True, 1)
    return A[:, :, 0], B[:, :, 0]


def _pair_fd(mh, oracle, radius, dx, omega, which, h=1e-6):
    if which == "dx":
        p, m = (radius, dx + h), (radius, dx - h)
    else:
        p, m = (radius + h, dx), (radius - h, dx)
    Ap, Bp = _pair_coefficients(mh, oracle, *p, omega)
    Am, Bm = _pair_coefficients(mh, oracle, *m, omega)
    return (Ap - Am) / (2 * h), (Bp - Bm) / (2 * h)


@pytest.mark.parametrize("table,which", [("pair_sensitivity_dx", "dx"), ("pair_sensitivity_dr", "r")])
def test_oracle_reproduces_reference_pair_gradients(mh, oracle, table, which):
    """The reference's own Zygote gradients of two 6 x 6 hemispheres
    (paper/Plots/11_heuristics_d{x,r}_DELhommeau.csv, written by
    paper/ArraySensitivities.jl:52-68 through the finite-difference mesh
    rrules of paper/meshGradients_pair.jl) against central differences
    (h = 1e-6) of the oracle on this package's hemisphere mesh.  Agreement to
    1e-6 of each column's scale pins the oracle, the mesh generator (the
    stand-in for Capytaine's sphere) and the solve at once."""
    p = PINS[table]
    dA_ref, dB_ref = np.array(p["dA11"]), np.array(p["dB11"])
    got = [_pair_fd(mh, oracle, p["radius"], dx, p["omega"], which) for dx in p["dx"]]
    dA = np.array([g[0][0, 0] for g in got])
    dB = np.array([g[1][0, 0] for g in got])
    assert np.max(np.abs(dA - dA_ref)) <= 1e-6 * np.max(np.abs(dA_ref))
    assert np.max(np.abs(dB - dB_ref)) <= 1e-6 * np.max(np.abs(dB_ref))


def test_oracle_reproduces_reference_dimensionless_gradients(mh, oracle):
    """dA21/dr and dB21/dr on the reference's (dx/r, kr) grid
    (paper/Plots/added_mass_data_dimensionless.csv and
    damping_data_dimensionless.csv; omega = sqrt(kr 9.8 / r), k = omega^2 / 9.81
    as in paper/ArraySensitivities.jl:71-97): every row."""
    p = PINS["pair_sensitivity_dimensionless"]
    r = p["radius"]
    dA, dB = [], []
    for dxr, kr in zip(p["dx_r_ratio"], p["kr"]):
        gA, gB = _pair_fd(mh, oracle, r, dxr * r, math.sqrt(kr * 9.8 / r), "r")
        dA.append(gA[1, 0])
        dB.append(gB[1, 0])
    dA_ref, dB_ref = np.array(p["dA21_dr"]), np.array(p["dB21_dr"])
    assert np.max(np.abs(np.array(dA) - dA_ref)) <= 1e-6 * np.max(np.abs(dA_ref))
    assert np.max(np.abs(np.array(dB) - dB_ref)) <= 1e-6 * np.max(np.abs(dB_ref))


@pytest.mark.parametrize("name", ["grad_fd_wu_direct", "grad_fd_delh_indirect"])
def test_gradient_fixture_reproduces(mh, oracle, name):
    """The committed gradient anchors are the oracle's own numbers: the
    objective value at the base point is recomputed here."""
    fx = np.load(pathlib.Path(__file__).parent / "golden" / f"{name}.npz")
    mesh = mh.mesh_hemisphere(1.0, (0.0, 0.0, 0.0), tuple(int(x) for x in fx["resolution"]))
    dofs = [np.tile([0.0, 0.0, 1.0], (mesh.nfaces, 1)), np.tile([1.0, 0.0, 0.0], (mesh.nfaces, 1))]
    A, B, Fd, Fk = oracle.hydro_coefficients(mesh, fx["omegas"], dofs, [0.0], 1000.0, 9.81, int(fx["gf_mask"]),
                                             bool(fx["direct"]))
    J = (np.sum(fx["wA"] * A) + np.sum(fx["wB"] * B) + np.real(np.sum(np.conj(fx["wF"]) * Fd))
         + np.real(np.sum(np.conj(fx["wK"]) * Fk)))
    assert abs(J - float(fx["J"])) <= 1e-12 * abs(float(fx["J"]))


def test_size_fixture_reproduces(mh, oracle):
    """The 1024-panel exact-Delhommeau fixture: A, B and two sampled S, D
    entries recomputed from the oracle."""
    fx = np.load(pathlib.Path(__file__).parent / "golden" / "hemisphere_1024p_delhommeau.npz")
    mesh = mh.mesh_hemisphere(1.0, (0.0, 0.0, 0.0), (32, 64))
    heave = np.tile([0.0, 0.0, 1.0], (mesh.nfaces, 1))
    A, B, _, _ = oracle.hydro_coefficients(mesh, fx["omegas"], [heave], [], 1000.0, 9.81, int(fx["gf_mask"]), True)
    assert abs(A[0, 0, 0] - fx["added_mass"][0, 0, 0]) <= 1e-12 * abs(fx["added_mass"][0, 0, 0])
    assert abs(B[0, 0, 0] - fx["damping"][0, 0, 0]) <= 1e-12 * abs(fx["damping"][0, 0, 0])
