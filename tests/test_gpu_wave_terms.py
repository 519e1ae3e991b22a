"""Wave terms on the device against the CPU oracle (GPU).

The tabulated Guevel-Delhommeau term is checked point-wise against the
oracle's adaptive quadrature over the whole tabulated region (polar patch,
Cartesian cells, their borders and the fallback outside), with tolerance
1e-10 * max(1, |value|); the Wu term against the oracle's restatement with
1e-12.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WU, DELH = 8, 16


def _points(rng, n):
    r = np.concatenate([rng.uniform(0, 1.5, n), rng.uniform(0, 16, n), rng.uniform(0, 3, n),
                        [0.0, 0.0, 1.0, 1.5, 1.49999, 15.99, 17.0, 20.0, 0.3]])
    z = -np.concatenate([rng.uniform(1e-3, 1.5, n), rng.uniform(1e-3, 16, n),
                         10 ** rng.uniform(-3, 0, n),
                         [0.01, 2.0, 1e-3, 1e-3, 0.5, 15.99, 1.0, 0.5, 18.0]])
    return r, z


def test_delhommeau_table_pointwise(mh, oracle, gpu):
    rng = np.random.default_rng(7)
    r, z = _points(rng, 150)
    G, Gr, Gz = gpu.wave_term(DELH, r, z)
    for q in range(r.shape[0]):
        g, gr, gz = oracle.delhommeau_dimless(r[q], z[q])
        for got, ref in ((G[q], g), (Gr[q], gr), (Gz[q], gz)):
            assert abs(got - ref) <= 1e-10 * max(1.0, abs(ref)), (r[q], z[q], got, ref)


def test_delhommeau_exact_method_pointwise(mh, oracle, gpu):
    rng = np.random.default_rng(8)
    r, z = _points(rng, 20)
    gpu.set_delhommeau_method("exact")
    try:
        G, Gr, _ = gpu.wave_term(DELH, r, z)
    finally:
        gpu.set_delhommeau_method("table")
    for q in range(r.shape[0]):
        g, gr, _ = oracle.delhommeau_dimless(r[q], z[q])
        assert abs(G[q] - g) <= 1e-11 * max(1.0, abs(g))
        assert abs(Gr[q] - gr) <= 1e-11 * max(1.0, abs(gr))


def test_wu_pointwise(mh, oracle, gpu):
    rng = np.random.default_rng(9)
    r, z = _points(rng, 100)
    G, Gr, Gz = gpu.wave_term(WU, r, z)
    for q in range(r.shape[0]):
        g, gr, gz = oracle.wu_dimless(r[q], z[q])
        for got, ref in ((G[q], g), (Gr[q], gr), (Gz[q], gz)):
            assert abs(got - ref) <= 1e-12 * max(1.0, abs(ref)), (r[q], z[q], got, ref)


def test_delhommeau_reference_goldens_on_device(mh, gpu):
    """test/greens_function.jl:81-83 through the device table."""
    import json
    import pathlib

    pins = json.loads((pathlib.Path(__file__).parent / "golden" /
                       "reference_pins.json").read_text())["delhommeau_dimless_r1_zm1"]
    G, Gr, _ = gpu.wave_term(DELH, [1.0], [-1.0])
    assert abs(G[0] - complex(*pins["G"])) < pins["atol"]
    assert abs(Gr[0] - complex(*pins["dG_dr"])) < pins["atol"]


def test_assembly_exact_vs_table(mh, oracle, gpu):
    mesh = mh.mesh_hemisphere(1.0, (0, 0, 0), (8, 12))
    gfs = (mh.Rankine(), mh.RankineReflected(), mh.ExactGuevelDelhommeau())
    So, Do = oracle.assemble(mesh, 0.8, mh.gf_mask(gfs), True)
    St, Dt = mh.assemble_matrices(gfs, mesh, 0.8, ctx=gpu)
    gpu.set_delhommeau_method("exact")
    try:
        Se, De = mh.assemble_matrices(gfs, mesh, 0.8, ctx=gpu)
    finally:
        gpu.set_delhommeau_method("table")
    scale = np.max(np.abs(So))
    assert np.max(np.abs(St - So)) / scale < 1e-11
    assert np.max(np.abs(Se - So)) / scale < 1e-11
    assert np.max(np.abs(Dt - Do)) / np.max(np.abs(Do)) < 1e-11
