"""C-ABI library loading/exports, mesh generation and host-side logic (CPU)."""
from __future__ import annotations

import ctypes
import pathlib
import re

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(mh_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol(mh):
    lib = mh.native.lib()
    declared = _declared_symbols()
    assert declared, "no declarations found in include/*.h"
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing
    # the ctypes signature table covers the same set
    assert set(mh.native.SIGNATURES) == declared


def test_version_and_device_count(mh):
    assert mh.native.lib().mh_version() >= 100
    assert mh.device_count() >= 0


def test_ctx_create_without_device_reports_error(mh):
    if mh.device_count() > 0:
        pytest.skip("a device is visible")
    with pytest.raises(mh.MarineHydroError) as ei:
        mh.Context(0)
    assert ei.value.code == mh.native.MH_ERR_NO_DEVICE


def test_null_arguments_rejected_without_device(mh):
    L = mh.native.lib()
    assert L.mh_ctx_create(0, None) == mh.native.MH_ERR_ARG
    assert L.mh_device_count(None) == mh.native.MH_ERR_ARG
    assert L.mh_ctx_destroy(None) == 0
    assert L.mh_mesh_nfaces(None, None) == mh.native.MH_ERR_ARG
    assert L.mh_mesh_nvertices(None, None) == mh.native.MH_ERR_ARG
    assert L.mh_mesh_nparams(None, None) == mh.native.MH_ERR_ARG
    assert L.mh_mesh_hemisphere(None, 1.0, 0.0, 0.0, 0.0, 10, 10, None) == mh.native.MH_ERR_ARG
    assert L.mh_mesh_wavebot(None, 0.88, 0.35, 0.16, 0.37, 5, 10, 5, 72, None) == mh.native.MH_ERR_ARG


@pytest.mark.parametrize("res,nf", [((10, 10), 50), ((32, 64), 1024), ((64, 64), 2048),
                                    ((9, 18), 90)])
def test_hemisphere_counts(mh, res, nf):
    m = mh.mesh_hemisphere(1.0, (0, 0, 0), res)
    assert m.nfaces == nf
    assert np.all(m.centers[:, 2] < 0)
    # outward normals: n . (c - centre) > 0
    assert np.all(np.sum(m.normals * m.centers, axis=1) > 0)
    assert np.allclose(np.linalg.norm(m.normals, axis=1), 1.0)
    assert m.areas.sum() < 2 * np.pi and m.areas.sum() > 0.9 * 2 * np.pi


def test_hemisphere_scaling_and_translation(mh):
    m1 = mh.mesh_hemisphere(1.0, (0, 0, 0), (8, 16))
    m2 = mh.mesh_hemisphere(2.0, (3.0, -1.0, 0.0), (8, 16))
    assert np.allclose(m2.areas, 4 * m1.areas)
    assert np.allclose(m2.radii, 2 * m1.radii)
    assert np.allclose(m2.centers, 2 * m1.centers + np.array([3.0, -1.0, 0.0]))
    assert np.allclose(m2.normals, m1.normals)


def test_combine_meshes_offsets_faces(mh):
    a = mh.mesh_hemisphere(1.0, (0, 0, 0), (4, 6))
    b = mh.mesh_hemisphere(1.0, (5, 0, 0), (4, 6))
    c = a + b
    assert c.nfaces == a.nfaces + b.nfaces
    assert c.nvertices == a.nvertices + b.nvertices
    assert np.array_equal(c.faces[a.nfaces:], b.faces + a.nvertices)
    assert np.allclose(c.vertices[c.faces[a.nfaces:]], b.vertices[b.faces])


def test_mesh_shape_checks(mh):
    m = mh.mesh_hemisphere(1.0, (0, 0, 0), (4, 6))
    with pytest.raises(ValueError):
        mh.Mesh(m.vertices[:, :2], m.faces, m.centers, m.normals, m.areas, m.radii)
    with pytest.raises(ValueError):
        mh.Mesh(m.vertices, m.faces[:, :3], m.centers, m.normals, m.areas, m.radii)
    with pytest.raises(ValueError):
        mh.Mesh(m.vertices, m.faces, m.centers[:-1], m.normals, m.areas, m.radii)
    with pytest.raises(ValueError):
        mh.Mesh(m.vertices, m.faces + 1000, m.centers, m.normals, m.areas, m.radii)


def test_gf_mask(mh):
    assert mh.gf_mask(mh.DEFAULT_GREEN_FUNCTIONS) == 1 | 2 | 8
    assert mh.gf_mask((mh.Rankine(), mh.RankineReflected(), mh.ExactGuevelDelhommeau())) == 19
    with pytest.raises(ValueError):
        mh.gf_mask((mh.Rankine(), mh.Rankine()))
    with pytest.raises(ValueError):
        mh.gf_mask(())


def test_host_helpers_match_oracle(mh, oracle):
    m = mh.mesh_hemisphere(1.0, (0.3, 0.1, 0), (8, 12))
    w = 1.03
    assert np.allclose(mh.radiation_bc(m, [0, 0, 1.0], w),
                       oracle.radiation_bc(m.normals, [0, 0, 1.0], w), rtol=1e-15)
    assert np.allclose(mh.AiryBC(m, w, 0.3), oracle.airy_bc(m.centers, m.normals, w, 0.3),
                       rtol=1e-14)
    p = np.random.default_rng(1).standard_normal(m.nfaces) + 0j
    assert np.isclose(mh.integrate_pressure(m, p, [0, 0, 1.0]),
                      oracle.integrate_pressure(m.normals, m.areas, p, [0, 0, 1.0]), rtol=1e-14)
    assert np.isclose(mh.FroudeKrylovForce(m, w, [0, 0, 1.0]),
                      oracle.froude_krylov_force(m, w, [0, 0, 1.0]), rtol=1e-14)


def test_mesh_is_hashable_and_snapshot_tracks_changes(mh):
    """The device-mesh cache is keyed by the mesh object and re-uploads when
    an array was changed in place or replaced by one of another shape."""
    import weakref

    m = mh.mesh_hemisphere(1.0, (0, 0, 0), (4, 6))
    d = weakref.WeakKeyDictionary()
    d[m] = 1
    assert d[m] == 1
    snap = mh.api._mesh_snapshot(m)
    assert mh.api._mesh_unchanged(snap, m)
    m.centers[0, 0] += 1e-3
    assert not mh.api._mesh_unchanged(snap, m)
    m.centers[0, 0] -= 1e-3
    assert mh.api._mesh_unchanged(mh.api._mesh_snapshot(m), m)
    m.areas = np.append(m.areas, 1.0)
    assert not mh.api._mesh_unchanged(snap, m)


def test_rigid_dofs_follow_reference(mh):
    """src/bodies.jl:63-89: translations are unit fields, rotations axis x (x - c)."""
    m = mh.mesh_hemisphere(1.0, (0, 0, 0), (6, 8))
    b = mh.FloatingBody.rigid(m, ["Surge", "Heave", "Pitch", "Yaw"], (1.0, 1.0, 0.0))
    assert np.array_equal(b.dofs["Surge"], np.tile([1.0, 0, 0], (m.nfaces, 1)))
    assert np.array_equal(b.dofs["Heave"], np.tile([0, 0, 1.0], (m.nfaces, 1)))
    pos = m.centers - np.array([1.0, 1.0, 0.0])
    assert np.allclose(b.dofs["Pitch"], np.cross([0, 1.0, 0], pos))
    assert np.allclose(b.dofs["Yaw"], np.cross([0, 0, 1.0], pos))
    with pytest.raises(ValueError):
        mh.FloatingBody.rigid(m, ["Wobble"])


def test_combine_floatingbodies_names(mh):
    """src/bodies.jl:102-170: unique names and zero-padded dof fields."""
    assert mh.make_body_name_list_unique(["a", "a", "a_2", "b"]) == ["a", "a_3", "a_2", "b"]
    m = mh.mesh_hemisphere(1.0, (0, 0, 0), (4, 6))
    b1 = mh.FloatingBody.rigid(m, ["Heave"], body_name="my body")
    b2 = mh.FloatingBody.rigid(m.translated((3, 0, 0)), ["Heave", "Surge"], body_name="my body")
    c = b1 + b2
    assert c.body_name == "my_body+my_body_2"
    assert list(c.dofs) == ["my_body__Heave", "my_body_2__Heave", "my_body_2__Surge"]
    assert np.all(c.dofs["my_body__Heave"][m.nfaces:] == 0)
    assert np.all(c.dofs["my_body_2__Heave"][:m.nfaces] == 0)
    assert np.all(c.dofs["my_body_2__Heave"][m.nfaces:, 2] == 1)
