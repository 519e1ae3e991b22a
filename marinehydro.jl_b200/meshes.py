"""Panel meshes: the ``Mesh`` container, multi-body concatenation and a
hemisphere generator.

``Mesh`` mirrors the reference's struct (src/meshes.jl:12-37): vertices
(V x 3), faces (N x 4, 0-based vertex indices; triangles repeat a vertex),
centers and normals (N x 3), areas and radii (N).  Arrays are held as numpy
float64 / int64; the C-ABI receives them column-major, as Julia stores them.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Sequence

import numpy as np


@dataclass(eq=False)
class Mesh:
    """Panel mesh (src/meshes.jl:12-37).  The constructor checks the same
    shapes as the reference's inner constructor (src/meshes.jl:27-34).
    Meshes compare and hash by identity (device uploads are cached per object)."""

    vertices: np.ndarray
    faces: np.ndarray
    centers: np.ndarray
    normals: np.ndarray
    areas: np.ndarray
    radii: np.ndarray
    nvertices: int = -1
    nfaces: int = -1

    def __post_init__(self):
        self.vertices = np.asarray(self.vertices, dtype=np.float64)
        self.faces = np.asarray(self.faces, dtype=np.int64)
        self.centers = np.asarray(self.centers, dtype=np.float64)
        self.normals = np.asarray(self.normals, dtype=np.float64)
        self.areas = np.asarray(self.areas, dtype=np.float64).reshape(-1)
        self.radii = np.asarray(self.radii, dtype=np.float64).reshape(-1)
        self.nvertices = int(self.vertices.shape[0])
        self.nfaces = int(self.faces.shape[0])
        if self.vertices.ndim != 2 or self.vertices.shape[1] != 3:
            raise ValueError("each vertex needs 3 coordinates")
        if self.faces.ndim != 2 or self.faces.shape[1] != 4:
            raise ValueError("only quadrilateral panels are allowed")
        if self.centers.shape != (self.nfaces, 3):
            raise ValueError("centers must be [nfaces x 3]")
        if self.normals.shape != (self.nfaces, 3):
            raise ValueError("normals must be [nfaces x 3]")
        if self.areas.shape[0] != self.nfaces:
            raise ValueError("areas vector must have length nfaces")
        if self.radii.shape[0] != self.nfaces:
            raise ValueError("radii vector must have length nfaces")
        if self.nfaces and (self.faces.min() < 0 or self.faces.max() >= self.nvertices):
            raise ValueError("face vertex index out of range")

    def __add__(self, other):
        if isinstance(other, Mesh):
            return combine_meshes([self, other])
        return combine_meshes([self, *other])

    def element(self, j: int) -> dict:
        """Panel j as the reference's element accessors see it
        (src/meshes.jl:171-179)."""
        return dict(center=self.centers[j].copy(), normal=self.normals[j].copy(),
                    area=float(self.areas[j]), radius=float(self.radii[j]),
                    vertices=self.vertices[self.faces[j]].copy())

    def translated(self, shift: Sequence[float]) -> "Mesh":
        s = np.asarray(shift, dtype=np.float64).reshape(1, 3)
        return Mesh(self.vertices + s, self.faces.copy(), self.centers + s,
                    self.normals.copy(), self.areas.copy(), self.radii.copy())


def combine_meshes(meshlist: Sequence[Mesh]) -> Mesh:
    """Concatenate meshes, re-offsetting face indices (src/meshes.jl:53-99).

    The reference offsets each mesh's faces by the vertex count of the mesh
    just before it only (``nvetrices_list[nfaces_index-1]``, meshes.jl:85),
    which is the cumulative count only for two meshes; here the cumulative
    vertex count is used, which agrees with the reference for two meshes."""
    offsets = np.cumsum([0] + [m.nvertices for m in meshlist[:-1]])
    return Mesh(
        np.concatenate([m.vertices for m in meshlist]),
        np.concatenate([m.faces + o for m, o in zip(meshlist, offsets)]),
        np.concatenate([m.centers for m in meshlist]),
        np.concatenate([m.normals for m in meshlist]),
        np.concatenate([m.areas for m in meshlist]),
        np.concatenate([m.radii for m in meshlist]),
    )


def panel_geometry(vertices: np.ndarray, faces: np.ndarray):
    """Centres, normals, areas and radii of quad panels from their vertices.

    Centre: area-weighted centroid of triangles (a,b,c) and (a,c,d)
    (src/meshes.jl:399-408); normal: normalize((b-a) x (c-a))
    (src/meshes.jl:413-414); area: sum of the two triangle areas; radius:
    the largest centre-to-vertex distance (Capytaine's ``faces_radiuses``,
    the convention of the meshes the reference's tests consume)."""
    v = vertices[faces]  # N x 4 x 3
    a, b, c, d = v[:, 0], v[:, 1], v[:, 2], v[:, 3]
    cr1 = np.cross(b - a, c - a)
    cr2 = np.cross(c - a, d - a)
    area1 = 0.5 * np.linalg.norm(cr1, axis=1)
    area2 = 0.5 * np.linalg.norm(cr2, axis=1)
    c1 = (a + b + c) / 3.0
    c2 = (a + c + d) / 3.0
    areas = area1 + area2
    centers = (c1 * area1[:, None] + c2 * area2[:, None]) / areas[:, None]
    normals = cr1 / np.linalg.norm(cr1, axis=1)[:, None]
    radii = np.max(np.linalg.norm(v - centers[:, None, :], axis=2), axis=1)
    return centers, normals, areas, radii


def mesh_hemisphere(radius: float = 1.0, center=(0.0, 0.0, 0.0),
                    resolution=(10, 10)) -> Mesh:
    """Immersed half (z <= centre) of a latitude-longitude sphere mesh.

    ``resolution = (ntheta, nphi)`` counts polar bands over the whole sphere
    and azimuthal sectors, as ``capytaine.mesh_sphere(...).immersed_part()``
    (src/meshes.jl:122-127) does: ceil(ntheta/2) bands cover the lower half,
    so (10, 10) gives 50 panels, (32, 64) gives 1024.  The bottom band is
    triangles stored as quads with a repeated vertex (src/meshes.jl:369-370).
    Vertex order (a, b, c, d) walks down the meridian first, so
    (b-a) x (c-a) points out of the body, into the fluid."""
    ntheta, nphi = int(resolution[0]), int(resolution[1])
    if ntheta < 2 or nphi < 3:
        raise ValueError("resolution must be at least (2, 3)")
    nb = (ntheta + 1) // 2
    thetas = 0.5 * math.pi + 0.5 * math.pi * np.arange(nb + 1) / nb
    phis = 2.0 * math.pi * np.arange(nphi) / nphi
    cx, cy, cz = (float(c) for c in center)
    verts = []
    for t in thetas[:-1]:
        st, ct = math.sin(t), math.cos(t)
        for p in phis:
            verts.append((cx + radius * st * math.cos(p), cy + radius * st * math.sin(p),
                          cz + radius * ct))
    pole = len(verts)
    verts.append((cx, cy, cz - radius))
    verts = np.asarray(verts, dtype=np.float64)
    faces = []
    for b in range(nb):
        for s in range(nphi):
            s2 = (s + 1) % nphi
            a_ = b * nphi + s
            d_ = b * nphi + s2
            if b + 1 < nb:
                b_ = (b + 1) * nphi + s
                c_ = (b + 1) * nphi + s2
                faces.append((a_, b_, c_, d_))
            else:
                faces.append((a_, pole, d_, d_))
    faces = np.asarray(faces, dtype=np.int64)
    centers, normals, areas, radii = panel_geometry(verts, faces)
    return Mesh(verts, faces, centers, normals, areas, radii)


def mesh_two_hemispheres(radius: float = 1.0, separation: float = 5.0,
                         resolution=(32, 64)) -> Mesh:
    """Two identical hemispheres, centres (0,0,0) and (separation,0,0)."""
    m1 = mesh_hemisphere(radius, (0.0, 0.0, 0.0), resolution)
    m2 = mesh_hemisphere(radius, (separation, 0.0, 0.0), resolution)
    return m1 + m2
