"""Panel meshes: the ``Mesh`` container, multi-body concatenation, a
hemisphere generator and the reference's axisymmetric / WaveBot generators.

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
    # band b, sector s -> vertex b * nphi + s (the sines and cosines of the
    # angles by the C library, the products in the same order per vertex)
    st = np.array([math.sin(t) for t in thetas[:-1]])
    ct = np.array([math.cos(t) for t in thetas[:-1]])
    cp = np.array([math.cos(p) for p in phis])
    sp = np.array([math.sin(p) for p in phis])
    rs = radius * st
    verts = np.empty((nb * nphi + 1, 3))
    verts[:-1, 0] = (cx + rs[:, None] * cp[None, :]).reshape(-1)
    verts[:-1, 1] = (cy + rs[:, None] * sp[None, :]).reshape(-1)
    verts[:-1, 2] = np.repeat(cz + radius * ct, nphi)
    pole = nb * nphi
    verts[pole] = (cx, cy, cz - radius)
    b = np.repeat(np.arange(nb), nphi)
    s = np.tile(np.arange(nphi), nb)
    s2 = (s + 1) % nphi
    a_ = b * nphi + s
    d_ = b * nphi + s2
    last = b + 1 == nb
    faces = np.stack([a_, np.where(last, pole, (b + 1) * nphi + s), np.where(last, d_, (b + 1) * nphi + s2), d_],
                     axis=1).astype(np.int64)
    centers, normals, areas, radii = panel_geometry(verts, faces)
    return Mesh(verts, faces, centers, normals, areas, radii)


def mesh_two_hemispheres(radius: float = 1.0, separation: float = 5.0,
                         resolution=(32, 64)) -> Mesh:
    """Two identical hemispheres, centres (0,0,0) and (separation,0,0)."""
    m1 = mesh_hemisphere(radius, (0.0, 0.0, 0.0), resolution)
    m2 = mesh_hemisphere(radius, (separation, 0.0, 0.0), resolution)
    return m1 + m2


# --------------------------------------------------------------------------
# Axisymmetric meshes and the WaveBot (src/meshes.jl:247-479)
# --------------------------------------------------------------------------

def wavebot_profile(cylinder_height: float = 0.16, frustum_height: float = 0.37,
                    top_radius: float = 0.88, bottom_radius: float = 0.35,
                    n_points=(5, 10, 5)) -> np.ndarray:
    """(r, z) points of the WaveBot profile, from the waterline down
    (src/meshes.jl:316-350): a cylinder of ``top_radius`` from z = 0 to
    -cylinder_height (n_cylinder points), a frustum narrowing to
    ``bottom_radius`` over ``frustum_height`` (n_frustum - 1 more) and the
    flat bottom to the axis (n_bottom - 1 more, the last at r = 0).
    ``n_points = (n_bottom, n_frustum, n_cylinder)`` as in the reference;
    lengths in metres."""
    n_bottom, n_frustum, n_cylinder = (int(x) for x in n_points)
    if min(n_bottom, n_frustum, n_cylinder) < 2:
        raise ValueError("each part of the profile needs at least 2 points")
    pts = []
    for j in range(n_cylinder):
        t = j / (n_cylinder - 1)
        pts.append((top_radius, -cylinder_height * t))
    for j in range(1, n_frustum):
        t = j / (n_frustum - 1)
        pts.append((top_radius + (bottom_radius - top_radius) * t, -cylinder_height - frustum_height * t))
    z_bottom = -cylinder_height - frustum_height
    for j in range(1, n_bottom):
        t = j / (n_bottom - 1)
        pts.append((bottom_radius * (1.0 - t), z_bottom))
    return np.asarray(pts, dtype=np.float64)


def axisymmetric_mesh(profile, n_theta: int = 72):
    """Vertices (V x 3) and 0-based faces (N x 4) of the surface swept by a
    profile of (r, z) points revolved about the z axis
    (src/meshes.jl:247-314).  Each profile point becomes a ring of n_theta
    vertices at theta = 2 pi i / n_theta, or one vertex on the axis when
    r = 0; consecutive rings are joined by quads (i1, i3, i4, i2) (upper ring
    i, lower ring i, lower ring i + 1, upper ring i + 1), and a ring next to
    an axis point by triangles, stored with their last vertex repeated
    (src/meshes.jl:366-368)."""
    prof = np.asarray(profile, dtype=np.float64)
    n_theta = int(n_theta)
    if n_theta < 3:
        raise ValueError("n_theta must be at least 3")
    if prof.ndim != 2 or prof.shape[1] != 2 or prof.shape[0] < 2:
        raise ValueError("profile must contain at least two (r, z) points")
    if np.any(prof[:, 0] < 0.0):
        raise ValueError("profile radii must be nonnegative")
    th = 2.0 * math.pi * np.arange(n_theta) / n_theta
    ct, st = np.cos(th), np.sin(th)
    verts, starts, sizes = [], [], []
    for r, z in prof:
        starts.append(len(verts))
        if r == 0.0:
            sizes.append(1)
            verts.append((0.0, 0.0, z))
        else:
            sizes.append(n_theta)
            verts.extend(zip(r * ct, r * st, np.full(n_theta, z)))
    faces = []
    for layer in range(len(prof) - 1):
        s1, s2 = starts[layer], starts[layer + 1]
        n1, n2 = sizes[layer], sizes[layer + 1]
        if n1 == 1 and n2 == 1:
            raise ValueError("adjacent points cannot both have radius 0")
        for i in range(n_theta):
            i2n = (i + 1) % n_theta
            if n1 == 1:
                faces.append((s1, s2 + i, s2 + i2n, s2 + i2n))
            elif n2 == 1:
                faces.append((s1 + i, s2, s1 + i2n, s1 + i2n))
            else:
                faces.append((s1 + i, s2 + i, s2 + i2n, s1 + i2n))
    return np.asarray(verts, dtype=np.float64), np.asarray(faces, dtype=np.int64)


def polygon_geometry(vertices: np.ndarray, faces: np.ndarray):
    """Centres, normals, areas and radii with the conventions of the
    reference's conversion of a polygon mesh (src/meshes.jl:353-423): the
    area-weighted centroid of triangles (a, b, c) and (a, c, d) (a triangle
    repeats c as d, so its second triangle has no area), the unit normal of
    (b - a) x (c - a), the area of the polygon (the two triangles) and the
    radius |a - centre| (distance to the first vertex; ``panel_geometry``
    takes the largest vertex distance instead)."""
    v = vertices[faces]
    a, b, c, d = v[:, 0], v[:, 1], v[:, 2], v[:, 3]
    cr1 = np.cross(b - a, c - a)
    cr2 = np.cross(c - a, d - a)
    area1 = 0.5 * np.linalg.norm(cr1, axis=1)
    area2 = 0.5 * np.linalg.norm(cr2, axis=1)
    areas = area1 + area2
    centers = ((a + b + c) / 3.0 * area1[:, None] + (a + c + d) / 3.0 * area2[:, None]) / areas[:, None]
    normals = cr1 / np.linalg.norm(cr1, axis=1)[:, None]
    radii = np.linalg.norm(a - centers, axis=1)
    return centers, normals, areas, radii


def wavebot_mesh(r1: float, r2: float, d1: float, d2: float, n_points=(5, 10, 5),
                 n_theta: int = 72) -> Mesh:
    """The WaveBot buoy (src/meshes.jl:458-479): top radius r1, bottom radius
    r2, cylinder height d1, frustum height d2 (metres), revolved with n_theta
    sectors.  The default (5, 10, 5) profile and 72 sectors give 17 x 72 =
    1224 panels, the last ring of them triangles at the bottom centre."""
    prof = wavebot_profile(d1, d2, r1, r2, n_points)
    verts, faces = axisymmetric_mesh(prof, n_theta)
    centers, normals, areas, radii = polygon_geometry(verts, faces)
    return Mesh(verts, faces, centers, normals, areas, radii)
