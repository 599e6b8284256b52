"""Synthetic inputs for the D3Q19 workloads (no dataset is involved).

* ``icosphere`` / ``write_binary_stl``: the obstacle of the duct workloads, an
  icosahedron subdivided ``levels`` times (4 -> 5,120 triangles), projected
  onto the unit sphere.
* ``duct_sphere_stl_params``: the STL stretch and the ``--voxel-scale`` /
  ``--voxel-translate`` values that make the reference voxelizer, which fits
  the mesh bounding box into the unit cube and then scales each axis by its
  own cell count (src/geom/voxelize.cpp:83-91,144), produce a sphere of a
  given radius in lattice units on a non-cubic grid.
* ``taylor_green_3d``: the 3-D Taylor-Green initial field evaluated at cell
  centres (i + 0.5), the convention of src/bench/main_taylor_green.cpp:68-70.
* ``taylor_green_2d``: the reference bench's own extruded 2-D field
  (src/bench/main_taylor_green.cpp:68-87).
* ``duct_mask``: y/z duct walls as solid mask cells marked "wall" (bit 3), so
  the momentum-exchange drag only sums over the obstacle.
"""
from __future__ import annotations

import math
import struct

import numpy as np

MASK_SOLID = 1
MASK_WALL = 8


def icosphere(levels: int = 4) -> np.ndarray:
    """Triangles (T, 3, 3) float64 of a unit icosphere with 20 * 4**levels faces."""
    p = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [(-1, p, 0), (1, p, 0), (-1, -p, 0), (1, -p, 0),
             (0, -1, p), (0, 1, p), (0, -1, -p), (0, 1, -p),
             (p, 0, -1), (p, 0, 1), (-p, 0, -1), (-p, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11),
             (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8),
             (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9),
             (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    v = [np.array(x, dtype=np.float64) / np.linalg.norm(x) for x in verts]
    for _ in range(levels):
        cache: dict = {}

        def mid(a: int, b: int) -> int:
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = (v[a] + v[b]) * 0.5
                v.append(m / np.linalg.norm(m))
                cache[key] = len(v) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    V = np.stack(v)
    return V[np.array(faces)]


def write_binary_stl(path: str, tris: np.ndarray, header: bytes = b"icosphere") -> None:
    """Binary STL: 80-byte header, uint32 count, 50-byte records (normal, 3 vertices, attr)."""
    t = np.asarray(tris, dtype=np.float32).reshape(-1, 3, 3)
    with open(path, "wb") as f:
        f.write(header.ljust(80, b"\0")[:80])
        f.write(struct.pack("<I", t.shape[0]))
        for tri in t:
            n = np.cross(tri[1] - tri[0], tri[2] - tri[0])
            nn = np.linalg.norm(n)
            n = (n / nn if nn > 0 else n).astype(np.float32)
            f.write(struct.pack("<3f", *n))
            f.write(tri.astype("<f4").tobytes())
            f.write(b"\0\0")


def write_ascii_stl(path: str, tris: np.ndarray, name: str = "obj") -> None:
    t = np.asarray(tris, dtype=np.float32).reshape(-1, 3, 3)
    with open(path, "w") as f:
        f.write(f"solid {name}\n")
        for tri in t:
            f.write("  facet normal 0 0 0\n    outer loop\n")
            for p in tri:
                f.write(f"      vertex {p[0]:.9g} {p[1]:.9g} {p[2]:.9g}\n")
            f.write("    endloop\n  endfacet\n")
        f.write(f"endsolid {name}\n")


def duct_sphere_stl_params(nx: int, ny: int, nz: int, radius: float, center):
    """(stretch, scale, translate) for a lattice-unit sphere through the reference voxelizer.

    The mesh is the unit sphere with axis k stretched by stretch[k]; the
    voxelizer maps the largest bbox extent to ``scale`` of the unit cube and
    multiplies each unit coordinate by that axis' cell count.
    """
    dims = np.array([nx, ny, nz], dtype=np.float64)
    m = dims.min()
    stretch = m / dims                       # axis k is scaled by n_min / n_k
    scale = 2.0 * radius / m                 # the largest extent (2) maps to 2r cells
    translate = np.asarray(center, dtype=np.float64) / dims
    return stretch, float(scale), tuple(float(t) for t in translate)


def duct_sphere_mesh(nx: int, ny: int, nz: int, radius: float, center, levels: int = 4):
    stretch, scale, translate = duct_sphere_stl_params(nx, ny, nz, radius, center)
    tris = icosphere(levels) * stretch[None, None, :]
    return tris.astype(np.float32), scale, translate


def duct_mask(nx: int, ny: int, nz: int, obstacle: np.ndarray | None = None) -> np.ndarray:
    """Mask (nz, ny, nx) uint8: walls on the y and z faces (1|8), obstacle cells 1."""
    m = np.zeros((nz, ny, nx), dtype=np.uint8)
    if obstacle is not None:
        m[obstacle.reshape(nz, ny, nx) != 0] = MASK_SOLID
    wall = MASK_SOLID | MASK_WALL
    m[:, 0, :] = wall
    m[:, ny - 1, :] = wall
    m[0, :, :] = wall
    m[nz - 1, :, :] = wall
    return m


def taylor_green_3d(nx: int, ny: int, nz: int, u0: float = 0.05, rho0: float = 1.0, k=None):
    """3-D TGV: u=u0 sin(kx)cos(ky)cos(kz), v=-u0 cos(kx)sin(ky)cos(kz), w=0,
    p=rho0 u0^2/16 (cos2kx+cos2ky)(cos2kz+2), rho=rho0+3p; FP64 -> float32."""
    if k is None:
        k = (2 * math.pi / nx, 2 * math.pi / ny, 2 * math.pi / nz)
    elif np.isscalar(k):
        k = (k, k, k)
    x = (np.arange(nx) + 0.5) * k[0]
    y = (np.arange(ny) + 0.5) * k[1]
    z = (np.arange(nz) + 0.5) * k[2]
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    u = u0 * np.sin(X) * np.cos(Y) * np.cos(Z)
    v = -u0 * np.cos(X) * np.sin(Y) * np.cos(Z)
    w = np.zeros_like(u)
    p = rho0 * u0 * u0 / 16.0 * (np.cos(2 * X) + np.cos(2 * Y)) * (np.cos(2 * Z) + 2.0)
    rho = rho0 + 3.0 * p
    f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)
    return f32(rho), f32(u), f32(v), f32(w)


def taylor_green_2d(nx: int, ny: int, nz: int, u0: float = 0.06, kx: float = 1.0, ky: float = 1.0):
    """The fluidsim_tgv initial field (2-D TGV extruded in z), main_taylor_green.cpp:68-87,126-136."""
    kxw = 2 * math.pi * kx / nx
    kyw = 2 * math.pi * ky / ny
    tx = (np.arange(nx) + 0.5) * kxw
    ty = (np.arange(ny) + 0.5) * kyw
    Y, X = np.meshgrid(ty, tx, indexing="ij")
    u = u0 * np.sin(X) * np.cos(Y)
    v = -u0 * np.cos(X) * np.sin(Y)
    rho = 1.0 + (u0 * u0 / (4.0 / 3.0)) * (np.cos(2 * X) + np.cos(2 * Y))
    rep = lambda a: np.ascontiguousarray(np.broadcast_to(a, (nz, ny, nx)), dtype=np.float32)
    return rep(rho), rep(u), rep(v), np.zeros((nz, ny, nx), np.float32)
