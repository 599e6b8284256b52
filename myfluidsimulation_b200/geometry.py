"""STL loading and GPU voxelization over the C-ABI.

Mirrors load_stl (src/geom/stl_loader.cpp:102-122), VoxelParams and
voxelize_mesh_to_mask (src/geom/voxelize.hpp:16-27, voxelize.cpp:228-243),
and the B0 band of src/apps/sim_runner.hpp:28-91 (computed on the GPU by a
Hybrid solver, see Solver.build_band).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from ._lib import VoxelParams as _VP
from ._lib import check, lib


@dataclass
class TriangleMesh:
    """Unindexed triangle soup (T, 3, 3) float32 and its bbox, like TriangleMesh (stl_loader.hpp:17-21)."""
    tris: np.ndarray
    bbmin: np.ndarray
    bbmax: np.ndarray


@dataclass
class VoxelParams:
    Nx: int = 128
    Ny: int = 128
    Nz: int = 128
    uniformScale: float = 0.9
    translate: tuple = field(default=(0.5, 0.5, 0.5))
    refine: int = 1
    coverageThreshold: float = 0.5


def load_stl(path: str) -> TriangleMesh:
    """Raises LBMError (LBM_ERR_IO) where the reference's load_stl returns false."""
    buf = C.c_void_p()
    n = C.c_int64()
    bb = np.zeros(6, np.float32)
    check(lib().lbm_load_stl(path.encode(), C.byref(buf), C.byref(n), bb.ctypes.data_as(C.c_void_p)))
    try:
        if n.value:
            arr = np.ctypeslib.as_array(C.cast(buf, C.POINTER(C.c_float)), shape=(n.value * 9,)).copy()
        else:
            arr = np.zeros(0, np.float32)
    finally:
        lib().lbm_free(buf)
    return TriangleMesh(arr.reshape(-1, 3, 3), bb[:3].copy(), bb[3:].copy())


def voxelize_mesh_to_mask(mesh: TriangleMesh, p: VoxelParams) -> np.ndarray:
    """Solid mask (Nz, Ny, Nx) uint8 from the GPU voxelizer."""
    tris = np.ascontiguousarray(mesh.tris, np.float32)
    bb = np.concatenate([mesh.bbmin, mesh.bbmax]).astype(np.float32)
    vp = _VP(int(p.Nx), int(p.Ny), int(p.Nz), float(p.uniformScale),
             (C.c_float * 3)(*[float(t) for t in p.translate]), int(p.refine), float(p.coverageThreshold))
    out = np.empty((p.Nz, p.Ny, p.Nx), np.uint8)
    check(lib().lbm_voxelize(tris.ctypes.data_as(C.c_void_p), tris.shape[0], bb.ctypes.data_as(C.c_void_p),
                             C.byref(vp), out.ctypes.data_as(C.c_void_p)))
    return out


def mesh_from_triangles(tris) -> TriangleMesh:
    t = np.ascontiguousarray(tris, np.float32).reshape(-1, 3, 3)
    v = t.reshape(-1, 3)
    if len(v):
        return TriangleMesh(t, v.min(0), v.max(0))
    big = np.finfo(np.float32).max
    return TriangleMesh(t, np.full(3, big, np.float32), np.full(3, -big, np.float32))
