"""GPU voxelizer and GPU band against the oracle (bit-exact) and the reference's own CPU build."""
import os

import numpy as np
import pytest

from myfluidsimulation_b200 import geometry as G
from myfluidsimulation_b200 import workloads as W
from myfluidsimulation_b200.solvers import METHOD_HYBRID, Solver
from oracle_bind import RefCPU, mesh_bbox

pytestmark = pytest.mark.gpu

VOX_CASES = [
    # dims, refine, radius, center
    ((256, 128, 128), 1, 16, (64, 64, 64)),
    ((64, 32, 32), 1, 6, (20, 16, 16)),
    ((48, 40, 24), 2, 7, (20, 20, 12)),
    ((37, 29, 31), 1, 9, (18, 14, 15)),
    ((33, 17, 19), 3, 5, (12, 8, 9)),
]


@pytest.mark.parametrize("dims,refine,radius,center", VOX_CASES)
def test_gpu_voxelizer_bit_exact(gpu, oracle, dims, refine, radius, center):
    tris, scale, tr = W.duct_sphere_mesh(*dims, radius, center)
    bb = mesh_bbox(tris)
    ref = oracle.voxelize(tris, bb, dims, scale, tr, refine)
    mesh = G.mesh_from_triangles(tris)
    got = G.voxelize_mesh_to_mask(mesh, G.VoxelParams(*dims, scale, tr, refine, 0.5))
    np.testing.assert_array_equal(got, ref)
    if RefCPU.available():
        np.testing.assert_array_equal(got, RefCPU().voxelize(tris, bb, dims, scale, tr, refine))


def test_gpu_voxelizer_concave_and_degenerate(gpu, oracle):
    """A cup-shaped (concave) mesh plus degenerate triangles; the flood fill must need several rounds."""
    rng = np.random.default_rng(0)
    ico = W.icosphere(2)
    inner = ico * 0.6
    cup = np.concatenate([ico[ico[:, :, 2].mean(1) < 0.3], inner[inner[:, :, 2].mean(1) < 0.3][:, ::-1]])
    degen = np.repeat(rng.standard_normal((5, 1, 3)) * 0.3, 3, axis=1)      # zero-area triangles
    tris = np.concatenate([cup, degen]).astype(np.float32)
    bb = mesh_bbox(tris)
    for dims in [(40, 36, 30), (21, 19, 23)]:
        ref = oracle.voxelize(tris, bb, dims, 0.8, (0.5, 0.5, 0.5), 1)
        got = G.voxelize_mesh_to_mask(G.mesh_from_triangles(tris), G.VoxelParams(*dims, 0.8, (0.5, 0.5, 0.5)))
        np.testing.assert_array_equal(got, ref)


def test_gpu_voxelizer_empty_mesh(gpu):
    m = G.mesh_from_triangles(np.zeros((0, 3, 3), np.float32))
    got = G.voxelize_mesh_to_mask(m, G.VoxelParams(8, 8, 8))
    assert not got.any()


@pytest.mark.parametrize("d0", [0, 1, 2, 3, 6])
def test_gpu_band_bit_exact(gpu, oracle, d0):
    dims = (64, 32, 32)
    tris, scale, tr = W.duct_sphere_mesh(*dims, 7, (24, 16, 16))
    mask = W.duct_mask(*dims, oracle.voxelize(tris, mesh_bbox(tris), dims, scale, tr, 1))
    _, ref = oracle.band(mask, d0)
    s = Solver(*dims, 0.6, method=METHOD_HYBRID)
    s.set_solid_mask(mask)
    n = s.build_band(d0)
    got = s.band()
    s.close()
    np.testing.assert_array_equal(got, ref)
    assert n == int(ref.sum())
    if RefCPU.available():
        np.testing.assert_array_equal(got, RefCPU().band(mask, d0)[1])


def test_gpu_stl_loader_matches(gpu, oracle, tmp_path):
    tris, _, _ = W.duct_sphere_mesh(64, 32, 32, 6, (20, 16, 16), levels=2)
    pb = os.path.join(tmp_path, "b.stl")
    pa = os.path.join(tmp_path, "a.stl")
    W.write_binary_stl(pb, tris)
    W.write_ascii_stl(pa, tris)
    for p in (pb, pa):
        m = G.load_stl(p)
        t, bb = oracle.load_stl(p)
        np.testing.assert_array_equal(m.tris, t)
        np.testing.assert_array_equal(np.concatenate([m.bbmin, m.bbmax]), bb)
