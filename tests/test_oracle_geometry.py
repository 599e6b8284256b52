"""The oracle's geometry (voxelizer, band BFS, STL loader) against the reference's own code.

Pinning: tests/golden/geometry_golden.npz holds masks, bands and loaded
meshes produced by the reference's voxelize.cpp / sim_runner.hpp /
stl_loader.cpp (tests/golden/make_golden.py).  Where the reference build is
present (oracle/_ref/libref_cpu.so) the oracle is also compared live on
random meshes.
"""
import os

import numpy as np
import pytest

from myfluidsimulation_b200 import workloads as W
from oracle_bind import RefCPU, mesh_bbox

GOLD = os.path.join(os.path.dirname(__file__), "golden", "geometry_golden.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def unpack(bits, shape):
    return np.unpackbits(bits)[: int(np.prod(shape))].reshape(shape)


@pytest.mark.parametrize("name", ["sphere_256x128x128", "sphere_64x32x32", "sphere_48x40x24_amr2",
                                  "sphere_37x29x31", "sphere_33x17x19_amr3"])
def test_oracle_voxelizer_matches_reference_golden(oracle, gold, name):
    meta = gold[f"{name}/meta"]
    dims = tuple(int(v) for v in meta[:3])
    refine, levels, r = int(meta[3]), int(meta[4]), float(meta[5])
    c = tuple(meta[6:9])
    tris, scale, tr = W.duct_sphere_mesh(*dims, r, c, levels=levels)
    assert np.float32(scale) == np.float32(meta[9])
    got = oracle.voxelize(tris, mesh_bbox(tris), dims, scale, tr, refine)
    want = unpack(gold[f"{name}/mask"], dims[::-1])
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("d0", [0, 1, 2, 3, 6])
def test_oracle_band_matches_reference_golden(oracle, gold, d0):
    m = gold["band/mask_raw"].reshape(32, 32, 64)
    dist, leg = oracle.band(m, d0)
    np.testing.assert_array_equal(leg, unpack(gold[f"band/d0_{d0}"], m.shape))
    np.testing.assert_array_equal(dist.astype(np.int8).ravel(), gold[f"band/dist_{d0}"])


def test_oracle_stl_loader_matches_reference_golden(oracle, gold, tmp_path):
    t2, _, _ = W.duct_sphere_mesh(64, 32, 32, 6, (20, 16, 16), levels=2)
    for kind, fn in (("binary", W.write_binary_stl), ("ascii", W.write_ascii_stl)):
        p = str(tmp_path / (kind + ".stl"))
        fn(p, t2)
        tt, bb = oracle.load_stl(p)
        np.testing.assert_array_equal(tt, gold[f"stl/{kind}_tris"])
        np.testing.assert_array_equal(bb, gold[f"stl/{kind}_bb"])


@pytest.mark.skipif(not RefCPU.available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("seed", range(6))
def test_oracle_voxelizer_matches_reference_live_random(oracle, seed):
    """Random triangle soups (open, overlapping, degenerate) at random sizes and AMR factors."""
    rng = np.random.default_rng(seed)
    nt = int(rng.integers(1, 300))
    tris = (rng.standard_normal((nt, 3, 3)) * rng.uniform(0.1, 2.0)).astype(np.float32)
    if seed % 2:
        tris[: nt // 4, 2] = tris[: nt // 4, 1]          # degenerate edges
    dims = tuple(int(v) for v in rng.integers(5, 40, size=3))
    refine = int(rng.integers(1, 3))
    scale = float(rng.uniform(0.3, 1.2))
    tr = tuple(float(v) for v in rng.uniform(0.2, 0.8, size=3))
    bb = mesh_bbox(tris)
    thr = float(rng.uniform(0, 1))
    a = oracle.voxelize(tris, bb, dims, scale, tr, refine, thr=thr)
    b = RefCPU().voxelize(tris, bb, dims, scale, tr, refine, thr=thr)
    np.testing.assert_array_equal(a, b)


@pytest.mark.skipif(not RefCPU.available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("seed", range(4))
def test_oracle_band_matches_reference_live_random(oracle, seed):
    rng = np.random.default_rng(100 + seed)
    dims = tuple(int(v) for v in rng.integers(3, 30, size=3))
    m = (rng.random(dims[::-1]) < rng.uniform(0.001, 0.2)).astype(np.uint8)
    d0 = int(rng.integers(0, 5))
    d1, l1 = oracle.band(m, d0)
    d2, l2 = RefCPU().band(m, d0)
    np.testing.assert_array_equal(d1, d2)
    np.testing.assert_array_equal(l1, l2)


@pytest.mark.skipif(not RefCPU.available(), reason="reference build (oracle/_ref) not present")
def test_oracle_stl_edge_cases_match_reference(oracle, tmp_path):
    """Truncated binary, empty binary, ASCII without vertices (falls back to binary), bad numbers."""
    ref = RefCPU()
    t = W.icosphere(1).astype(np.float32)
    good = str(tmp_path / "g.stl")
    W.write_binary_stl(good, t)
    raw = open(good, "rb").read()
    cases = {
        "trunc.stl": raw[: 84 + 50 * 3 + 10],
        "empty.stl": raw[:80] + b"\0\0\0\0",
        "short.stl": raw[:50],
        "solid_binary.stl": b"solid" + raw[5:],
        "ascii_bad.stl": b"solid x\n vertex 1 2 3\n vertex 1 zz 3\n vertex 4 5 6\n vertex 7 8 9\nendsolid\n",
        "ascii_none.stl": b"solid x\n facet\nendsolid\n" + b"\0" * 100,
    }
    for name, data in cases.items():
        p = str(tmp_path / name)
        open(p, "wb").write(data)
        ta, ba = oracle.load_stl(p)
        tb, bb = ref.load_stl(p)
        assert (ta is None) == (tb is None), name
        if ta is not None:
            np.testing.assert_array_equal(ta, tb)
            np.testing.assert_array_equal(ba, bb)
    assert oracle.load_stl(str(tmp_path / "missing.stl"))[0] is None
