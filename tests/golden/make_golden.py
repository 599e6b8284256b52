"""Generates the CPU golden fixtures of tests/golden from the reference's OWN code.

Run here, where the reference sources exist: oracle/build_ref.sh compiles the
reference's src/geom/stl_loader.cpp, src/geom/voxelize.cpp and the band BFS of
src/apps/sim_runner.hpp into oracle/_ref/libref_cpu.so; this script drives it
on synthetic icosphere meshes and stores its masks and bands (bit-packed) in
geometry_golden.npz.  The oracle and the GPU voxelizer are tested against it.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from myfluidsimulation_b200 import workloads as W  # noqa: E402
from oracle_bind import RefCPU, mesh_bbox  # noqa: E402

# (name, dims, radius, center, refine, levels)
VOX = [
    ("sphere_256x128x128", (256, 128, 128), 16, (64, 64, 64), 1, 4),
    ("sphere_64x32x32", (64, 32, 32), 6, (20, 16, 16), 1, 4),
    ("sphere_48x40x24_amr2", (48, 40, 24), 7, (20, 20, 12), 2, 3),
    ("sphere_37x29x31", (37, 29, 31), 9, (18, 14, 15), 1, 3),
    ("sphere_33x17x19_amr3", (33, 17, 19), 5, (12, 8, 9), 3, 2),
]
BAND_D0 = [0, 1, 2, 3, 6]


def main():
    ref = RefCPU()
    out = {}
    for name, dims, r, c, refine, levels in VOX:
        tris, scale, tr = W.duct_sphere_mesh(*dims, r, c, levels=levels)
        bb = mesh_bbox(tris)
        mask = ref.voxelize(tris, bb, dims, scale, tr, refine)
        out[f"{name}/mask"] = np.packbits(mask.ravel())
        out[f"{name}/meta"] = np.array([*dims, refine, levels, r, *c, scale, *tr], np.float64)
        print(name, int(mask.sum()))
    # the band on the duct mask of the 64x32x32 sphere
    dims = (64, 32, 32)
    tris, scale, tr = W.duct_sphere_mesh(*dims, 6, (20, 16, 16), levels=4)
    m = W.duct_mask(*dims, ref.voxelize(tris, mesh_bbox(tris), dims, scale, tr, 1))
    out["band/mask"] = np.packbits(m.ravel())
    out["band/mask_raw"] = m.ravel()
    for d0 in BAND_D0:
        dist, leg = ref.band(m, d0)
        out[f"band/d0_{d0}"] = np.packbits(leg.ravel())
        out[f"band/dist_{d0}"] = dist.ravel().astype(np.int8)
    # the reference loader on the binary and ASCII icosphere STLs
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        t2, _, _ = W.duct_sphere_mesh(64, 32, 32, 6, (20, 16, 16), levels=2)
        for kind, fn in (("binary", W.write_binary_stl), ("ascii", W.write_ascii_stl)):
            p = os.path.join(td, kind + ".stl")
            fn(p, t2)
            tt, bb = ref.load_stl(p)
            out[f"stl/{kind}_tris"] = tt
            out[f"stl/{kind}_bb"] = bb
    np.savez_compressed(os.path.join(HERE, "geometry_golden.npz"), **out)
    print("wrote", os.path.join(HERE, "geometry_golden.npz"))


if __name__ == "__main__":
    main()
