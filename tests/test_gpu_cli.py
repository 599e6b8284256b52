"""The command-line tools against the reference's own tools, built from its sources.

oracle/_ref/bin/fluidsim_{legacy,home,hybrid,tgv} are the reference's
src/apps/main_*.cpp and src/bench/main_taylor_green.cpp linked with its own
solvers, geometry and VTK writer.  Both are run with the same arguments on the
same generated STL; stdout lines, the set of VTK files, their headers, and the
field values (relative L2, written in each case) must agree.  The library's
tools run with --bounce reference where a solid is present, because the
reference's opposite table is part of what it computes.  Velocities that start
from rest are small differences of O(0.05) populations, so two FP32 orders of
the same sums differ by ~1e-4 of them: the field tolerance is 3e-4 relative L2.
"""
import os
import subprocess

import numpy as np
import pytest

from myfluidsimulation_b200 import build as B
from myfluidsimulation_b200 import workloads as W
from oracle_bind import REF_DIR

pytestmark = pytest.mark.gpu
REF_BIN = os.path.join(REF_DIR, "bin")


@pytest.fixture(scope="module")
def bins(gpu):
    if not os.path.exists(os.path.join(REF_BIN, "fluidsim_legacy")):
        pytest.skip("reference tools not built")
    B.build_lib()
    B.build_apps()
    return True


@pytest.fixture(scope="module")
def stl(tmp_path_factory):
    """An icosphere of radius 6 cells at (16,16,16) in a 48x32x32 box, with its voxel options."""
    tris, scale, tr = W.duct_sphere_mesh(48, 32, 32, 6.0, (16, 16, 16), levels=3)
    p = str(tmp_path_factory.mktemp("stl") / "ball.stl")
    W.write_binary_stl(p, tris)
    return p, ["--voxel-scale", repr(scale), "--voxel-translate"] + [repr(t) for t in tr]


def run(exe, args, cwd):
    r = subprocess.run([exe] + args, capture_output=True, text=True, cwd=cwd, timeout=600)
    assert r.returncode == 0, f"{exe} failed:\n{r.stdout}\n{r.stderr}"
    return r


def read_vtk(path):
    lines = open(path).read().split("\n")
    k = next(i for i, l in enumerate(lines) if l.startswith("LOOKUP_TABLE") or l.startswith("VECTORS"))
    vals = np.array(" ".join(lines[k + 1:]).split(), dtype=np.float64)
    return lines[:k + 1], vals


def rl2(a, b):
    d = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (d if d > 0 else 1.0)


def compare_runs(tmp_path, name, args, mine_extra, tol):
    dm, dr = tmp_path / "mine", tmp_path / "ref"
    dm.mkdir()
    dr.mkdir()
    rm = run(os.path.join(B.BIN, name), args + ["--vtk-dir", str(dm / "vtk")] + mine_extra, str(dm))
    rr = run(os.path.join(REF_BIN, name), args + ["--vtk-dir", str(dr / "vtk")], str(dr))
    # stdout: the same [vtk]/[run] lines, with the directory names swapped
    assert rm.stdout.replace(str(dm), "X") == rr.stdout.replace(str(dr), "X")
    files = sorted(os.listdir(dr / "vtk"))
    assert files and sorted(os.listdir(dm / "vtk")) == files
    worst = 0.0
    for f in files:
        hm, vm = read_vtk(dm / "vtk" / f)
        hr, vr = read_vtk(dr / "vtk" / f)
        assert hm == hr, f
        assert vm.shape == vr.shape
        if f.startswith("rho"):
            # values near 1 are printed with 6 significant digits (steps of 1e-5):
            # two printed steps, plus the tolerance on the deviation from rest
            e = float(np.max(np.abs(vm - vr)))
            bound = 2.05e-5 + tol * float(np.max(np.abs(vr - 1.0)))
            assert e <= bound, f"{f}: max abs diff {e:.3e} > {bound:.3e}"
            continue
        e = rl2(vm, vr)
        worst = max(worst, e)
        assert e < tol, f"{f}: rel L2 {e:.3e}"
    print(f"{name}: {len(files)} files, worst rel L2 {worst:.3e}")


BOX = ["--nx", "48", "--ny", "32", "--nz", "32", "--tau", "0.56", "--force", "1e-5", "0", "0"]
GAUSS = ["--init", "gauss", "--amp", "0.01", "--sigma", "0.15"]


def test_legacy_tool_matches_reference_tool(bins, stl, tmp_path):
    """The reference's Legacy kernel writes some slots next to a solid twice from
    two threads (a race, see test_gpu_reference_build), so next to the obstacle
    its fields vary from run to run.  Checked: the same stdout and files, the
    same solid cells (zero velocity, unit density), and the fields agree away
    from the cells the race can have reached (3 cells after 2 steps)."""
    path, vox = stl
    args = BOX + ["--stl", path] + vox + ["--steps", "2", "--vtk-every", "1"]
    dm, dr = tmp_path / "mine", tmp_path / "ref"
    dm.mkdir()
    dr.mkdir()
    rm = run(os.path.join(B.BIN, "fluidsim_legacy"), args + ["--vtk-dir", str(dm / "vtk"), "--bounce", "reference"],
             str(dm))
    rr = run(os.path.join(REF_BIN, "fluidsim_legacy"), args + ["--vtk-dir", str(dr / "vtk")], str(dr))
    assert rm.stdout.replace(str(dm), "X") == rr.stdout.replace(str(dr), "X")
    files = sorted(os.listdir(dr / "vtk"))
    assert files and sorted(os.listdir(dm / "vtk")) == files
    shape = (32, 32, 48)
    for step in (1, 2):
        _, sm_ = read_vtk(dm / "vtk" / f"speed_legacy_{step:06d}.vtk")
        _, sr_ = read_vtk(dr / "vtk" / f"speed_legacy_{step:06d}.vtk")
        solid_m = (sm_ == 0).reshape(shape)
        solid_r = (sr_ == 0).reshape(shape)
        assert solid_r.sum() > 100
        np.testing.assert_array_equal(solid_m, solid_r)
        near = solid_r.copy()
        for _ in range(3):
            grown = near.copy()
            for ax in range(3):
                grown |= np.roll(near, 1, ax) | np.roll(near, -1, ax)
            near = grown
        far = ~near.ravel()
        assert rl2(sm_[far], sr_[far]) < 1e-4
    for f in files:
        assert read_vtk(dm / "vtk" / f)[0] == read_vtk(dr / "vtk" / f)[0], f


def test_home_tool_matches_reference_tool(bins, stl, tmp_path):
    path, vox = stl
    args = BOX + GAUSS + ["--stl", path] + vox + ["--steps", "20", "--vtk-every", "10", "--substeps", "2"]
    compare_runs(tmp_path, "fluidsim_home", args, ["--bounce", "reference"], 3e-4)


def test_hybrid_tool_matches_reference_tool(bins, stl, tmp_path):
    # one step from rest: after that the reference's own race (and its zero-filled
    # second buffer, see test_gpu_reference_build) decides
    path, vox = stl
    args = BOX + ["--stl", path] + vox + ["--steps", "1", "--vtk-every", "1", "--hybrid-band", "3"]
    compare_runs(tmp_path, "fluidsim_hybrid", args, ["--bounce", "reference"], 1e-5)


def test_tools_without_obstacle_match(bins, tmp_path):
    args = ["--nx", "40", "--ny", "24", "--nz", "16", "--init", "slab", "--amp", "0.02", "--axis", "y",
            "--steps", "30", "--vtk-every", "15"]
    compare_runs(tmp_path, "fluidsim_legacy", args, [], 3e-4)


def test_unreadable_stl_runs_without_obstacle(bins, tmp_path):
    args = BOX + GAUSS + ["--stl", str(tmp_path / "missing.stl"), "--steps", "4", "--vtk-every", "4"]
    compare_runs(tmp_path, "fluidsim_home", args, [], 3e-4)


def test_tgv_tool_matches_reference_tool(bins, tmp_path):
    args = ["--nx", "32", "--ny", "32", "--nz", "4", "--steps", "60", "--sample-every", "10", "--tau", "0.6"]
    rm = run(os.path.join(B.BIN, "fluidsim_tgv"), args + ["--csv", str(tmp_path / "m.csv")], str(tmp_path))
    rr = run(os.path.join(REF_BIN, "fluidsim_tgv"), args + ["--csv", str(tmp_path / "r.csv")], str(tmp_path))
    cfg = lambda out: [l for l in out.splitlines() if l.startswith("[cfg ]") and "csv=" not in l]
    assert cfg(rm.stdout) == cfg(rr.stdout)
    nstep = lambda out: sum(l.startswith("[step") for l in out.splitlines())
    assert nstep(rm.stdout) == nstep(rr.stdout) == 7
    mh, *mrows = open(tmp_path / "m.csv").read().splitlines()
    rh, *rrows = open(tmp_path / "r.csv").read().splitlines()
    assert mh == rh
    m = np.array([[float(x) for x in r.split(",")] for r in mrows])
    r = np.array([[float(x) for x in r.split(",")] for r in rrows])
    np.testing.assert_array_equal(m[:, :3], r[:, :3])          # step, time, exact energy
    np.testing.assert_allclose(m[:, 3:5], r[:, 3:5], rtol=2e-5)  # energies
    np.testing.assert_allclose(m[:, 5:], r[:, 5:], rtol=2e-3, atol=1e-9)  # errors vs analytic
