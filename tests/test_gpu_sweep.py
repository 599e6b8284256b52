"""The headless B0 sweep (bin/fluidsim_sweep) against the FP64 oracle.

fluidsim_compare --hybrid-sweep-max M (src/main_compare.cpp:505-699) runs Legacy
and HOME once and Hybrid(B0) for d0 = 0..M from the same initial density and
prints one CSV line per d0.  The reference tool needs OpenGL/GLFW and is not
built here; its sweep is restated below on the oracle: the same obstacle mask,
the same near-wall cell list (fluid cells with a solid 6-neighbour inside the
box, main_compare.cpp:359-386), the band of every d0, and the three runs, with
the reference's opposite table (--bounce reference, Hybrid runs one at a time)
and with halfway bounce-back (the default, Hybrid runs batched).

Integer columns (band size, fluid and near-wall counts) must be equal; the
float columns are FP32 (tool) against FP64 (oracle) after 30 steps: mean |u|
within 1e-4 relative, the mean |u| differences within 2e-4 of mean |u|, the mean
densities within 1e-6 (plus 1e-7 on the velocities: FP32 populations of ~1/18
round at ~4e-9, so a velocity carries ~1e-8 of absolute rounding).
"""
import os
import subprocess

import numpy as np
import pytest
import torch

from myfluidsimulation_b200 import build as B
from myfluidsimulation_b200 import lib
from myfluidsimulation_b200 import workloads as W

pytestmark = pytest.mark.gpu

HEADER = ("d0,legacy_cells,legacy_ratio,mean_u_legacy,mean_u_home,mean_u_hybrid,mean_absdiff_home,"
          "mean_absdiff_hybrid,mean_rho_legacy,mean_rho_home,mean_rho_hybrid,absdiff_rho_home,"
          "absdiff_rho_hybrid,ms_per_step_legacy,ms_per_step_home,ms_per_step_hybrid,amr_factor,"
          "amr_threshold,fluid_cells,near_wall_cells")


def near_wall(mask):
    m = mask.astype(bool)
    nb = np.zeros_like(m)
    nb[:, :, 1:] |= m[:, :, :-1]
    nb[:, :, :-1] |= m[:, :, 1:]
    nb[:, 1:, :] |= m[:, :-1, :]
    nb[:, :-1, :] |= m[:, 1:, :]
    nb[1:, :, :] |= m[:-1, :, :]
    nb[:-1, :, :] |= m[1:, :, :]
    return np.flatnonzero((nb & ~m).ravel())


def gauss_rho(dims, cen, sigma, amp):
    nx, ny, nz = dims
    d = torch.empty(nx * ny * nz, device="cuda")
    torch.cuda.synchronize()
    lib().make_rho_gauss(d.data_ptr(), nx, ny, nz, *cen, sigma, amp)
    torch.cuda.synchronize()
    return d.cpu().numpy().reshape(nz, ny, nx)


DIMS = (48, 32, 32)
TAU, FORCE, STEPS, DMAX = 0.58, 2e-4, 30, 3
CEN, SIGMA, AMP = (0.4, 0.5, 0.5), 0.1, 1e-2


@pytest.fixture(scope="module")
def ball(tmp_path_factory):
    B.build_lib()
    B.build_apps()
    nx, ny, nz = DIMS
    tris, scale, tr = W.duct_sphere_mesh(nx, ny, nz, 6.0, (16, 16, 16), levels=3)
    stl = str(tmp_path_factory.mktemp("sweep") / "ball.stl")
    W.write_binary_stl(stl, tris)
    return stl, scale, tr


def sweep(ball, *extra):
    stl, scale, tr = ball
    nx, ny, nz = DIMS
    args = ["--stl", stl, "--nx", str(nx), "--ny", str(ny), "--nz", str(nz), "--tau", repr(TAU),
            "--voxel-scale", repr(scale), "--voxel-translate", *[repr(t) for t in tr],
            "--init", "gauss", "--center", *[repr(c) for c in CEN], "--sigma", repr(SIGMA), "--amp", repr(AMP),
            "--force", repr(FORCE), "--hybrid-sweep-max", str(DMAX), "--sweep-steps", str(STEPS), *extra]
    r = subprocess.run([os.path.join(B.BIN, "fluidsim_sweep")] + args, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.strip().split("\n")
    k = lines.index(HEADER)
    rows = [l.split(",") for l in lines[k + 1:]]
    assert [int(x[0]) for x in rows] == list(range(DMAX + 1))
    return lines, rows


def test_batched_sweep_equals_one_by_one(gpu, ball):
    """The batched Hybrid runs give the same CSV as one solver at a time, timings aside."""
    _, a = sweep(ball)
    _, b = sweep(ball, "--no-batch")
    for ra, rb in zip(a, b):
        assert ra[:13] == rb[:13] and ra[16:] == rb[16:]


@pytest.mark.parametrize("bounce", ["reference", "halfway"])
def test_sweep_matches_oracle(gpu, oracle, ball, bounce):
    stl, scale, tr = ball
    dims, tau, force, steps, dmax, cen, sigma, amp = DIMS, TAU, FORCE, STEPS, DMAX, CEN, SIGMA, AMP
    bb = 1 if bounce == "reference" else 0
    lines, rows = sweep(ball, "--bounce", bounce)

    # the oracle's sweep
    t2, box = oracle.load_stl(stl)
    mask = oracle.voxelize(t2, box, dims, scale, tr)
    near = near_wall(mask)
    fluid = mask.size - int(mask.sum())
    assert f"[wall] near-wall fluid cells: {near.size}" in lines
    rho0 = gauss_rho(dims, cen, sigma, amp)
    zero = np.zeros_like(rho0)
    fields = (rho0, zero, zero, zero)
    frc = (force, 0.0, 0.0)

    def stats(rho, u, v, w):
        sp = np.sqrt(u.astype(np.float64) ** 2 + v ** 2 + w ** 2).ravel()[near]
        return sp, sp.mean(), rho.astype(np.float64).ravel()[mask.ravel() == 0].mean()

    f0 = oracle.reinit_eq(*fields)
    _, *mac, _ = oracle.bgk_run(f0, mask, steps, tau, frc, bb=bb)
    sp_l, mu_l, mr_l = stats(*mac)
    m0 = np.zeros((10,) + rho0.shape)
    m0[0] = rho0
    m, _ = oracle.home_run(m0, mask, steps, tau, frc, bb=bb)
    sp_h, mu_h, mr_h = stats(m[0], m[1], m[2], m[3])
    for d0, row in zip(range(dmax + 1), rows):
        _, band = oracle.band(mask, d0)
        nb = int(band.sum())
        _, *mac, _ = oracle.bgk_run(f0, mask, steps, tau, frc, mode=1, band=band, bb=bb,
                                    fnext=np.zeros_like(f0) if bb else None)
        sp_y, mu_y, mr_y = stats(*mac)
        want = [d0, nb, nb / fluid, mu_l, mu_h, mu_y, np.abs(sp_h - sp_l).mean(), np.abs(sp_y - sp_l).mean(),
                mr_l, mr_h, mr_y, abs(mr_h - mr_l), abs(mr_y - mr_l)]
        got = [float(x) for x in row[:13]]
        print(f"d0 {d0}: band {nb}, mean|u| tool {got[3]:.6e} {got[4]:.6e} {got[5]:.6e} "
              f"oracle {mu_l:.6e} {mu_h:.6e} {mu_y:.6e}, absdiff {got[6]:.3e}/{want[6]:.3e} {got[7]:.3e}/{want[7]:.3e}")
        assert int(row[1]) == nb
        assert abs(got[2] - nb / fluid) < 1e-6
        for j in (3, 4, 5):
            assert abs(got[j] - want[j]) <= 1e-4 * want[j] + 1e-7, (d0, j)
        for j in (6, 7):
            assert abs(got[j] - want[j]) <= 2e-4 * mu_l + 1e-7, (d0, j)
        for j in (8, 9, 10, 11, 12):
            assert abs(got[j] - want[j]) <= 1e-6, (d0, j)
        assert all(float(x) > 0 for x in row[13:16])
        assert row[16:] == ["1", "0.500000", str(fluid), str(near.size)]
