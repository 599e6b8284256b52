"""Self-consistency of the FP64 oracle (it is the checker, so it is checked first).

Physical invariants the reference's algorithm must satisfy: rest equilibrium
is a fixed point, mass is conserved on periodic grids, the Taylor-Green
vortex decays at the viscosity nu = (tau - 1/2)/3 (the analytic rate the
reference's fluidsim_tgv reports against, main_taylor_green.cpp:68-87,188-190),
the Hybrid form equals BGK when omega_s == omega_h, and HOME reproduces the
BGK macro field of a smooth flow closely (both are second-order schemes).
"""
import numpy as np

from myfluidsimulation_b200 import workloads as W


def test_rest_state_is_fixed_point(oracle):
    n = 6
    one = np.ones((n, n, n))
    f0 = oracle.reinit_eq(one, None, None, None)
    f, rho, u, v, w, _ = oracle.bgk_run(f0, None, 5, 0.6)
    np.testing.assert_allclose(f, f0, atol=1e-15)
    m0 = np.zeros((10, n, n, n)); m0[0] = 1
    m, _ = oracle.home_run(m0, None, 5, 0.6)
    np.testing.assert_allclose(m, m0, atol=1e-15)


def test_mass_conserved_periodic(oracle):
    n = 12
    rho, u, v, w = W.taylor_green_3d(n, n, n, 0.05)
    f0 = oracle.reinit_eq(rho, u, v, w)
    f, *_ = oracle.bgk_run(f0, None, 50, 0.6)
    assert abs(f.sum() - f0.sum()) < 1e-10 * f0.sum()
    mask = np.zeros((n, n, n), np.uint8); mask[4:7, 4:7, 4:7] = 1
    f, *_ = oracle.bgk_run(f0, mask, 50, 0.6)
    fl = mask == 0
    assert abs(f[:, fl].sum() - f0[:, fl].sum()) < 1e-10 * f0.sum()


def test_tgv_decay_rate(oracle):
    n, tau, u0 = 32, 0.6, 0.02
    rho, u, v, w = W.taylor_green_2d(n, n, 1, u0)
    f, rho, ux, uy, uz, _ = oracle.bgk_run(oracle.reinit_eq(rho, u, v, w), None, 201, tau)
    # macros after 201 calls are the moments of the state after 200 streams
    nu = (tau - 0.5) / 3
    k2 = 2 * (2 * np.pi / n) ** 2
    e = 0.5 * (ux ** 2 + uy ** 2).mean()
    e_exact = 0.25 * u0 ** 2 * np.exp(-2 * nu * k2 * 200)
    assert abs(e / e_exact - 1) < 0.02


def test_hybrid_forms_agree_when_rates_equal(oracle):
    n = 10
    rho, u, v, w = W.taylor_green_3d(n, n, n, 0.05)
    f0 = oracle.reinit_eq(rho, u, v, w)
    mask = np.zeros((n, n, n), np.uint8); mask[3:5, 3:6, 2:5] = 1
    a = oracle.bgk_run(f0, mask, 20, 0.6, mode=0)[0]
    _, band = oracle.band(mask, 2)
    b = oracle.bgk_run(f0, mask, 20, 0.6, mode=1, band=band)[0]
    c = oracle.bgk_run(f0, mask, 20, 0.6, mode=1, band=None)[0]
    np.testing.assert_allclose(b, a, rtol=0, atol=1e-14)
    np.testing.assert_allclose(c, a, rtol=0, atol=1e-14)
    d = oracle.bgk_run(f0, mask, 20, 0.6, mode=1, band=band, omega_s=1.2)[0]
    assert np.abs(d - a).max() > 1e-8                        # the shear rate does act


def test_home_close_to_bgk_on_smooth_flow(oracle):
    n = 24
    rho, u, v, w = W.taylor_green_3d(n, n, n, 0.03)
    fb, rb, ub, vb, wb, _ = oracle.bgk_run(oracle.reinit_eq(rho, u, v, w), None, 41, 0.6)
    m0 = np.zeros((10, n, n, n)); m0[0], m0[1], m0[2], m0[3] = rho, u, v, w
    m, _ = oracle.home_run(m0, None, 40, 0.6)
    err = np.linalg.norm(m[1] - ub) / np.linalg.norm(ub)
    assert err < 0.02


def test_duct_inflow_reaches_outlet(oracle):
    nx, ny, nz = 30, 10, 10
    mask = W.duct_mask(nx, ny, nz)
    one = np.ones((nz, ny, nx))
    f0 = oracle.reinit_eq(one, None, None, None)
    f, rho, ux, *_ = oracle.bgk_run(f0, mask, 300, 0.6, bc=1, u_in=0.03)
    fl = mask == 0
    assert np.all(np.isfinite(f))
    assert ux[fl].mean() > 0.01                          # flow established along the duct
    assert ux[:, :, -1][fl[:, :, -1]].mean() > 0.01      # and leaves through the outlet


def test_fp32_twin_tracks_fp64(oracle):
    n = 16
    rho, u, v, w = W.taylor_green_3d(n, n, n, 0.05)
    a = oracle.bgk_run(oracle.reinit_eq(rho, u, v, w), None, 20, 0.6)
    b = oracle.bgk_run(oracle.reinit_eq(rho, u, v, w, np.float32), None, 20, 0.6, dtype=np.float32)
    assert np.linalg.norm(b[0] - a[0]) / np.linalg.norm(a[0]) < 1e-5
