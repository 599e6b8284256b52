"""Parity of the CUDA path (through the C-ABI) with the FP64 oracle.

Each case runs the same seeded input through liblbm_b200 and through the C
restatement of the reference's step functions in FP64, and compares the
macro fields, the full state and (where enabled) the FP64 statistics.
Tolerances are relative L2 (FP32 arithmetic against FP64 over <= 100 steps:
the reference's own FP32 kernels drift by ~2e-6..5e-6 over that span).
"""
import numpy as np
import pytest

from myfluidsimulation_b200 import workloads as W
from myfluidsimulation_b200.solvers import (BC_DUCT, BC_PERIODIC, BOUNCE_HALFWAY, BOUNCE_REFERENCE, METHOD_HOME,
                                            METHOD_HYBRID, METHOD_LEGACY, STORE_F16, STORE_F32, Solver)

pytestmark = pytest.mark.gpu

TOL_F = 2e-5      # populations, rho, u (FP32 vs FP64, <= 100 steps)
TOL_S = 5e-4      # HOME non-equilibrium stress (small, cancellation-limited)


def rl2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    d = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (d if d > 0 else 1.0)


def vel_err(us, ur):
    """relative L2 of the velocity vector field"""
    return rl2(np.stack(us), np.stack(ur))


def obstacle_mask(nx, ny, nz, seed=0, duct=False):
    rng = np.random.default_rng(seed)
    m = np.zeros((nz, ny, nx), np.uint8)
    # a block obstacle and a few scattered solid cells
    m[nz // 3: nz // 3 + 3, ny // 3: ny // 3 + 4, nx // 3: nx // 3 + 3] = 1
    idx = rng.integers(0, m.size, size=max(3, m.size // 200))
    m.ravel()[idx] = 1
    if duct:
        m = W.duct_mask(nx, ny, nz, m)
    return m


def init_fields(nx, ny, nz, seed=1, u0=0.04):
    rng = np.random.default_rng(seed)
    rho, u, v, w = W.taylor_green_3d(nx, ny, nz, u0)
    rho = rho + (1e-3 * rng.standard_normal(rho.shape)).astype(np.float32)
    w = (0.01 * rng.standard_normal(w.shape)).astype(np.float32)
    return rho, u, v, w


def run_gpu(method, dims, tau, fields, mask, steps, force=(0, 0, 0), bc=BC_PERIODIC, u_in=0.0, band=None,
            omega_s=None, stats=False, chunks=None, bounce=BOUNCE_HALFWAY):
    nx, ny, nz = dims
    s = Solver(nx, ny, nz, tau, force, method=method, bc=bc, inlet_u=u_in, bounce=bounce)
    if mask is not None:
        s.set_solid_mask(mask)
    if band is not None:
        s.set_legacy_mapping(band)
    if omega_s is not None:
        s.set_shear_omega(omega_s)
    s.reinit_from_host(*fields)
    s.enable_stats(stats)
    for c in (chunks or [steps]):
        s.step(c)
    s.synchronize()
    out = dict(macros=s.macros(), state=s.state(), stats=s.stats() if stats else None)
    s.close()
    return out


def oracle_bgk(oracle, dims, tau, fields, mask, steps, force=(0, 0, 0), mode=0, band=None, omega_s=None, bc=0,
               u_in=0.0, bb=0, fnext=None):
    f0 = oracle.reinit_eq(*fields)
    f, rho, u, v, w, drag = oracle.bgk_run(f0, mask, steps, tau, force, mode=mode, band=band, omega_s=omega_s,
                                           bc=bc, u_in=u_in, bb=bb, fnext=fnext)
    return f, (rho, u, v, w), drag


CASES = [
    # (dims, tau, steps, with_mask, force)
    ((16, 16, 16), 0.6, 1, False, (0, 0, 0)),
    ((16, 16, 16), 0.6, 2, False, (0, 0, 0)),
    ((16, 16, 16), 0.6, 37, False, (0, 0, 0)),
    ((24, 10, 12), 0.56, 20, True, (1e-5, 0, 0)),
    ((17, 9, 11), 0.7, 15, True, (2e-6, -1e-6, 3e-6)),   # odd sizes: scalar even path, wraps
    ((32, 8, 1), 0.6, 9, True, (0, 0, 0)),               # a single z plane
    ((136, 5, 4), 0.6, 7, True, (1e-5, 0, 0)),           # 128-cell staged tiles, a partial second tile
    ((260, 3, 3), 0.58, 6, False, (0, 2e-6, 0)),         # three tiles per row, periodic x wrap
]


@pytest.mark.parametrize("bounce", [BOUNCE_HALFWAY, BOUNCE_REFERENCE])
@pytest.mark.parametrize("dims,tau,steps,with_mask,force", CASES)
def test_legacy_vs_oracle(gpu, oracle, dims, tau, steps, with_mask, force, bounce):
    nx, ny, nz = dims
    fields = init_fields(nx, ny, nz)
    mask = obstacle_mask(nx, ny, nz) if with_mask else None
    g = run_gpu(METHOD_LEGACY, dims, tau, fields, mask, steps, force, bounce=bounce)
    f, mac, _ = oracle_bgk(oracle, dims, tau, fields, mask, steps, force, bb=bounce)
    assert rl2(g["state"], f) < TOL_F
    assert rl2(g["macros"][0], mac[0]) < TOL_F
    assert vel_err(g["macros"][1:], mac[1:]) < TOL_F


@pytest.mark.parametrize("storage", [STORE_F32, STORE_F16])
def test_home_zchunk_does_not_change_results(gpu, storage):
    """The z-chunk only splits the planes among blocks: every chunk length gives the same bits."""
    dims = (40, 20, 23)
    fields = init_fields(*dims, seed=11)
    mask = obstacle_mask(*dims, seed=12)
    out = []
    for zc in (None, 1, 5, 23, 100):
        s = Solver(*dims, 0.6, (1e-5, 0, 0), method=METHOD_HOME, storage=storage)
        if zc is not None:
            s.home_zchunk = zc
            assert s.home_zchunk == min(zc, dims[2])
        s.set_solid_mask(mask)
        s.reinit_from_host(*fields)
        s.enable_stats(True)
        s.step(9)
        s.synchronize()
        out.append((s.state(), s.stats()))
        s.close()
    for st, sts in out[1:]:
        np.testing.assert_array_equal(st, out[0][0])
        for k in ("mass", "ke_sum"):
            assert abs(sts[k] - out[0][1][k]) <= 1e-12 * abs(out[0][1][k])
    with pytest.raises(RuntimeError):
        Solver(*dims, 0.6, method=METHOD_LEGACY).home_zchunk = 4


def test_legacy_split_calls_match_one_call(gpu):
    """step(3)+step(4) == step(7): the parity of the in-place pattern is carried across calls."""
    dims = (20, 12, 8)
    fields = init_fields(*dims)
    mask = obstacle_mask(*dims)
    a = run_gpu(METHOD_LEGACY, dims, 0.6, fields, mask, 7)
    b = run_gpu(METHOD_LEGACY, dims, 0.6, fields, mask, 7, chunks=[3, 4])
    np.testing.assert_array_equal(a["state"], b["state"])
    for x, y in zip(a["macros"], b["macros"]):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("bounce", [BOUNCE_HALFWAY, BOUNCE_REFERENCE])
@pytest.mark.parametrize("omega_s", [None, 1.3])
def test_hybrid_vs_oracle(gpu, oracle, omega_s, bounce):
    dims = (24, 14, 10)
    nx, ny, nz = dims
    fields = init_fields(nx, ny, nz, seed=3)
    mask = obstacle_mask(nx, ny, nz, seed=4)
    _, band = oracle.band(mask, 2)
    g = run_gpu(METHOD_HYBRID, dims, 0.6, fields, mask, 12, force=(1e-5, 0, 0), band=band, omega_s=omega_s,
                bounce=bounce)
    om = None if omega_s is None else omega_s
    # the Hybrid's second buffer is never initialised by its reinit (hybrid.cu:245-257): zeros here
    fn = np.zeros((19,) + fields[0].shape) if bounce == BOUNCE_REFERENCE else None
    f, mac, _ = oracle_bgk(oracle, dims, 0.6, fields, mask, 12, (1e-5, 0, 0), mode=1, band=band, omega_s=om,
                           bb=bounce, fnext=fn)
    assert rl2(g["state"], f) < TOL_F
    assert rl2(g["macros"][0], mac[0]) < TOL_F
    assert vel_err(g["macros"][1:], mac[1:]) < TOL_F


def test_hybrid_equals_legacy_by_default(gpu):
    """omega_s = omega_h makes the two collision forms the same arithmetic (hybrid.cu:264-267)."""
    dims = (16, 12, 10)
    fields = init_fields(*dims, seed=5)
    mask = obstacle_mask(*dims, seed=6)
    s = Solver(*dims, 0.6, method=METHOD_HYBRID)
    s.set_solid_mask(mask)
    nb = s.build_band(2)
    assert nb > 0
    s.reinit_from_host(*fields)
    s.step(10)
    s.synchronize()
    h = s.state()
    s.close()
    leg = run_gpu(METHOD_LEGACY, dims, 0.6, fields, mask, 10)
    assert rl2(h, leg["state"]) < 1e-6


@pytest.mark.parametrize("bounce", [BOUNCE_HALFWAY, BOUNCE_REFERENCE])
@pytest.mark.parametrize("dims,tau,steps,with_mask,force", CASES)
def test_home_vs_oracle(gpu, oracle, dims, tau, steps, with_mask, force, bounce):
    nx, ny, nz = dims
    rho, u, v, w = init_fields(nx, ny, nz, seed=7)
    mask = obstacle_mask(nx, ny, nz, seed=8) if with_mask else None
    g = run_gpu(METHOD_HOME, dims, tau, (rho, u, v, w), mask, steps, force, bounce=bounce)
    m0 = np.zeros((10,) + rho.shape)
    m0[0], m0[1], m0[2], m0[3] = rho, u, v, w
    m, _ = oracle.home_run(m0, mask, steps, tau, force, bb=bounce)
    st = g["state"]
    assert rl2(st[0], m[0]) < TOL_F
    assert rl2(st[1:4], m[1:4]) < TOL_F
    assert rl2(st[4:], m[4:]) < TOL_S
    assert rl2(g["macros"][0], m[0]) < TOL_F


# (30, 10, 9): nx not a multiple of the even step's 4-cell vectors, so vectors
# run across row ends, where the inlet and outlet cells sit; (31, 10, 9): odd nx
# (two-cell vectors across row ends; HOME's unpaired last column)
@pytest.mark.parametrize("dims", [(40, 18, 14), (136, 10, 8), (30, 10, 9), (31, 10, 9)])
@pytest.mark.parametrize("method", [METHOD_LEGACY, METHOD_HYBRID, METHOD_HOME])
def test_duct_vs_oracle(gpu, oracle, method, dims):
    """Velocity inlet / zero-gradient outlet / wall cells / obstacle; drag of the last step."""
    nx, ny, nz = dims
    sphere = np.zeros((nz, ny, nx), np.uint8)
    Z, Y, X = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    sphere[(X - 12) ** 2 + (Y - ny // 2) ** 2 + (Z - nz // 2) ** 2 <= 9] = 1
    mask = W.duct_mask(nx, ny, nz, sphere)
    rho = np.ones((nz, ny, nx), np.float32)
    u = np.full((nz, ny, nx), 0.04, np.float32)
    zero = np.zeros_like(u)
    steps = 30
    band = None
    if method == METHOD_HYBRID:
        _, band = oracle.band(mask, 2)
    g = run_gpu(method, dims, 0.58, (rho, u, zero, zero), mask, steps, bc=BC_DUCT, u_in=0.04, band=band,
                stats=True)
    if method == METHOD_HOME:
        m0 = np.zeros((10, nz, ny, nx))
        m0[0], m0[1] = rho, u
        m, drag = oracle.home_run(m0, mask, steps, 0.58, bc=1, u_in=0.04)
        assert rl2(g["state"][0], m[0]) < TOL_F
        assert rl2(g["state"][1:4], m[1:4]) < TOL_F
        mac = (m[0], m[1], m[2], m[3])
    else:
        f, mac, drag = oracle_bgk(oracle, dims, 0.58, (rho, u, zero, zero), mask, steps,
                                  mode=1 if method == METHOD_HYBRID else 0, band=band, bc=1, u_in=0.04)
        assert rl2(g["state"], f) < TOL_F
    assert rl2(g["macros"][0], mac[0]) < TOL_F
    assert vel_err(g["macros"][1:], mac[1:]) < TOL_F
    st = g["stats"]
    gd = np.array([st["drag_x"], st["drag_y"], st["drag_z"]])
    assert abs(drag[0]) > 0
    assert np.linalg.norm(gd - drag) / np.linalg.norm(drag) < 1e-4
    fluid = mask == 0
    assert abs(st["mass"] - np.float64(mac[0])[fluid].sum()) / st["mass"] < 1e-6


@pytest.mark.parametrize("method", [METHOD_LEGACY, METHOD_HOME])
def test_stats_match_macros(gpu, method):
    dims = (32, 16, 12)
    fields = init_fields(*dims, seed=11)
    mask = obstacle_mask(*dims, seed=12)
    g = run_gpu(method, dims, 0.6, fields, mask, 5, stats=True)
    rho, u, v, w = [np.float64(a) for a in g["macros"]]
    fluid = mask == 0
    st = g["stats"]
    assert abs(st["mass"] - rho[fluid].sum()) <= 1e-9 * rho.sum()
    ke = 0.5 * (u * u + v * v + w * w).sum()
    assert abs(st["ke_sum"] - ke) <= 1e-7 * ke
    assert abs(st["mom_x"] - (rho * u)[fluid].sum()) <= 1e-6 * np.abs(rho * u).sum()


def test_reset_and_null_reinit(gpu):
    dims = (12, 8, 6)
    for method in (METHOD_LEGACY, METHOD_HOME, METHOD_HYBRID):
        s = Solver(*dims, 0.6, method=method)
        s.reinit_from_host(*init_fields(*dims))
        s.step(3)
        s.reset()
        s.synchronize()
        rho, u, v, w = s.macros()
        assert np.all(rho == 1.0) and not u.any() and not v.any() and not w.any()
        st = s.state()
        if method == METHOD_HOME:
            assert np.all(st[0] == 1.0) and not st[1:].any()
        else:
            w19 = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, np.float32)
            np.testing.assert_array_equal(st, np.broadcast_to(w19[:, None, None, None], st.shape))
        s.close()


def test_periodic_mass_conservation_long(gpu):
    dims = (32, 32, 32)
    s = Solver(*dims, 0.6)
    s.reinit_from_host(*W.taylor_green_3d(*dims, 0.05))
    s.enable_stats(True)
    s.step(1)
    m0 = s.stats()["mass"]
    s.step(400)
    m1 = s.stats()["mass"]
    s.close()
    assert abs(m1 - m0) / m0 < 1e-5


@pytest.mark.parametrize("method", [METHOD_LEGACY, METHOD_HOME])
def test_pipelined_host_io_matches_synchronous(gpu, method):
    """lbm_stage_from_host / lbm_reinit_from_stage / lbm_read_macros_async give the
    fields that lbm_reinit_from_host / lbm_step / lbm_get_macros give, run by run."""
    import ctypes as C
    from myfluidsimulation_b200._lib import check, lib
    dims = (40, 18, 14)
    nx, ny, nz = dims
    mask = obstacle_mask(*dims, duct=True)
    runs = [init_fields(*dims, seed=k) for k in range(3)]
    L = lib()
    vp = lambda a: a.ctypes.data_as(C.c_void_p)

    def solver():
        s = Solver(*dims, 0.58, method=method, bc=BC_DUCT, inlet_u=0.05)
        s.set_solid_mask(mask)
        return s

    s = solver()
    want = []
    for f in runs:
        s.reinit_from_host(*f)
        s.step(7)
        want.append([x.copy() for x in s.macros()])
    s.close()
    s = solver()
    host = [[np.ascontiguousarray(x, np.float32) for x in f] for f in runs]
    outs = [[np.zeros((nz, ny, nx), np.float32) for _ in range(4)] for _ in range(3)]
    check(L.lbm_stage_from_host(s._h, *[vp(x) for x in host[0]]))
    for k in range(3):
        check(L.lbm_reinit_from_stage(s._h))
        if k + 1 < 3:
            check(L.lbm_stage_from_host(s._h, *[vp(x) for x in host[k + 1]]))
        check(L.lbm_step(s._h, 7))
        check(L.lbm_read_macros_async(s._h, *[vp(o) for o in outs[k]]))
    check(L.lbm_wait_reads(s._h))
    s.synchronize()
    s.close()
    for k in range(3):
        for a, b in zip(outs[k], want[k]):
            np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("storage,tol", [(1, 5e-3), (2, 4e-2)])
@pytest.mark.parametrize("method", [METHOD_LEGACY, METHOD_HYBRID])
@pytest.mark.parametrize("dims,bc", [((128, 12, 10), BC_DUCT), ((30, 10, 9), BC_DUCT), ((31, 10, 9), BC_DUCT),
                                     ((64, 10, 9), BC_PERIODIC), ((42, 9, 7), BC_PERIODIC)])
def test_narrow_storage_vs_oracle(gpu, oracle, storage, tol, method, dims, bc):
    """F16/BF16 populations (shifted, FP32 arithmetic) against the FP64 oracle:
    duct and periodic grids; cell counts divisible by 4 (four cells per thread
    in the even step) and not (42x9x7: two cells per thread)."""
    nx, ny, nz = dims
    duct = bc == BC_DUCT
    mask = obstacle_mask(*dims, seed=3, duct=duct)
    fields = init_fields(*dims, seed=4)
    steps = 21
    s = Solver(nx, ny, nz, 0.6, (0, 0, 0) if duct else (1e-5, 0, 0), method=method, storage=storage, bc=bc,
               inlet_u=0.04)
    s.set_solid_mask(mask)
    s.reinit_from_host(*fields)
    s.step(steps)
    s.synchronize()
    rho, u, v, w = s.macros()
    s.close()
    f0 = oracle.reinit_eq(*fields)
    _, r_o, u_o, v_o, w_o, _ = oracle.bgk_run(f0, mask, steps, 0.6, (0, 0, 0) if duct else (1e-5, 0, 0),
                                              mode=1 if method == METHOD_HYBRID else 0, bc=1 if duct else 0,
                                              u_in=0.04, band=np.zeros_like(mask) if method == METHOD_HYBRID else None)
    fl = mask == 0
    e_u = vel_err([u[fl], v[fl], w[fl]], [u_o[fl], v_o[fl], w_o[fl]])
    e_r = rl2(rho[fl] - 1.0, r_o[fl] - 1.0)
    print(f"storage {storage} method {method} dims {dims}: u rel L2 {e_u:.3e}, rho-1 rel L2 {e_r:.3e}")
    assert e_u < tol


@pytest.mark.parametrize("storage,tol", [(1, 2e-3), (2, 2e-2)])
@pytest.mark.parametrize("dims", [(64, 12, 10), (128, 8, 6), (192, 5, 4)])
def test_narrow_periodic_vs_oracle(gpu, oracle, storage, tol, dims):
    """F16/BF16 on periodic grids without solid cells (the 512^3 TGV's case):
    odd and even step counts, forces on all three axes, against the FP64 oracle
    and against the FP32 run (the error stays at the storage's rounding level)."""
    nx, ny, nz = dims
    fields = init_fields(*dims, seed=31)
    frc = (1e-5, -2e-6, 3e-6)
    for steps in (1, 8):
        s = Solver(nx, ny, nz, 0.6, frc, storage=storage)
        s.reinit_from_host(*fields)
        s.enable_stats(True)
        s.step(steps)
        s.synchronize()
        rho, u, v, w = s.macros()
        st = s.stats()
        s.close()
        ref = Solver(nx, ny, nz, 0.6, frc)
        ref.reinit_from_host(*fields)
        ref.enable_stats(True)
        ref.step(steps)
        ref.synchronize()
        r32 = ref.macros()
        st32 = ref.stats()
        ref.close()
        _, r_o, u_o, v_o, w_o, _ = oracle.bgk_run(oracle.reinit_eq(*fields), None, steps, 0.6, frc)
        e_u = vel_err([u, v, w], [u_o, v_o, w_o])
        e_32 = vel_err([u, v, w], list(r32[1:]))
        print(f"storage {storage} dims {dims} steps {steps}: u rel L2 {e_u:.3e} (vs FP32 {e_32:.3e})")
        assert e_u < tol and e_32 < tol
        assert abs(st["mass"] - st32["mass"]) <= 1e-4 * abs(st32["mass"])


def test_stats_async_equals_sync(gpu):
    """lbm_get_stats_async queues the same copy that lbm_get_stats waits for."""
    import ctypes as C
    import torch
    from myfluidsimulation_b200 import lib
    dims = (24, 16, 12)
    s = Solver(*dims, 0.6, (1e-5, 0, 0))
    s.set_solid_mask(obstacle_mask(*dims, seed=21))
    s.reinit_from_host(*init_fields(*dims, seed=22))
    s.enable_stats(True)
    got = []
    for k in range(3):
        s.step(5)
        buf = torch.zeros(8, dtype=torch.float64, pin_memory=True).numpy()
        assert lib().lbm_get_stats_async(s._h, buf.ctypes.data_as(C.c_void_p)) == 0
        got.append(buf)
    s.synchronize()
    final = s.stats()
    np.testing.assert_array_equal(got[-1], np.array([final[k] for k in ("mass", "ke_sum", "drag_x", "drag_y", "drag_z",
                                                                        "mom_x", "mom_y", "mom_z")]))
    assert not np.array_equal(got[0], got[-1])
    s.close()


@pytest.mark.parametrize("method", [METHOD_LEGACY, METHOD_HYBRID])
@pytest.mark.parametrize("bc", [BC_PERIODIC, BC_DUCT])
def test_f64_storage_vs_oracle(gpu, oracle, method, bc):
    """FP64 storage and arithmetic (the reference form of the precision
    measurements) against the FP64 oracle: the FP64 statistics agree to FP64
    rounding (1e-11 relative over 20 steps), the FP32 read-out of the state to
    FP32 rounding (1e-7)."""
    from myfluidsimulation_b200.solvers import STORE_F64
    dims = (40, 18, 14)
    nx, ny, nz = dims
    mask = obstacle_mask(*dims, seed=31, duct=bc == BC_DUCT)
    fields = init_fields(*dims, seed=32)
    band = oracle.band(mask, 2)[1] if method == METHOD_HYBRID else None
    steps, tau, u_in = 20, 0.58, 0.04 if bc == BC_DUCT else 0.0
    force = (1e-5, 0, 0) if bc == BC_PERIODIC else (0, 0, 0)
    s = Solver(*dims, tau, force, method=method, storage=STORE_F64, bc=bc, inlet_u=u_in)
    s.set_solid_mask(mask)
    if band is not None:
        s.set_legacy_mapping(band)
        s.set_shear_omega(1.0 / 0.61)
    s.reinit_from_host(*fields)
    s.step(steps - 1)
    s.enable_stats(True)
    s.step(1)
    s.synchronize()
    st, state = s.stats(), s.state()
    s.close()
    # the solver's parameters are FP32 (omega = 1/tau in FP32, force, inlet
    # speed): the oracle gets exactly those values
    f32 = lambda x: float(np.float32(x))
    tau_eff = 1.0 / float(np.float32(1.0) / np.float32(tau))
    f0 = oracle.reinit_eq(*[np.float64(a) for a in fields])
    f, r, u, v, w, drag = oracle.bgk_run(f0, mask, steps, tau_eff, tuple(f32(x) for x in force),
                                        mode=1 if band is not None else 0, band=band,
                                        omega_s=f32(1.0 / 0.61) if band is not None else None,
                                        bc=1 if bc == BC_DUCT else 0, u_in=f32(u_in))
    assert rl2(state, f) < 1e-7
    fluid = mask == 0
    mass = r[fluid].sum()
    ke = 0.5 * (u * u + v * v + w * w)[fluid].sum()
    mom = (r * u)[fluid].sum()
    assert abs(st["mass"] - mass) <= 1e-11 * mass
    assert abs(st["ke_sum"] - ke) <= 1e-11 * ke
    assert abs(st["mom_x"] - mom) <= 1e-11 * np.abs(r * u)[fluid].sum()
    if bc == BC_DUCT:
        assert np.linalg.norm(np.array([st["drag_x"], st["drag_y"], st["drag_z"]]) - drag) <= 1e-11 * np.linalg.norm(drag)
