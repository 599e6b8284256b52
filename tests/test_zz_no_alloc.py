"""lbm_macro_stats_static (the statistics entry point that allocates nothing)
against the statistics lbm_step computes on the same fields.

Both sum the same FP32 values in FP64, in a different order, so they agree to
a relative 1e-10; two consecutive static calls agree bit for bit."""
import ctypes as C

import numpy as np
import pytest

from myfluidsimulation_b200 import _lib
from myfluidsimulation_b200 import workloads as W
from myfluidsimulation_b200.solvers import METHOD_HOME, METHOD_LEGACY, Solver

pytestmark = pytest.mark.gpu

SLOTS = [0, 1, 5, 6, 7]          # mass, KE, momentum x/y/z


def static_stats(ptrs, mask_dev, n, out_dev, stream=None):
    import torch
    rc = _lib.lib().lbm_macro_stats_static(*[C.c_void_p(p) for p in ptrs],
                                           None if mask_dev is None else C.c_void_p(mask_dev.data_ptr()),
                                           C.c_int64(n), C.c_void_p(out_dev.data_ptr()), stream)
    _lib.check(rc)
    torch.cuda.synchronize()
    return out_dev.cpu().numpy().copy()


def sphere_mask(dims, r):
    nx, ny, nz = dims
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    return (((x - nx / 2) ** 2 + (y - ny / 2) ** 2 + (z - nz / 2) ** 2) < r * r).astype(np.uint8)


@pytest.mark.parametrize("method", [METHOD_LEGACY, METHOD_HOME])
def test_static_stats_match_step_statistics(gpu, method):
    import torch
    dims = (48, 40, 36)
    n = int(np.prod(dims))
    mask = sphere_mask(dims, 7)
    s = Solver(*dims, 0.6, (1e-5, 0, 0), method=method)
    try:
        s.set_solid_mask(mask)
        rho, ux, uy, uz = W.taylor_green_3d(*dims, 0.05)
        s.reinit_from_host(rho, ux + 0.01, uy, uz)
        s.enable_stats(True)
        s.step(3)
        s.synchronize()
        want = s.stats()
        want = np.array([want[k] for k in ("mass", "ke_sum", "drag_x", "drag_y", "drag_z",
                                           "mom_x", "mom_y", "mom_z")])
        mask_dev = torch.from_numpy(mask.ravel()).cuda()
        out_dev = torch.full((_lib.NSTAT,), np.nan, dtype=torch.float64, device="cuda")
        first = static_stats(s.macro_ptrs(), mask_dev, n, out_dev)
        second = static_stats(s.macro_ptrs(), mask_dev, n, out_dev)
    finally:
        s.close()
    np.testing.assert_array_equal(first, second)
    scale = np.abs(want[SLOTS]).max()
    np.testing.assert_allclose(first[SLOTS], want[SLOTS], rtol=1e-10, atol=1e-12 * scale)
    assert np.all(first[2:5] == 0.0)


def test_static_stats_small_and_empty_inputs(gpu):
    import torch
    rng = np.random.default_rng(3)
    out_dev = torch.zeros(_lib.NSTAT, dtype=torch.float64, device="cuda")
    for n in (0, 1, 8191, 8192, 8193, 70001):
        f = [rng.standard_normal(max(n, 1)).astype(np.float32) for _ in range(4)]
        dev = [torch.from_numpy(a).cuda() for a in f]
        got = static_stats([t.data_ptr() for t in dev], None, n, out_dev)
        r, u, v, w = [a[:n].astype(np.float64) for a in f]
        want = np.array([r.sum(), 0.5 * (u * u + v * v + w * w).sum(), 0, 0, 0,
                         (r * u).sum(), (r * v).sum(), (r * w).sum()])
        np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-9)


def test_static_stats_rejects_oversized_and_null_inputs(gpu):
    import torch
    L = _lib.lib()
    buf = torch.zeros(16, device="cuda")
    out = torch.zeros(_lib.NSTAT, dtype=torch.float64, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    rc = L.lbm_macro_stats_static(p, p, p, p, None, C.c_int64(268435456 + 1), C.c_void_p(out.data_ptr()), None)
    assert rc == 4 and b"static scratch limit" in L.lbm_last_error()
    rc = L.lbm_macro_stats_static(p, None, p, p, None, C.c_int64(16), C.c_void_p(out.data_ptr()), None)
    assert rc == 1
    rc = L.lbm_macro_stats_static(p, p, p, p, None, C.c_int64(-1), C.c_void_p(out.data_ptr()), None)
    assert rc == 1
