"""lbm_step_graph: replayed CUDA graphs against plain lbm_step calls.

A solver stepped through lbm_step_graph must end in the state a twin stepped
through lbm_step reaches, bit for bit, whatever the substep count's parity,
with statistics on or off, and across setters that change the captured work
(force, mask, statistics, macro output).  A read-back queued on the copy
stream before a replay must see the fields as they were before the replay.
"""
import ctypes as C

import numpy as np
import pytest

from myfluidsimulation_b200 import workloads as W
from myfluidsimulation_b200.solvers import BC_DUCT, METHOD_HOME, METHOD_HYBRID, METHOD_LEGACY, STORE_F16, Solver

pytestmark = pytest.mark.gpu

DIMS = (40, 18, 14)


def _mask(seed):
    nx, ny, nz = DIMS
    rng = np.random.default_rng(seed)
    m = np.zeros((nz, ny, nx), np.uint8)
    m[5:8, 6:10, 12:16] = 1
    m.ravel()[rng.integers(0, m.size, size=20)] = 1
    return W.duct_mask(nx, ny, nz, m)


def _fields(seed):
    rng = np.random.default_rng(seed)
    rho, u, v, w = W.taylor_green_3d(*DIMS, 0.04)
    return rho + (1e-3 * rng.standard_normal(rho.shape)).astype(np.float32), u, v, w


def _twin(method, storage):
    s = Solver(*DIMS, 0.58, method=method, storage=storage, bc=BC_DUCT, inlet_u=0.05)
    s.set_solid_mask(_mask(1))
    if method == METHOD_HYBRID:
        s.build_band(2)
        s.set_shear_omega(1.0 / 0.62)
    s.reinit_from_host(*_fields(2))
    return s


@pytest.mark.parametrize("method,storage", [(METHOD_LEGACY, 0), (METHOD_HYBRID, 0), (METHOD_HOME, 0),
                                            (METHOD_LEGACY, STORE_F16), (METHOD_HOME, STORE_F16)])
def test_step_graph_matches_step(gpu, method, storage):
    a, b = _twin(method, storage), _twin(method, storage)

    def both(fn):
        fn(a, False)
        fn(b, True)

    def adv(n):
        return lambda s, g: s.step_graph(n) if g else s.step(n)

    script = [adv(5), adv(4), adv(5),                                   # odd, even, odd again (graph reused)
              lambda s, g: s.enable_stats(True), adv(3), adv(3),
              lambda s, g: s.set_force(2e-5, 0, 0), adv(4),
              lambda s, g: s.set_macro_output(False), adv(3),
              lambda s, g: s.set_macro_output(True), adv(2),
              lambda s, g: s.set_solid_mask(_mask(7)), adv(5),
              lambda s, g: s.enable_stats(False), adv(6)]
    for k, op in enumerate(script):
        both(op)
        if k in (2, 5, 9, 13):
            a.synchronize()
            b.synchronize()
            np.testing.assert_array_equal(b.state(), a.state())
    a.synchronize()
    b.synchronize()
    assert a.steps == b.steps == 5 + 4 + 5 + 3 + 3 + 4 + 3 + 2 + 5 + 6
    np.testing.assert_array_equal(b.state(), a.state())
    for x, y in zip(b.macros(), a.macros()):
        np.testing.assert_array_equal(x, y)
    a.enable_stats(True)
    b.enable_stats(True)
    a.step(2)
    b.step_graph(2)
    sa, sb = a.stats(), b.stats()
    assert sa == sb
    a.close()
    b.close()


@pytest.mark.parametrize("method", [METHOD_LEGACY, METHOD_HOME])
def test_step_graph_waits_for_async_read(gpu, method):
    """lbm_read_macros_async, then lbm_step_graph, then lbm_wait_reads: the host
    copy holds the fields from before the replayed steps."""
    import torch
    from myfluidsimulation_b200._lib import check, lib
    L = lib()
    s = _twin(method, 0)
    s.step_graph(4)          # capture once, so the replay below launches at once
    s.synchronize()
    want = [x.copy() for x in s.macros()]
    nx, ny, nz = DIMS
    outs = [torch.zeros(nx * ny * nz, dtype=torch.float32, pin_memory=True).numpy() for _ in range(4)]
    stats = torch.zeros(8, dtype=torch.float64, pin_memory=True).numpy()
    s.enable_stats(True)
    s.step(2)
    s.synchronize()
    want_stats = np.array(list(s.stats().values())[:8])
    want = [x.copy() for x in s.macros()]
    for rep in range(3):
        check(L.lbm_read_macros_async(s._h, *[o.ctypes.data_as(C.c_void_p) for o in outs]))
        check(L.lbm_get_stats_async(s._h, stats.ctypes.data_as(C.c_void_p)))
        for _ in range(5):
            s.step_graph(4)
        check(L.lbm_wait_reads(s._h))
        s.synchronize()
        for o, w in zip(outs, want):
            np.testing.assert_array_equal(o.reshape(nz, ny, nx), w)
        np.testing.assert_array_equal(stats, want_stats)
        want = [x.copy() for x in s.macros()]
        want_stats = np.array(list(s.stats().values())[:8])
    s.close()
