"""Batched instances (lbm_batch_*): one persistent launch per step over many
uneven Legacy/Hybrid instances must give, bit for bit, the states that
stepping each instance on its own gives (the same per-cell code runs), and
per-instance statistics equal to the single-instance ones up to the order of
the FP64 sums."""
import numpy as np
import pytest

from myfluidsimulation_b200 import workloads as W
from myfluidsimulation_b200._lib import LBMError
from myfluidsimulation_b200.solvers import (BC_DUCT, BC_PERIODIC, METHOD_HOME, METHOD_HYBRID, METHOD_LEGACY,
                                            STORE_BF16, STORE_F16, STORE_F32, STORE_F64, Batch, Solver)

pytestmark = pytest.mark.gpu

SPECS = [
    # (dims, tau, method, bc, b0)
    ((48, 32, 32), 0.56, METHOD_HYBRID, BC_DUCT, 2),
    ((64, 16, 48), 0.7, METHOD_LEGACY, BC_DUCT, 0),
    ((32, 48, 16), 0.52, METHOD_HYBRID, BC_DUCT, 0),
    ((80, 32, 32), 0.6, METHOD_HYBRID, BC_DUCT, 6),
    ((24, 20, 18), 0.65, METHOD_LEGACY, BC_PERIODIC, 0),
    ((300, 8, 6), 0.58, METHOD_HYBRID, BC_PERIODIC, 1),    # rows longer than a block
]


def make(spec, seed, storage=STORE_F32):
    dims, tau, method, bc, b0 = spec
    nx, ny, nz = dims
    rng = np.random.default_rng(seed)
    mask = np.zeros((nz, ny, nx), np.uint8)
    mask[nz // 3: nz // 3 + 3, ny // 3: ny // 3 + 4, nx // 4: nx // 4 + 3] = 1
    mask.ravel()[rng.integers(0, mask.size, size=mask.size // 150)] = 1
    if bc == BC_DUCT:
        mask = W.duct_mask(nx, ny, nz, mask)
    s = Solver(nx, ny, nz, tau, (1e-6, 0, 0) if bc == BC_PERIODIC else (0, 0, 0), method=method, bc=bc,
               inlet_u=0.04, storage=storage)
    s.set_solid_mask(mask)
    if method == METHOD_HYBRID:
        s.build_band(b0)
    rho = (1.0 + 1e-3 * rng.standard_normal((nz, ny, nx))).astype(np.float32)
    u = (0.02 * rng.standard_normal((nz, ny, nx))).astype(np.float32)
    s.reinit_from_host(rho, u, None, None)
    return s


# cell counts that are odd (1575), even but not a multiple of 4 (4050) and multiples of 4 (2700, 1512)
SPECS_ODD = [
    ((25, 9, 7), 0.6, METHOD_LEGACY, BC_PERIODIC, 0),
    ((18, 15, 15), 0.57, METHOD_HYBRID, BC_DUCT, 1),
    ((30, 10, 9), 0.62, METHOD_LEGACY, BC_DUCT, 0),
    ((27, 8, 7), 0.6, METHOD_LEGACY, BC_DUCT, 0),      # odd nx in a duct, 1512 cells
]


def run_single(steps_list, stats=False, storage=STORE_F32, specs=SPECS):
    out = []
    for i, spec in enumerate(specs):
        s = make(spec, i, storage)
        s.enable_stats(stats)
        for n in steps_list:
            s.step(n)
        s.synchronize()
        out.append((s.state(), s.stats() if stats else None))
        s.close()
    return out


@pytest.mark.parametrize("steps_list", [[1], [1, 1, 1], [7], [3, 20, 1]])
def test_batch_bit_identical_to_single(gpu, steps_list):
    ref = run_single(steps_list)
    solvers = [make(spec, i) for i, spec in enumerate(SPECS)]
    b = Batch(solvers)
    for n in steps_list:
        b.step(n)
    b.synchronize()
    for (st, _), s in zip(ref, solvers):
        np.testing.assert_array_equal(s.state(), st)
    b.close()
    for s in solvers:
        s.close()


@pytest.mark.parametrize("storage", [STORE_F16, STORE_BF16])
def test_narrow_batch_bit_identical_to_single(gpu, storage):
    """F16/BF16 instances: the batch's even step takes the single solver's
    four-cell vectors, and the stochastic rounding draws its bits by cell index,
    so batched states equal the single-instance ones bit for bit."""
    ref = run_single([3, 20, 1], stats=True, storage=storage)
    solvers = [make(spec, i, storage) for i, spec in enumerate(SPECS)]
    b = Batch(solvers)
    b.enable_stats(True)
    for n in (3, 20, 1):
        b.step(n)
    st = b.stats()
    for i, ((state, sref), s) in enumerate(zip(ref, solvers)):
        np.testing.assert_array_equal(s.state(), state)
        assert st[i, 0] == pytest.approx(sref["mass"], rel=1e-11), i
    b.close()
    for s in solvers:
        s.close()


@pytest.mark.parametrize("storage", [STORE_F32, STORE_F16, STORE_BF16])
def test_any_cell_count_batch_bit_identical_to_single(gpu, storage):
    """Instances whose cell counts are odd or not multiples of 4: each one's even
    step takes the vector width its own step takes for that count."""
    ref = run_single([5, 2], storage=storage, specs=SPECS_ODD)
    solvers = [make(spec, i, storage) for i, spec in enumerate(SPECS_ODD)]
    b = Batch(solvers)
    b.step(5)
    b.step(2)
    b.synchronize()
    for (state, _), s in zip(ref, solvers):
        np.testing.assert_array_equal(s.state(), state)
    b.close()
    for s in solvers:
        s.close()


@pytest.mark.parametrize("tuning", [dict(threads=128, blocks_per_sm=2, even_unit=128, odd_unit=1),
                                    dict(threads=256, blocks_per_sm=8, even_unit=4096, odd_unit=16)])
def test_batch_launch_shapes_and_stats(gpu, tuning):
    ref = run_single([5, 4], stats=True)
    solvers = [make(spec, i) for i, spec in enumerate(SPECS)]
    b = Batch(solvers)
    b.set_tuning(**tuning)
    b.enable_stats(True)
    b.step(5)
    b.step(4)
    st = b.stats()
    for i, ((state, sref), s) in enumerate(zip(ref, solvers)):
        np.testing.assert_array_equal(s.state(), state)
        for k, name in enumerate(("mass", "ke_sum", "drag_x", "drag_y", "drag_z", "mom_x", "mom_y", "mom_z")):
            assert st[i, k] == pytest.approx(sref[name], rel=1e-11, abs=1e-12), (i, name)
    b.close()
    for s in solvers:
        s.close()


def test_batch_tune_and_refresh(gpu):
    solvers = [make(spec, i) for i, spec in enumerate(SPECS)]
    b = Batch(solvers)
    t = b.tune(1)
    assert t["threads"] in (128, 256) and t["us_per_step"] > 0
    # reinitialise everything, then the batch must be refreshed before stepping
    fresh = [make(spec, i) for i, spec in enumerate(SPECS)]
    for s, f in zip(solvers, fresh):
        s.reinit_from_host(*[x for x in f.macros()])
        f.close()
    s0 = solvers[0]
    s0.step(1)                      # one instance out of step
    with pytest.raises(LBMError):
        b.step(1)
    with pytest.raises(LBMError):
        b.refresh()                 # parities differ
    s0.step(1)
    b.refresh()
    b.step(2)
    b.synchronize()
    b.close()
    for s in solvers:
        s.close()


def test_batch_rejects_unsupported_instances(gpu):
    a = Solver(16, 16, 16, 0.6, method=METHOD_HOME)
    c = Solver(16, 16, 16, 0.6, method=METHOD_LEGACY, storage=STORE_F16)
    d = Solver(16, 16, 16, 0.6, method=METHOD_LEGACY)
    f = Solver(16, 16, 16, 0.6, method=METHOD_LEGACY, storage=STORE_F64)
    g = Solver(18, 15, 15, 0.6, method=METHOD_LEGACY, storage=STORE_BF16)   # 4050 cells: any count is fine
    h = Solver(17, 15, 15, 0.6, method=METHOD_LEGACY)                        # odd count
    for bad in ([a], [d, a], [d, c], [f]):
        with pytest.raises(LBMError):
            Batch(bad)
    for ok in ([c], [g], [h]):
        Batch(ok).close()
    for s in (c, f, g, h):
        s.close()
    d.step(1)
    e = Solver(16, 16, 16, 0.6, method=METHOD_LEGACY)
    with pytest.raises(LBMError):
        Batch([d, e])               # different parities
    for s in (a, d, e):
        s.close()
