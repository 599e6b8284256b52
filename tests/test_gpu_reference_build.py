"""Parity with the reference's OWN CUDA build (oracle/_ref/libref_cuda.so, compiled
from the reference's src/lbm, src/fields and src/moment_vtk_writer.cu by
oracle/build_ref.sh), run on the same GPU with the same FP32 inputs.

The library is driven with LBM_BOUNCE_REFERENCE where solid cells are present,
so both sides use the reference's reflection table.  Near solid cells the
reference's Legacy/Hybrid step writes some slots from two threads (a data race,
see lbm_push.cu); its results then vary from run to run (measured on a B200:
the same 64x32x32 Hybrid input gave 5004 and 6092 populations differing from a
fixed-rule emulation after 2 steps in two runs).  Those cases are compared over
the first steps, where the race has not yet changed any value beyond FP32
rounding, and bounded over longer runs by the spread the race produces.
"""
import os

import numpy as np
import pytest

from myfluidsimulation_b200 import workloads as W
from myfluidsimulation_b200.solvers import (BOUNCE_REFERENCE, METHOD_HOME, METHOD_HYBRID, METHOD_LEGACY, Solver)
from oracle_bind import RefCUDA

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not RefCUDA.available(), reason="reference CUDA build (oracle/_ref) not present")]


def rl2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel())


@pytest.fixture(scope="module")
def ref(gpu):
    return RefCUDA()


def run_mine(method, dims, tau, fields, mask=None, steps=1, force=(0, 0, 0), band=None, bounce=BOUNCE_REFERENCE):
    s = Solver(*dims, tau, force, method=method, bounce=bounce)
    if mask is not None:
        s.set_solid_mask(mask)
    if band is not None:
        s.set_legacy_mapping(band)
    s.reinit_from_host(*fields)
    s.step(steps)
    s.synchronize()
    out = s.macros(), s.state()
    s.close()
    return out


def run_ref(ref, method, dims, tau, fields, mask=None, steps=1, force=(0, 0, 0), band=None):
    h = ref.create(method, dims, tau, force)
    try:
        ref.set_mask(h, np.zeros(dims[::-1], np.uint8) if mask is None else mask)
        if band is not None:
            ref.set_legacy(h, band)
        ref.init_fields(h, *fields)
        for _ in range(steps):       # the reference's drivers call step(1) per outer step
            ref.step(h, 1)
        shape = dims[::-1]
        mac = ref.macros(h, shape)
        st = ref.state(h, 10 if method == 1 else 19, shape)
    finally:
        ref.destroy(h)
    return mac, st


@pytest.mark.parametrize("method", [METHOD_LEGACY, METHOD_HOME])
@pytest.mark.parametrize("steps", [1, 2, 25, 200])
def test_tgv64_matches_reference_build(ref, method, steps):
    """The 64^3 periodic Taylor-Green vortex, tau 0.6, u0 0.05."""
    dims = (64, 64, 64)
    fields = W.taylor_green_3d(*dims, 0.05)
    (mr, mu, mv, mw), sm = run_mine(method, dims, 0.6, fields, steps=steps)
    (rr, ru, rv, rw), sr = run_ref(ref, method, dims, 0.6, fields, steps=steps)
    # two FP32 evaluations of the same arithmetic in a different order: both
    # drift from the FP64 trajectory by ~2e-6 over 25 steps
    tol = 1e-5 if steps <= 25 else 5e-5
    assert rl2(mr, rr) < tol
    assert rl2(np.stack([mu, mv, mw]), np.stack([ru, rv, rw])) < tol
    assert rl2(sm, sr) < tol


def duct_like(dims, radius, center):
    """The reference-comparable duct: y/z faces as solid cells, a sphere, periodic x."""
    tris, scale, tr = W.duct_sphere_mesh(*dims, radius, center, levels=3)
    from myfluidsimulation_b200 import geometry as G
    sph = G.voxelize_mesh_to_mask(G.mesh_from_triangles(tris), G.VoxelParams(*dims, scale, tr))
    return (W.duct_mask(*dims, sph) != 0).astype(np.uint8)


def test_masked_home_matches_reference_build(ref, oracle):
    """HOME's reflection is deterministic in the reference: both the reference build
    and the library sit within FP32 rounding of the FP64 oracle (reference table)."""
    dims = (64, 32, 32)
    mask = duct_like(dims, 6, (20, 16, 16))
    rho = np.ones(dims[::-1], np.float32)
    zero = np.zeros_like(rho)
    fields = (rho, zero, zero, zero)
    (mr, mu, mv, mw), sm = run_mine(METHOD_HOME, dims, 0.56, fields, mask, 60, force=(1e-5, 0, 0))
    (rr, ru, rv, rw), sr = run_ref(ref, METHOD_HOME, dims, 0.56, fields, mask, 60, force=(1e-5, 0, 0))
    m0 = np.zeros((10,) + rho.shape)
    m0[0] = rho
    mo, _ = oracle.home_run(m0, mask, 60, 0.56, (1e-5, 0, 0), bb=1)
    e_ref = rl2(np.stack([ru, rv, rw]), mo[1:4])          # the reference build against the oracle
    e_mine = rl2(np.stack([mu, mv, mw]), mo[1:4])
    assert e_ref < 3e-4 and e_mine < 3e-4                  # u ~ 5e-4 here: FP32 noise ~1e-4 relative
    assert rl2(rr, mo[0]) < 3e-6 and rl2(mr, mo[0]) < 3e-6
    assert rl2(np.stack([mu, mv, mw]), np.stack([ru, rv, rw])) < 2 * max(e_ref, e_mine) + 1e-5


# (method, steps, bound on the relative L2 of the full population state)
PUSH_CASES = [
    (METHOD_LEGACY, 1, 1e-5), (METHOD_LEGACY, 2, 1e-5), (METHOD_LEGACY, 60, 3e-4),
    (METHOD_HYBRID, 1, 1e-5), (METHOD_HYBRID, 60, 5e-2),
]


@pytest.mark.parametrize("method,steps,bound", PUSH_CASES)
def test_masked_push_matches_reference_build(ref, oracle, method, steps, bound):
    """Legacy/Hybrid with solids: same reflection table, stale slots, two buffers.
    Exact to FP32 rounding over the first steps; afterwards the reference's own
    race (and, for Hybrid, its zero-filled second buffer, which makes a lost race
    replace a population by 0) bounds the agreement (measured 8.5e-5 / 2.1e-2
    after 60 steps)."""
    dims = (64, 32, 32)
    mask = duct_like(dims, 6, (20, 16, 16))
    rho = np.ones(dims[::-1], np.float32)
    zero = np.zeros_like(rho)
    fields = (rho, zero, zero, zero)
    band = oracle.band(mask, 2)[1] if method == METHOD_HYBRID else None
    (mr, mu, mv, mw), sm = run_mine(method, dims, 0.56, fields, mask, steps, force=(1e-5, 0, 0), band=band)
    (rr, ru, rv, rw), sr = run_ref(ref, method, dims, 0.56, fields, mask, steps, force=(1e-5, 0, 0), band=band)
    e = rl2(sm, sr)
    print(f"method {method} steps {steps}: rel L2 state {e:.3e}")
    assert e < bound


def test_free_functions_match_reference(ref):
    import ctypes as C
    import torch
    rng = np.random.default_rng(0)
    n = 5000
    u, v, w = [rng.standard_normal(n).astype(np.float32) * 0.05 for _ in range(3)]
    from myfluidsimulation_b200 import lib
    L = lib()
    du, dv, dw = [torch.from_numpy(a).cuda() for a in (u, v, w)]
    out = torch.empty(n, device="cuda")
    torch.cuda.synchronize()
    L.launch_speed(du.data_ptr(), dv.data_ptr(), dw.data_ptr(), out.data_ptr(), n)
    torch.cuda.synchronize()
    want = np.empty(n, np.float32)
    assert ref.lib.refcu_speed(*[C.c_void_p(a.ctypes.data) for a in (u, v, w, want)], C.c_int(n)) == 0
    np.testing.assert_array_equal(out.cpu().numpy(), want)
    dims = (23, 17, 9)
    N = int(np.prod(dims))
    d = torch.empty(N, device="cuda")
    for kind, params in ((0, [0.6, 0.5, 0.4, 0.08, 1e-3]), (1, [1, 2e-3, 0.45, 0.2])):
        if kind == 0:
            L.make_rho_gauss(d.data_ptr(), *dims, *params)
        else:
            L.make_rho_slab(d.data_ptr(), *dims, int(params[0]), *params[1:])
        torch.cuda.synchronize()
        want = np.empty(N, np.float32)
        pp = np.array(params, np.float32)
        ref.lib.refcu_rho_profile(C.c_int(kind), C.c_int(dims[0]), C.c_int(dims[1]), C.c_int(dims[2]),
                                  pp.ctypes.data_as(C.c_void_p), want.ctypes.data_as(C.c_void_p))
        np.testing.assert_array_equal(d.cpu().numpy(), want)


def test_reinit_free_function_matches_reference_state(ref):
    """reinit_equilibrium_from_macro (lbm_reinit.cu:52-61) == the reference Legacy's f after reinit."""
    import torch
    from myfluidsimulation_b200 import lib
    dims = (16, 12, 10)
    fields = W.taylor_green_3d(*dims, 0.05)
    N = int(np.prod(dims))
    dev = [torch.from_numpy(np.ascontiguousarray(a).ravel()).cuda() for a in fields]
    f = torch.empty(19 * N, device="cuda")
    torch.cuda.synchronize()
    lib().reinit_equilibrium_from_macro(*[t.data_ptr() for t in dev], f.data_ptr(), N)
    torch.cuda.synchronize()
    _, sr = run_ref(ref, 0, dims, 0.6, fields, steps=0)
    np.testing.assert_array_equal(f.cpu().numpy().reshape(sr.shape), sr)


def test_vtk_files_byte_identical(ref, tmp_path):
    import ctypes as C
    import torch
    from myfluidsimulation_b200 import lib
    dims = (7, 5, 3)
    rng = np.random.default_rng(1)
    a, b, c = [(rng.standard_normal(dims[::-1]) * 10.0 ** rng.integers(-9, 3, dims[::-1])).astype(np.float32)
               for _ in range(3)]
    a.ravel()[:3] = [0.0, -0.0, 1e-30]
    da, db, dc = [torch.from_numpy(x.ravel().copy()).cuda() for x in (a, b, c)]
    torch.cuda.synchronize()
    L = lib()
    mine_s, ref_s = str(tmp_path / "m_s.vtk"), str(tmp_path / "r_s.vtk")
    mine_v, ref_v = str(tmp_path / "m_v.vtk"), str(tmp_path / "r_v.vtk")
    L.write_scalar_vtk(mine_s.encode(), da.data_ptr(), *dims)
    L.write_vector_vtk(mine_v.encode(), da.data_ptr(), db.data_ptr(), dc.data_ptr(), *dims)
    vp = lambda x: C.c_void_p(x.ctypes.data)
    assert ref.lib.refcu_write_vtk(ref_s.encode(), vp(a), None, None, *dims) == 0
    assert ref.lib.refcu_write_vtk(ref_v.encode(), vp(a), vp(b), vp(c), *dims) == 0
    assert open(mine_s, "rb").read() == open(ref_s, "rb").read()
    assert open(mine_v, "rb").read() == open(ref_v, "rb").read()
