"""Solver classes over the C-ABI.

``Solver`` is the general handle (method, storage precision, boundary).  The
classes ``LBM3D_Legacy``, ``LBM3D_Home`` and ``LBM3D_Hybrid`` mirror the
reference's solver classes (src/lbm/lbm3d_legacy.hpp:19-56,
src/lbm/lbm3d_home.hpp:15-46, src/lbm/lbm3d_hybrid.hpp:18-58): the same method
names, argument meanings and null semantics, with ``step`` synchronous as in
the reference.  Device pointers are plain integers (or objects with a
``data_ptr()`` method, such as torch tensors).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import (BC_DUCT, BC_PERIODIC, BOUNCE_HALFWAY, BOUNCE_REFERENCE, METHOD_HOME, METHOD_HYBRID,
                   METHOD_LEGACY, NSTAT, STORE_BF16, STORE_F16, STORE_F32, STORE_F64, check, lib)

STAT_NAMES = ("mass", "ke_sum", "drag_x", "drag_y", "drag_z", "mom_x", "mom_y", "mom_z")


@dataclass
class Domain:
    """struct Domain (src/lbm/lbm_common.hpp:6-10), same field names and defaults."""
    Nx: int = 128
    Ny: int = 128
    Nz: int = 96
    tau: float = 0.6
    forceX: float = 0.0
    forceY: float = 0.0
    forceZ: float = 0.0


def _ptr(x):
    if x is None:
        return None
    if hasattr(x, "data_ptr"):
        return C.c_void_p(x.data_ptr())
    return C.c_void_p(int(x))


def _host(a, dtype, n):
    if a is None:
        return None, None
    arr = np.ascontiguousarray(a, dtype=dtype)
    if arr.size != n:
        raise ValueError(f"expected {n} elements, got {arr.size}")
    return arr, arr.ctypes.data_as(C.c_void_p)


class Solver:
    """One D3Q19 solver on the GPU (Legacy, HOME or Hybrid; F32/F16/BF16; periodic or duct)."""

    def __init__(self, nx, ny, nz, tau, force=(0.0, 0.0, 0.0), method=METHOD_LEGACY, storage=STORE_F32,
                 bc=BC_PERIODIC, inlet_u=0.0, rho0=1.0, stream=None, bounce=BOUNCE_HALFWAY):
        L = lib()
        d = _lib.Domain(int(nx), int(ny), int(nz), float(tau), *[float(f) for f in force])
        o = _lib.Options(int(method), int(storage), int(bc), int(bounce), float(inlet_u), float(rho0),
                         None if stream is None else C.c_void_p(int(stream)))
        h = C.c_void_p()
        check(L.lbm_create(C.byref(d), C.byref(o), C.byref(h)))
        self._h = h
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.N = self.nx * self.ny * self.nz
        self.shape = (self.nz, self.ny, self.nx)
        self.method, self.storage, self.bc, self.bounce = method, storage, bc, bounce

    # -- lifecycle -------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            lib().lbm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- set-up ------------------------------------------------------------------
    def set_solid_mask(self, mask):
        arr, p = _host(mask, np.uint8, self.N)
        check(lib().lbm_set_solid_mask(self._h, p))

    def set_legacy_mapping(self, band):
        if band is None:
            check(lib().lbm_set_legacy_mapping(self._h, None))
        else:
            arr, p = _host(band, np.uint8, self.N)
            check(lib().lbm_set_legacy_mapping(self._h, p))

    def build_band(self, d0: int) -> int:
        n = C.c_int64()
        check(lib().lbm_build_band(self._h, int(d0), C.byref(n)))
        return n.value

    def band(self) -> np.ndarray:
        out = np.empty(self.shape, np.uint8)
        check(lib().lbm_get_band(self._h, out.ctypes.data_as(C.c_void_p)))
        return out

    def reset(self):
        check(lib().lbm_reset(self._h))

    def reinit_from_macro(self, d_rho=None, d_ux=None, d_uy=None, d_uz=None):
        check(lib().lbm_reinit_from_macro(self._h, _ptr(d_rho), _ptr(d_ux), _ptr(d_uy), _ptr(d_uz)))

    def reinit_from_host(self, rho=None, ux=None, uy=None, uz=None):
        keep = [_host(a, np.float32, self.N) for a in (rho, ux, uy, uz)]
        check(lib().lbm_reinit_from_host(self._h, *[k[1] for k in keep]))
        self.synchronize()

    def set_force(self, fx, fy=0.0, fz=0.0):
        check(lib().lbm_set_force(self._h, float(fx), float(fy), float(fz)))

    def set_shear_omega(self, omega_s):
        check(lib().lbm_set_shear_omega(self._h, float(omega_s)))

    @property
    def home_zchunk(self):
        z = C.c_int()
        check(lib().lbm_home_zchunk(self._h, C.byref(z)))
        return z.value

    @home_zchunk.setter
    def home_zchunk(self, zchunk):
        check(lib().lbm_set_home_zchunk(self._h, int(zchunk)))

    def enable_stats(self, on=True):
        check(lib().lbm_enable_stats(self._h, 1 if on else 0))

    def set_macro_output(self, on=True):
        check(lib().lbm_set_macro_output(self._h, 1 if on else 0))

    # -- stepping ----------------------------------------------------------------
    def step(self, n: int = 1):
        """Queue n steps (asynchronous)."""
        check(lib().lbm_step(self._h, int(n)))

    def step_graph(self, n: int):
        check(lib().lbm_step_graph(self._h, int(n)))

    def synchronize(self):
        check(lib().lbm_synchronize(self._h))

    @property
    def steps(self) -> int:
        v = C.c_int64()
        check(lib().lbm_step_count(self._h, C.byref(v)))
        return v.value

    # -- outputs -----------------------------------------------------------------
    @property
    def stream(self) -> int:
        """The cudaStream_t this solver runs on."""
        p = C.c_void_p()
        check(lib().lbm_solver_stream(self._h, C.byref(p)))
        return p.value or 0

    def macro_ptrs(self):
        p = [C.c_void_p() for _ in range(4)]
        check(lib().lbm_macro_ptrs(self._h, *[C.byref(x) for x in p]))
        return tuple(x.value for x in p)

    def macros(self):
        out = [np.empty(self.shape, np.float32) for _ in range(4)]
        check(lib().lbm_get_macros(self._h, *[o.ctypes.data_as(C.c_void_p) for o in out]))
        return tuple(out)

    def state(self) -> np.ndarray:
        nc = 10 if self.method == METHOD_HOME else 19
        out = np.empty((nc,) + self.shape, np.float32)
        check(lib().lbm_get_state(self._h, out.ctypes.data_as(C.c_void_p)))
        return out

    def stats(self) -> dict:
        out = np.zeros(NSTAT, np.float64)
        check(lib().lbm_get_stats(self._h, out.ctypes.data_as(C.c_void_p)))
        d = dict(zip(STAT_NAMES, out.tolist()))
        d["ke_mean"] = d["ke_sum"] / self.N
        return d


class _RefSolver:
    """Common surface of the reference's solver classes.

    bounce defaults to BOUNCE_REFERENCE, the reference's own reflection table,
    so that results match the reference's; BOUNCE_HALFWAY selects true
    halfway bounce-back (and, for Legacy/Hybrid, the in-place AA kernels)."""

    _method = METHOD_LEGACY

    def __init__(self, storage=STORE_F32, bc=BC_PERIODIC, inlet_u=0.0, bounce=BOUNCE_REFERENCE):
        self._opts = dict(storage=storage, bc=bc, inlet_u=inlet_u, bounce=bounce)
        self._s = None

    def init(self, d: Domain):
        self._s = Solver(d.Nx, d.Ny, d.Nz, d.tau, (d.forceX, d.forceY, d.forceZ), method=self._method,
                         **self._opts)

    def setSolidMask(self, h_mask):
        self._s.set_solid_mask(h_mask)

    def reset(self):
        self._s.reset()
        self._s.synchronize()

    def reinitEquilibriumFromMacro(self, d_rho, d_ux, d_uy, d_uz):
        self._s.reinit_from_macro(d_rho, d_ux, d_uy, d_uz)
        self._s.synchronize()

    def step(self, substeps: int = 1):
        self._s.step(substeps)
        self._s.synchronize()

    def setForce(self, fx, fy=0.0, fz=0.0):
        self._s.set_force(fx, fy, fz)

    def d_rho(self):
        return self._s.macro_ptrs()[0]

    def d_u(self):
        return self._s.macro_ptrs()[1]

    def d_v(self):
        return self._s.macro_ptrs()[2]

    def d_w(self):
        return self._s.macro_ptrs()[3]

    def Nx(self):
        return self._s.nx

    def Ny(self):
        return self._s.ny

    def Nz(self):
        return self._s.nz

    def N(self):
        return self._s.N

    @property
    def solver(self) -> Solver:
        return self._s


class LBM3D_Legacy(_RefSolver):
    _method = METHOD_LEGACY


class LBM3D_Home(_RefSolver):
    _method = METHOD_HOME


class LBM3D_Hybrid(_RefSolver):
    _method = METHOD_HYBRID

    def init(self, d: Domain, nLegacyCells: int = 0):   # the count is ignored, as in the reference
        super().init(d)

    def setLegacyMapping(self, h_isLegacy, h_legacySlot_ignored=None):
        self._s.set_legacy_mapping(h_isLegacy)


__all__ = ["Domain", "Solver", "LBM3D_Legacy", "LBM3D_Home", "LBM3D_Hybrid", "METHOD_LEGACY", "METHOD_HOME",
           "METHOD_HYBRID", "STORE_F32", "STORE_F16", "STORE_BF16", "STORE_F64", "BC_PERIODIC", "BC_DUCT", "BOUNCE_HALFWAY",
           "BOUNCE_REFERENCE"]


class Batch:
    """Many Legacy/Hybrid solvers advanced together by one persistent launch per
    substep (lbm_batch_* in include/lbm_capi.h).  The solvers stay owned by the
    caller and must outlive the batch."""

    def __init__(self, solvers, stream=None):
        L = lib()
        self._solvers = list(solvers)
        arr = (C.c_void_p * len(self._solvers))(*[s._h.value for s in self._solvers])
        h = C.c_void_p()
        check(L.lbm_batch_create(arr, len(self._solvers), None if stream is None else C.c_void_p(int(stream)),
                                 C.byref(h)))
        self._h = h
        self.n = len(self._solvers)
        self.cells = sum(s.N for s in self._solvers)

    def close(self):
        if getattr(self, "_h", None):
            lib().lbm_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def refresh(self):
        check(lib().lbm_batch_refresh(self._h))

    def tune(self, trial_pairs: int = 2) -> dict:
        t = _lib.BatchTuning()
        check(lib().lbm_batch_tune(self._h, int(trial_pairs), C.byref(t)))
        return {k: getattr(t, k) for k, _ in _lib.BatchTuning._fields_}

    def set_tuning(self, threads=256, blocks_per_sm=4, even_unit=512, odd_unit=8):
        t = _lib.BatchTuning(threads, blocks_per_sm, even_unit, odd_unit, 0.0)
        check(lib().lbm_batch_set_tuning(self._h, C.byref(t)))

    def tuning(self) -> dict:
        t = _lib.BatchTuning()
        check(lib().lbm_batch_get_tuning(self._h, C.byref(t)))
        return {k: getattr(t, k) for k, _ in _lib.BatchTuning._fields_}

    def step(self, n: int = 1):
        check(lib().lbm_batch_step(self._h, int(n)))

    def synchronize(self):
        check(lib().lbm_batch_synchronize(self._h))

    def enable_stats(self, on=True):
        check(lib().lbm_batch_enable_stats(self._h, 1 if on else 0))

    def stats(self) -> np.ndarray:
        out = np.zeros((self.n, NSTAT), np.float64)
        check(lib().lbm_batch_get_stats(self._h, out.ctypes.data_as(C.c_void_p)))
        return out
