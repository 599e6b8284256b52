"""ctypes bindings to the checkers under oracle/ (test infrastructure only).

* ``Oracle``: oracle/liblbm_oracle.so, the C restatement (FP64 + FP32 twin).
* ``RefCPU``: oracle/_ref/libref_cpu.so, the reference's own geometry code.
* ``RefCUDA``: oracle/_ref/libref_cuda.so, the reference's own CUDA solvers.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
REF_DIR = os.path.join(ORACLE_DIR, "_ref")

_p = lambda a: a.ctypes.data_as(C.c_void_p) if a is not None else None


def _ensure_oracle():
    so = os.path.join(ORACLE_DIR, "liblbm_oracle.so")
    src = os.path.join(ORACLE_DIR, "lbm_oracle.c")
    if not os.path.exists(so) or os.path.getmtime(so) < max(
            os.path.getmtime(src), os.path.getmtime(os.path.join(ORACLE_DIR, "lbm_oracle_impl.h"))):
        subprocess.check_call(["bash", os.path.join(ORACLE_DIR, "build_ref.sh")])
    return so


class Oracle:
    """FP64 (or FP32 twin) CPU restatement of the reference step functions."""

    def __init__(self):
        self.lib = C.CDLL(_ensure_oracle())
        L = self.lib
        for sfx in ("f64", "f32"):
            getattr(L, "orc_bgk_step_" + sfx).restype = None
            getattr(L, "orc_home_step_" + sfx).restype = None
        L.orc_load_stl.restype = C.c_int64
        L.orc_load_stl.argtypes = [C.c_char_p, C.POINTER(C.c_void_p), C.c_void_p]
        L.orc_num_threads.restype = C.c_int

    # -- LBM ---------------------------------------------------------------
    @staticmethod
    def _rt(dtype):
        return (C.c_double, "f64") if dtype == np.float64 else (C.c_float, "f32")

    def reinit_eq(self, rho, ux, uy, uz, dtype=np.float64):
        ct, s = self._rt(dtype)
        N = rho.size
        f = np.empty((19,) + rho.shape, dtype)
        cv = lambda a: None if a is None else np.ascontiguousarray(a, dtype)
        r, u, v, w = cv(rho), cv(ux), cv(uy), cv(uz)
        getattr(self.lib, "orc_reinit_eq_" + s)(_p(r), _p(u), _p(v), _p(w), _p(f), C.c_int64(N))
        return f

    def bgk_run(self, f, mask, nsteps, tau, force=(0, 0, 0), mode=0, band=None, omega_s=None,
                bc=0, u_in=0.0, bb=0, dtype=np.float64, fnext=None):
        """Run nsteps Legacy (mode 0) / Hybrid (mode 1) steps; returns (f, rho, u, v, w, drag_of_last).

        bb=1 uses the reference's opposite table and buffer semantics; `fnext` is
        the second buffer's content on entry (default: a copy of f, as after the
        reference's reinitEquilibriumFromMacro)."""
        ct, s = self._rt(dtype)
        nz, ny, nx = f.shape[1:]
        a = np.ascontiguousarray(f, dtype).copy()
        b = a.copy() if fnext is None else np.ascontiguousarray(fnext, dtype).copy()
        mac = [np.zeros((nz, ny, nx), dtype) for _ in range(4)]
        m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
        bd = None if band is None else np.ascontiguousarray(band, np.uint8)
        om = ct(1.0 / np.float32(tau)) if dtype == np.float32 else ct(1.0 / tau)
        if dtype == np.float32:
            om = ct(np.float32(1.0) / np.float32(tau))
        oms = om if omega_s is None else ct(omega_s)
        drag = np.zeros(3, np.float64)
        getattr(self.lib, "orc_bgk_run_" + s)(
            _p(a), _p(b), *[_p(x) for x in mac], _p(m), _p(bd), C.c_int(mode),
            C.c_int(nx), C.c_int(ny), C.c_int(nz), om, om, oms,
            ct(force[0]), ct(force[1]), ct(force[2]), C.c_int(bc), ct(u_in), C.c_int(bb), C.c_int(nsteps),
            _p(drag))
        self.last_fnext = b
        return a, mac[0], mac[1], mac[2], mac[3], drag

    def home_run(self, m0, mask, nsteps, tau, force=(0, 0, 0), bc=0, u_in=0.0, bb=0, dtype=np.float64):
        ct, s = self._rt(dtype)
        nz, ny, nx = m0.shape[1:]
        a = np.ascontiguousarray(m0, dtype).copy()
        b = np.empty_like(a)
        mk = None if mask is None else np.ascontiguousarray(mask, np.uint8)
        om = ct(np.float32(1.0) / np.float32(tau)) if dtype == np.float32 else ct(1.0 / tau)
        drag = np.zeros(3, np.float64)
        getattr(self.lib, "orc_home_run_" + s)(
            _p(a), _p(b), _p(mk), C.c_int(nx), C.c_int(ny), C.c_int(nz), om,
            ct(force[0]), ct(force[1]), ct(force[2]), C.c_int(bc), ct(u_in), C.c_int(bb), C.c_int(nsteps),
            _p(drag))
        return a, drag

    # -- volume view -----------------------------------------------------------
    def raymarch(self, field, inv_pv, cam, step, scale, thresh, width, height):
        """The shader of src/render/Vis3D.cpp:30-78 on the CPU -> (rgba[h, w, 4], samples)."""
        f = np.ascontiguousarray(field, np.float32)
        nz, ny, nx = f.shape
        m = np.ascontiguousarray(inv_pv, np.float32).ravel()
        c = np.ascontiguousarray(cam, np.float32).ravel()
        out = np.empty((height, width, 4), np.float32)
        ns = C.c_int64()
        self.lib.orc_raymarch_f32(_p(f), C.c_int(nx), C.c_int(ny), C.c_int(nz), _p(m), _p(c), C.c_float(step),
                                  C.c_float(scale), C.c_float(thresh), C.c_int(width), C.c_int(height), _p(out),
                                  C.byref(ns))
        return out, ns.value

    # -- geometry ------------------------------------------------------------
    def band(self, mask, d0):
        m = np.ascontiguousarray(mask, np.uint8)
        nz, ny, nx = m.shape
        dist = np.empty(m.shape, np.int32)
        leg = np.empty(m.shape, np.uint8)
        self.lib.orc_band(_p(m), C.c_int(nx), C.c_int(ny), C.c_int(nz), C.c_int(d0), _p(dist), _p(leg))
        return dist, leg

    def load_stl(self, path):
        buf = C.c_void_p()
        bb = np.zeros(6, np.float32)
        n = self.lib.orc_load_stl(path.encode(), C.byref(buf), _p(bb))
        if n < 0:
            return None, None
        arr = np.ctypeslib.as_array(C.cast(buf, C.POINTER(C.c_float)), shape=(n * 9,)).copy()
        self.lib.orc_free(buf)
        return arr.reshape(n, 3, 3), bb

    def voxelize(self, tris, bb, dims, scale, translate, refine=1, thr=0.5):
        t = np.ascontiguousarray(tris, np.float32)
        bbv = np.ascontiguousarray(bb, np.float32)
        nx, ny, nz = dims
        out = np.empty((nz, ny, nx), np.uint8)
        self.lib.orc_voxelize(_p(t), C.c_int64(t.shape[0]), _p(bbv), C.c_int(nx), C.c_int(ny), C.c_int(nz),
                              C.c_float(scale), C.c_float(translate[0]), C.c_float(translate[1]),
                              C.c_float(translate[2]), C.c_int(refine), C.c_float(thr), _p(out))
        return out


def mesh_bbox(tris):
    """bbox exactly as the reference loader accumulates it (min/max over all vertices, float)."""
    v = np.asarray(tris, np.float32).reshape(-1, 3)
    return np.concatenate([v.min(0), v.max(0)]).astype(np.float32)


class RefCPU:
    """The reference's own stl_loader.cpp / voxelize.cpp / band BFS (compiled from its sources)."""

    path = os.path.join(REF_DIR, "libref_cpu.so")

    @classmethod
    def available(cls):
        return os.path.exists(cls.path)

    def __init__(self):
        self.lib = C.CDLL(self.path)
        self.lib.ref_load_stl.restype = C.c_int64

    def load_stl(self, path):
        bb = np.zeros(6, np.float32)
        n = self.lib.ref_load_stl(path.encode(), None, C.c_int64(0), _p(bb))
        if n < 0:
            return None, None
        out = np.empty((n, 3, 3), np.float32)
        self.lib.ref_load_stl(path.encode(), _p(out), C.c_int64(n), _p(bb))
        return out, bb

    def voxelize(self, tris, bb, dims, scale, translate, refine=1, thr=0.5):
        t = np.ascontiguousarray(tris, np.float32)
        bbv = np.ascontiguousarray(bb, np.float32)
        nx, ny, nz = dims
        out = np.empty((nz, ny, nx), np.uint8)
        self.lib.ref_voxelize(_p(t), C.c_int64(t.shape[0]), _p(bbv), C.c_int(nx), C.c_int(ny), C.c_int(nz),
                              C.c_float(scale), C.c_float(translate[0]), C.c_float(translate[1]),
                              C.c_float(translate[2]), C.c_int(refine), C.c_float(thr), _p(out))
        return out

    def build_obstacle(self, stl_path, dims, scale=0.5, translate=(0.5, 0.5, 0.5), amr=1, thr=0.5):
        nx, ny, nz = dims
        out = np.empty((nz, ny, nx), np.uint8)
        has = self.lib.ref_build_obstacle(stl_path.encode() if stl_path else None, C.c_int(nx), C.c_int(ny),
                                          C.c_int(nz), C.c_float(scale), C.c_float(translate[0]),
                                          C.c_float(translate[1]), C.c_float(translate[2]), C.c_int(amr),
                                          C.c_float(thr), _p(out))
        return has, out

    def band(self, mask, d0):
        m = np.ascontiguousarray(mask, np.uint8)
        nz, ny, nx = m.shape
        dist = np.empty(m.shape, np.int32)
        leg = np.empty(m.shape, np.uint8)
        self.lib.ref_band(_p(m), C.c_int(nx), C.c_int(ny), C.c_int(nz), C.c_int(d0), _p(dist), _p(leg))
        return dist, leg


class RefCUDA:
    """The reference's own CUDA solver classes (GPU only)."""

    path = os.path.join(REF_DIR, "libref_cuda.so")

    @classmethod
    def available(cls):
        return os.path.exists(cls.path)

    def __init__(self):
        self.lib = C.CDLL(self.path)
        self.lib.refcu_create.restype = C.c_void_p
        self.lib.refcu_last_error.restype = C.c_char_p
        for n in ("refcu_destroy", "refcu_set_mask", "refcu_set_legacy", "refcu_init_fields", "refcu_init_rho",
                  "refcu_step", "refcu_time_steps", "refcu_get_macros", "refcu_get_state"):
            getattr(self.lib, n).argtypes = None

    def _ck(self, rc):
        if rc != 0:
            raise RuntimeError(self.lib.refcu_last_error().decode())

    def create(self, method, dims, tau, force=(0, 0, 0)):
        nx, ny, nz = dims
        h = self.lib.refcu_create(C.c_int(method), C.c_int(nx), C.c_int(ny), C.c_int(nz), C.c_float(tau),
                                  C.c_float(force[0]), C.c_float(force[1]), C.c_float(force[2]))
        if not h:
            raise RuntimeError(self.lib.refcu_last_error().decode())
        return C.c_void_p(h)

    def destroy(self, h):
        self.lib.refcu_destroy(h)

    def set_mask(self, h, mask):
        m = np.ascontiguousarray(mask, np.uint8)
        self._ck(self.lib.refcu_set_mask(h, _p(m)))

    def set_legacy(self, h, leg):
        m = None if leg is None else np.ascontiguousarray(leg, np.uint8)
        self._ck(self.lib.refcu_set_legacy(h, _p(m)))

    def init_fields(self, h, rho, u, v, w):
        a = [np.ascontiguousarray(x, np.float32) for x in (rho, u, v, w)]
        self._ck(self.lib.refcu_init_fields(h, *[_p(x) for x in a]))

    def init_rho(self, h, rho=None):
        r = None if rho is None else np.ascontiguousarray(rho, np.float32)
        self._ck(self.lib.refcu_init_rho(h, _p(r)))

    def step(self, h, n=1):
        self._ck(self.lib.refcu_step(h, C.c_int(n)))

    def time_steps(self, h, calls, substeps=1):
        ms = C.c_float()
        self._ck(self.lib.refcu_time_steps(h, C.c_int(calls), C.c_int(substeps), C.byref(ms)))
        return ms.value

    def macros(self, h, shape):
        out = [np.empty(shape, np.float32) for _ in range(4)]
        self._ck(self.lib.refcu_get_macros(h, *[_p(x) for x in out]))
        return out

    def state(self, h, ncomp, shape):
        out = np.empty((ncomp,) + tuple(shape), np.float32)
        self._ck(self.lib.refcu_get_state(h, _p(out)))
        return out
