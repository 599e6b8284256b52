"""ctypes binding of liblbm_b200.so (the C-ABI declared in include/lbm_capi.h).

The library is the only implementation: if it is missing and cannot be built,
or no CUDA device is present when a solver is created, calls raise instead of
falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "liblbm_b200.so")

LBM_OK = 0
ERRORS = {1: "LBM_ERR_INVALID", 2: "LBM_ERR_CUDA", 3: "LBM_ERR_ALLOC", 4: "LBM_ERR_SIZE",
          5: "LBM_ERR_IO", 6: "LBM_ERR_UNSUPPORTED", 7: "LBM_ERR_TIMEOUT"}

METHOD_LEGACY, METHOD_HOME, METHOD_HYBRID = 0, 1, 2
STORE_F32, STORE_F16, STORE_BF16, STORE_F64 = 0, 1, 2, 3
VTK_SCALAR, VTK_SPEED, VTK_VECTOR = 0, 1, 2
FILTER_EXACT, FILTER_TEXTURE = 0, 1
BC_PERIODIC, BC_DUCT = 0, 1
BOUNCE_HALFWAY, BOUNCE_REFERENCE = 0, 1
NSTAT = 8


class LBMError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Domain(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("tau", C.c_float),
                ("force_x", C.c_float), ("force_y", C.c_float), ("force_z", C.c_float)]


class Options(C.Structure):
    _fields_ = [("method", C.c_int32), ("storage", C.c_int32), ("bc", C.c_int32), ("bounce", C.c_int32),
                ("inlet_u", C.c_float), ("rho0", C.c_float), ("stream", C.c_void_p)]


class VoxelParams(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("uniform_scale", C.c_float),
                ("translate", C.c_float * 3), ("refine", C.c_int32), ("coverage_threshold", C.c_float)]


class BatchTuning(C.Structure):
    _fields_ = [("threads", C.c_int32), ("blocks_per_sm", C.c_int32), ("even_unit", C.c_int32),
                ("odd_unit", C.c_int32), ("us_per_step", C.c_float)]


class AdjProblem(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("tau", C.c_double),
                ("force", C.c_double * 3), ("n_steps", C.c_int32), ("window_begin", C.c_int32),
                ("window_end", C.c_int32), ("checkpoint_every", C.c_int32), ("precision", C.c_int32)]


# (name, restype, argtypes)
class RenderParams(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("inv_pv", C.c_float * 16), ("cam_pos", C.c_float * 3),
                ("step", C.c_float), ("scale", C.c_float), ("threshold", C.c_float), ("filter", C.c_int32)]


_P = C.c_void_p
_PROTOS = [
    ("lbm_last_error", C.c_char_p, []),
    ("lbm_version", C.c_char_p, []),
    ("lbm_create", C.c_int, [C.POINTER(Domain), C.POINTER(Options), C.POINTER(_P)]),
    ("lbm_destroy", C.c_int, [_P]),
    ("lbm_set_solid_mask", C.c_int, [_P, _P]),
    ("lbm_set_legacy_mapping", C.c_int, [_P, _P]),
    ("lbm_build_band", C.c_int, [_P, C.c_int, C.POINTER(C.c_int64)]),
    ("lbm_get_band", C.c_int, [_P, _P]),
    ("lbm_reset", C.c_int, [_P]),
    ("lbm_reinit_from_macro", C.c_int, [_P, _P, _P, _P, _P]),
    ("lbm_reinit_from_host", C.c_int, [_P, _P, _P, _P, _P]),
    ("lbm_stage_from_host", C.c_int, [_P, _P, _P, _P, _P]),
    ("lbm_reinit_from_stage", C.c_int, [_P]),
    ("lbm_read_macros_async", C.c_int, [_P, _P, _P, _P, _P]),
    ("lbm_wait_reads", C.c_int, [_P]),
    ("lbm_step", C.c_int, [_P, C.c_int]),
    ("lbm_step_graph", C.c_int, [_P, C.c_int]),
    ("lbm_synchronize", C.c_int, [_P]),
    ("lbm_set_force", C.c_int, [_P, C.c_float, C.c_float, C.c_float]),
    ("lbm_set_shear_omega", C.c_int, [_P, C.c_float]),
    ("lbm_set_home_zchunk", C.c_int, [_P, C.c_int]),
    ("lbm_home_zchunk", C.c_int, [_P, C.POINTER(C.c_int)]),
    ("lbm_macro_ptrs", C.c_int, [_P, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P), C.POINTER(_P)]),
    ("lbm_get_macros", C.c_int, [_P, _P, _P, _P, _P]),
    ("lbm_get_state", C.c_int, [_P, _P]),
    ("lbm_dims", C.c_int, [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                           C.POINTER(C.c_int64)]),
    ("lbm_step_count", C.c_int, [_P, C.POINTER(C.c_int64)]),
    ("lbm_enable_stats", C.c_int, [_P, C.c_int]),
    ("lbm_get_stats", C.c_int, [_P, _P]),
    ("lbm_get_stats_async", C.c_int, [_P, _P]),
    ("lbm_set_macro_output", C.c_int, [_P, C.c_int]),
    ("lbm_macro_stats_static", C.c_int, [_P, _P, _P, _P, _P, C.c_int64, _P, _P]),
    ("lbm_batch_create", C.c_int, [C.POINTER(_P), C.c_int32, _P, C.POINTER(_P)]),
    ("lbm_batch_refresh", C.c_int, [_P]),
    ("lbm_batch_destroy", C.c_int, [_P]),
    ("lbm_batch_tune", C.c_int, [_P, C.c_int32, C.POINTER(BatchTuning)]),
    ("lbm_batch_set_tuning", C.c_int, [_P, C.POINTER(BatchTuning)]),
    ("lbm_batch_get_tuning", C.c_int, [_P, C.POINTER(BatchTuning)]),
    ("lbm_batch_step", C.c_int, [_P, C.c_int32]),
    ("lbm_batch_synchronize", C.c_int, [_P]),
    ("lbm_batch_enable_stats", C.c_int, [_P, C.c_int]),
    ("lbm_batch_get_stats", C.c_int, [_P, _P]),
    ("lbm_adjoint_run", C.c_int, [C.POINTER(AdjProblem), _P, _P, _P, _P, _P, _P]),
    ("lbm_load_stl", C.c_int, [C.c_char_p, C.POINTER(_P), C.POINTER(C.c_int64), _P]),
    ("lbm_free", None, [_P]),
    ("lbm_voxelize", C.c_int, [_P, C.c_int64, _P, C.POINTER(VoxelParams), _P]),
    ("reinit_equilibrium_from_macro", None, [_P, _P, _P, _P, _P, C.c_int]),
    ("launch_speed", None, [_P, _P, _P, _P, C.c_int]),
    ("make_rho_gauss", None, [_P, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float,
                              C.c_float]),
    ("make_rho_slab", None, [_P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float]),
    ("write_scalar_vtk", None, [C.c_char_p, _P, C.c_int, C.c_int, C.c_int]),
    ("write_vector_vtk", None, [C.c_char_p, _P, _P, _P, C.c_int, C.c_int, C.c_int]),
    ("lbm_write_scalar_vtk", C.c_int, [C.c_char_p, _P, C.c_int, C.c_int, C.c_int]),
    ("lbm_write_vector_vtk", C.c_int, [C.c_char_p, _P, _P, _P, C.c_int, C.c_int, C.c_int]),
    ("lbm_vtk_text_bound", C.c_int64, [C.c_int32, C.c_int64]),
    ("lbm_vtk_format", C.c_int, [C.c_int32, _P, _P, _P, C.c_int64, _P, C.c_int64, C.POINTER(C.c_int64), _P]),
    ("lbm_vtk_writer_create", C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.POINTER(_P)]),
    ("lbm_vtk_writer_submit", C.c_int, [_P, C.c_int32, _P, _P, _P, C.c_char_p, _P]),
    ("lbm_vtk_writer_flush", C.c_int, [_P]),
    ("lbm_vtk_writer_bytes", C.c_int, [_P, C.POINTER(C.c_uint64)]),
    ("lbm_vtk_writer_destroy", C.c_int, [_P]),
    ("lbm_format_g6", C.c_int, [_P, C.c_int64, _P, C.c_int32, _P]),
    ("lbm_solver_stream", C.c_int, [_P, C.POINTER(_P)]),
    ("lbm_step_parity", C.c_int, [_P, C.POINTER(C.c_int)]),
    ("lbm_set_z_ghosts", C.c_int, [_P, C.c_int]),
    ("lbm_zslab_slots", C.c_int, [_P, C.c_int, C.c_int, C.POINTER(_P), C.POINTER(C.c_int64)]),
    ("lbm_zslab_exchange", C.c_int, [_P, _P, C.c_int, _P]),
    ("lbm_zslab_merge", C.c_int, [_P, C.c_int, C.c_int, C.POINTER(_P), _P]),
    ("lbm_zslab_moment_planes", C.c_int, [_P, C.c_int, C.POINTER(_P), C.POINTER(C.c_int64)]),
    ("lbm_set_index_base", C.c_int, [_P, C.c_int64]),
    ("lbm_zslab_step_planes", C.c_int, [_P, C.c_int, C.c_int, C.c_int]),
    ("lbm_zslab_plan_create", C.c_int, [C.POINTER(_P), C.c_int32, C.POINTER(_P)]),
    ("lbm_zslab_plan_exchange", C.c_int, [_P, C.c_int, _P]),
    ("lbm_zslab_plan_destroy", C.c_int, [_P]),
    ("launch_diff", None, [_P, _P, _P, C.c_int]),
    ("launch_shift", None, [_P, C.c_float, _P, C.c_int]),
    ("lbm_renderer_create", C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.POINTER(_P)]),
    ("lbm_render_volume", C.c_int, [_P, _P, C.POINTER(RenderParams), _P, _P]),
    ("lbm_renderer_destroy", C.c_int, [_P]),
    ("lbm_render_orbit_camera", C.c_int, [C.c_float, C.c_float, C.c_float, _P, C.c_int32, C.c_int32, _P, _P]),
    ("lbm_write_ppm", C.c_int, [C.c_char_p, _P, C.c_int32, C.c_int32]),
]

EXPORTED = [n for n, _, _ in _PROTOS]

_lock = threading.Lock()
_lib = None


def _sources_newer() -> bool:
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    csrc = os.path.join(PKG, "csrc")
    for f in os.listdir(csrc):
        if os.path.getmtime(os.path.join(csrc, f)) > t:
            return True
    return False


def lib():
    """Load (building it first if it is missing or stale) the CUDA library."""
    global _lib
    with _lock:
        if _lib is None:
            if _sources_newer():
                from . import build
                build.build_lib()
            L = C.CDLL(LIB_PATH)
            for name, res, args in _PROTOS:
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
    return _lib


def check(code: int):
    if code != LBM_OK:
        raise LBMError(code, lib().lbm_last_error().decode(errors="replace"))
