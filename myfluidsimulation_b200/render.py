"""Headless volume view: the reference's ray-march shader as a CUDA kernel.

src/render/Vis3D.cpp draws the field with a GLSL fragment shader in an OpenGL
window; `VolumeRenderer.render` produces the same frame into a device RGBA
buffer (row 0 at the bottom, as in GL), and `write_ppm` stores it as an image.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import FILTER_EXACT, FILTER_TEXTURE, RenderParams, check, lib

__all__ = ["FILTER_EXACT", "FILTER_TEXTURE", "orbit_camera", "VolumeRenderer", "write_ppm"]


def orbit_camera(yaw=0.0, pitch=0.3, radius=2.5, target=(0.5, 0.5, 0.5), width=1280, height=720):
    """inverse(P V) (column-major, 16 floats) and the eye of the viewer's orbit camera
    (main_compare.cpp:51-60,972-981; its defaults)."""
    inv = np.zeros(16, np.float32)
    cam = np.zeros(3, np.float32)
    t = np.asarray(target, np.float32)
    check(lib().lbm_render_orbit_camera(float(yaw), float(pitch), float(radius), t.ctypes.data_as(C.c_void_p),
                                        int(width), int(height), inv.ctypes.data_as(C.c_void_p),
                                        cam.ctypes.data_as(C.c_void_p)))
    return inv, cam


class VolumeRenderer:
    def __init__(self, nx, ny, nz):
        h = C.c_void_p()
        check(lib().lbm_renderer_create(nx, ny, nz, C.byref(h)))
        self._h = h
        self.dims = (nx, ny, nz)

    def render(self, field, inv_pv, cam, width=1280, height=720, step=0.005, scale=150.0, threshold=0.15,
               filter=FILTER_EXACT, out=None, stream=None):
        """field: device float32 tensor of Nz*Ny*Nx cells -> device tensor [height, width, 4]."""
        import torch
        p = RenderParams(int(width), int(height), (C.c_float * 16)(*np.asarray(inv_pv, np.float32).ravel()),
                         (C.c_float * 3)(*np.asarray(cam, np.float32).ravel()), float(step), float(scale),
                         float(threshold), int(filter))
        if out is None:
            out = torch.empty((height, width, 4), dtype=torch.float32, device=field.device)
        st = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        check(lib().lbm_render_volume(self._h, C.c_void_p(field.data_ptr()), C.byref(p), C.c_void_p(out.data_ptr()),
                                      C.c_void_p(st)))
        return out

    def close(self):
        if self._h:
            h, self._h = self._h, None
            check(lib().lbm_renderer_destroy(h))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def write_ppm(path, rgba):
    """Host float RGBA image [h, w, 4] (row 0 at the bottom) -> binary PPM."""
    a = np.ascontiguousarray(rgba, np.float32)
    check(lib().lbm_write_ppm(str(path).encode(), a.ctypes.data_as(C.c_void_p), a.shape[1], a.shape[0]))
