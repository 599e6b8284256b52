"""Legacy-ASCII VTK output formatted on the GPU.

The reference writes fields with `ofstream << float` on the host
(src/moment_vtk_writer.cu:8-48).  Here the text is produced on the device,
byte for byte the same, and `VtkWriter` writes whole files from a background
thread while the solver keeps stepping.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import VTK_SCALAR, VTK_SPEED, VTK_VECTOR, check, lib

__all__ = ["VTK_SCALAR", "VTK_SPEED", "VTK_VECTOR", "format_host", "format_device", "VtkWriter"]


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def format_host(values) -> list[str]:
    """The text of each float (host build of the device formatter)."""
    v = np.ascontiguousarray(values, np.float32).ravel()
    out = np.zeros((v.size, 16), np.uint8)
    lens = np.zeros(v.size, np.uint8)
    check(lib().lbm_format_g6(v.ctypes.data_as(C.c_void_p), v.size, out.ctypes.data_as(C.c_void_p), 16,
                              lens.ctypes.data_as(C.c_void_p)))
    return [bytes(out[i, :lens[i]]).decode() for i in range(v.size)]


def format_device(kind, a, b=None, c=None, stream=None) -> bytes:
    """Lines of `kind` for device tensors (float32, contiguous) -> bytes."""
    import torch
    n = a.numel()
    cap = lib().lbm_vtk_text_bound(kind, n)
    text = torch.empty(cap, dtype=torch.uint8, device=a.device)
    ln = C.c_int64()
    st = C.c_void_p(stream if stream is not None else torch.cuda.current_stream().cuda_stream)
    check(lib().lbm_vtk_format(kind, _ptr(a), _ptr(b), _ptr(c), n, _ptr(text), cap, C.byref(ln), st))
    return bytes(text[:ln.value].cpu().numpy())


class VtkWriter:
    """Asynchronous VTK files: submit() queues the formatting on a CUDA stream
    and returns; a writer thread copies and writes; flush() waits."""

    def __init__(self, nx, ny, nz, depth=3):
        h = C.c_void_p()
        check(lib().lbm_vtk_writer_create(nx, ny, nz, depth, C.byref(h)))
        self._h = h

    def submit(self, kind, path, a, b=None, c=None, stream=None):
        """a, b, c: device pointers (int) or tensors; stream: cudaStream_t (int)."""
        p = [x if x is None or isinstance(x, int) else x.data_ptr() for x in (a, b, c)]
        check(lib().lbm_vtk_writer_submit(self._h, kind, *[None if x is None else C.c_void_p(x) for x in p],
                                          str(path).encode(), C.c_void_p(stream or 0)))

    def flush(self):
        check(lib().lbm_vtk_writer_flush(self._h))

    @property
    def bytes_written(self) -> int:
        b = C.c_uint64()
        check(lib().lbm_vtk_writer_bytes(self._h, C.byref(b)))
        return b.value

    def close(self):
        if self._h:
            h, self._h = self._h, None
            check(lib().lbm_vtk_writer_destroy(h))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
