"""VTK text formatted on the GPU (lbm_vtk.cu) and the asynchronous writer.

- The device text equals the host build of the same formatter, which
  tests/test_vtk_format.py checks against printf "%g", for random bit patterns,
  LBM-like values and special values, at sizes that end inside a block.
- write_scalar_vtk / write_vector_vtk files equal those of the reference's own
  writer (src/moment_vtk_writer.cu, built into oracle/_ref) byte for byte.
- VtkWriter files, queued on a solver's stream between steps, hold the fields
  of the step they were queued after.
"""
import ctypes as C
import os

import numpy as np
import pytest
import torch

from myfluidsimulation_b200 import lib
from myfluidsimulation_b200.solvers import METHOD_HOME, METHOD_LEGACY, Solver
from myfluidsimulation_b200.vtk import VTK_SCALAR, VTK_SPEED, VTK_VECTOR, VtkWriter, format_device, format_host
from oracle_bind import RefCUDA

pytestmark = pytest.mark.gpu


def header(kind, nx, ny, nz):
    h = ("# vtk DataFile Version 3.0\n" + ("vector" if kind == VTK_VECTOR else "scalar") +
         "\nASCII\nDATASET STRUCTURED_POINTS\n" + f"DIMENSIONS {nx} {ny} {nz}\nORIGIN 0 0 0\nSPACING 1 1 1\n" +
         f"POINT_DATA {nx * ny * nz}\n")
    return h + ("VECTORS vec float\n" if kind == VTK_VECTOR else "SCALARS s float 1\nLOOKUP_TABLE default\n")


def lines(kind, a, b=None, c=None):
    if kind == VTK_VECTOR:
        return "".join(f"{x} {y} {z}\n" for x, y, z in zip(format_host(a), format_host(b), format_host(c)))
    return "".join(s + "\n" for s in format_host(a))


def mixed(n, seed):
    rng = np.random.default_rng(seed)
    a = (1.0 + 1e-3 * rng.standard_normal(n)).astype(np.float32)
    k = n // 3
    a[:k] = rng.integers(0, 2 ** 32, size=k, dtype=np.uint64).astype(np.uint32).view(np.float32)
    a[k:2 * k] = (0.05 * rng.standard_normal(k)).astype(np.float32)
    sp = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 1e-45, 3.4028235e38, 1234565.0, 0.0001, 1e6], np.float32)
    a[:min(sp.size, n)] = sp[:n]
    return a


def speed_of(u, v, w):
    du, dv, dw = [torch.from_numpy(x).cuda() for x in (u, v, w)]
    out = torch.empty_like(du)
    torch.cuda.synchronize()
    lib().launch_speed(du.data_ptr(), dv.data_ptr(), dw.data_ptr(), out.data_ptr(), du.numel())
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("n", [1, 255, 256, 257, 300_001])
def test_device_text_equals_host_formatter(gpu, n):
    a, b, c = mixed(n, 1), mixed(n, 2), mixed(n, 3)
    da, db, dc = [torch.from_numpy(x).cuda() for x in (a, b, c)]
    assert format_device(VTK_SCALAR, da) == lines(VTK_SCALAR, a).encode()
    assert format_device(VTK_VECTOR, da, db, dc) == lines(VTK_VECTOR, a, b, c).encode()
    # |u| fused into the formatting: the same bits as launch_speed
    u, v, w = [(0.05 * np.random.default_rng(s).standard_normal(n)).astype(np.float32) for s in (4, 5, 6)]
    du, dv, dw = [torch.from_numpy(x).cuda() for x in (u, v, w)]
    assert format_device(VTK_SPEED, du, dv, dw) == lines(VTK_SCALAR, speed_of(u, v, w)).encode()


def test_empty_field(gpu):
    z = torch.empty(0, device="cuda")
    assert format_device(VTK_SCALAR, z) == b""


@pytest.mark.skipif(not RefCUDA.available(), reason="reference CUDA build (oracle/_ref) not present")
def test_files_equal_reference_writer(gpu, tmp_path):
    ref = RefCUDA()
    dims = (23, 17, 9)
    n = int(np.prod(dims))
    a, b, c = mixed(n, 7), mixed(n, 8), mixed(n, 9)
    da, db, dc = [torch.from_numpy(x).cuda() for x in (a, b, c)]
    pa = [x.ctypes.data_as(C.c_void_p) for x in (a, b, c)]
    for kind in (VTK_SCALAR, VTK_VECTOR):
        mine, theirs = tmp_path / f"mine{kind}.vtk", tmp_path / f"ref{kind}.vtk"
        torch.cuda.synchronize()
        if kind == VTK_SCALAR:
            assert lib().lbm_write_scalar_vtk(str(mine).encode(), da.data_ptr(), *dims) == 0
            assert ref.lib.refcu_write_vtk(str(theirs).encode(), pa[0], None, None, *[C.c_int(d) for d in dims]) == 0
        else:
            assert lib().lbm_write_vector_vtk(str(mine).encode(), da.data_ptr(), db.data_ptr(), dc.data_ptr(),
                                              *dims) == 0
            assert ref.lib.refcu_write_vtk(str(theirs).encode(), *pa, *[C.c_int(d) for d in dims]) == 0
        assert mine.read_bytes() == theirs.read_bytes()
        assert mine.read_bytes() == (header(kind, *dims) + lines(kind, a, b, c)).encode()


@pytest.mark.parametrize("method", [METHOD_LEGACY, METHOD_HOME])
def test_async_writer_files_hold_the_queued_step(gpu, tmp_path, method):
    dims = (48, 40, 36)
    nx, ny, nz = dims
    rng = np.random.default_rng(3)
    rho = (1 + 1e-3 * rng.standard_normal((nz, ny, nx))).astype(np.float32)
    u = (0.03 * rng.standard_normal((nz, ny, nx))).astype(np.float32)
    zero = np.zeros_like(u)
    s = Solver(nx, ny, nz, 0.6, (1e-5, 0, 0), method=method)
    s.reinit_from_host(rho, u, zero, zero)
    want = []
    with VtkWriter(nx, ny, nz, depth=2) as w:
        for k in range(4):
            s.step(3)
            r, ux, uy, uz = s.macro_ptrs()
            names = [tmp_path / f"{t}_{k}.vtk" for t in ("rho", "speed", "vel")]
            w.submit(VTK_SCALAR, names[0], r, stream=s.stream)
            w.submit(VTK_SPEED, names[1], ux, uy, uz, stream=s.stream)
            w.submit(VTK_VECTOR, names[2], ux, uy, uz, stream=s.stream)
            want.append((names, [m.ravel().copy() for m in s.macros()]))
        w.flush()
        total = w.bytes_written
    s.close()
    size = 0
    for names, (mr, mu, mv, mw) in want:
        assert names[0].read_bytes() == (header(VTK_SCALAR, *dims) + lines(VTK_SCALAR, mr)).encode()
        assert names[1].read_bytes() == (header(VTK_SCALAR, *dims) + lines(VTK_SCALAR, speed_of(mu, mv, mw))).encode()
        assert names[2].read_bytes() == (header(VTK_VECTOR, *dims) + lines(VTK_VECTOR, mu, mv, mw)).encode()
        size += sum(os.path.getsize(p) for p in names)
    assert total == size


def test_writer_reports_unwritable_path(gpu, tmp_path):
    d = torch.ones(8 * 4 * 2, device="cuda")
    with VtkWriter(8, 4, 2, depth=1) as w:
        w.submit(VTK_SCALAR, tmp_path / "missing_dir" / "a.vtk", d)
        w.submit(VTK_SCALAR, tmp_path / "b.vtk", d)
        with pytest.raises(RuntimeError, match="missing_dir"):
            w.flush()
        w.flush()   # the error was reported once
    assert (tmp_path / "b.vtk").read_bytes() == (header(VTK_SCALAR, 8, 4, 2) + "1\n" * 64).encode()
