"""The headless volume view (lbm_render.cu) against the oracle's restatement of
the reference's fragment shader (src/render/Vis3D.cpp:30-78).

With LBM_FILTER_EXACT every operation is rounded as written on both sides, so
the frames must be equal bit for bit, for odd frame sizes, cameras outside and
inside the box, axis-aligned rays (direction components of zero) and fields
whose samples cross the threshold.  The texture-unit filter (8-bit weights, as
GL_LINEAR on this hardware) is held to a bound on the displayed (clamped)
colours instead.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from myfluidsimulation_b200 import lib
from myfluidsimulation_b200.render import FILTER_EXACT, FILTER_TEXTURE, VolumeRenderer, orbit_camera
from oracle_bind import RefCUDA

pytestmark = pytest.mark.gpu


def blob_field(nx, ny, nz, seed=0):
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid((np.arange(nz) + 0.5) / nz, (np.arange(ny) + 0.5) / ny, (np.arange(nx) + 0.5) / nx,
                          indexing="ij")
    f = 0.004 * np.exp(-((x - 0.45) ** 2 + (y - 0.5) ** 2 + (z - 0.55) ** 2) / 0.04)
    f += 0.0015 * np.sin(9 * x) * np.cos(7 * y) + 3e-4 * rng.standard_normal(f.shape)
    return f.astype(np.float32)


CAMERAS = [
    # (yaw, pitch, radius, width, height, step, scale)
    (0.0, 0.3, 2.5, 97, 61, 0.005, 150.0),      # the viewer's default orbit
    (0.0, 0.0, 2.5, 64, 48, 0.005, 150.0),      # level view: rays with zero y/z components
    (2.3, -0.6, 1.9, 80, 80, 0.01, 300.0),
    (0.7, 0.2, 0.3, 50, 40, 0.004, 150.0),      # eye inside the box: tNear < 0
]


@pytest.mark.parametrize("cam_args", CAMERAS)
def test_exact_filter_equals_oracle(gpu, oracle, cam_args):
    yaw, pitch, radius, w, h, step, scale = cam_args
    nx, ny, nz = 40, 24, 32
    f = blob_field(nx, ny, nz)
    inv, cam = orbit_camera(yaw, pitch, radius, (0.5, 0.5, 0.5), w, h)
    want, ns = oracle.raymarch(f, inv, cam, step, scale, 0.15, w, h)
    with VolumeRenderer(nx, ny, nz) as r:
        got = r.render(torch.from_numpy(f).cuda(), inv, cam, w, h, step, scale, 0.15, FILTER_EXACT).cpu().numpy()
    assert ns > 0
    lit = (want[..., :3] > 0.05).any(axis=2)
    assert lit.mean() > 0.05                            # samples above the threshold in the frame
    np.testing.assert_array_equal(got, want)


def test_texture_filter_close_to_oracle(gpu, oracle):
    nx, ny, nz = 40, 24, 32
    f = blob_field(nx, ny, nz, 1)
    inv, cam = orbit_camera(0.4, 0.35, 2.2, (0.5, 0.5, 0.5), 120, 90)
    want, _ = oracle.raymarch(f, inv, cam, 0.005, 150.0, 0.15, 120, 90)
    with VolumeRenderer(nx, ny, nz) as r:
        got = r.render(torch.from_numpy(f).cuda(), inv, cam, 120, 90, 0.005, 150.0, 0.15,
                       FILTER_TEXTURE).cpu().numpy()
    d = np.abs(np.clip(got[..., :3], 0, 1) - np.clip(want[..., :3], 0, 1)).max(axis=2)
    print(f"texture filter: mean |d| {d.mean():.2e}, pixels > 0.1: {(d > 0.1).mean():.3%}")
    assert d.mean() < 0.01
    assert (d > 0.1).mean() < 0.02


@pytest.mark.skipif(not RefCUDA.available(), reason="reference CUDA build (oracle/_ref) not present")
def test_field_helpers_match_reference(gpu):
    ref = RefCUDA()
    n = 10007
    rng = np.random.default_rng(5)
    a, b = [torch.from_numpy(rng.standard_normal(n).astype(np.float32)).cuda() for _ in range(2)]
    mine, theirs = torch.empty_like(a), torch.empty_like(a)
    torch.cuda.synchronize()
    lib().launch_diff(a.data_ptr(), b.data_ptr(), mine.data_ptr(), n)
    ref.lib.launch_diff(C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()), C.c_void_p(theirs.data_ptr()), C.c_int(n))
    torch.cuda.synchronize()
    assert torch.equal(mine, theirs)
    lib().launch_shift(a.data_ptr(), -1.0, mine.data_ptr(), n)
    ref.lib.launch_shift(C.c_void_p(a.data_ptr()), C.c_float(-1.0), C.c_void_p(theirs.data_ptr()), C.c_int(n))
    torch.cuda.synchronize()
    assert torch.equal(mine, theirs)
