"""The hand-written adjoint (lbm_adjoint_run) against torch FP64 autodiff of the
same step on a 32x16x16 copy of the duct, against central finite differences
of the FP64 objective (eps = 1e-3, random control directions, bound 1e-4
relative), and against the product's own forward (the AA kernels) for the
objective itself."""
import numpy as np
import pytest

from myfluidsimulation_b200 import workloads as W
from myfluidsimulation_b200.adjoint import DuctProblem, drag_objective, objective

pytestmark = pytest.mark.gpu


def duct(nx, ny, nz, radius, center):
    z, y, x = np.meshgrid(np.arange(nz) + 0.5, np.arange(ny) + 0.5, np.arange(nx) + 0.5, indexing="ij")
    ball = (x - center[0]) ** 2 + (y - center[1]) ** 2 + (z - center[2]) ** 2 <= radius ** 2
    return W.duct_mask(nx, ny, nz, ball.astype(np.uint8))


def controls(nx, ny, nz, seed):
    rng = np.random.default_rng(seed)
    raw = 0.04 + 0.005 * rng.standard_normal((nz + 4, ny + 4))
    # 5x5 box filter, periodic-free (valid part of the padded field)
    k = np.ones(5) / 5
    sm = np.apply_along_axis(lambda r: np.convolve(r, k, "valid"), 1, raw)
    sm = np.apply_along_axis(lambda c: np.convolve(c, k, "valid"), 0, sm)
    u0 = np.zeros((3, nz, ny, nx))
    u0[0] = 0.04
    u0 += 1e-3 * rng.standard_normal(u0.shape)
    return sm, u0


@pytest.fixture(scope="module")
def tiny():
    nx, ny, nz = 32, 16, 16
    mask = duct(nx, ny, nz, 3.0, (8, 8, 8))
    prob = DuctProblem(nx, ny, nz, 0.6, mask, n_steps=40, window=(31, 40), checkpoint_every=8)
    ui, u0 = controls(nx, ny, nz, 7)
    return prob, ui, u0


def test_adjoint_matches_fp64_autodiff(gpu, tiny):
    import torch
    from torch_duct import TorchDuct
    prob, ui, u0 = tiny
    td = TorchDuct(prob.mask, prob.tau)
    tui = torch.tensor(ui, requires_grad=True)
    tu0 = torch.tensor(u0, requires_grad=True)
    Jt = td.objective(tui, tu0, prob.n_steps, prob.window)
    Jt.backward()
    J64, gi64, gu64 = objective(prob, ui, u0, "f64", grad=True)
    J32, gi32, gu32 = objective(prob, ui, u0, "f32", grad=True)
    rl = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    print(f"J torch {Jt.item():.12e} f64 {J64:.12e} f32 {J32:.12e}")
    print(f"grad inlet: f64 {rl(gi64, tui.grad.numpy()):.3e}, f32 {rl(gi32, tui.grad.numpy()):.3e}; "
          f"grad u0: f64 {rl(gu64, tu0.grad.numpy()):.3e}, f32 {rl(gu32, tu0.grad.numpy()):.3e}")
    assert J64 == pytest.approx(Jt.item(), rel=1e-11)
    assert rl(gi64, tui.grad.numpy()) < 1e-9
    assert rl(gu64, tu0.grad.numpy()) < 1e-9
    assert J32 == pytest.approx(Jt.item(), rel=1e-4)
    assert rl(gi32, tui.grad.numpy()) < 1e-3
    assert rl(gu32, tu0.grad.numpy()) < 1e-3


def test_checkpoint_interval_does_not_change_the_gradient(gpu, tiny):
    prob, ui, u0 = tiny
    ref = objective(prob, ui, u0, "f64", grad=True)
    for k in (1, 5, 40, 100):
        p = DuctProblem(prob.nx, prob.ny, prob.nz, prob.tau, prob.mask, prob.n_steps, prob.window, k)
        J, gi, gu = objective(p, ui, u0, "f64", grad=True)
        assert J == ref[0]
        np.testing.assert_array_equal(gi, ref[1])
        np.testing.assert_array_equal(gu, ref[2])


def test_adjoint_matches_central_differences(gpu):
    """A 64x32x32 copy of the adjoint case (sphere r=5 at (16,16,16)), 120 steps,
    drag averaged over steps 100-120: directional derivatives along random
    control directions against central differences of the FP64 objective."""
    nx, ny, nz = 64, 32, 32
    prob = DuctProblem(nx, ny, nz, 0.6, duct(nx, ny, nz, 5.0, (16, 16, 16)), n_steps=120, window=(100, 120),
                       checkpoint_every=30)
    ui, u0 = controls(nx, ny, nz, 11)
    J, gi, gu = objective(prob, ui, u0, "f64", grad=True)
    rng = np.random.default_rng(5)
    eps = 1e-3
    worst = 0.0
    for _ in range(6):
        di = rng.standard_normal(ui.shape)
        du = rng.standard_normal(u0.shape)
        scale = 1.0 / np.sqrt((di ** 2).sum() + (du ** 2).sum())
        di *= scale
        du *= scale
        Jp = objective(prob, ui + eps * di, u0 + eps * du, "f64")
        Jm = objective(prob, ui - eps * di, u0 - eps * du, "f64")
        fd = (Jp - Jm) / (2 * eps)
        ad = float((gi * di).sum() + (gu * du).sum())
        err = abs(fd - ad) / abs(fd)
        worst = max(worst, err)
        assert err < 1e-4, (fd, ad)
    print(f"central differences: worst relative difference {worst:.3e}")


def test_full_case_matches_central_differences(gpu):
    """The adjoint case at full size: duct 128x64x64, tau 0.6, sphere r = 10 at
    (32,32,32), 500 steps, drag averaged over steps 400-500, checkpoints every
    50 steps; inlet profile 0.04 + 0.005 N(0,1) smoothed by a 5x5 box filter and
    initial velocity 0.04 + 1e-3 N(0,1).  Along 32 random unit directions in
    control space, the FP64 and the FP32 adjoint gradients against central
    differences of the FP64 objective (eps 1e-3): relative 1e-6 (FP64) and 1e-4
    (FP32, the stated bound)."""
    nx, ny, nz = 128, 64, 64
    prob = DuctProblem(nx, ny, nz, 0.6, duct(nx, ny, nz, 10.0, (32, 32, 32)), n_steps=500, window=(400, 500),
                       checkpoint_every=50)
    import torch
    gen = torch.Generator().manual_seed(4)          # the draws of `bench.py --study adjoint`
    raw = (0.04 + 0.005 * torch.randn((nz + 4, ny + 4), generator=gen, dtype=torch.float64)).numpy()
    k = np.ones(5) / 5
    ui = np.apply_along_axis(lambda r: np.convolve(r, k, "valid"), 1, raw)
    ui = np.apply_along_axis(lambda c: np.convolve(c, k, "valid"), 0, ui)
    u0 = 1e-3 * torch.randn((3, nz, ny, nx), generator=gen, dtype=torch.float64).numpy()
    u0[0] += 0.04
    _, gi64, gu64 = objective(prob, ui, u0, "f64", grad=True)
    _, gi32, gu32 = objective(prob, ui, u0, "f32", grad=True)
    rng = np.random.default_rng(2026)
    eps = 1e-3
    worst64 = worst32 = 0.0
    for _ in range(32):
        di = rng.standard_normal(ui.shape)
        du = rng.standard_normal(u0.shape)
        scale = 1.0 / np.sqrt((di ** 2).sum() + (du ** 2).sum())
        di *= scale
        du *= scale
        fd = (objective(prob, ui + eps * di, u0 + eps * du, "f64") -
              objective(prob, ui - eps * di, u0 - eps * du, "f64")) / (2 * eps)
        worst64 = max(worst64, abs(float((gi64 * di).sum() + (gu64 * du).sum()) - fd) / abs(fd))
        worst32 = max(worst32, abs(float((gi32 * di).sum() + (gu32 * du).sum()) - fd) / abs(fd))
    print(f"full case: worst relative difference FP64 {worst64:.3e}, FP32 {worst32:.3e}")
    assert worst64 < 1e-6
    assert worst32 < 1e-4


def test_objective_matches_the_product_forward(gpu):
    """With a uniform inlet the adjoint's forward model is the AA duct step of
    lbm_step: the windowed drag agrees within FP32 rounding."""
    from myfluidsimulation_b200.solvers import BC_DUCT, METHOD_LEGACY, Solver
    nx, ny, nz = 48, 24, 24
    mask = duct(nx, ny, nz, 4.0, (12, 12, 12))
    prob = DuctProblem(nx, ny, nz, 0.58, mask, n_steps=60, window=(41, 60), checkpoint_every=20)
    rng = np.random.default_rng(3)
    u0 = np.zeros((3, nz, ny, nx))
    u0[0] = 0.04
    u0 += 1e-3 * rng.standard_normal(u0.shape)
    u0[:, mask != 0] = 0.0
    ui = np.full((nz, ny), 0.04)
    J = objective(prob, ui, u0, "f32")
    s = Solver(nx, ny, nz, 0.58, method=METHOD_LEGACY, bc=BC_DUCT, inlet_u=0.04)
    s.set_solid_mask(mask)
    s.reinit_from_host(np.ones((nz, ny, nx), np.float32), *[u0[k].astype(np.float32) for k in range(3)])
    s.step(40)
    s.enable_stats(True)
    drags = []
    for _ in range(20):
        s.step(1)
        drags.append(s.stats()["drag_x"])
    s.close()
    assert J == pytest.approx(np.mean(drags), rel=1e-4)


def test_torch_autograd_function(gpu, tiny):
    import torch
    prob, ui, u0 = tiny
    tui = torch.tensor(ui, requires_grad=True)
    tu0 = torch.tensor(u0, requires_grad=True)
    loss = 3.0 * drag_objective(tui, tu0, prob, "f64") + (tui ** 2).sum()
    loss.backward()
    J, gi, gu = objective(prob, ui, u0, "f64", grad=True)
    np.testing.assert_allclose(tui.grad.numpy(), 3.0 * gi + 2.0 * ui, rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(tu0.grad.numpy(), 3.0 * gu, rtol=1e-12, atol=1e-18)
