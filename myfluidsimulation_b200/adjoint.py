"""Drag objective of the duct and its gradient by the hand-written adjoint.

``objective`` runs ``lbm_adjoint_run`` (include/lbm_capi.h): the Legacy BGK duct
step from f^0 = feq(1, u0) with a per-(y,z) inlet velocity profile, the
objective J = mean x-drag on the obstacle over a window of steps, and -- on
request -- dJ/du_inlet and dJ/du0 from the discrete adjoint with checkpointing.
``DragObjective`` wraps it as a ``torch.autograd.Function`` so the controls
can sit in a torch graph.  The gradient is always the library's adjoint; torch
only carries it.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import check, lib


@dataclass
class DuctProblem:
    """Grid, relaxation time, solid mask (nz, ny, nx) uint8 (walls 1|8 are left
    out of the drag), number of steps, the 1-based drag window and the
    checkpoint interval of the reverse pass."""
    nx: int
    ny: int
    nz: int
    tau: float
    mask: np.ndarray
    n_steps: int = 500
    window: tuple = (400, 500)
    checkpoint_every: int = 50
    force: tuple = field(default=(0.0, 0.0, 0.0))

    def _c(self, precision: str) -> "_lib.AdjProblem":
        p = _lib.AdjProblem()
        p.nx, p.ny, p.nz = self.nx, self.ny, self.nz
        p.tau = float(self.tau)
        for k in range(3):
            p.force[k] = float(self.force[k])
        p.n_steps = int(self.n_steps)
        p.window_begin, p.window_end = int(self.window[0]), int(self.window[1])
        p.checkpoint_every = int(self.checkpoint_every)
        p.precision = {"f32": 0, "f64": 1}[precision]
        return p


def objective(problem: DuctProblem, u_inlet, u0, precision: str = "f32", grad: bool = False):
    """J, or (J, dJ/du_inlet (nz, ny), dJ/du0 (3, nz, ny, nx)) when grad is set.

    u_inlet: (nz, ny) inlet x-velocity profile; u0: (3, nz, ny, nx) initial velocity."""
    L = lib()
    nx, ny, nz = problem.nx, problem.ny, problem.nz
    mask = np.ascontiguousarray(problem.mask, np.uint8)
    ui = np.ascontiguousarray(u_inlet, np.float64)
    u = np.ascontiguousarray(u0, np.float64)
    if mask.size != nx * ny * nz or ui.size != ny * nz or u.size != 3 * nx * ny * nz:
        raise ValueError("mask, u_inlet or u0 has the wrong size")
    J = C.c_double(0.0)
    gi = np.zeros((nz, ny), np.float64) if grad else None
    gu = np.zeros((3, nz, ny, nx), np.float64) if grad else None
    vp = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)
    pc = problem._c(precision)
    check(L.lbm_adjoint_run(C.byref(pc), vp(mask), vp(ui), vp(u), C.byref(J), vp(gi), vp(gu)))
    return (J.value, gi, gu) if grad else J.value


def _autograd_function():
    import torch

    class DragObjective(torch.autograd.Function):
        """J(u_inlet, u0) with the library's adjoint as its backward."""

        @staticmethod
        def forward(ctx, u_inlet, u0, problem, precision="f32"):
            J, gi, gu = objective(problem, u_inlet.detach().cpu().numpy(), u0.detach().cpu().numpy(), precision,
                                  grad=True)
            ctx.save_for_backward(torch.from_numpy(gi).to(u_inlet.device, u_inlet.dtype),
                                  torch.from_numpy(gu).to(u0.device, u0.dtype))
            return torch.tensor(J, dtype=torch.float64, device=u_inlet.device)

        @staticmethod
        def backward(ctx, gJ):
            gi, gu = ctx.saved_tensors
            return gJ.to(gi.dtype) * gi, gJ.to(gu.dtype) * gu, None, None

    return DragObjective


_DRAG = None


def drag_objective(u_inlet, u0, problem: DuctProblem, precision: str = "f32"):
    """torch entry point: DragObjective.apply(u_inlet, u0, problem, precision)."""
    global _DRAG
    if _DRAG is None:
        _DRAG = _autograd_function()
    return _DRAG.apply(u_inlet, u0, problem, precision)
