"""Test infrastructure: the duct BGK push step written in plain torch (FP64),
the model that lbm_adjoint_run differentiates by hand, so that torch's
automatic differentiation gives an independent gradient on small grids.

Step (D3Q19, reference direction order, src/lbm/lbm3d_legacy.cu:16-32):
f* = f + w (feq(rho, u) - f); incoming population q of cell x is
  f*_q(x - c_q)                       if that link streams,
  f*_opp(q)(x)                        if x - c_q is solid (halfway bounce-back),
  w_q rho(x) (1 + 3 u_in + 3 u_in^2)  if x - c_q lies before the inlet plane,
  f*_q(x)                             if x - c_q lies past the outlet plane;
solid cells keep their populations; y and z are periodic.  Drag of a step:
sum of 2 c_qx f*_q(x) over fluid cells x and directions q whose target x + c_q
is an obstacle cell (solid, not a wall).
"""
import torch

CX = [0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0]
CY = [0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1]
CZ = [0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1]
OPP = [0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15]
W = [1 / 3] + [1 / 18] * 6 + [1 / 36] * 12


class TorchDuct:
    def __init__(self, mask, tau, force=(0.0, 0.0, 0.0), dtype=torch.float64):
        m = torch.as_tensor(mask)
        self.nz, self.ny, self.nx = m.shape
        self.solid = m != 0
        self.obst = (m != 0) & ((m & 8) == 0)
        self.omega = 1.0 / tau
        self.force = force
        self.dtype = dtype
        self.c = torch.tensor([CX, CY, CZ], dtype=dtype)          # (3, 19)
        self.w = torch.tensor(W, dtype=dtype)
        x = torch.arange(self.nx).view(1, 1, self.nx).expand(self.nz, self.ny, self.nx)
        # per incoming direction q: where its source x - c_q lies
        self.src_solid, self.src_in, self.src_out = [], [], []
        for q in range(19):
            sx = x - CX[q]
            inlet = sx < 0
            outlet = sx >= self.nx
            # the source cell with periodic y, z (x is not wrapped: those links are inlet/outlet)
            src = torch.roll(self.solid, shifts=(CZ[q], CY[q], CX[q]), dims=(0, 1, 2))
            self.src_solid.append(src & ~inlet & ~outlet)
            self.src_in.append(inlet)
            self.src_out.append(outlet)
        # drag: x + c_q is an obstacle (inside the duct)
        self.to_obst = []
        for q in range(19):
            tx = x + CX[q]
            tgt = torch.roll(self.obst, shifts=(-CZ[q], -CY[q], -CX[q]), dims=(0, 1, 2))
            self.to_obst.append(tgt & (tx >= 0) & (tx < self.nx) & ~self.solid)

    def feq(self, rho, ux, uy, uz):
        uu = ux * ux + uy * uy + uz * uz
        out = []
        for q in range(19):
            cu = CX[q] * ux + CY[q] * uy + CZ[q] * uz
            out.append(W[q] * rho * (1 + 3 * cu + 4.5 * cu * cu - 1.5 * uu))
        return torch.stack(out)

    def init(self, u0):
        return self.feq(torch.ones_like(u0[0]), u0[0], u0[1], u0[2])

    def step(self, f, u_inlet):
        rho = f.sum(0)
        jx = sum(CX[q] * f[q] for q in range(19))
        jy = sum(CY[q] * f[q] for q in range(19))
        jz = sum(CZ[q] * f[q] for q in range(19))
        ux, uy, uz = jx / rho + self.force[0], jy / rho + self.force[1], jz / rho + self.force[2]
        fs = f + self.omega * (self.feq(rho, ux, uy, uz) - f)
        drag = sum((2 * CX[q] * fs[q] * self.to_obst[q]).sum() for q in range(19) if CX[q] != 0)
        kin = 1 + 3 * u_inlet + 3 * u_inlet * u_inlet                      # (nz, ny)
        out = []
        for q in range(19):
            streamed = torch.roll(fs[q], shifts=(CZ[q], CY[q], CX[q]), dims=(0, 1, 2))
            v = torch.where(self.src_solid[q], fs[OPP[q]], streamed)
            v = torch.where(self.src_in[q], W[q] * rho * kin.unsqueeze(-1), v)
            v = torch.where(self.src_out[q], fs[q], v)
            out.append(torch.where(self.solid, f[q], v))
        return torch.stack(out), drag

    def objective(self, u_inlet, u0, n_steps, window):
        f = self.init(u0)
        J = 0.0
        for n in range(1, n_steps + 1):
            f, drag = self.step(f, u_inlet)
            if window[0] <= n <= window[1]:
                J = J + drag
        return J / (window[1] - window[0] + 1)
