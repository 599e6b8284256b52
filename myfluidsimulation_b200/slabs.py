"""z-slab decomposition of the Legacy/Hybrid (AA) step.

The domain's z planes are split into slabs.  Each slab solver holds its planes
plus one ghost plane at each end (`lbm_set_z_ghosts`), and steps only its own
planes.  The AA even step is local.  Around each odd step the 5 slot planes
crossing each slab face (directions with c_z = +-1) travel twice:
  phase 0, before the odd step: boundary plane -> the neighbour's ghost plane;
  phase 1, after it: ghost plane -> its owner's boundary plane, for the cells
           whose link across the face streams (a population that a boundary
           cell bounced back off a solid neighbour stays where it is).
Nothing else is exchanged, and every cell computes exactly what it would in one
grid, so a decomposed run equals the single-grid run bit for bit.

HOME pulls whole planes of moments instead: before every step the 10 moment
planes of each boundary plane go to the neighbour's ghost plane (phase 0 only),
and each slab draws its stochastic-rounding bits by global cell index
(`lbm_set_index_base`), so HOME slabs match the single grid bit for bit too.

`SlabSet` keeps all slabs on one GPU, with device copies as the exchange.
`DistSlab` keeps one slab per process (torch.distributed, NCCL between GPUs;
any backend works for the plan), exchanging with point-to-point sends.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import BC_PERIODIC, METHOD_HOME, METHOD_LEGACY, STORE_F32, check, lib
from .solvers import Solver

__all__ = ["slab_bounds", "exchange_plan", "exchange", "with_ghosts", "reduce_stats", "SlabSet", "DistSlab"]

# FP64 statistics of a solver, in the order of lbm_get_stats (LBM_STAT_* in lbm_capi.h)
STAT_KEYS = ("mass", "ke_sum", "drag_x", "drag_y", "drag_z", "mom_x", "mom_y", "mom_z")


def slab_bounds(nz: int, parts: int):
    """[z0, z1) of each slab: nz planes in `parts` nearly equal runs."""
    if parts < 1 or parts > nz:
        raise ValueError("need 1 <= parts <= nz")
    cuts = [nz * k // parts for k in range(parts + 1)]
    return [(cuts[k], cuts[k + 1]) for k in range(parts)]


def with_ghosts(a, z0: int, z1: int, axis: int = 0):
    """Planes z0-1 .. z1 of a periodic field (the slab and its two ghosts)."""
    a = np.asarray(a)
    nz = a.shape[axis]
    idx = [(z0 - 1) % nz] + list(range(z0, z1)) + [z1 % nz]
    return np.ascontiguousarray(np.take(a, idx, axis=axis))


def reduce_stats(local: dict, cells: int, dist, group=None) -> dict:
    """The whole grid's statistics from every rank's own sums: one FP64
    all-reduce (sum) of the 8 values over the group.  A slab's sums cover its
    own planes only (ghost planes are never stepped), so the sum over the ranks
    counts every cell once.  The tensor lives on the GPU for NCCL and on the
    host for other backends (gloo)."""
    import torch
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    v = torch.tensor([float(local[k]) for k in STAT_KEYS], dtype=torch.float64, device=dev)
    dist.all_reduce(v, op=dist.ReduceOp.SUM, group=group)
    out = dict(zip(STAT_KEYS, v.cpu().tolist()))
    out["ke_mean"] = out["ke_sum"] / cells
    return out


# planes of a slab solver with L planes: 0 ghost below, 1 first own, L-2 last own, L-1 ghost above
def exchange_plan(phase: int, rank: int, world: int):
    """Point-to-point transfers of one rank for one phase:
    (kind, peer, plane, cz): kind 'send' or 'recv'; plane one of
    'ghost_lo', 'first', 'last', 'ghost_hi'; cz the direction set (+1/-1).
    Sends precede receives in the list; a pair of ranks posts matching ops."""
    lo, hi = (rank - 1) % world, (rank + 1) % world
    if phase == 0:
        return [("send", hi, "last", -1), ("send", lo, "first", +1),
                ("recv", lo, "ghost_lo", -1), ("recv", hi, "ghost_hi", +1)]
    if phase == 1:
        return [("send", lo, "ghost_lo", -1), ("send", hi, "ghost_hi", +1),
                ("recv", hi, "last", -1), ("recv", lo, "first", +1)]
    raise ValueError("phase is 0 or 1")


def exchange(views, phase: int, rank: int, world: int, dist, group=None, recv_views=None, wait=True):
    """Run one phase of the plan with torch.distributed point-to-point ops.
    views[(plane, cz)]: the 5 tensors (slot planes) of that plane and
    direction set, in direction order, on this rank; recv_views (optional)
    redirects receives of a (plane, cz) into other tensors (staging).
    wait=False returns the works instead of waiting for them (with NCCL, a
    work's wait() makes the current stream wait: the transfers overlap with
    whatever the stream runs until then)."""
    ops = []
    for kind, peer, plane, cz in exchange_plan(phase, rank, world):
        fn = dist.isend if kind == "send" else dist.irecv
        peer_g = dist.get_global_rank(group, peer) if group is not None else peer
        ts = views[(plane, cz)]
        if kind == "recv" and recv_views and (plane, cz) in recv_views:
            ts = recv_views[(plane, cz)]
        for t in ts:
            ops.append(dist.P2POp(fn, t, peer_g, group))
    works = dist.batch_isend_irecv(ops)
    if not wait:
        return works
    for w in works:
        w.wait()
    return []


def _slot_ptrs(solver: Solver, plane: int, cz: int):
    ptrs = (C.c_void_p * 5)()
    nb = C.c_int64()
    check(lib().lbm_zslab_slots(solver._h, int(plane), int(cz), ptrs, C.byref(nb)))
    return [p for p in ptrs], nb.value


def _parity(solver: Solver) -> int:
    v = C.c_int()
    check(lib().lbm_step_parity(solver._h, C.byref(v)))
    return v.value


class SlabSet:
    """All slabs of one grid on this GPU (one stream); the single-device image of
    the multi-GPU layout.  Fields are given and returned for the whole grid."""

    def __init__(self, nx, ny, nz, tau, parts, force=(0.0, 0.0, 0.0), method=METHOD_LEGACY, storage=STORE_F32,
                 bc=BC_PERIODIC, inlet_u=0.0, stream=None):
        import torch
        self.shape = (nz, ny, nx)
        self.bounds = slab_bounds(nz, parts)
        self.stream = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        self.slabs = []
        self._plan = None
        self._stats, self._macro = False, True
        self.home = method == METHOD_HOME
        for z0, z1 in self.bounds:
            s = Solver(nx, ny, z1 - z0 + 2, tau, force, method=method, storage=storage, bc=bc, inlet_u=inlet_u,
                       stream=self.stream)
            check(lib().lbm_set_z_ghosts(s._h, 1))
            check(lib().lbm_set_index_base(s._h, (z0 - 1) * nx * ny))
            self.slabs.append(s)

    def _drop_plan(self):
        if self._plan:
            check(lib().lbm_zslab_plan_destroy(self._plan))
            self._plan = None

    def set_solid_mask(self, mask):
        m = np.asarray(mask, np.uint8).reshape(self.shape)
        for s, (z0, z1) in zip(self.slabs, self.bounds):
            s.set_solid_mask(with_ghosts(m, z0, z1))
        self._drop_plan()

    def set_legacy_mapping(self, band):
        b = np.asarray(band, np.uint8).reshape(self.shape)
        for s, (z0, z1) in zip(self.slabs, self.bounds):
            s.set_legacy_mapping(with_ghosts(b, z0, z1))
        self._drop_plan()

    def reinit_from_host(self, rho=None, ux=None, uy=None, uz=None):
        for s, (z0, z1) in zip(self.slabs, self.bounds):
            s.reinit_from_host(*[None if a is None else with_ghosts(np.asarray(a, np.float32).reshape(self.shape),
                                                                     z0, z1) for a in (rho, ux, uy, uz)])

    def enable_stats(self, on=True):
        self._stats = bool(on)
        for s in self.slabs:
            s.enable_stats(on)

    def set_shear_omega(self, omega_s):
        for s in self.slabs:
            s.set_shear_omega(omega_s)

    def set_macro_output(self, on=True):
        self._macro = bool(on)
        for s in self.slabs:
            s.set_macro_output(on)

    def _outputs(self, on):
        """Statistics and macro fields as set (on) or off: the slabs step one
        substep per call, so n steps leave them off for all but the last, as
        lbm_step(n) does."""
        for s in self.slabs:
            s.enable_stats(self._stats and on)
            s.set_macro_output(self._macro and on)

    def _ensure_plan(self):
        # every face in one launch per phase (lbm_zslab_plan_*), built after the mask and band
        if self._plan is None:
            hs = (C.c_void_p * len(self.slabs))(*[s._h.value for s in self.slabs])
            p = C.c_void_p()
            check(lib().lbm_zslab_plan_create(hs, len(self.slabs), C.byref(p)))
            self._plan = p

    def _exchange(self, phase):
        if self.home:   # the moment planes move between buffers every step: per face
            self.exchange_pairwise(phase)
            return
        self._ensure_plan()
        check(lib().lbm_zslab_plan_exchange(self._plan, phase, C.c_void_p(self.stream)))

    def exchange_pairwise(self, phase):
        """The same transfers as one lbm_zslab_exchange per face."""
        n = len(self.slabs)
        for k in range(n):
            check(lib().lbm_zslab_exchange(self.slabs[k]._h, self.slabs[(k + 1) % n]._h, phase,
                                           C.c_void_p(self.stream)))

    def graph(self, n: int = 2):
        """A torch CUDA graph of n steps (n even: the step parity comes back).
        Needs a stream other than the legacy default one; replay() advances the
        device state by n steps (the solvers' host-side step counters do not move)."""
        import torch
        if n % 2 or n < 2:
            raise ValueError("n must be even")
        if not self.home:
            self._ensure_plan()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=torch.cuda.ExternalStream(self.stream)):
            self.step(n)
        return g

    def step(self, n: int = 1):
        quiet = n > 1 and (self._stats or self._macro)
        if quiet:
            self._outputs(False)
        for k in range(n):
            if quiet and k == n - 1:
                self._outputs(True)
            ex = self.home or _parity(self.slabs[0]) == 1
            if ex:
                self._exchange(0)
            for s in self.slabs:
                s.step(1)
            if ex and not self.home:
                self._exchange(1)

    def synchronize(self):
        for s in self.slabs:
            s.synchronize()

    def macros(self):
        parts = [s.macros() for s in self.slabs]
        return tuple(np.concatenate([p[k][1:-1] for p in parts], axis=0) for k in range(4))

    def state(self):
        """The whole grid's state: populations in the natural layout (after an even
        step count), or HOME's 10 moments."""
        return np.concatenate([s.state()[:, 1:-1] for s in self.slabs], axis=1)

    def stats(self) -> dict:
        out = {}
        for s in self.slabs:
            for k, v in s.stats().items():
                out[k] = out.get(k, 0.0) + v
        out["ke_mean"] = out["ke_sum"] / int(np.prod(self.shape))
        return out

    def close(self):
        self._drop_plan()
        for s in self.slabs:
            s.close()
        self.slabs = []


def _device_view(ptr: int, nbytes: int, device):
    """A uint8 torch tensor over raw device memory (no copy)."""
    import torch

    class _Mem:
        __cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False), "version": 3,
                                    "strides": None}

    return torch.as_tensor(_Mem(), device=device)


class DistSlab:
    """This process's slab of a grid split across the ranks of a torch.distributed
    group (one GPU per rank).  The solver runs on torch's current stream, so the
    point-to-point transfers (queued by torch on its communication stream after
    the work already on the current stream) order correctly with the steps."""

    def __init__(self, nx, ny, nz, tau, force=(0.0, 0.0, 0.0), method=METHOD_LEGACY, storage=STORE_F32,
                 bc=BC_PERIODIC, inlet_u=0.0, group=None, dist=None):
        import torch
        if dist is None:
            import torch.distributed as dist
        self.dist, self.group = dist, group
        self.rank, self.world = dist.get_rank(group), dist.get_world_size(group)
        self.shape = (nz, ny, nx)
        self.z0, self.z1 = slab_bounds(nz, self.world)[self.rank]
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.solver = Solver(nx, ny, self.z1 - self.z0 + 2, tau, force, method=method, storage=storage, bc=bc,
                             inlet_u=inlet_u, stream=torch.cuda.current_stream().cuda_stream)
        check(lib().lbm_set_z_ghosts(self.solver._h, 1))
        check(lib().lbm_set_index_base(self.solver._h, (self.z0 - 1) * nx * ny))
        self.home = method == METHOD_HOME
        L = self.z1 - self.z0 + 2
        planes = {"ghost_lo": 0, "first": 1, "last": L - 2, "ghost_hi": L - 1}
        self.planes = planes
        self.views = {}
        self._home_views = {}
        self._pending = []          # phase-1 works of an overlapped odd step, merged before the next use
        self._plan = None           # one rank: the self-exchange plan (lbm_zslab_plan_*)
        self._stats, self._macro = False, True
        if not self.home:
            for name, pl in planes.items():
                for cz in (+1, -1):
                    ptrs, nb = _slot_ptrs(self.solver, pl, cz)
                    self.views[(name, cz)] = [_device_view(p, nb, self.device) for p in ptrs]
            # phase 1 lands in staging first: only the values the neighbour's cells
            # wrote are taken (lbm_zslab_merge), a bounced-back population stays
            self.staging = {key: [torch.empty_like(t) for t in self.views[key]]
                            for key in (("last", -1), ("first", 1))}

    def _moment_views(self):
        """HOME: views of the 10 moment planes of each named plane in the current
        buffer (the plan's direction sets both map to all 10 planes)."""
        ptrs = {}
        for name, pl in self.planes.items():
            arr = (C.c_void_p * 10)()
            nb = C.c_int64()
            check(lib().lbm_zslab_moment_planes(self.solver._h, pl, arr, C.byref(nb)))
            ptrs[name] = ([p for p in arr], nb.value)
        key = tuple(ptrs["first"][0])
        if key not in self._home_views:
            v = {}
            for name, (ps, nb) in ptrs.items():
                ts = [_device_view(p, nb, self.device) for p in ps]
                v[(name, 1)] = ts
                v[(name, -1)] = ts
            self._home_views[key] = v
        return self._home_views[key]

    def _merge_staging(self):
        for (name, cz), ts in self.staging.items():
            src = (C.c_void_p * 5)(*[t.data_ptr() for t in ts])
            check(lib().lbm_zslab_merge(self.solver._h, self.planes[name], cz, src,
                                        C.c_void_p(self.solver.stream)))

    def _flush(self):
        """Complete a phase-1 exchange left in flight by an overlapped odd step."""
        if self._pending:
            for w in self._pending:
                w.wait()
            self._pending = []
            self._merge_staging()

    def _planes(self, z0, z1, finish):
        check(lib().lbm_zslab_step_planes(self.solver._h, int(z0), int(z1), 1 if finish else 0))

    def _step_overlapped(self):
        """One step with the face exchange overlapped with the interior planes
        (Legacy/Hybrid, 2 or more ranks, at least 3 own planes).  In the AA
        pattern every cell reads exactly the slots it writes, so planes can be
        stepped in any order.  Odd step: phase 0 goes out, the interior planes
        2..L-3 compute meanwhile (they touch neither the ghost planes nor the
        boundary slots that phase 0 sends), then the two boundary planes; phase 1
        is left in flight.  Even step: the interior computes while phase 1
        lands, then the merge and the two boundary planes."""
        L = self.planes["ghost_hi"] + 1
        if _parity(self.solver) == 1:
            self._flush()
            works = exchange(self.views, 0, self.rank, self.world, self.dist, self.group, wait=False)
            self._planes(2, L - 2, False)
            for w in works:
                w.wait()
            self._planes(1, 2, False)
            self._planes(L - 2, L - 1, True)
            self._pending = exchange(self.views, 1, self.rank, self.world, self.dist, self.group,
                                     recv_views=self.staging, wait=False)
        else:
            self._planes(2, L - 2, False)
            self._flush()
            self._planes(1, 2, False)
            self._planes(L - 2, L - 1, True)

    def _drop_plan(self):
        if self._plan:
            check(lib().lbm_zslab_plan_destroy(self._plan))
            self._plan = None

    def _exchange(self, phase):
        if self.world == 1:
            # one self-neighbouring slab: both faces of a phase in one launch of the
            # exchange plan (HOME's moment planes move per face, between buffers that swap)
            if self.home:
                check(lib().lbm_zslab_exchange(self.solver._h, self.solver._h, phase,
                                               C.c_void_p(self.solver.stream)))
                return
            if self._plan is None:
                hs = (C.c_void_p * 1)(self.solver._h.value)
                p = C.c_void_p()
                check(lib().lbm_zslab_plan_create(hs, 1, C.byref(p)))
                self._plan = p
            check(lib().lbm_zslab_plan_exchange(self._plan, phase, C.c_void_p(self.solver.stream)))
            return
        if self.home:
            if phase == 0:
                exchange(self._moment_views(), 0, self.rank, self.world, self.dist, self.group)
            return
        if phase == 0:
            exchange(self.views, 0, self.rank, self.world, self.dist, self.group)
            return
        exchange(self.views, 1, self.rank, self.world, self.dist, self.group, recv_views=self.staging)
        self._merge_staging()

    def set_solid_mask(self, mask):
        self.solver.set_solid_mask(with_ghosts(np.asarray(mask, np.uint8).reshape(self.shape), self.z0, self.z1))
        self._drop_plan()           # the plan holds the flag and link planes of the mask it was built for

    def set_legacy_mapping(self, band):
        self.solver.set_legacy_mapping(with_ghosts(np.asarray(band, np.uint8).reshape(self.shape), self.z0, self.z1))
        self._drop_plan()

    def reinit_from_host(self, rho=None, ux=None, uy=None, uz=None):
        self.solver.reinit_from_host(*[None if a is None else with_ghosts(
            np.asarray(a, np.float32).reshape(self.shape), self.z0, self.z1) for a in (rho, ux, uy, uz)])

    def step(self, n: int = 1, overlap: bool = False):
        """n steps.  overlap=True overlaps the face exchange with the interior
        planes (Legacy/Hybrid on 2 or more ranks, 3 or more own planes) for every
        step but the last, which runs whole, so that its statistics and macro
        fields come out as from lbm_step."""
        can = overlap and not self.home and self.world > 1 and self.planes["ghost_hi"] - 1 >= 3
        # one substep per call: statistics and macro fields only on the last, as lbm_step(n)
        quiet = n > 1 and (self._stats or self._macro)
        if quiet:
            self._outputs(False)
        for k in range(n):
            if can and k < n - 1:
                self._step_overlapped()
                continue
            if quiet and k == n - 1:
                self._outputs(True)
            self._flush()
            ex = self.home or _parity(self.solver) == 1
            if ex:
                self._exchange(0)
            self.solver.step(1)
            if ex and not self.home:
                self._exchange(1)

    def set_shear_omega(self, omega_s):
        self.solver.set_shear_omega(omega_s)

    def enable_stats(self, on=True):
        self._stats = bool(on)
        self.solver.enable_stats(on)

    def set_macro_output(self, on=True):
        self._macro = bool(on)
        self.solver.set_macro_output(on)

    def _outputs(self, on):
        self.solver.enable_stats(self._stats and on)
        self.solver.set_macro_output(self._macro and on)

    def synchronize(self):
        self._flush()
        self.solver.synchronize()

    def stats(self) -> dict:
        """Mass, kinetic energy, momentum-exchange drag and momentum of the whole
        grid (FP64, from the last step with statistics on): this rank's sums
        over its own planes, added over the ranks by one FP64 all-reduce.  Every
        rank must call it (a collective)."""
        self._flush()
        return reduce_stats(self.solver.stats(), int(np.prod(self.shape)), self.dist, self.group)

    def macros(self):
        """This rank's planes z0..z1-1 of rho, ux, uy, uz."""
        self._flush()
        return tuple(m[1:-1] for m in self.solver.macros())

    def state(self):
        """This rank's populations (natural layout after an even step count)."""
        self._flush()
        return self.solver.state()[:, 1:-1]

    def close(self):
        self._flush()
        self._drop_plan()
        self.solver.close()
