"""z-slab decomposition (slabs.py, lbm_set_z_ghosts / lbm_zslab_exchange) against
the single-grid run.

Every cell of a slab computes exactly what it computes in the whole grid, and
the exchange moves exactly the slots that cross the slab faces, so the
decomposed run must equal the single-grid run bit for bit: populations and
macro fields after an even number of steps, for Legacy and Hybrid, FP32 and
F16, periodic and duct boundaries, obstacles cut by the slab faces, uneven
slabs and a single slab exchanging with itself.  The FP64 statistics are sums
in another order: equal to 1e-12.
"""
import numpy as np
import pytest

from myfluidsimulation_b200.slabs import SlabSet
from myfluidsimulation_b200.solvers import (BC_DUCT, BC_PERIODIC, METHOD_HOME, METHOD_HYBRID, METHOD_LEGACY,
                                            STORE_BF16, STORE_F16, STORE_F32, Solver)

pytestmark = pytest.mark.gpu


def fields(nx, ny, nz, seed=1):
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    rho = (1 + 1e-3 * rng.standard_normal((nz, ny, nx))).astype(np.float32)
    u = (0.04 * np.sin(2 * np.pi * x / nx) * np.cos(2 * np.pi * z / nz)).astype(np.float32)
    v = (0.02 * rng.standard_normal((nz, ny, nx))).astype(np.float32)
    w = (0.03 * np.cos(2 * np.pi * y / ny)).astype(np.float32)
    return rho, u, v, w


def obstacle(nx, ny, nz, seed=2):
    rng = np.random.default_rng(seed)
    m = np.zeros((nz, ny, nx), np.uint8)
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    m[(x - nx // 3) ** 2 + (y - ny // 2) ** 2 + (z - nz // 2) ** 2 <= 16] = 1   # cut by the middle slab faces
    m.ravel()[rng.integers(0, m.size, m.size // 150)] = 1
    m[0, :3, :3] = 1                                                          # on the periodic z seam
    return m


CASES = [
    # (dims, parts, method, storage, bc)
    ((36, 20, 30), 3, METHOD_LEGACY, STORE_F32, BC_PERIODIC),
    ((36, 20, 30), 4, METHOD_LEGACY, STORE_F32, BC_PERIODIC),      # slabs of 7 and 8 planes
    ((36, 20, 30), 1, METHOD_LEGACY, STORE_F32, BC_PERIODIC),      # one slab, its own neighbour
    ((36, 20, 30), 2, METHOD_HYBRID, STORE_F32, BC_PERIODIC),
    ((40, 16, 18), 3, METHOD_LEGACY, STORE_F16, BC_PERIODIC),
    ((48, 18, 21), 3, METHOD_LEGACY, STORE_F32, BC_DUCT),
    ((17, 9, 12), 3, METHOD_LEGACY, STORE_F32, BC_PERIODIC),       # odd plane size: scalar even step
    ((36, 20, 30), 3, METHOD_HOME, STORE_F32, BC_PERIODIC),
    ((40, 16, 18), 4, METHOD_HOME, STORE_F16, BC_PERIODIC),         # stochastic rounding by global index
    ((48, 18, 21), 2, METHOD_HOME, STORE_BF16, BC_DUCT),
    ((36, 20, 30), 1, METHOD_HOME, STORE_F32, BC_PERIODIC),
]


@pytest.mark.parametrize("dims,parts,method,storage,bc", CASES)
def test_slabs_equal_single_grid(gpu, oracle, dims, parts, method, storage, bc):
    nx, ny, nz = dims
    f = fields(nx, ny, nz)
    m = obstacle(nx, ny, nz)
    band = oracle.band(m, 2)[1] if method == METHOD_HYBRID else None
    kw = dict(force=(1e-5, 2e-6, 0.0), method=method, storage=storage, bc=bc, inlet_u=0.04 if bc == BC_DUCT else 0.0)
    one = Solver(nx, ny, nz, 0.58, **kw)
    sl = SlabSet(nx, ny, nz, 0.58, parts, **kw)
    for obj in (one, sl):
        obj.set_solid_mask(m)
        if band is not None:
            obj.set_legacy_mapping(band)
            obj.set_shear_omega(1.4)
        obj.reinit_from_host(*f)
        obj.enable_stats(True)
        obj.step(7)
        obj.step(7)
        obj.synchronize()
    np.testing.assert_array_equal(sl.state(), one.state())
    for a, b in zip(sl.macros(), one.macros()):
        np.testing.assert_array_equal(a, b)
    s1, s2 = one.stats(), sl.stats()
    for k in ("mass", "ke_sum", "mom_x"):
        assert abs(s1[k] - s2[k]) <= 1e-12 * max(abs(s1[k]), 1e-30) + 1e-18, k
    one.close()
    sl.close()


def test_slab_setter_rejects(gpu):
    from myfluidsimulation_b200 import lib
    from myfluidsimulation_b200.solvers import BOUNCE_REFERENCE
    s = Solver(8, 8, 8, 0.6, bounce=BOUNCE_REFERENCE)      # the two-buffer push form
    assert lib().lbm_set_z_ghosts(s._h, 1) != 0
    s.close()
    s = Solver(8, 8, 2, 0.6)
    assert lib().lbm_set_z_ghosts(s._h, 1) != 0
    s.close()


class _Mailbox:
    """In-process point-to-point transport for emulated ranks on one GPU: a send
    stores a copy of its tensor; a receive waits (host side, with a time limit)
    for the matching send and copies it.  All ranks share the default stream, so
    the copies sit in stream order between the senders' and receivers' kernels;
    no kernel ever waits on another."""

    def __init__(self):
        import threading
        self.cv = threading.Condition()
        self.box = {}

    def put(self, key, t):
        with self.cv:
            self.box[key] = t.clone()
            self.cv.notify_all()

    def take(self, key, timeout=60.0):
        with self.cv:
            if not self.cv.wait_for(lambda: key in self.box, timeout):
                raise TimeoutError(f"no send for {key}")
            return self.box.pop(key)


class _FakeDist:
    """The torch.distributed calls DistSlab makes, over a _Mailbox."""

    class _Work:
        def wait(self):
            return True

    def __init__(self, rank, world, box):
        self.rank, self.world, self.mb = rank, world, box
        self.nsend, self.nrecv = {}, {}

    def get_rank(self, group=None):
        return self.rank

    def get_world_size(self, group=None):
        return self.world

    def get_backend(self, group=None):
        return "gloo"

    class ReduceOp:
        SUM = "sum"

    def all_reduce(self, t, op=None, group=None):
        """Sum over the emulated ranks, added in rank order."""
        k = self.nsend.get("ar", 0)
        self.nsend["ar"] = k + 1
        for r in range(self.world):
            if r != self.rank:
                self.mb.put(("ar", self.rank, r, k), t)
        parts = {self.rank: t.clone()}
        for r in range(self.world):
            if r != self.rank:
                parts[r] = self.mb.take(("ar", r, self.rank, k))
        acc = parts[0].clone()
        for r in range(1, self.world):
            acc += parts[r]
        t.copy_(acc)

    def isend(self, *a):
        raise AssertionError("used only as a P2POp tag")

    def irecv(self, *a):
        raise AssertionError("used only as a P2POp tag")

    class P2POp:
        def __init__(self, op, tensor, peer, group=None):
            self.op, self.tensor, self.peer = op, tensor, peer

    def batch_isend_irecv(self, ops):
        for o in ops:
            if o.op == self.isend:
                k = self.nsend.get(o.peer, 0)
                self.nsend[o.peer] = k + 1
                self.mb.put((self.rank, o.peer, k), o.tensor)
        for o in ops:
            if o.op == self.irecv:
                k = self.nrecv.get(o.peer, 0)
                self.nrecv[o.peer] = k + 1
                o.tensor.copy_(self.mb.take((o.peer, self.rank, k)))
        return [self._Work() for _ in ops]


@pytest.mark.parametrize("world,method,overlap", [(1, METHOD_LEGACY, False), (1, METHOD_HOME, False),
                                                  (2, METHOD_LEGACY, False), (3, METHOD_HYBRID, False),
                                                  (3, METHOD_HOME, False), (2, METHOD_LEGACY, True),
                                                  (3, METHOD_HYBRID, True)])
def test_dist_slabs_equal_single_grid(gpu, oracle, world, method, overlap):
    """DistSlab's multi-rank path (views of the slot planes, point-to-point plan,
    staging and merge) with `world` ranks emulated by threads on this GPU; with
    overlap, the steps that split each slab into interior and boundary planes
    around the exchange (lbm_zslab_step_planes)."""
    import threading
    from myfluidsimulation_b200.slabs import DistSlab, slab_bounds
    nx, ny, nz = 32, 18, 27
    f = fields(nx, ny, nz, 4)
    m = obstacle(nx, ny, nz, 5)
    band = oracle.band(m, 2)[1] if method == METHOD_HYBRID else None
    kw = dict(force=(1e-5, 0.0, 3e-6), method=method)
    one = Solver(nx, ny, nz, 0.6, **kw)
    one.set_solid_mask(m)
    if band is not None:
        one.set_legacy_mapping(band)
    one.reinit_from_host(*f)
    one.step(9)
    one.enable_stats(True)
    one.step(1)
    one.synchronize()
    box = _Mailbox()
    out, errs = {}, []

    def rank_main(r):
        try:
            d = DistSlab(nx, ny, nz, 0.6, dist=_FakeDist(r, world, box), **kw)
            d.set_solid_mask(m)
            if band is not None:
                d.set_legacy_mapping(band)
            d.reinit_from_host(*f)
            d.step(9, overlap=overlap)
            d.enable_stats(True)
            d.step(1)
            d.synchronize()
            out[r] = (d.state(), d.macros(), d.stats())
            d.close()
        except Exception as e:   # reported by the main thread
            errs.append(e)

    th = [threading.Thread(target=rank_main, args=(r,)) for r in range(world)]
    for t in th:
        t.start()
    for t in th:
        t.join(300)
    assert not errs, errs
    st = np.concatenate([out[r][0] for r in range(world)], axis=1)
    np.testing.assert_array_equal(st, one.state())
    mac = [np.concatenate([out[r][1][k] for r in range(world)], axis=0) for k in range(4)]
    for a, b in zip(mac, one.macros()):
        np.testing.assert_array_equal(a, b)
    # the FP64 statistics: every rank's own sums, added over the ranks
    want = one.stats()
    for r in range(world):
        got = out[r][2]
        for k in ("mass", "ke_sum", "mom_x", "mom_y", "mom_z", "drag_x", "drag_y", "drag_z"):
            assert abs(got[k] - want[k]) <= 1e-12 * max(abs(want[k]), abs(want["mass"]) * 1e-6), (k, got[k], want[k])
    assert [b for b in slab_bounds(nz, world)][-1][1] == nz
    one.close()


def test_plan_exchange_equals_pairwise_and_graph_replay(gpu):
    """The one-launch exchange plan moves what the per-face exchange moves, and
    a captured graph of the slab steps replays the same state."""
    import torch
    nx, ny, nz = 24, 16, 20
    f = fields(nx, ny, nz, 6)
    m = obstacle(nx, ny, nz, 7)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        runs = []
        for mode in ("plan", "pairwise", "graph"):
            sl = SlabSet(nx, ny, nz, 0.6, 3, force=(1e-5, 0, 0), stream=stream.cuda_stream)
            sl.set_solid_mask(m)
            sl.reinit_from_host(*f)
            if mode == "pairwise":
                sl._exchange = sl.exchange_pairwise
            sl.step(2)
            if mode == "graph":
                g = sl.graph(4)
                g.replay()
                g.replay()
            else:
                sl.step(8)
            sl.synchronize()
            runs.append(sl.state())
            if mode == "graph":
                del g
            sl.close()
    np.testing.assert_array_equal(runs[0], runs[1])
    np.testing.assert_array_equal(runs[0], runs[2])
