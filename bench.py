#!/usr/bin/env python
"""D3Q19 MLUPS and HBM-roofline fraction on the duct-past-a-sphere workloads.

Two workloads share one grid and one solid mask: a 256x128x128 duct with
solid wall cells on its y/z faces and an icosphere (5,120 triangles, radius
16 cells, centre (64,64,64)) voxelized by ray parity, tau = 0.56.
  * "periodic": x periodic, driven by a body force (1e-5, 0, 0), started
    from rho = 1, u = 0.  This is the form the reference's own solvers can
    run (they have no inlet/outlet), so both arms time the same work.
  * "inlet": uniform velocity inlet u = 0.05 at x = 0, zero-gradient outflow
    at x = 255, started from rho = 1, u = 0.05.
One bench step = 50 LBM steps (one drag interval) with the FP64 statistics
(mass, energy, momentum, momentum-exchange drag) taken at the last one.
Inputs are synthetic (generated from fixed parameters; no dataset).  The
state (319 MB of FP32 populations) is larger than L2, so no flush is needed
between steps.

`value` is Legacy BGK FP32 on the periodic workload; every method on both
workloads is reported under "methods" (keys `legacy`, `home`, `hybrid` for the
periodic workload, `*_inlet` for the inlet duct).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

With --gpus N (under torchrun) every rank runs its own duct instance (weak
scaling, no data-path collective); time is the max over ranks.  With
--decomp zslab the ranks instead hold z-slabs of ONE duct of 128 x N planes
and exchange their face slots around every odd step through NCCL.
--impl reference times the reference's own CUDA solvers (compiled from its
sources into oracle/_ref) on the periodic workload, Legacy, HOME and
Hybrid(B0=2), with the mask built by the reference's own STL loader and
voxelizer (oracle/_ref/libref_cpu.so); it loads nothing of this library.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import math
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX, NY, NZ = 256, 128, 128
TAU = 0.56
U_IN = 0.05
FORCE = (1e-5, 0.0, 0.0)
DRAG_EVERY = 50
RADIUS, CENTER = 16, (64, 64, 64)
B0 = 2
# algorithmic bytes per cell-update (state read once + written once, plus the mask/flag byte)
BYTES = {"legacy": 19 * 4 * 2 + 1, "hybrid": 19 * 4 * 2 + 1, "home": 10 * 4 * 2 + 1}
KERNEL = {"legacy": "aa_even/aa_odd", "hybrid": "aa_even/aa_odd", "home": "home_step"}
METRIC = "D3Q19 MLUPS (Legacy BGK FP32, duct 256x128x128 past a voxelized sphere)"
WORKLOAD_TEXT = {
    "periodic": "duct 256x128x128, y/z walls as solid cells, icosphere (5120 triangles, r=16, centre (64,64,64)) "
                "voxelized by ray parity, x periodic, body force (1e-5,0,0), tau 0.56, start rho=1 u=0; "
                "one step = 50 LBM steps + FP64 statistics",
    "inlet": "duct 256x128x128, inlet u=0.05 at x=0, zero-gradient outflow, y/z walls as solid cells, icosphere "
             "(5120 triangles, r=16) voxelized by ray parity, tau 0.56, start rho=1 u=0.05; one step = 50 LBM "
             "steps + FP64 statistics (drag)",
}
# the configuration both arms print for the headline (Legacy, periodic workload)
HEAD_CONFIG = {"workload": WORKLOAD_TEXT["periodic"], "method": "legacy", "storage": "f32",
               "l2": "state larger than L2 (no flush needed)"}
RUNS = [("legacy", "periodic"), ("home", "periodic"), ("hybrid", "periodic"),
        ("legacy", "inlet"), ("home", "inlet"), ("hybrid", "inlet")]


def run_key(method, workload):
    return method if workload == "periodic" else f"{method}_inlet"


def load_workloads():
    """The input generator (pure numpy), loaded from its file so that nothing of
    the library's package (and no native code) is imported with it."""
    spec = importlib.util.spec_from_file_location(
        "_bench_workloads", os.path.join(ROOT, "myfluidsimulation_b200", "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(method):
    """DRAM bytes per cell of the dominant kernel from the committed ncu summary, or None."""
    p = os.path.join(ROOT, "profiles", "traffic.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        m = re.match(r"\|\s*%s\s*\|\s*([0-9.]+)\s*\|" % method, line)
        if m:
            return float(m.group(1))
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 8:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[4 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def build_mask(tmpdir):
    """Icosphere STL -> the library's STL loader -> its GPU voxelizer -> duct walls."""
    from myfluidsimulation_b200 import geometry as G
    W = load_workloads()
    tris, scale, tr = W.duct_sphere_mesh(NX, NY, NZ, RADIUS, CENTER)
    path = os.path.join(tmpdir, "icosphere.stl")
    W.write_binary_stl(path, tris)
    mesh = G.load_stl(path)
    sphere = G.voxelize_mesh_to_mask(mesh, G.VoxelParams(NX, NY, NZ, scale, tr))
    return W.duct_mask(NX, NY, NZ, sphere), int(mesh.tris.shape[0]), int(sphere.sum())


def initial_fields(workload, mask):
    rho = np.ones((NZ, NY, NX), np.float32)
    u = np.full((NZ, NY, NX), U_IN if workload == "inlet" else 0.0, np.float32)
    u[mask != 0] = 0
    return rho, u


def make_solver(method, workload, mask, stream):
    from myfluidsimulation_b200.solvers import (BC_DUCT, BC_PERIODIC, METHOD_HOME, METHOD_HYBRID, METHOD_LEGACY,
                                                Solver)
    m = {"legacy": METHOD_LEGACY, "home": METHOD_HOME, "hybrid": METHOD_HYBRID}[method]
    if workload == "inlet":
        s = Solver(NX, NY, NZ, TAU, method=m, bc=BC_DUCT, inlet_u=U_IN, stream=stream)
    else:
        s = Solver(NX, NY, NZ, TAU, FORCE, method=m, bc=BC_PERIODIC, stream=stream)
    s.set_solid_mask(mask)
    nb = s.build_band(B0) if method == "hybrid" else 0
    rho, u = initial_fields(workload, mask)
    s.reinit_from_host(rho, u, None, None)
    s.enable_stats(True)
    return s, nb


def kernel_split(s, method, torch, launches=40):
    """Per-kernel device time, summing to the time of back-to-back steps.

    The total is ONE lbm_step(launches) call (no macro fields, no statistics)
    between two CUDA events, so nothing sits between the launches.  For the AA
    methods the even/odd shares come from a second pass of single-step
    launches with a CUDA event between every two (no synchronisation inside
    the loop), whose median intervals split that total.  Returns
    {kernel: us per launch}."""
    st = torch.cuda.current_stream()
    s.enable_stats(False)
    s.set_macro_output(False)
    s.step(2)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(st)
    s.step(launches)                   # an even count: as many even as odd launches
    e1.record(st)
    torch.cuda.synchronize()
    mean_us = 1e3 * e0.elapsed_time(e1) / launches
    if method == "home":
        s.set_macro_output(True)
        s.enable_stats(True)
        return {"home_step": round(mean_us, 2)}
    par = s.steps % 2                  # parity of the first launch below
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(launches + 1)]
    ev[0].record(st)
    for i in range(launches):
        s.step(1)
        ev[i + 1].record(st)
    torch.cuda.synchronize()
    t = [1e3 * ev[i].elapsed_time(ev[i + 1]) for i in range(launches)]
    s.set_macro_output(True)
    s.enable_stats(True)
    a, b = statistics.median(t[0::2]), statistics.median(t[1::2])
    names = ("aa_even", "aa_odd") if par == 0 else ("aa_odd", "aa_even")
    return {names[0]: round(2 * mean_us * a / (a + b), 2), names[1]: round(2 * mean_us * b / (a + b), 2)}


def run_method(method, workload, mask, args, torch, dist=None):
    st = torch.cuda.current_stream()
    s, nb = make_solver(method, workload, mask, st.cuda_stream)
    for _ in range(args.warmup):
        s.step(DRAG_EVERY)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
        torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(args.steps):
        s.step(DRAG_EVERY)
    e1.record(st)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    st_ = s.stats()
    res = {"ms_total": ms, "launches": args.steps * (DRAG_EVERY + 1), "band_cells": nb,
           "drag_last": [st_["drag_x"], st_["drag_y"], st_["drag_z"]], "mass": st_["mass"],
           "kernel_us": kernel_split(s, method, torch)}
    return s, res


def e2e_run(method, workload, mask, args, torch, dist=None):
    """Through the public C-ABI with host buffers: every step uploads the macro
    fields from pinned host memory, reinitialises from them, runs one drag
    interval and reads the macro fields and the statistics back.  The copies of
    consecutive steps are pipelined against the compute (lbm_stage_from_host /
    lbm_reinit_from_stage / lbm_read_macros_async / lbm_get_stats_async): the
    upload of step k+1 and the read-back of step k run while step k+1 computes,
    and the timed region ends after the last read-back."""
    st = torch.cuda.current_stream()
    s, _ = make_solver(method, workload, mask, st.cuda_stream)
    N = NX * NY * NZ
    pin = lambda: torch.empty(N, dtype=torch.float32, pin_memory=True).numpy().reshape(NZ, NY, NX)
    rho_h, u_h, v_h, w_h = pin(), pin(), pin(), pin()
    r0, u0 = initial_fields(workload, mask)
    rho_h[:] = r0
    u_h[:] = u0
    v_h[:] = 0
    w_h[:] = 0
    outs = [[pin() for _ in range(4)] for _ in range(2)]
    import ctypes as C
    from myfluidsimulation_b200._lib import check, lib
    L = lib()
    vp = lambda a: a.ctypes.data_as(C.c_void_p)
    stats = [torch.zeros(8, dtype=torch.float64, pin_memory=True).numpy() for _ in range(2)]

    def run(k_steps):
        # every step's macro fields and statistics come back to pinned host
        # buffers asynchronously; the loop waits for all of them at its end
        check(L.lbm_stage_from_host(s._h, vp(rho_h), vp(u_h), vp(v_h), vp(w_h)))
        for k in range(k_steps):
            check(L.lbm_reinit_from_stage(s._h))
            if k + 1 < k_steps:
                check(L.lbm_stage_from_host(s._h, vp(rho_h), vp(u_h), vp(v_h), vp(w_h)))
            check(L.lbm_step(s._h, DRAG_EVERY))
            check(L.lbm_read_macros_async(s._h, *[vp(o) for o in outs[k % 2]]))
            check(L.lbm_get_stats_async(s._h, vp(stats[k % 2])))
        check(L.lbm_wait_reads(s._h))
        check(L.lbm_synchronize(s._h))

    run(max(2, args.warmup // 2))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
        torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(st)
    run(args.steps)
    e1.record(st)
    torch.cuda.synchronize()
    wall = (time.perf_counter() - t0) * 1e3
    ms = max(e0.elapsed_time(e1), 0.0)
    # the read-back of the last step ends on the copy stream after e1: use the wall clock if longer
    ms = max(ms, wall)
    s.close()
    return ms, wall, 4 * 4 * N, 4 * 4 * N + 8 * 8


def cpu_baseline(mask, gpu_state_fn):
    """The FP64 oracle (the C restatement, OpenMP over the host cores) on a bounded
    sample of the headline workload: the full grid for a few steps."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_bind import Oracle
    o = Oracle()
    nthreads = o.lib.orc_num_threads()
    rho = np.ones((NZ, NY, NX))
    u = np.zeros((NZ, NY, NX))
    f0 = o.reinit_eq(rho, u, None, None)
    force = tuple(float(np.float32(x)) for x in FORCE)
    # size the sample to ~10-20 s: time one step first
    t = time.perf_counter()
    o.bgk_run(f0, mask, 1, TAU, force=force)
    t1 = time.perf_counter() - t
    steps = int(max(2, min(40, 12.0 / max(t1, 1e-3))))
    t = time.perf_counter()
    f, r, ux, uy, uz, drag = o.bgk_run(f0, mask, steps, TAU, force=force)
    dt = time.perf_counter() - t
    mlups = NX * NY * NZ * steps / dt / 1e6
    # the same sample on the GPU: relative L2 of the state against FP64
    g = gpu_state_fn(steps)
    err = float(np.linalg.norm(g - f) / np.linalg.norm(f))
    return {"value": round(mlups, 2), "unit": "MLUPS", "cores": int(nthreads), "kind": "port",
            "sample": f"FP64 oracle (C, OpenMP) Legacy BGK, periodic duct {NX}x{NY}x{NZ}, {steps} steps"}, err, steps


def reference_mask(tmpdir):
    """The duct mask built by the reference's own code (oracle/_ref/libref_cpu.so:
    its stl_loader.cpp and voxelize.cpp) from the same generated icosphere."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_bind import RefCPU
    W = load_workloads()
    tris, scale, tr = W.duct_sphere_mesh(NX, NY, NZ, RADIUS, CENTER)
    path = os.path.join(tmpdir, "icosphere.stl")
    W.write_binary_stl(path, tris)
    R = RefCPU()
    t, bb = R.load_stl(path)
    sphere = R.voxelize(t, bb, (NX, NY, NZ), scale, tr)
    return W.duct_mask(NX, NY, NZ, sphere), R


def reference_arm(args, torch, rank, world):
    """The reference's own CUDA solvers on the periodic workload: Legacy (the
    headline), HOME and Hybrid(B0=2), each timed over `steps` calls of step(50)
    with cudaEvents on the default stream, as its own sweep times them
    (src/main_compare.cpp:539-553).  Nothing of this library is loaded."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_bind import RefCPU, RefCUDA
    base = {"metric": METRIC, "unit": "MLUPS", "impl": "reference", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic"}
    if not (RefCUDA.available() and RefCPU.available()):
        if rank == 0:
            base["unavailable"] = "the reference's build oracle/_ref/libref_cuda.so / libref_cpu.so is not present"
            print(json.dumps(base))
        return
    if rank != 0:
        return
    with tempfile.TemporaryDirectory() as td:
        mask, RC = reference_mask(td)
    solid = (mask != 0).astype(np.uint8)
    R = RefCUDA()
    N = NX * NY * NZ
    methods = {}
    clocks = None
    for name, mid in (("legacy", 0), ("home", 1), ("hybrid", 2)):
        h = R.create(mid, (NX, NY, NZ), TAU, FORCE)
        R.set_mask(h, solid)
        if name == "hybrid":
            _, leg = RC.band(solid, B0)        # the reference's own band BFS (sim_runner.hpp)
            R.set_legacy(h, leg)
        R.init_rho(h, None)                    # rho = 1, u = 0 (sim_runner.hpp:135-137)
        R.time_steps(h, args.warmup, DRAG_EVERY)
        if name == "legacy":
            with ClockSampler(int(os.environ.get("LOCAL_RANK", 0))) as clk:
                ms = R.time_steps(h, args.steps, DRAG_EVERY)
            clocks = clk.summary()
        else:
            ms = R.time_steps(h, args.steps, DRAG_EVERY)
        R.destroy(h)
        mlups = N * DRAG_EVERY * args.steps / (ms * 1e-3) / 1e6
        methods[name] = {"mlups": round(mlups, 1), "ms_per_step": round(ms / args.steps, 4),
                         "call": {"legacy": "LBM3D_Legacy::step(50)", "home": "LBM3D_Home::step(50)",
                                  "hybrid": "LBM3D_Hybrid::step(50)"}[name]}
    h = methods["legacy"]
    base.update({
        "value": h["mlups"], "ms_per_step": h["ms_per_step"], "config": dict(HEAD_CONFIG),
        "methods": methods,
        "cpu_baseline": {"value": h["mlups"], "unit": "MLUPS", "cores": 0, "kind": "reference", "device": "cuda:0",
                         "sample": f"the reference's CUDA solvers (oracle/_ref/libref_cuda.so), {args.steps} x 50 "
                                   "steps per method; mask from its own STL loader and voxelizer"},
        "e2e": {"value": h["mlups"], "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "clocks": clocks,
    })
    print(json.dumps(base))


def tgv_fields(n, torch):
    """The 3-D Taylor-Green field of n^3 cells (u0 0.05, k 2 pi / n) at cell
    centres, built on the device in FP64 and cast to FP32: rho, u, v, w."""
    k = 2 * math.pi / n
    c = (torch.arange(n, device="cuda", dtype=torch.float64) + 0.5) * k
    z, y, x = c.view(n, 1, 1), c.view(1, n, 1), c.view(1, 1, n)
    u = (0.05 * torch.sin(x) * torch.cos(y) * torch.cos(z)).float().contiguous()
    v = (-0.05 * torch.cos(x) * torch.sin(y) * torch.cos(z)).float().contiguous()
    w = torch.zeros_like(u)
    rho = (1.0 + 3.0 * (0.05 ** 2 / 16.0) * (torch.cos(2 * x) + torch.cos(2 * y)) * (torch.cos(2 * z) + 2.0)).float().contiguous()
    return rho, u, v, w


def _device_field(ptr, n, torch):
    """A float32 torch view of n values of device memory (no copy)."""
    class _Mem:
        __cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (int(ptr), False), "version": 3,
                                    "strides": None}
    return torch.as_tensor(_Mem(), device="cuda")


def _rel_l2(a, b):
    d = (a.double() - b.double()).norm().item()
    return d / max(b.double().norm().item(), 1e-300)


def precision_study(args, torch):
    """512^3 periodic Taylor-Green vortex (tau 0.51, u0 0.05, k 2pi/512), Legacy and
    HOME, in FP64 (storage and arithmetic: the reference form), FP32, F16 and BF16:
      * MLUPS over --steps steps after 4 warm-up steps (CUDA events, macro output
        off), with the roofline fraction of the algorithmic bytes, and the
        even/odd launch split (events between back-to-back launches);
      * from the initial field, the kinetic energy (FP64 reduction on the GPU)
        every --tgv-every steps up to --tgv-steps, and the fields at the end;
      * every form's energy curve (max relative error over the samples) and
        final fields (relative L2 of rho - 1 and of u) against the FP64 run of
        the same method.
    The reference's own HOME (FP32, oracle/_ref/libref_cuda.so) runs the same
    case for its time and error; its Legacy cannot (its int32 indices overflow
    above about 483^3 cells)."""
    from myfluidsimulation_b200.solvers import (METHOD_HOME, METHOD_LEGACY, STORE_BF16, STORE_F16, STORE_F32,
                                                STORE_F64, Solver)
    n = args.tgv_n
    N = n ** 3
    steps, every = args.tgv_steps, args.tgv_every
    st = torch.cuda.current_stream()
    rho, u, v, w = tgv_fields(n, torch)
    out = {}
    forms = (("f64", STORE_F64, 8), ("f32", STORE_F32, 4), ("f16", STORE_F16, 2), ("bf16", STORE_BF16, 2))
    peak, peak_kind = measured_peaks()
    ref_fields, ref_ke_end = {}, {}
    for mname, m, ncomp in (("legacy", METHOD_LEGACY, 19), ("home", METHOD_HOME, 10)):
        ref_curve = None
        for sname, sto, esz in forms:
            s = Solver(n, n, n, 0.51, method=m, storage=sto, stream=st.cuda_stream)
            s.reinit_from_macro(rho, u, v, w)
            s.set_macro_output(False)
            for _ in range(4):
                s.step(1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(st)
            s.step(args.steps)
            e1.record(st)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            mlups = N * args.steps / (ms * 1e-3) / 1e6
            # per-launch split: Legacy alternates the local (even) and neighbour (odd) kernels
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(9)]
            ev[0].record(st)
            for i in range(8):
                s.step(1)
                ev[i + 1].record(st)
            torch.cuda.synchronize()
            t = [1e3 * ev[i].elapsed_time(ev[i + 1]) for i in range(8)]
            # accuracy run from the initial field
            s.reinit_from_macro(rho, u, v, w)
            s.set_macro_output(True)
            s.enable_stats(True)
            curve = []
            done = 0
            while done < steps:
                k = min(every, steps - done)
                s.step(k)
                done += k
                curve.append(s.stats()["ke_sum"] / N)
            s.synchronize()
            fields = [_device_field(p_, N, torch) for p_ in s.macro_ptrs()]
            b = ncomp * esz * 2
            res = {"mlups": round(mlups, 1), "us_per_step": round(ms * 1e3 / args.steps, 1),
                   "roofline_frac": round(N * b / (ms * 1e-3 / args.steps) / 1e9 / peak, 4), "bytes_per_cell": b,
                   "us_launch_a_b": [round(statistics.median(t[0::2]), 1), round(statistics.median(t[1::2]), 1)],
                   "ke_final_over_initial": curve[-1] / (curve[0] if curve else 1.0)}
            if sto == STORE_F64:
                ref_curve = np.array(curve)
                ref_ke_end[mname] = curve[-1]
                ref_fields[mname] = [f.clone() for f in fields]
            else:
                c = np.array(curve)
                res["ke_max_rel_err_vs_f64"] = float(np.max(np.abs(c - ref_curve) / ref_curve))
                rf = ref_fields[mname]
                res["rho_minus_1_rel_l2_vs_f64"] = _rel_l2(fields[0] - 1.0, rf[0] - 1.0)
                res["u_rel_l2_vs_f64"] = _rel_l2(torch.stack(fields[1:]), torch.stack(rf[1:]))
            del fields
            s.close()
            out[f"{mname}_{sname}"] = res
        for sname in ("f16", "bf16"):
            out[f"{mname}_{sname}"]["speedup_vs_f32"] = round(
                out[f"{mname}_{sname}"]["mlups"] / out[f"{mname}_f32"]["mlups"], 3)
    # the reference's own HOME on the same case (FP32): time and error against FP64
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_bind import RefCUDA
    if RefCUDA.available():
        R = RefCUDA()
        h = R.create(1, (n, n, n), 0.51)
        try:
            host = [x.cpu().numpy() for x in (rho, u, v, w)]
            R.set_mask(h, np.zeros((n, n, n), np.uint8))
            R.init_fields(h, *host)
            ms = R.time_steps(h, args.steps, 1)
            R.init_fields(h, *host)
            R.time_steps(h, steps, 1)
            rr, ru, rv, rw = [torch.from_numpy(a.ravel()).cuda() for a in R.macros(h, (n, n, n))]
            rf = ref_fields["home"]
            ke = 0.5 * float((ru.double() ** 2 + rv.double() ** 2 + rw.double() ** 2).sum().item()) / N
            out["home_reference_build"] = {
                "mlups": round(N * args.steps / (ms * 1e-3) / 1e6, 1), "us_per_step": round(ms * 1e3 / args.steps, 1),
                "call": "LBM3D_Home::step(1) per step (synchronous)",
                "ke_rel_err_vs_f64_at_end": abs(ke - ref_ke_end["home"]) / ref_ke_end["home"],
                "rho_minus_1_rel_l2_vs_f64": _rel_l2(rr - 1.0, rf[0] - 1.0),
                "u_rel_l2_vs_f64": _rel_l2(torch.stack([ru, rv, rw]), torch.stack(rf[1:]))}
        finally:
            R.destroy(h)
    out["legacy_reference_build"] = {"unavailable": "the reference's Legacy step indexes populations with int32 "
                                                    "(src/lbm/lbm3d_legacy.cu:73,94-106): 19 x 512^3 overflows"}
    print(json.dumps({"study": "precision", "workload": f"TGV {n}^3 periodic, tau 0.51, u0 0.05, "
                      f"{args.steps} timed steps; KE every {every} steps up to {steps}, fields at {steps}",
                      "hbm_peak_gbs": {"value": peak, "source": peak_kind}, "results": out}))


def batch_instances(count=64, seed=20261203):
    """The batched Hybrid(B0) sweep: `count` duct-with-sphere instances drawn from a
    seeded numpy generator: nx in {64,80,..,192}, ny, nz in {32,48,..,96}, B0 in
    {0,1,2,3,4,6}, tau uniform in [0.51, 0.8], sphere radius 0.15 min(ny,nz) at
    x = nx/4 (y, z centred), inlet u = 0.04."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        nx = int(rng.choice(np.arange(64, 193, 16)))
        ny = int(rng.choice(np.arange(32, 97, 16)))
        nz = int(rng.choice(np.arange(32, 97, 16)))
        out.append({"dims": (nx, ny, nz), "b0": int(rng.choice([0, 1, 2, 3, 4, 6])),
                    "tau": float(rng.uniform(0.51, 0.8)), "radius": 0.15 * min(ny, nz),
                    "center": (nx / 4, ny / 2, nz / 2), "u_in": 0.04})
    return out


def batch_study(args, torch):
    """64 uneven Hybrid(B0) duct instances: one persistent launch per step over all
    of them (autotuned, graph-replayed) against stepping them one by one."""
    from myfluidsimulation_b200 import geometry as G
    from myfluidsimulation_b200 import workloads as W
    from myfluidsimulation_b200.solvers import BC_DUCT, METHOD_HYBRID, Batch, Solver
    st = torch.cuda.current_stream()
    specs = batch_instances(args.batch_count)
    steps = args.batch_steps

    def make_all():
        solvers = []
        for sp in specs:
            nx, ny, nz = sp["dims"]
            tris, scale, tr = W.duct_sphere_mesh(nx, ny, nz, sp["radius"], sp["center"], levels=3)
            sph = G.voxelize_mesh_to_mask(G.mesh_from_triangles(tris), G.VoxelParams(nx, ny, nz, scale, tr))
            mask = W.duct_mask(nx, ny, nz, sph)
            s = Solver(nx, ny, nz, sp["tau"], method=METHOD_HYBRID, bc=BC_DUCT, inlet_u=sp["u_in"],
                       stream=st.cuda_stream)
            s.set_solid_mask(mask)
            s.build_band(sp["b0"])
            u = np.full((nz, ny, nx), sp["u_in"], np.float32)
            u[mask != 0] = 0
            sp["u0"] = u
            s.reinit_from_host(np.ones((nz, ny, nx), np.float32), u, None, None)
            s.set_macro_output(False)
            solvers.append(s)
        return solvers

    cells = sum(int(np.prod(sp["dims"])) for sp in specs)
    ev = lambda: torch.cuda.Event(enable_timing=True)
    # one by one: every instance advanced through its own captured graph
    solvers = make_all()
    for s in solvers:
        s.step_graph(50)
    torch.cuda.synchronize()
    e0, e1 = ev(), ev()
    e0.record(st)
    for s in solvers:
        for _ in range(steps // 50):
            s.step_graph(50)
    e1.record(st)
    torch.cuda.synchronize()
    ms_seq = e0.elapsed_time(e1)
    drag_seq = []
    for s in solvers:
        s.enable_stats(True)
        s.step(2)
        drag_seq.append(s.stats()["drag_x"])
        s.close()
    # batched
    solvers = make_all()
    b = Batch(solvers, stream=st.cuda_stream)
    tuning = b.tune(2)
    for s, sp in zip(solvers, specs):   # restart from the initial state after tuning
        nx, ny, nz = sp["dims"]
        s.reinit_from_host(np.ones((nz, ny, nx), np.float32), sp["u0"], None, None)
    b.refresh()
    b.step(50)
    torch.cuda.synchronize()
    e0, e1 = ev(), ev()
    e0.record(st)
    for _ in range(steps // 50):
        b.step(50)
    e1.record(st)
    torch.cuda.synchronize()
    ms_b = e0.elapsed_time(e1)
    b.enable_stats(True)
    b.step(2)
    drag_b = b.stats()[:, 2]
    b.close()
    for s in solvers:
        s.close()
    done = cells * (steps // 50) * 50
    print(json.dumps({"study": "batch", "instances": len(specs), "cells": cells, "steps": (steps // 50) * 50,
                      "batched": {"mlups": round(done / (ms_b * 1e-3) / 1e6, 1), "ms": round(ms_b, 2),
                                  "launch": "one persistent launch per step, graph-replayed 50 at a time",
                                  "tuning": tuning},
                      "one_by_one": {"mlups": round(done / (ms_seq * 1e-3) / 1e6, 1), "ms": round(ms_seq, 2)},
                      "drag_x_batched": [round(float(d), 6) for d in drag_b],
                      "drag_x_max_abs_diff_vs_one_by_one": float(np.max(np.abs(np.array(drag_seq) - drag_b))),
                      "b0": [sp["b0"] for sp in specs], "dims": [sp["dims"] for sp in specs]}))


def adjoint_study(args, torch):
    """The adjoint case: BGK duct 128x64x64, tau 0.6, sphere r=10 at (32,32,32);
    controls = inlet profile u_x(y,z) = 0.04 + 0.005 N(0,1) smoothed by a 5x5 box
    filter and the initial velocity (0.04 + 1e-3 N(0,1) in x, 1e-3 N(0,1) in y, z);
    objective = mean drag over steps 400-500; checkpoints every 50 steps.  Times
    the FP32 and FP64 forward+adjoint and checks the gradient against central
    differences of the FP64 objective (eps 1e-3) on random unit directions."""
    from myfluidsimulation_b200 import workloads as W
    from myfluidsimulation_b200.adjoint import DuctProblem, objective
    nx, ny, nz = 128, 64, 64
    z, y, x = np.meshgrid(np.arange(nz) + 0.5, np.arange(ny) + 0.5, np.arange(nx) + 0.5, indexing="ij")
    ball = ((x - 32) ** 2 + (y - 32) ** 2 + (z - 32) ** 2 <= 100).astype(np.uint8)
    mask = W.duct_mask(nx, ny, nz, ball)
    gen = torch.Generator().manual_seed(4)
    raw = (0.04 + 0.005 * torch.randn((nz + 4, ny + 4), generator=gen, dtype=torch.float64)).numpy()
    k = np.ones(5) / 5
    ui = np.apply_along_axis(lambda r: np.convolve(r, k, "valid"), 1, raw)
    ui = np.apply_along_axis(lambda c: np.convolve(c, k, "valid"), 0, ui)
    u0 = 1e-3 * torch.randn((3, nz, ny, nx), generator=gen, dtype=torch.float64).numpy()
    u0[0] += 0.04
    prob = DuctProblem(nx, ny, nz, 0.6, mask, n_steps=500, window=(400, 500), checkpoint_every=50)
    out = {"study": "adjoint", "workload": "duct 128x64x64, sphere r=10 at (32,32,32), tau 0.6, 500 steps, "
                                           "J = mean drag over steps 400-500, checkpoints every 50"}
    for prec in ("f32", "f64"):
        objective(prob, ui, u0, prec, grad=True)          # warm-up
        t0 = time.perf_counter()
        J, gi, gu = objective(prob, ui, u0, prec, grad=True)
        dt = time.perf_counter() - t0
        t0 = time.perf_counter()
        objective(prob, ui, u0, prec)
        dtf = time.perf_counter() - t0
        out[prec] = {"J": J, "seconds_forward_and_adjoint": round(dt, 3), "seconds_forward": round(dtf, 3),
                     "grad_inlet_norm": float(np.linalg.norm(gi)), "grad_u0_norm": float(np.linalg.norm(gu))}
        if prec == "f32":
            g32 = (gi, gu)
        else:
            g64 = (gi, gu)
    rl = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    out["f32_vs_f64_grad_rel_l2"] = {"inlet": rl(g32[0], g64[0]), "u0": rl(g32[1], g64[1])}
    rng = np.random.default_rng(2026)
    eps = 1e-3
    errs = []
    for _ in range(args.fd_directions):
        di = rng.standard_normal(ui.shape)
        du = rng.standard_normal(u0.shape)
        sc = 1.0 / np.sqrt((di ** 2).sum() + (du ** 2).sum())
        di, du = di * sc, du * sc
        fd = (objective(prob, ui + eps * di, u0 + eps * du, "f64") -
              objective(prob, ui - eps * di, u0 - eps * du, "f64")) / (2 * eps)
        ad64 = float((g64[0] * di).sum() + (g64[1] * du).sum())
        ad32 = float((g32[0] * di).sum() + (g32[1] * du).sum())
        errs.append((abs(ad64 - fd) / abs(fd), abs(ad32 - fd) / abs(fd)))
    e = np.array(errs)
    out["central_differences"] = {"directions": len(errs), "eps": eps,
                                  "max_rel_err_f64_adjoint": float(e[:, 0].max()),
                                  "max_rel_err_f32_adjoint": float(e[:, 1].max()),
                                  "median_rel_err_f64_adjoint": float(np.median(e[:, 0]))}
    print(json.dumps(out))


def vtk_study(args, torch):
    """VTK snapshots of the bench duct (256x128x128, Legacy): rho, |u| and u,
    the three files the command-line tools write every --vtk-every steps.
    (a) the reference's own writer (src/moment_vtk_writer.cu, built into
        oracle/_ref: cudaMemcpy + ofstream) and its launch_speed, one snapshot;
    (b) the library's synchronous writers (text formatted on the GPU);
    (c) the asynchronous writer in a step loop: the loop's time with a snapshot
        every --vtk-every steps minus the same loop without, per snapshot, and
        the wait for the last file at the end;
    (d) the formatting kernels alone (CUDA events), with their algorithmic bytes
        (fields read + text written) against the measured HBM copy peak.
    The first snapshot of (b) must be byte-identical to (a)'s files."""
    import ctypes as C
    import shutil
    from myfluidsimulation_b200 import lib
    from myfluidsimulation_b200.vtk import VTK_SCALAR, VTK_SPEED, VTK_VECTOR, VtkWriter
    L = lib()
    st = torch.cuda.current_stream()
    with tempfile.TemporaryDirectory() as td:
        mask, _, _ = build_mask(td)
    s, _ = make_solver("legacy", mask, st.cuda_stream)
    s.step(50)
    torch.cuda.synchronize()
    N = NX * NY * NZ
    r, u, v, w = s.macro_ptrs()
    speed = torch.empty(N, device="cuda")
    out = {"study": "vtk", "workload": f"duct {NX}x{NY}x{NZ} Legacy after 50 steps; rho, |u| and u per snapshot"}
    root = tempfile.mkdtemp(prefix="vtk_study_")
    try:
        def files(tag):
            d = os.path.join(root, tag)
            os.makedirs(d, exist_ok=True)
            return [os.path.join(d, f"{k}.vtk").encode() for k in ("rho", "speed", "vel")]

        # the baseline leg: the reference's own writer, built from its sources
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from oracle_bind import RefCUDA
        ref_files = None
        if RefCUDA.available():
            R = C.CDLL(RefCUDA.path)
            f = files("ref")
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            R.launch_speed(C.c_void_p(u), C.c_void_p(v), C.c_void_p(w), C.c_void_p(speed.data_ptr()), C.c_int(N))
            R.write_scalar_vtk(f[0], C.c_void_p(r), NX, NY, NZ)
            R.write_scalar_vtk(f[1], C.c_void_p(speed.data_ptr()), NX, NY, NZ)
            R.write_vector_vtk(f[2], C.c_void_p(u), C.c_void_p(v), C.c_void_p(w), NX, NY, NZ)
            out["reference_writer_s_per_snapshot"] = round(time.perf_counter() - t0, 3)
            out["cpu_baseline"] = {"kind": "reference", "cores": 1,
                                   "sample": "one snapshot: src/moment_vtk_writer.cu (cudaMemcpy + ofstream <<) "
                                             "and launch_speed, built into oracle/_ref"}
            ref_files = f
        else:
            out["reference_writer_s_per_snapshot"] = None
        times = []
        for k in range(3):
            f = files(f"sync{k}")
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            L.launch_speed(u, v, w, speed.data_ptr(), N)
            assert L.lbm_write_scalar_vtk(f[0], r, NX, NY, NZ) == 0
            assert L.lbm_write_scalar_vtk(f[1], speed.data_ptr(), NX, NY, NZ) == 0
            assert L.lbm_write_vector_vtk(f[2], u, v, w, NX, NY, NZ) == 0
            times.append(time.perf_counter() - t0)
            if k == 0:
                out["text_bytes_per_snapshot"] = sum(os.path.getsize(x) for x in f)
                if ref_files:
                    out["bytes_identical_to_reference"] = all(
                        open(a, "rb").read() == open(b, "rb").read() for a, b in zip(f, ref_files))
            shutil.rmtree(os.path.dirname(f[0]))
        out["sync_gpu_writer_s_per_snapshot"] = round(statistics.median(times), 4)
        if out["reference_writer_s_per_snapshot"]:
            out["sync_speedup_vs_reference_writer"] = round(out["reference_writer_s_per_snapshot"] /
                                                            out["sync_gpu_writer_s_per_snapshot"], 1)
        # (c) asynchronous snapshots inside the step loop
        steps, every = args.vtk_steps, args.vtk_every
        s.step(10)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(steps):
            s.step(1)
        torch.cuda.synchronize()
        plain = time.perf_counter() - t0
        with VtkWriter(NX, NY, NZ, depth=3) as wr:
            nsnap = 0
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for k in range(1, steps + 1):
                s.step(1)
                if k % every == 0:
                    f = files(f"async{nsnap}")
                    rr, uu, vv, ww = s.macro_ptrs()
                    wr.submit(VTK_SCALAR, f[0].decode(), rr, stream=s.stream)
                    wr.submit(VTK_SPEED, f[1].decode(), uu, vv, ww, stream=s.stream)
                    wr.submit(VTK_VECTOR, f[2].decode(), uu, vv, ww, stream=s.stream)
                    nsnap += 1
            torch.cuda.synchronize()
            loop = time.perf_counter() - t0
            wr.flush()
            done = time.perf_counter() - t0
            written = wr.bytes_written
        out["async"] = {"steps": steps, "every": every, "snapshots": nsnap, "loop_s_without": round(plain, 4),
                        "loop_s_with": round(loop, 4),
                        "loop_overhead_ms_per_snapshot": round(1e3 * (loop - plain) / max(nsnap, 1), 2),
                        "all_files_written_s": round(done, 4), "bytes_written": written}
        # (d) the formatting kernels alone
        text = torch.empty(int(L.lbm_vtk_text_bound(VTK_VECTOR, N)), dtype=torch.uint8, device="cuda")
        peak, peak_kind = measured_peaks()
        kern = {}
        for name, kind, ptrs, nin in (("rho", VTK_SCALAR, (r, None, None), 1), ("speed", VTK_SPEED, (u, v, w), 3),
                                      ("vel", VTK_VECTOR, (u, v, w), 3)):
            ln = C.c_int64()
            ts = []
            for it in range(6):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(st)
                assert L.lbm_vtk_format(kind, *[None if p is None else C.c_void_p(p) for p in ptrs], N,
                                        text.data_ptr(), text.numel(), C.byref(ln), st.cuda_stream) == 0
                e1.record(st)
                torch.cuda.synchronize()
                if it >= 2:
                    ts.append(e0.elapsed_time(e1))
            ms = statistics.median(ts)
            gbs = (4 * nin * N + ln.value) / (ms * 1e-3) / 1e9
            kern[name] = {"ms": round(ms, 3), "text_bytes": ln.value, "gvalues_per_s": round(nin * N / ms / 1e6, 2),
                          "gb_s": round(gbs, 1), "frac_of_hbm": round(gbs / peak, 3) if peak else None}
        out["format_kernels"] = kern
        out["hbm_peak_gbs"] = {"value": peak, "source": peak_kind}
    finally:
        shutil.rmtree(root, ignore_errors=True)
        s.close()
    print(json.dumps(out))


def render_study(args, torch):
    """The viewer's volume view of the bench duct (256x128x128, Legacy after
    200 steps) at 1280x720 with the viewer's default orbit camera and uStep
    0.005 (main_compare.cpp:999), in its two displays: |u| with uScale 150
    (opaque within a few samples) and rho-1 with uScale 1000 (mostly below the
    0.15 threshold: long rays).  Frame time of the exact and texture-unit
    samplers (CUDA events, median of 20), samples per second (the sample count
    from the oracle, which marches the same rays), and the oracle itself on
    the host cores as the baseline leg (one frame)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_bind import Oracle
    from myfluidsimulation_b200 import lib
    from myfluidsimulation_b200.render import FILTER_EXACT, FILTER_TEXTURE, VolumeRenderer, orbit_camera
    st = torch.cuda.current_stream()
    with tempfile.TemporaryDirectory() as td:
        mask, _, _ = build_mask(td)
    s, _ = make_solver("legacy", mask, st.cuda_stream)
    s.step(200)
    r, u, v, w = s.macro_ptrs()
    N = NX * NY * NZ
    speed = torch.empty(N, device="cuda")
    torch.cuda.synchronize()
    lib().launch_speed(u, v, w, speed.data_ptr(), N)
    torch.cuda.synchronize()
    W_, H_ = 1280, 720
    inv, cam = orbit_camera(0.0, 0.3, 2.5, (0.5, 0.5, 0.5), W_, H_)
    pres = torch.empty(N, device="cuda")
    lib().launch_shift(r, -1.0, pres.data_ptr(), N)
    torch.cuda.synchronize()
    out = {"study": "render", "workload": f"duct {NX}x{NY}x{NZ} (Legacy, 200 steps), {W_}x{H_}, orbit yaw 0 "
                                          "pitch 0.3 radius 2.5, uStep 0.005, uThresh 0.15"}
    orc = Oracle()
    with VolumeRenderer(NX, NY, NZ) as rr:
        img = None
        for view, field, scale in (("speed", speed, 150.0), ("pressure", pres, 1000.0)):
            host = field.cpu().numpy().reshape(NZ, NY, NX)
            t0 = time.perf_counter()
            ref_img, samples = orc.raymarch(host, inv, cam, 0.005, scale, 0.15, W_, H_)
            dt = time.perf_counter() - t0
            res_v = {"uScale": scale, "samples_per_frame": samples,
                     "cpu_baseline": {"value": round(dt * 1e3, 1), "unit": "ms per frame",
                                      "cores": orc.lib.orc_num_threads(), "kind": "port",
                                      "sample": "one frame, the oracle's FP32 restatement of the shader"}}
            for name, flt in (("exact", FILTER_EXACT), ("texture", FILTER_TEXTURE)):
                ts = []
                for it in range(25):
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record(st)
                    img = rr.render(field, inv, cam, W_, H_, 0.005, scale, 0.15, flt, out=img)
                    e1.record(st)
                    torch.cuda.synchronize()
                    if it >= 5:
                        ts.append(e0.elapsed_time(e1))
                ms = statistics.median(ts)
                res = {"ms_per_frame": round(ms, 3), "fps": round(1e3 / ms, 1),
                       "gsamples_per_s": round(samples / ms / 1e6, 2)}
                got = img.cpu().numpy()
                if flt == FILTER_EXACT:
                    res["bit_identical_to_oracle"] = bool(np.array_equal(got, ref_img))
                else:
                    d = np.abs(np.clip(got[..., :3], 0, 1) - np.clip(ref_img[..., :3], 0, 1)).max(axis=2)
                    res["displayed_mean_abs_diff_vs_oracle"] = float(d.mean())
                res["speedup_vs_cpu_baseline"] = round(dt * 1e3 / ms, 1)
                res_v[name] = res
            out[view] = res_v
    s.close()
    print(json.dumps(out))


def slab_study(args, torch):
    """The bench duct (256x128x128, Legacy, FP32) split into z-slabs on this one
    GPU: the single-device image of the multi-GPU decomposition.  Per slab count:
    MLUPS over 200 steps (CUDA events) against the single grid, the bytes that
    cross the slab faces per step pair (the 5 slot planes of each face, out in
    phase 0 and back in phase 1), and the time those bytes would take over
    NVLink at the measured 770 GB/s per direction between two GPUs."""
    from myfluidsimulation_b200.slabs import SlabSet
    from myfluidsimulation_b200.solvers import BC_DUCT, METHOD_LEGACY, Solver
    with tempfile.TemporaryDirectory() as td:
        mask, _, _ = build_mask(td)
    rho = np.ones((NZ, NY, NX), np.float32)
    u = np.full((NZ, NY, NX), U_IN, np.float32)
    u[mask != 0] = 0
    st = torch.cuda.Stream()
    N = NX * NY * NZ
    steps = 200
    out = {"study": "slab", "workload": f"duct {NX}x{NY}x{NZ} Legacy FP32, {steps} steps, z-slabs on one GPU, "
                                        "every run replayed from a CUDA graph of 20 steps"}
    base = None
    for parts in (1, 2, 4, 8):
        with torch.cuda.stream(st):
            if parts == 1:
                obj = Solver(NX, NY, NZ, TAU, method=METHOD_LEGACY, bc=BC_DUCT, inlet_u=U_IN,
                             stream=st.cuda_stream)
            else:
                obj = SlabSet(NX, NY, NZ, TAU, parts, method=METHOD_LEGACY, bc=BC_DUCT, inlet_u=U_IN,
                              stream=st.cuda_stream)
            obj.set_solid_mask(mask)
            obj.reinit_from_host(rho, u, None, None)
            obj.set_macro_output(False)
            obj.step(10)
            torch.cuda.synchronize()
            if parts == 1:
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, stream=st):
                    obj.step(20)
            else:
                g = obj.graph(20)
            g.replay()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(steps // 20):
                g.replay()
            e1.record(st)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            del g
        mlups = N * steps / (ms * 1e-3) / 1e6
        face = 5 * NX * NY * 4
        r = {"mlups": round(mlups, 1), "us_per_step": round(ms * 1e3 / steps, 1)}
        if parts == 1:
            base = mlups
        else:
            # per odd step each face moves 5 slot planes each way (phase 0), and back (phase 1)
            r["face_bytes_per_step_pair"] = 4 * face
            r["nvlink_us_per_step_pair_at_770GBs"] = round(2 * face / 770e9 * 1e6 * 2, 1)
            r["vs_single_grid"] = round(mlups / base, 3)
        out[f"slabs_{parts}"] = r
        obj.close()
    print(json.dumps(out))


def profile_tgv(args, torch):
    """Set-up of the periodic Taylor-Green vortex of --profile-n^3 cells (tau 0.51,
    u0 0.05; the precision study's field), --profile-method in --profile-storage,
    macro output off, then 6 single steps: the case the narrow-storage ncu
    captures run (`-k regex:aa_odd -s 1 -c 1` takes the second odd step)."""
    from myfluidsimulation_b200.solvers import METHOD_HOME, METHOD_LEGACY, STORE_BF16, STORE_F16, STORE_F32, Solver
    n = args.profile_n
    rho, u, v, w = tgv_fields(n, torch)
    sto = {"f32": STORE_F32, "f16": STORE_F16, "bf16": STORE_BF16}[args.profile_storage]
    m = METHOD_HOME if args.profile_method == "home" else METHOD_LEGACY
    st = torch.cuda.current_stream()
    s = Solver(n, n, n, 0.51, method=m, storage=sto, stream=st.cuda_stream)
    s.reinit_from_macro(rho, u, v, w)
    s.set_macro_output(False)
    for _ in range(6):
        s.step(1)
    s.synchronize()
    s.close()
    print(json.dumps({"profile": "tgv", "n": n, "method": args.profile_method, "storage": args.profile_storage,
                      "steps": 6}))


def decomp_run(args, torch, dist, rank, world):
    """The periodic duct stretched along z to 128 x N planes and split into N
    z-slabs, one per rank (DistSlab: ghost planes, the 5 crossing slot planes of
    each face exchanged point to point through NCCL around every odd step,
    overlapped with the slab's interior planes).  Weak scaling: 128 planes per
    GPU.  One bench step = 50 LBM steps, the last one with the FP64 statistics
    all-reduced over the ranks."""
    from myfluidsimulation_b200.slabs import DistSlab
    from myfluidsimulation_b200.solvers import METHOD_LEGACY
    W = load_workloads()
    nzg = NZ * world
    with tempfile.TemporaryDirectory() as td:
        box, ntri, nsph = build_mask(td)          # one 256x128x128 box: walls + sphere
    sphere = (box != 0) & (W.duct_mask(NX, NY, NZ) == 0)
    obstacle = np.zeros((nzg, NY, NX), np.uint8)
    obstacle[:NZ][sphere] = 1
    mask = W.duct_mask(NX, NY, nzg, obstacle)
    rho = np.ones(mask.shape, np.float32)
    zero = np.zeros(mask.shape, np.float32)
    d = DistSlab(NX, NY, nzg, TAU, FORCE, method=METHOD_LEGACY, dist=dist if world > 1 else _SoloDist())
    d.set_solid_mask(mask)
    d.reinit_from_host(rho, zero, None, None)
    d.enable_stats(True)
    st = torch.cuda.current_stream()
    for _ in range(args.warmup):
        d.step(DRAG_EVERY, overlap=True)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(int(os.environ.get("LOCAL_RANK", 0))) as clk:
        e0.record(st)
        for _ in range(args.steps):
            d.step(DRAG_EVERY, overlap=True)
        e1.record(st)
        torch.cuda.synchronize()
    ms = torch.tensor([e0.elapsed_time(e1)], device="cuda")
    if dist:
        dist.barrier()
        dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    ms = float(ms.item())
    stats = d.stats()
    d.close()
    N = NX * NY * nzg
    mlups = N * DRAG_EVERY * args.steps / (ms * 1e-3) / 1e6
    per_launch = ms / (DRAG_EVERY * args.steps)
    peak, peak_kind = measured_peaks()
    achieved = NX * NY * NZ * BYTES["legacy"] / (per_launch * 1e-3) / 1e9
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": round(mlups, 1), "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"periodic duct {NX}x{NY}x{nzg} (128 planes per GPU), y/z walls as solid cells, "
                                   "icosphere r=16 at (64,64,64), x periodic, body force (1e-5,0,0), tau 0.56; "
                                   "one step = 50 LBM steps + FP64 statistics all-reduced",
                       "method": "legacy", "storage": "f32", "l2": HEAD_CONFIG["l2"],
                       "parallelism": f"zslab x{world}"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": None, "kernel": "aa_even/aa_odd per GPU",
                         "bytes_per_cell": BYTES["legacy"], "peak_kind": peak_kind},
            "exchange": {"bytes_per_face_per_odd_step": 2 * 5 * NX * NY * 4,
                         "transport": "NCCL point to point, overlapped with interior planes" if world > 1 else
                                      "self-exchange (one slab, device copies)"},
            # per step pair: the even and odd kernels (3 parts each when overlapped) and the
            # 10 merge kernels of phase 1 (one rank: the two steps and one exchange-plan launch
            # per phase); plus the statistics' final pass per bench step
            "gpu_launches": args.steps * ((DRAG_EVERY // 2) * (16 if world > 1 else 4) + 1),
            "stats": {"mass": stats["mass"], "drag": [stats["drag_x"], stats["drag_y"], stats["drag_z"]]},
            "clocks": clk.summary()}))


class _SoloDist:
    """The torch.distributed calls a one-rank DistSlab makes, without a process group."""

    def get_rank(self, group=None):
        return 0

    def get_world_size(self, group=None):
        return 1

    def get_backend(self, group=None):
        return "gloo"

    class ReduceOp:
        SUM = "sum"

    def all_reduce(self, t, op=None, group=None):
        return None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--methods", default=",".join(run_key(m, w) for m, w in RUNS),
                    help="comma list of run keys: legacy, home, hybrid (periodic workload), *_inlet (inlet duct); "
                         "the first is the headline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--decomp", default=None, choices=["zslab"],
                    help="zslab: one periodic duct of 128 x N planes split into z-slabs over the N ranks "
                         "(NCCL face exchange overlapped with the interior planes) instead of N replicas")
    ap.add_argument("--profile", default=None,
                    help="set up one run key (e.g. legacy, home_inlet) on the duct, or 'tgv' (the periodic "
                         "Taylor-Green vortex of --profile-n^3 cells, Legacy, --profile-storage), and run 4 plain LBM "
                         "steps only (for ncu captures)")
    ap.add_argument("--profile-n", type=int, default=256)
    ap.add_argument("--profile-storage", default="f32", choices=["f32", "f16", "bf16"])
    ap.add_argument("--profile-method", default="legacy", choices=["legacy", "home"])
    ap.add_argument("--study", default=None, choices=["precision", "batch", "adjoint", "vtk", "render", "slab"],
                    help="precision: 512^3 TGV MLUPS and kinetic-energy error of F32/F16/BF16 storage; "
                         "batch: 64 uneven Hybrid(B0) ducts in one persistent launch per step; "
                         "adjoint: drag gradient of the 128x64x64 duct against central differences; "
                         "vtk: snapshot cost of the GPU VTK writers against the reference's writer; "
                         "render: the viewer's volume ray-march of the duct's |u| at 1280x720; "
                         "slab: the duct split into z-slabs on one GPU (the multi-GPU decomposition)")
    ap.add_argument("--vtk-steps", type=int, default=1000)
    ap.add_argument("--vtk-every", type=int, default=200)
    ap.add_argument("--fd-directions", type=int, default=32)
    ap.add_argument("--batch-count", type=int, default=64)
    ap.add_argument("--batch-steps", type=int, default=2000)
    ap.add_argument("--tgv-n", type=int, default=512)
    ap.add_argument("--tgv-steps", type=int, default=2000)
    ap.add_argument("--tgv-every", type=int, default=100)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    if args.impl == "reference":
        reference_arm(args, torch, rank, world)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    import myfluidsimulation_b200 as P
    P.lib()
    studies = {"precision": precision_study, "batch": batch_study, "adjoint": adjoint_study, "vtk": vtk_study,
               "render": render_study, "slab": slab_study}
    if args.study:
        studies[args.study](args, torch)
        return
    if args.profile == "tgv":
        profile_tgv(args, torch)
        return
    if args.decomp == "zslab":
        decomp_run(args, torch, dist, rank, world)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    with tempfile.TemporaryDirectory() as td:
        mask, ntri, nsph = build_mask(td)
    keys = {run_key(m, w): (m, w) for m, w in RUNS}
    if args.profile:
        st = torch.cuda.current_stream()
        m, w = keys[args.profile]
        s, _ = make_solver(m, w, mask, st.cuda_stream)
        s.enable_stats(False)
        s.set_macro_output(False)      # the plain launches that make up 49 of every 50 bench steps
        for _ in range(4):
            s.step(1)
        s.synchronize()
        s.close()
        print(json.dumps({"profile": args.profile, "steps": 4}))
        return
    runs = [k for k in args.methods.split(",") if k]
    for k in runs:
        if k not in keys:
            raise SystemExit(f"unknown run key {k!r}; known: {', '.join(keys)}")
    peak, peak_kind = measured_peaks()
    N = NX * NY * NZ
    results = {}
    head = runs[0]
    clk = ClockSampler(local).__enter__()   # spans the timed regions of all runs
    for key in runs:
        mth, wl = keys[key]
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        s, r = run_method(mth, wl, mask, args, torch, dist)
        ms = torch.tensor([r["ms_total"]], device="cuda")
        if dist:
            dist.all_reduce(ms, op=dist.ReduceOp.MAX)
        ms = float(ms.item())
        cell_updates = N * DRAG_EVERY * args.steps * world
        mlups = cell_updates / (ms * 1e-3) / 1e6
        per_launch_ms = r["ms_total"] / (DRAG_EVERY * args.steps)
        achieved = N * BYTES[mth] / (per_launch_ms * 1e-3) / 1e9
        tr = profile_traffic(mth)
        ku = r["kernel_us"]
        split_ms = DRAG_EVERY * sum(ku.values()) / len(ku) / 1e3
        results[key] = {"mlups": round(mlups, 1), "ms_per_step": round(ms / args.steps, 4),
                        "workload": wl, "kernel_us": ku,
                        "kernel_split_ms_per_step": round(split_ms, 4),
                        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                                     "frac": round(achieved / peak, 4),
                                     "traffic": None if tr is None else int(round(tr * N)),
                                     "kernel": KERNEL[mth], "bytes_per_cell": BYTES[mth]},
                        "kernel_frac": {k: round(N * BYTES[mth] / (v * 1e-6) / 1e9 / peak, 4) for k, v in ku.items()},
                        "drag": [round(x, 6) for x in r["drag_last"]], "mass": round(r["mass"], 3),
                        "launches": r["launches"]}
        if mth == "hybrid":
            results[key]["band_cells"] = r["band_cells"]
        if key == head:
            head_solver = s
        else:
            s.close()

    clk.__exit__()
    clocks = clk.summary()
    # end to end through the C-ABI with host buffers (headline run)
    hm, hw = keys[head]
    e2e_ms, e2e_wall, h2d, d2h = e2e_run(hm, hw, mask, args, torch, dist)
    e2e_t = torch.tensor([e2e_ms], device="cuda")
    if dist:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_mlups = N * DRAG_EVERY * args.steps * world / (float(e2e_t.item()) * 1e-3) / 1e6

    cpu = None
    l2 = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and head == "legacy":
        def gpu_state(steps):
            st = torch.cuda.current_stream()
            g, _ = make_solver("legacy", "periodic", mask, st.cuda_stream)
            g.enable_stats(False)
            g.step(steps)
            g.synchronize()
            out = g.state()
            g.close()
            return out
        try:
            cpu, l2, l2_steps = cpu_baseline(mask, gpu_state)
        except Exception as e:  # the checker is optional on a box without it
            cpu = {"value": None, "unavailable": f"{type(e).__name__}: {e}"}
    head_solver.close()

    if rank == 0:
        h = results[head]
        config = dict(HEAD_CONFIG) if head == "legacy" else {
            "workload": WORKLOAD_TEXT[hw], "method": hm, "storage": "f32", "l2": HEAD_CONFIG["l2"]}
        if world > 1:
            config["parallelism"] = f"replicas x{world}"
        line = {
            "metric": METRIC,
            "value": h["mlups"], "unit": "MLUPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": h["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic", "config": config,
            "bounce": "halfway bounce-back, AA pattern in place",
            "roofline": dict(h["roofline"], peak_kind=peak_kind),
            "e2e": {"value": round(e2e_mlups, 1), "unit": "MLUPS", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "wall_ms": round(e2e_wall, 2)},
            "gpu_launches": sum(r["launches"] for r in results.values()),
            "methods": results,
            "clocks": clocks,
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        if l2 is not None:
            line["l2_vs_fp64"] = {"value": l2, "what": "relative L2 of the Legacy state vs the FP64 oracle "
                                                       "(periodic workload)", "steps": l2_steps}
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
