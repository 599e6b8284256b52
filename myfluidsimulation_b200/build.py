"""Build recipe of liblbm_b200.so (hand-written CUDA for sm_100a, in-tree).

``python -m myfluidsimulation_b200.build`` compiles every source under csrc/
with nvcc for ``sm_100a`` (``-gencode arch=compute_100a,code=sm_100a``) in
parallel and links the shared library next to this file, plus the C++
command-line tools under apps/ (fluidsim_legacy/home/hybrid/tgv/sweep) into bin/.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
APPS = os.path.join(PKG, "apps")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "liblbm_b200.so")
BIN = os.path.join(PKG, "bin")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
           "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include")]

SOURCES = ["lbm_aa.cu", "lbm_push.cu", "lbm_home.cu", "lbm_aux.cu", "lbm_geom.cu", "lbm_capi.cu", "lbm_static.cu", "lbm_adjoint.cu", "lbm_vtk.cu", "lbm_render.cu", "lbm_io.cpp"]
HEADERS = ["lbm_common.cuh", "lbm_internal.h"]
APP_NAMES = ["fluidsim_legacy", "fluidsim_home", "fluidsim_hybrid", "fluidsim_tgv", "fluidsim_sweep"]


def nvcc() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return p


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d))


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r


def build_lib(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "lbm_capi.h")]
    objs, jobs = [], []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or not _newer(o, [s] + hdrs):
            jobs.append([nvcc(), *NVFLAGS, *ARCH, "-c", s, "-o", o])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            list(ex.map(lambda c: _run(c, verbose), jobs))
    if force or jobs or not _newer(LIB, objs):
        _run([nvcc(), "-shared", *ARCH, "-Xlinker", "-Bsymbolic", "-o", LIB + ".tmp", *objs, "-lcudart"], verbose)
        os.replace(LIB + ".tmp", LIB)
    return LIB


def build_apps(force: bool = False, verbose: bool = False):
    os.makedirs(BIN, exist_ok=True)
    common = os.path.join(APPS, "sim_host.hpp")
    outs = []
    jobs = []
    for name in APP_NAMES:
        src = os.path.join(APPS, name + ".cpp")
        if not os.path.exists(src):
            continue
        out = os.path.join(BIN, name)
        outs.append(out)
        deps = [src, common, LIB, os.path.join(ROOT, "include", "lbm_capi.h"),
                os.path.join(ROOT, "include", "lbm3d_compat.hpp")]
        if force or not _newer(out, deps):
            jobs.append(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I", APPS,
                         "-I", "/usr/local/cuda/include", src, "-o", out, "-L", PKG, "-llbm_b200",
                         f"-Wl,-rpath,$ORIGIN/..", "-L/usr/local/cuda/lib64", "-lcudart"])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(len(jobs), 4)) as ex:
            list(ex.map(lambda c: _run(c, verbose), jobs))
    return outs


def build(force: bool = False, verbose: bool = False) -> str:
    lib = build_lib(force, verbose)
    build_apps(force, verbose)
    return lib


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build(force=force, verbose="-v" in sys.argv))
