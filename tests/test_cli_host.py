"""Command-line tools: build, and argument parsing against the reference's own parser.

The tools' --print-config prints the parsed settings without touching a GPU;
the reference's parse_common_args (src/apps/sim_common.hpp:115-192), compiled
from its sources into oracle/_ref/libref_cpu.so, prints the same fields for
the same argv.  Flags, aliases, defaults and clamps must agree exactly.
"""
import ctypes as C
import os
import subprocess

import pytest

from myfluidsimulation_b200 import build as B
from oracle_bind import RefCPU

ARGVS = [
    [],
    ["--nx", "64", "--ny", "32", "--nz", "16", "--tau", "0.6", "--steps", "10"],
    ["--nx", "4", "--ny", "-3", "--nz", "0", "--tau", "0.3", "--substeps", "0", "--steps", "-5"],
    ["--force", "1e-5", "2", "-3", "--force-y", "7", "--force-z", "0.25"],
    ["--stl", "a b.stl", "--voxel-scale", "0.25", "--voxel-translate", "0.25", "0.5", "0.75"],
    ["--amr", "--amr-threshold", "1.7"],
    ["--amr-factor", "3", "--amr", "--amr-refine", "0", "--amr-threshold", "-2"],
    ["--vtk-dir", "out", "--vtk-every", "25", "--vtk-interval", "-1"],
    ["--init", "gauss", "--amp", "0.01", "--sigma", "0.1", "--center", "0.1", "0.2", "0.3"],
    ["--init", "slab", "--axis", "y", "--width", "0.4", "--slab-center", "0.3"],
    ["--axis", "zz", "--axis", "q"],
    ["--hybrid-band", "5"],
    ["--hybrid-d0", "-4", "--unknown", "--nx", "12"],
    ["--nx"],                               # a flag without its value is ignored
    ["--force", "1", "2"],                  # too few values: ignored
    ["--precision", "f16", "--bounce", "reference", "--bc", "duct", "--inlet-u", "0.04", "--walls",
     "--stats-every", "10"],               # extensions: the reference ignores them
]


def tool(name):
    return os.path.join(B.BIN, name)


@pytest.fixture(scope="module")
def tools():
    B.build_lib()
    outs = B.build_apps()
    assert sorted(os.path.basename(o) for o in outs) == sorted(B.APP_NAMES)
    return outs


@pytest.fixture(scope="module")
def ref_parse():
    if not RefCPU.available():
        pytest.skip("reference build not present")
    L = C.CDLL(RefCPU.path)
    L.ref_parse_common_args.restype = C.c_int

    def parse(argv, hybrid):
        args = [b"prog"] + [a.encode() for a in argv]
        arr = (C.c_char_p * len(args))(*args)
        buf = C.create_string_buffer(8192)
        n = L.ref_parse_common_args(len(args), arr, int(hybrid), buf, 8192)
        return None if n < 0 else buf.value.decode()

    return parse


def test_tools_build_and_link(tools):
    for t in tools:
        assert os.access(t, os.X_OK)


@pytest.mark.parametrize("argv", ARGVS, ids=lambda a: " ".join(a)[:40] or "defaults")
@pytest.mark.parametrize("name,hybrid", [("fluidsim_legacy", 0), ("fluidsim_home", 0), ("fluidsim_hybrid", 1)])
def test_parse_matches_reference(tools, ref_parse, name, hybrid, argv):
    want = ref_parse(argv, hybrid)
    r = subprocess.run([tool(name), "--print-config"] + argv, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert r.stdout == want


@pytest.mark.parametrize("argv", [["--nx", "abc"], ["--tau", "x"], ["--force", "1", "2", "--tau"]])
def test_bad_numbers_fail_like_the_reference(tools, ref_parse, argv):
    # the reference's std::stoi/stof throw out of main; the tools exit non-zero too
    assert ref_parse(argv, 0) is None
    r = subprocess.run([tool("fluidsim_legacy"), "--print-config"] + argv, capture_output=True, text=True)
    assert r.returncode != 0


def test_sweep_tool_args_lines(tools):
    """fluidsim_sweep prints fluidsim_compare's [args]/[amr ] lines (src/main_compare.cpp:312-315) and,
    without --hybrid-sweep-max, exits 1 before touching a GPU (the viewer is not provided)."""
    import numpy as np
    f = lambda x: float(np.float32(x))
    argv = ["--init", "gauss", "--amp", "0.01", "--center", "0.1", "0.2", "0.3", "--axis", "y", "--width", "0.4",
            "--force", "2e-5", "--force-z", "-3e-6", "--amr", "--amr-threshold", "1.7"]
    r = subprocess.run([tool("fluidsim_sweep")] + argv, capture_output=True, text=True)
    assert r.returncode == 1
    want = ["[args] init=%s amp=%.3g sigma=%.3g center=(%.3f,%.3f,%.3f) axis=%d width=%.3f forceX=%.3g"
            % ("gauss", f(0.01), f(0.08), f(0.1), f(0.2), f(0.3), 1, f(0.4), f(2e-5)),
            "[args] force=(%.3g, %.3g, %.3g)" % (f(2e-5), 0.0, f(-3e-6)),
            "[amr ] refine=%d threshold=%.2f" % (2, 1.0)]
    assert r.stdout.split("\n")[:3] == want
    assert "--hybrid-sweep-max" in r.stderr
