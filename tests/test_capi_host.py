"""The C-ABI library on the CPU: it loads, exports every declared symbol, and its
host-only paths (argument checks, STL loader) behave like the reference's.
No CUDA compute is called here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from myfluidsimulation_b200 import _lib
from myfluidsimulation_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(inc, fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([a-z_][a-z0-9_]*)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    names.discard("if")
    return sorted(names)


def test_library_exports_every_declared_symbol():
    L = C.CDLL(_lib.LIB_PATH if os.path.exists(_lib.LIB_PATH) else _lib.lib()._name)
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # and the Python binding covers them all
    assert set(names) <= set(_lib.EXPORTED)


def test_create_rejects_bad_arguments_without_touching_the_gpu():
    L = _lib.lib()
    h = C.c_void_p()
    d = _lib.Domain(0, 8, 8, 0.6, 0, 0, 0)
    assert L.lbm_create(C.byref(d), None, C.byref(h)) == 1
    assert b"dimensions" in L.lbm_last_error()
    d = _lib.Domain(8, 8, 8, 0.5, 0, 0, 0)
    assert L.lbm_create(C.byref(d), None, C.byref(h)) == 1
    d = _lib.Domain(8, 8, 8, 0.6, 0, 0, 0)
    o = _lib.Options(7, 0, 0, 0, 0.0, 1.0, None)
    assert L.lbm_create(C.byref(d), C.byref(o), C.byref(h)) == 1
    o = _lib.Options(0, 0, 1, 0, 0.0, 1.0, None)
    d = _lib.Domain(2, 8, 8, 0.6, 0, 0, 0)
    assert L.lbm_create(C.byref(d), C.byref(o), C.byref(h)) == 1          # duct needs nx >= 3
    d = _lib.Domain(1 << 20, 1 << 20, 1 << 10, 0.6, 0, 0, 0)
    assert L.lbm_create(C.byref(d), None, C.byref(h)) == 4                # LBM_ERR_SIZE
    assert L.lbm_create(None, None, C.byref(h)) == 1
    assert L.lbm_step(None, 1) == 1
    assert L.lbm_destroy(None) == 0


def test_library_stl_loader_matches_oracle(oracle, tmp_path):
    from myfluidsimulation_b200 import geometry as G
    t = W.duct_sphere_mesh(64, 32, 32, 6, (20, 16, 16), levels=2)[0]
    for fn in (W.write_binary_stl, W.write_ascii_stl):
        p = str(tmp_path / "m.stl")
        fn(p, t)
        m = G.load_stl(p)
        tt, bb = oracle.load_stl(p)
        np.testing.assert_array_equal(m.tris, tt)
        np.testing.assert_array_equal(np.concatenate([m.bbmin, m.bbmax]), bb)


def test_library_stl_loader_errors(tmp_path):
    from myfluidsimulation_b200 import geometry as G
    with pytest.raises(_lib.LBMError) as e:
        G.load_stl(str(tmp_path / "nope.stl"))
    assert e.value.code == 5
    p = str(tmp_path / "t.stl")
    W.write_binary_stl(p, W.icosphere(1))
    raw = open(p, "rb").read()
    open(p, "wb").write(raw[:200])
    with pytest.raises(_lib.LBMError):
        G.load_stl(p)
    open(p, "wb").write(raw[:80] + b"\0\0\0\0")       # zero triangles: loads, empty (as the reference)
    assert G.load_stl(p).tris.shape == (0, 3, 3)
