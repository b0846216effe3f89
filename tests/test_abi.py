"""The C-ABI library loads and exports every entry point include/gvh.h declares (no GPU
needed: only argument checks that fail before any CUDA call are exercised)."""
import ctypes
import os
import re

import pytest

import gvh
from gvh import build as gbuild

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in sorted(os.listdir(os.path.join(ROOT, "include")))
           if f.endswith(".h")]


@pytest.fixture(scope="module")
def lib():
    if gbuild.needs_rebuild():
        gbuild.build(verbose=False)
    return ctypes.CDLL(gbuild.LIB)


def declared_functions(path):
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    names = re.findall(r"\b(gvh_[A-Za-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions(os.path.join(ROOT, "include", "gvh.h"))
    for must in ("gvh_create", "gvh_rk2_step", "gvh_set_state", "gvh_get_state", "gvh_destroy", "gvh_status"):
        assert must in names


@pytest.mark.parametrize("header", HEADERS, ids=os.path.basename)
def test_every_declared_symbol_is_exported(lib, header):
    missing = [n for n in declared_functions(header) if not hasattr(lib, n)]
    assert not missing, f"{os.path.basename(header)}: not exported by libgvh.so: {missing}"


def test_python_binding_covers_exports(lib):
    declared = set(declared_functions(os.path.join(ROOT, "include", "gvh.h")))
    assert set(gvh.EXPORTS) <= declared


def test_create_rejects_bad_lattice_without_gpu(lib):
    L = gvh.load()
    lat = gvh.LatticeParams(0, 5, 5, 4, 9, 9, 0, 0.1, 0.1, 0.1, 0.01)
    hyd = gvh.HydroParams(0.5, 0.2, 0.15, 0, 0.0)
    h = ctypes.c_void_p()
    rc = L.gvh_create(ctypes.byref(lat), ctypes.byref(hyd), None, ctypes.byref(h))
    assert rc == -1 and not h.value
    assert b"lattice" in L.gvh_last_error()
    o = gvh.Options()
    L.gvh_default_options(ctypes.byref(o))
    assert (o.eos, o.shear, o.bulk, o.precision, o.theta) == (gvh.GVH_EOS_QCD, 1, 1, gvh.GVH_PRECISION_FP64, 2.0)
    lat = gvh.LatticeParams(5, 5, 5, 9, 9, 9, 0, 0.1, 0.1, 0.1, 0.01)
    o.shear, o.bulk = 0, 1
    assert L.gvh_create(ctypes.byref(lat), ctypes.byref(hyd), ctypes.byref(o), ctypes.byref(h)) == -1
    assert b"bulk" in L.gvh_last_error()
    # the limiter's closed form takes theta > 0 (minmod of theta-scaled differences)
    o.shear, o.bulk = 1, 1
    for bad in (0.0, -1.8, float("nan")):
        o.theta = bad
        assert L.gvh_create(ctypes.byref(lat), ctypes.byref(hyd), ctypes.byref(o), ctypes.byref(h)) == -1
        assert b"theta" in L.gvh_last_error()
