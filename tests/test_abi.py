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


def test_null_and_bad_arguments_are_rejected_without_gpu(lib):
    """Every entry point that takes a handle, batch or surface refuses a null one (and bad
    sizes or ids) with a negative code and a message, before any CUDA call; destroying null
    is a no-op, as free(NULL) is."""
    L = gvh.load()
    gvh._bind_batch(L)
    gvh._bind_surface(L)
    d = ctypes.c_double()
    u = ctypes.c_uint()
    t = ctypes.c_longlong()
    n = ctypes.c_int()
    calls = [
        ("gvh_rk2_step", (None, 0.5, 0.01, 0.0)),
        ("gvh_set_state", (None, None, 25)),
        ("gvh_get_state", (None, None, 25)),
        ("gvh_set_state_async", (None, None, 25)),
        ("gvh_get_state_async", (None, None, 25)),
        ("gvh_join_async", (None,)),
        ("gvh_status", (None, ctypes.byref(u))),
        ("gvh_clear_status", (None,)),
        ("gvh_synchronize", (None,)),
        ("gvh_max_energy_density", (None, ctypes.byref(d))),
        ("gvh_max_propagation_speed", (None, ctypes.byref(d))),
        ("gvh_set_hotspot_state", (None, None)),
        ("gvh_gather_state_device", (None, None, 25, 8)),
        ("gvh_scatter_state_device", (None, None, 25, 8)),
        ("gvh_enable_validity", (None, 1)),
        ("gvh_set_stream", (None, None)),
        ("gvh_save_state", (None, b"/nonexistent/x", 0.5, 0)),
        ("gvh_load_state", (None, b"/nonexistent/x", ctypes.byref(d), ctypes.byref(t))),
    ]
    for name, args in calls:
        rc = getattr(L, name)(*args)
        assert rc < 0, (name, rc)
        assert L.gvh_last_error(), name
    batch_calls = [
        ("gvh_batch_step", (None, 1)),
        ("gvh_batch_round", (None, 1, ctypes.byref(t))),
        ("gvh_batch_poll", (None, 0, 0, None, None, ctypes.byref(n), None)),
        ("gvh_batch_remove_event", (None, 0)),
        ("gvh_batch_synchronize", (None,)),
    ]
    for name, args in batch_calls:
        rc = getattr(L, name)(*args)
        assert rc < 0, (name, rc)
        assert L.gvh_batch_last_error(), name
    zero, one = ctypes.c_double(0.0), ctypes.c_double(1.0)
    for name, args in [("gvh_surface_find", (None, zero, one, ctypes.byref(t))),
                       ("gvh_surface_find_begin", (None, zero, one)),
                       ("gvh_surface_find_end", (None, ctypes.byref(t))),
                       ("gvh_surface_set_lower", (None,))]:
        rc = getattr(L, name)(*args)
        assert rc < 0, (name, rc)
        assert L.gvh_surface_last_error(), name
    assert L.gvh_destroy(None) == 0
