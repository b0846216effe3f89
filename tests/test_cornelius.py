"""The library's surface-element finder (gvh_cornelius) against the reference's cornelius.

1. The reference's own examples (freezeout/cornelius-c++-1.3/output_{2,3,4}d.dat, kept for
   the first 2500 cubes of each dimension in tests/golden/cornelius_examples.npz): the
   elements, written with the reference's ostream format, are the same text.
2. The reference's cornelius compiled from its tree (oracle/_ref/libref_cornelius.so):
   identical bits on random, ambiguous and degenerate cubes (corners exactly on the
   iso-value, unequal edges), and an error exactly where the reference exits.
"""
import ctypes
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import gvh

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "cornelius_examples.npz")
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libref_cornelius.so")
RAND_MAX = 2147483647
dp = ctypes.POINTER(ctypes.c_double)


def lib():
    L = gvh.load()
    L.gvh_cornelius.argtypes = [ctypes.c_int, dp, dp, ctypes.c_double, dp, dp, ctypes.c_int,
                                ctypes.POINTER(ctypes.c_int)]
    return L


def ours(L, dim, v, dx, iso):
    v = np.ascontiguousarray(v, dtype=np.float64)
    dx = np.ascontiguousarray(dx, dtype=np.float64)
    c = np.zeros(10 * dim)
    n = np.zeros(10 * dim)
    k = ctypes.c_int()
    rc = L.gvh_cornelius(dim, v.ctypes.data_as(dp), dx.ctypes.data_as(dp), iso, c.ctypes.data_as(dp),
                         n.ctypes.data_as(dp), 10, ctypes.byref(k))
    return rc, c[:k.value * dim].reshape(-1, dim), n[:k.value * dim].reshape(-1, dim)


@pytest.mark.parametrize("dim", [2, 3, 4])
def test_reference_examples_same_text(dim):
    L = lib()
    g = np.load(GOLDEN)
    draws, expect = g[f"draws_{dim}d"], [str(s) for s in g[f"lines_{dim}d"]]
    lines = []
    for d in draws:
        rc, c, n = ours(L, dim, d / float(RAND_MAX), np.ones(dim), 0.5)
        assert rc == 0
        for i in range(len(c)):
            lines.append(" ".join("%g" % x for x in list(c[i]) + list(n[i])) + " ")
    assert len(lines) == len(expect)
    assert lines == expect


def cube_cases(rng, dim, count):
    for t in range(count):
        kind = t % 4
        if kind == 0:
            v = rng.random(2 ** dim)
        elif kind == 1:
            v = rng.choice([0.25, 0.5, 0.75, 0.5], 2 ** dim)  # corners on the iso-value
        elif kind == 2:
            v = rng.choice([0.1, 0.9], 2 ** dim) + rng.normal(0, 0.05, 2 ** dim)  # saddles, ambiguous faces
        else:
            v = 0.5 + rng.normal(0, 1e-3, 2 ** dim)
        yield v, rng.choice([1.0, 0.1, 0.01, 0.3], dim)


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference cornelius not built (oracle/_ref)")
@pytest.mark.parametrize("dim", [2, 3, 4])
def test_bit_identical_to_reference_build(dim):
    L = lib()
    R = ctypes.CDLL(REF_LIB)
    R.gvh_refc_find.argtypes = [ctypes.c_int, dp, dp, ctypes.c_double, dp, dp, ctypes.c_int]
    rng = np.random.default_rng(100 + dim)
    checked = elements = 0
    for v, dx in cube_cases(rng, dim, 6000):
        rc, c, n = ours(L, dim, v, dx, 0.5)
        if rc != 0:
            continue  # the reference exits on these (checked in test_error_where_reference_exits)
        rc_ = np.zeros(10 * dim)
        rn = np.zeros(10 * dim)
        k = R.gvh_refc_find(dim, v.ctypes.data_as(dp), dx.ctypes.data_as(dp), 0.5, rc_.ctypes.data_as(dp),
                            rn.ctypes.data_as(dp), 10)
        assert k == len(c), (v, dx)
        assert np.array_equal(c, rc_[:k * dim].reshape(-1, dim)), (v, dx)
        assert np.array_equal(n, rn[:k * dim].reshape(-1, dim)), (v, dx)
        checked += 1
        elements += k
    assert checked > 5000 and elements > 4000


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference cornelius not built (oracle/_ref)")
@pytest.mark.parametrize("dim,v,dx", [
    (3, [0.25, 0.5, 0.5, 0.25, 0.75, 0.25, 0.5, 0.25], [0.01, 0.01, 0.1]),
    (4, [0.75, 0.5, 0.25, 0.25, 0.5, 0.25, 0.25, 0.5, 0.5, 0.75, 0.25, 0.25, 0.5, 0.75, 0.25, 0.25], [0.01] * 4),
])
def test_error_where_reference_exits(dim, v, dx):
    """Segments shorter than the end-point tolerance: the reference prints an error and
    calls exit(1) (cornelius.cpp:1552); the library returns GVH_ERR_NUMERIC instead."""
    L = lib()
    rc, _, _ = ours(L, dim, np.array(v), np.array(dx), 0.5)
    assert rc == gvh.GVH_ERR_NUMERIC
    # the reference in a separate process: its exit must not end the test process
    child = ("import ctypes, json, sys\n"
             "import numpy as np\n"
             "dp = ctypes.POINTER(ctypes.c_double)\n"
             "R = ctypes.CDLL(sys.argv[1])\n"
             "R.gvh_refc_find.argtypes = [ctypes.c_int, dp, dp, ctypes.c_double, dp, dp, ctypes.c_int]\n"
             "va, da, buf = np.array(json.loads(sys.argv[2])), np.array(json.loads(sys.argv[3])), np.zeros(40)\n"
             "R.gvh_refc_find(int(sys.argv[4]), va.ctypes.data_as(dp), da.ctypes.data_as(dp), 0.5,\n"
             "                buf.ctypes.data_as(dp), buf.ctypes.data_as(dp), 10)\n")
    r = subprocess.run([sys.executable, "-c", child, REF_LIB, json.dumps(list(v)), json.dumps(list(dx)), str(dim)],
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL, timeout=60)
    assert r.returncode == 1


def test_normals_point_to_lower_values_and_close():
    """A linear field crossing the 4-cube: one element whose normal is the gradient's
    direction reversed, with the cut's 3-volume; its centroid lies on the surface."""
    L = lib()
    dx = np.array([0.02, 0.1, 0.1, 0.1])
    grad = np.array([-3.0, 1.0, 2.0, -0.5])
    corners = np.zeros((2, 2, 2, 2))
    for idx in np.ndindex(2, 2, 2, 2):
        corners[idx] = 1.0 + np.dot(grad, np.array(idx) * dx)
    iso = float(np.mean(corners))
    rc, c, n = ours(L, 4, corners.reshape(-1), dx, iso)
    assert rc == 0 and len(c) == 1
    assert np.dot(n[0], grad) < 0
    cos = np.dot(n[0], -grad) / np.linalg.norm(n[0]) / np.linalg.norm(grad)
    assert cos > 1 - 1e-12
    assert abs(1.0 + np.dot(grad, c[0]) - iso) < 1e-12


def test_bad_arguments():
    L = lib()
    k = ctypes.c_int()
    v = np.zeros(16)
    assert L.gvh_cornelius(5, v.ctypes.data_as(dp), v.ctypes.data_as(dp), 0.5, None, None, 0,
                           ctypes.byref(k)) == gvh.GVH_ERR_INVALID
    v[0] = 1.0  # one element, but no room for it
    assert L.gvh_cornelius(4, v.ctypes.data_as(dp), np.ones(4).ctypes.data_as(dp), 0.5, None, None, 0,
                           ctypes.byref(k)) == gvh.GVH_ERR_INVALID
    assert k.value == 1
