"""Fixture for the surface finder: the reference's own cornelius examples.

The reference ships freezeout/cornelius-c++-1.3/example_cornelius.cpp together with its
output files output_2d.dat, output_3d.dat and output_4d.dat: 10000 cubes each of 2, 3 and 4
dimensions with corner values rand()/RAND_MAX (glibc rand, default seed, drawn in the order
example_2d, example_3d, example_4d), unit edges, iso-value 0.5, one line per surface element
(centroid then normal, ostream default format). This script keeps the first CUBES cubes of
each dimension: their rand() draws and the lines the reference wrote for them. The number of
lines per cube comes from the reference's own cornelius (oracle/_ref/libref_cornelius.so).

Run in a container that has the reference tree and the built oracle:
    python tests/golden/make_cornelius_golden.py
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle.build_ref import REF_ROOT as REF  # noqa: E402

CUBES = 2500
RAND_MAX = 2147483647


def main():
    libc = ctypes.CDLL("libc.so.6")
    libc.srand(1)
    ref = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_cornelius.so"))
    dp = ctypes.POINTER(ctypes.c_double)
    ref.gvh_refc_find.argtypes = [ctypes.c_int, dp, dp, ctypes.c_double, dp, dp, ctypes.c_int]
    out = {}
    for dim in (2, 3, 4):
        draws = np.array([libc.rand() for _ in range(10000 * 2 ** dim)], dtype=np.uint32).reshape(10000, 2 ** dim)
        lines = open(os.path.join(REF, "freezeout", "cornelius-c++-1.3", f"output_{dim}d.dat")).read().splitlines()
        nlines = 0
        c = np.zeros(10 * dim)
        n = np.zeros(10 * dim)
        for i in range(CUBES):
            v = draws[i] / float(RAND_MAX)
            nlines += ref.gvh_refc_find(dim, v.ctypes.data_as(dp), np.ones(dim).ctypes.data_as(dp), 0.5,
                                        c.ctypes.data_as(dp), n.ctypes.data_as(dp), 10)
        out[f"draws_{dim}d"] = draws[:CUBES]
        out[f"lines_{dim}d"] = np.array(lines[:nlines])
    np.savez_compressed(os.path.join(HERE, "cornelius_examples.npz"), **out)
    print("wrote", os.path.join(HERE, "cornelius_examples.npz"))


if __name__ == "__main__":
    sys.exit(main())
