"""The bounds-checked build (gpu-vh_b200/libgvh_bounds.so, GVH_BOUNDS_CHECK): on a lattice
every cell's stencil indices lie inside its arrays, so no GVH_STATUS_BOUNDS bit is raised and
the values are those of the plain build (run in a child process, which loads the other
library through GVH_LIBRARY)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from gvh import build as gbuild

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

CHILD = r"""
import json, sys
import numpy as np
sys.path[:0] = [sys.argv[1], sys.argv[1] + "/gpu-vh_b200", sys.argv[1] + "/tests"]
import gvh
from helpers import rich_state
out = {}
for name, kw in [("qcd", dict(conformal=False, shear=True, bulk=True, theta=2.0)),
                 ("line", dict(conformal=True, shear=True, bulk=False, theta=1.8))]:
    shape = dict(nx=11, ny=9, nz=6) if name == "qcd" else dict(nx=1, ny=1, nz=12)
    L = gvh.Lattice(dx=0.3, dy=0.3, dz=0.3, dt=0.01, etabar=0.16, **shape, **kw)
    L.set_primitive(rich_state(L, seed=4))
    for n in range(3):
        L.step(0.5 + 0.01 * n, 0.01)
    st = L.get_state()
    out[name] = {"status": L.status(), "e": L.interior(st["e"]).ravel().tolist(),
                 "pixy": L.interior(st["pixy"]).ravel().tolist()}
print(json.dumps(out))
"""


def _run(lib):
    env = dict(os.environ, GVH_LIBRARY=lib)
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_bounds_checked_build_raises_nothing_and_matches():
    if not os.path.exists(gbuild.BOUNDS_LIB):
        pytest.skip("libgvh_bounds.so not built (__graft_entry__.build builds it)")
    checked, plain = _run(gbuild.BOUNDS_LIB), _run(gbuild.LIB)
    for name in checked:
        assert checked[name]["status"] == 0, (name, checked[name]["status"])
        for k in ("e", "pixy"):
            assert np.array_equal(np.array(checked[name][k]), np.array(plain[name][k])), (name, k)
