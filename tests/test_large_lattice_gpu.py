"""Maximum sizes. A 385 x 385 x 225 lattice (33.4 M interior cells, QCD EoS, shear + bulk:
12 GB of state, the 15 conserved components alone 4 GB, so every byte offset beyond 2^32 is
taken) against the benchmark's 131 x 131 x 61 lattice, both with the same spacing and a
hotspot at the origin filled on the device.

Cell centres sit at (i - (n - 1)/2) dx on both grids (odd n), so the small grid's cell i is
the large grid's cell i + 127 (x, y) and k + 82 (eta), with bit-identical initial values. A
stage reads at most two cells away along each axis, so after two RK2 steps (four stages) a
cell more than 8 cells from the small grid's edge has seen nothing of that edge: those cells
must agree bit for bit between the two lattices (size independence of the per-cell
arithmetic, in FP64 and in mixed precision). The single centred source is even under
x -> -x, y -> -y, eta -> -eta, and the large lattice's state must stay exactly even."""
import numpy as np
import pytest

import gvh
from gvh import workloads

pytestmark = pytest.mark.gpu

SMALL = (131, 131, 61)
LARGE = (385, 385, 225)
STEPS = 2
MARGIN = 4 * STEPS  # two cells per stage, two stages per step


def lattice(shape, precision):
    nx, ny, nz = shape
    w = workloads.CONFIG2
    kw = dict(w.lattice_kwargs(), nx=nx, ny=ny, nz=nz)
    return gvh.Lattice(precision=precision, tau0=w.tau0, **kw)


def centred_hotspot():
    return workloads.Hotspots(x=np.array([0.0]), y=np.array([0.0]), w=np.array([1.0]), sigma=1.0,
                              scale=40.0 / workloads.HBARC, eta_flat=1.0, sigma_eta=0.6,
                              background=0.05 / workloads.HBARC, meta={})


def run(shape, precision, fields):
    L = lattice(shape, precision)
    L.set_hotspots(centred_hotspot())
    w = workloads.CONFIG2
    t = w.tau0
    for n in range(1, STEPS + 1):
        L.step(t, w.dtau)
        t = w.tau0 + n * w.dtau
    flags = L.status()
    s = L.get_state(fields)
    out = {k: L.interior(s[k]) for k in fields}
    L.close()
    return out, flags


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_large_lattice_matches_small_lattice_away_from_edges(precision):
    fields = ["e", "ux", "ttt", "pixy", "Pi"]
    big, flags_big = run(LARGE, precision, fields)
    small, flags_small = run(SMALL, precision, fields)
    assert not flags_big & gvh.GVH_STATUS_ERRORS and not flags_small & gvh.GVH_STATUS_ERRORS
    ox = (LARGE[0] - SMALL[0]) // 2
    oz = (LARGE[2] - SMALL[2]) // 2
    m = MARGIN
    # interior() returns [k][j][i]
    core = (slice(m, SMALL[2] - m), slice(m, SMALL[1] - m), slice(m, SMALL[0] - m))
    shifted = (slice(oz + m, oz + SMALL[2] - m), slice(ox + m, ox + SMALL[1] - m), slice(ox + m, ox + SMALL[0] - m))
    for k in fields:
        assert np.isfinite(big[k]).all(), k
        np.testing.assert_array_equal(big[k][shifted], small[k][core], err_msg=k)
    E = big["e"]
    np.testing.assert_array_equal(E, E[::-1, :, :])
    np.testing.assert_array_equal(E, E[:, ::-1, :])
    np.testing.assert_array_equal(E, E[:, :, ::-1])
    UX = big["ux"]
    np.testing.assert_array_equal(UX, -UX[:, :, ::-1])
    assert np.abs(UX).max() > 0
