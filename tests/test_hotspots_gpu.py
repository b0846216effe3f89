"""The hotspot initial state generated on the device (gvh_set_hotspot_state,
gvh_batch_add_event_hotspots) against the host generator (gvh/workloads.py hotspot_field) on
the same seeded sources: the benchmark event's lattice, a 2+1D and a 3+1D grid of the serving
mix. The device follows the host's operations one by one, each rounded on its own; the values
are rounded to float, so they agree exactly wherever the device's exp agrees with the host's
and otherwise by at most one float rounding step (relative 2^-23 of the stored value)."""
import dataclasses

import numpy as np
import pytest

import gvh
from gvh import workloads

pytestmark = pytest.mark.gpu

FLOAT_STEP = 2.0 ** -23

GRIDS = [
    workloads.CONFIG2,
    dataclasses.replace(workloads.CONFIG2, name="mix_61x61x1", nx=61, ny=61, nz=1, dx=0.2, dy=0.2, dtau=0.02, seed=7),
    dataclasses.replace(workloads.CONFIG2, name="mix_101x101x31", nx=101, ny=101, nz=31, dx=0.15, dy=0.15,
                        dtau=0.015, seed=8),
]


@pytest.mark.parametrize("w", GRIDS, ids=lambda w: w.name)
def test_device_fill_matches_host_generator(w):
    hs = workloads.hotspot_sources(w)
    e_host = workloads.hotspot_field(w, hs).reshape(-1)
    D = gvh.Lattice(**w.lattice_kwargs())
    D.set_hotspots(hs)
    H = gvh.Lattice(**w.lattice_kwargs())
    prim = workloads._primitive(w, e_host)
    H.set_primitive(prim)
    sd, sh = D.get_state(), H.get_state()
    ed, eh = D.interior(sd["e"]), H.interior(sh["e"])
    rel = np.abs(ed - eh) / eh
    differing = int(np.count_nonzero(rel))
    assert rel.max() <= FLOAT_STEP, (rel.max(), differing)
    assert differing <= ed.size // 1000, differing  # a float-rounding tie is rare
    # the rest of the state is the same function of e
    same = rel == 0
    for k in D.field_names:
        a, b = D.interior(sd[k]), H.interior(sh[k])
        assert np.array_equal(a[same], b[same]), k
    for k in ["ux", "uy", "un"] + D.qnames[4:]:
        assert not np.any(D.interior(sd[k])), k
    assert np.all(D.interior(sd["ut"]) == 1.0)


def test_batch_admission_from_sources_matches_primitive_admission():
    w = GRIDS[2]
    hs = workloads.hotspot_sources(w)
    B = gvh.Batch(1 << 30, precision="fp64")
    lat = dict(nx=w.nx, ny=w.ny, nz=w.nz, dx=w.dx, dy=w.dy, dz=w.dz, dt=w.dtau, etabar=w.etabar)
    a = B.add_event_hotspots(**lat, hs=hs, tau0=w.tau0)
    # the device's own values as primitive arrays, admitted the ordinary way
    D = gvh.Lattice(**w.lattice_kwargs())
    D.set_hotspots(hs)
    sd = D.get_state()
    b = B.add_event(**lat, prim={k: sd[k] for k in ["e", "ut", "ux", "uy", "un"]}, tau0=w.tau0)
    B.step(3)
    sa, sb = B.get_state(a), B.get_state(b)
    for k in B.field_names:
        np.testing.assert_array_equal(sa[k], sb[k])
