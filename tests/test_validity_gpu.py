"""Validity diagnostics (gvh_enable_validity / gvh_get_validity) against the reference's own
checkValidityKernel (HydrodynamicValidity.cu, compiled into the CPU build and launched where
twoStepRungeKutta launches it) and its regulation factor, after a few steps on the same state."""
import numpy as np
import pytest

import gvh
import oracle
from helpers import rich_state

pytestmark = pytest.mark.gpu

CASES = {
    "conformal_shear": (dict(nx=12, ny=11, nz=7, dx=0.3, dy=0.3, dz=0.3, dt=0.02, etabar=0.2, theta=1.8,
                             conformal=True, shear=True, bulk=False), 0.0),
    "qcd_bulk": (dict(nx=12, ny=11, nz=7, dx=0.3, dy=0.3, dz=0.3, dt=0.02, etabar=0.16, theta=2.0, conformal=False,
                      shear=True, bulk=True), 0.0),
    # T_reg above the hot region's temperature: every cell is regulated
    "qcd_bulk_regulated": (dict(nx=10, ny=9, nz=5, dx=0.3, dy=0.3, dz=0.3, dt=0.02, etabar=0.16, theta=2.0,
                                conformal=False, shear=True, bulk=True), 2.0),
    "qcd_ideal": (dict(nx=10, ny=9, nz=5, dx=0.3, dy=0.3, dz=0.3, dt=0.02, etabar=0.16, theta=2.0, conformal=False,
                       shear=False, bulk=False), 0.0),
}
REL_TOL = 1e-9


@pytest.mark.parametrize("case", sorted(CASES))
def test_validity_matches_reference(case):
    lat, T_reg_GeV = CASES[case]
    R = oracle.RefLattice(**lat)
    prim = rich_state(R, seed=21)
    R.set_primitive(prim)
    G = gvh.Lattice(**lat)
    G.set_state(R.get_state())
    G.enable_validity()
    T_reg = T_reg_GeV / 0.197326938
    t = 0.5
    for n in range(4):
        R.step(t, lat["dt"], T_reg)
        G.step(t, lat["dt"], T_reg)
        t = 0.5 + (n + 1) * lat["dt"]
    want, got = R.get_validity(), G.get_validity()
    checked = 0
    for name in G.VALIDITY_NAMES:
        a, b = G.interior(got[name]), G.interior(want[name])
        fin = np.isfinite(b)
        assert np.array_equal(np.isfinite(a), fin), name
        if not fin.any():
            continue
        scale = max(np.max(np.abs(b[fin])), 1e-300)
        err = np.max(np.abs(a[fin] - b[fin])) / scale
        assert err <= REL_TOL, (name, err)
        checked += 1
    assert checked >= (4 if not lat["shear"] else 10)
    if T_reg_GeV > 0:
        reg = G.interior(got["regulations"])
        assert np.any(reg < 1.0)  # the regulation acted, and its factor matches


def test_validity_off_by_default_and_rejected():
    lat = CASES["qcd_ideal"][0]
    G = gvh.Lattice(**lat)
    with pytest.raises(gvh.GvhError):
        G.get_validity()
