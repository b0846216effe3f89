"""Pins the oracle (oracle/kt_oracle.c, the CPU restatement) to the reference.

The reference ships no stored outputs for the KT step, so the pins are (a) the golden
fixtures in tests/golden, produced by the reference's own rhic/src sources compiled for
the CPU (tests/golden/make_golden.py), and (b) where that build is present (oracle/_ref),
live comparisons on further seeded cases. Both compare bit for bit.
"""
import os

import numpy as np
import pytest

import oracle
from helpers import rich_state

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
import importlib.util

_spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
make_golden = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(make_golden)

CASES = sorted(make_golden.CASES)


@pytest.fixture(scope="session", autouse=True)
def _oracle_built():
    oracle.build_oracle(verbose=False)


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_golden(case):
    lat_kw, steps, T_reg, st_kw = make_golden.CASES[case]
    g = load_golden(case)
    L, prim, s0, s1 = make_golden.run_case(oracle.OracleLattice, lat_kw, steps, T_reg, st_kw)
    for k in L.field_names:
        np.testing.assert_array_equal(L.interior(s0[k]), g["init_" + k], err_msg=f"{case} init {k}")
        np.testing.assert_array_equal(L.interior(s1[k]), g["final_" + k], err_msg=f"{case} final {k}")


def test_golden_cases_exercise_their_branches():
    """The fixtures cover the branches they are named for."""
    reg = load_golden("qcd_shear_regulated")
    lat_kw, steps, _, st_kw = make_golden.CASES["qcd_shear_regulated"]
    L, _, _, s1 = make_golden.run_case(oracle.OracleLattice, lat_kw, steps, 0.0, st_kw)
    # regulation shrinks pi: the unregulated run has larger |pi|
    assert np.abs(reg["final_pixx"]).max() < 0.9 * np.abs(L.interior(s1["pixx"])).max()
    dil = load_golden("qcd_bulk_dilute_2d")
    assert (dil["init_e"] <= 0.1).any(), "dilute case must reach the e <= 0.1 branch"
    assert (dil["init_e"] > 0.1).any()


@pytest.mark.parametrize("conformal", [True, False])
def test_oracle_scalars_match_golden(conformal):
    g = load_golden("scalars")
    tag = "conf" if conformal else "qcd"
    L = oracle.OracleLattice(nx=1, ny=1, nz=1, dx=0.1, dy=0.1, dz=0.1, dt=0.01, etabar=0.2, theta=2.0,
                             conformal=conformal, shear=True, bulk=True)
    np.testing.assert_array_equal([L.pressure(x) for x in g[f"{tag}_e"]], g[f"{tag}_p"])
    np.testing.assert_array_equal([L.temperature(x) for x in g[f"{tag}_e"]], g[f"{tag}_T"])
    np.testing.assert_array_equal([L.energy_density(x) for x in g[f"{tag}_Tgrid"]], g[f"{tag}_eofT"])
    out = np.array([L.inferred(0.6, q, ep) for q, ep in zip(g[f"{tag}_inf_q"], g[f"{tag}_inf_eprev"])])
    np.testing.assert_array_equal(out, g[f"{tag}_inf_out"])


needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference CPU build (oracle/_ref) not built")


@needs_ref
@pytest.mark.parametrize("conformal", [True, False])
@pytest.mark.parametrize("phys", ["ideal", "shear", "bulk"])
def test_oracle_matches_reference_build_live(conformal, phys):
    kw = dict(nx=10, ny=7, nz=8, dx=0.25, dy=0.3, dz=0.2, dt=0.015, etabar=0.12, theta=1.6, conformal=conformal,
              shear=phys != "ideal", bulk=phys == "bulk")
    A = oracle.OracleLattice(**kw)
    B = oracle.RefLattice(**kw)
    prim = rich_state(A, seed=11, vel=0.2)
    A.set_primitive(prim)
    B.set_primitive(prim)
    t = 0.6
    for n in range(1, 7):
        A.step(t, kw["dt"], 0.0)
        B.step(t, kw["dt"], 0.0)
        t = 0.6 + n * kw["dt"]
    sa, sb = A.get_state(), B.get_state()
    for k in A.field_names:
        np.testing.assert_array_equal(A.interior(sa[k]), A.interior(sb[k]), err_msg=k)


@pytest.mark.parametrize("variant", ["fp64_conf_ideal_cart", "fp64_conf_shear_cart", "fp64_qcd_bulk_cart"])
@pytest.mark.skipif(not oracle.ref_available("fp64_conf_ideal_cart"), reason="Cartesian reference builds not built")
def test_oracle_cartesian_matches_reference_build_live(variant):
    """The reference compiled with USE_CARTESIAN_COORDINATES defined (SourceTerms.cu:738-743)
    against the oracle's Cartesian switch, bit for bit."""
    _, eos, phys, _ = variant.split("_")
    kw = dict(nx=9, ny=6, nz=5, dx=0.25, dy=0.3, dz=0.2, dt=0.015, etabar=0.12, theta=1.6, conformal=eos == "conf",
              shear=phys != "ideal", bulk=phys == "bulk", cartesian=True)
    A = oracle.OracleLattice(**kw)
    B = oracle.RefLattice(**kw)
    assert B.variant == variant
    prim = rich_state(A, seed=12, vel=0.2)
    A.set_primitive(prim)
    B.set_primitive(prim)
    t = 0.6
    for n in range(1, 6):
        A.step(t, kw["dt"], 0.0)
        B.step(t, kw["dt"], 0.0)
        t = 0.6 + n * kw["dt"]
    sa, sb = A.get_state(), B.get_state()
    for k in A.field_names:
        np.testing.assert_array_equal(A.interior(sa[k]), A.interior(sb[k]), err_msg=k)
