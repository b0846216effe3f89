"""Mixed-precision path (FP32 limiter, fluxes, sources and face-state recovery; FP64
state, cell-centre recovery, RK accumulation and regulation) against the FP64 oracle.

Stated tolerances (max over cells): relative error in e <= 1e-4, |delta u^mu| <= 1e-4
(u^tau >= 1, so this is relative to u^tau), |delta pi^{mu nu}| / (e + p) <= 1e-3.
"""
import numpy as np
import pytest

import gvh
import oracle
from gvh import workloads

pytestmark = pytest.mark.gpu

E_TOL = 1e-4
U_TOL = 1e-4
PI_TOL = 1e-3


def mixed_errors(G, sg, so):
    e_g, e_o = G.interior(sg["e"]), G.interior(so["e"])
    p_o = G.interior(so["p"])
    err = {"e": float(np.max(np.abs(e_g - e_o) / np.abs(e_o)))}
    err["u"] = max(float(np.max(np.abs(G.interior(sg[k]) - G.interior(so[k])))) for k in ("ut", "ux", "uy", "un"))
    if G.shear:
        wpp = np.abs(e_o + p_o)
        err["pi"] = max(float(np.max(np.abs(G.interior(sg[k]) - G.interior(so[k])) / wpp))
                        for k in G.qnames[4:14])
    return err


def run_pair(w, prim, steps):
    kw = w.lattice_kwargs()
    G = gvh.Lattice(precision="mixed", **kw)
    O = oracle.OracleLattice(**kw)
    G.set_primitive(prim)
    O.set_primitive(prim)
    t = w.tau0
    for n in range(1, steps + 1):
        G.step(t, w.dtau)
        O.step(t, w.dtau)
        t = w.tau0 + n * w.dtau
    assert G.status() == 0
    return G, G.get_state(), O.get_state()


def test_mixed_config1_100_steps():
    w = workloads.CONFIG1
    G, sg, so = run_pair(w, workloads.gaussian_profile(w), w.steps)
    err = mixed_errors(G, sg, so)
    assert err["e"] <= E_TOL and err["u"] <= U_TOL and err["pi"] <= PI_TOL, err


def test_mixed_config2_lattice_10_steps():
    w = workloads.CONFIG2
    prim = workloads.glauber_hotspots(w)
    prim.pop("_meta")
    G, sg, so = run_pair(w, prim, 10)
    err = mixed_errors(G, sg, so)
    assert err["e"] <= E_TOL and err["u"] <= U_TOL and err["pi"] <= PI_TOL, err


def test_mixed_config1_event_at_100_freezeout_and_500_steps():
    """Configuration 3 (the config-1 event in mixed precision) against the FP64 oracle at
    step 100, at freeze-out (the step after which the oracle's maximum e has been at or below
    e(T_fo = 150 MeV) for 11 checks, the reference's stop rule, HydroPlugin.cpp:396-413:
    step 297) and at step 500, within the stated tolerances. Measured on a B200: e 9.7e-8,
    6.5e-7, 7.7e-6; u 2.4e-8, 7.1e-8, 1.7e-6; pi/(e+p) 1.2e-8, 2.9e-8, 1.1e-6."""
    w = workloads.CONFIG1
    kw = w.lattice_kwargs()
    G = gvh.Lattice(precision="mixed", **kw)
    O = oracle.OracleLattice(**kw)
    prim = workloads.gaussian_profile(w)
    G.set_primitive(prim)
    O.set_primitive(prim)
    e_fo = O.energy_density(w.T_fo_GeV / 0.197326938)
    t, n, frozen, checked = w.tau0, 0, 0, []
    while True:
        so = O.get_state()
        if frozen < 11 and float(np.max(O.interior(so["e"]))) <= e_fo:
            frozen += 1
            if frozen == 11:
                checked.append(("freezeout", n))
        if n in (100, 500):
            checked.append((n, n))
        if checked and checked[-1][1] == n:
            err = mixed_errors(G, G.get_state(), so)
            assert err["e"] <= E_TOL and err["u"] <= U_TOL and err["pi"] <= PI_TOL, (checked[-1], err)
        if n == 500:
            break
        G.step(t, w.dtau)
        O.step(t, w.dtau)
        n += 1
        t = w.tau0 + n * w.dtau
    assert [c[0] for c in checked] == [100, "freezeout", 500], checked


def test_mixed_benchmark_event_at_100_and_500_steps():
    """The 131x131x61 QCD + bulk event in mixed precision against the plain FP64 path (which
    the reference's FP64 CUDA build pins to 1e-10 over these steps, test_ref_gpu.py) after
    100 and 500 steps, within the stated tolerances. Measured on a B200: e 2.5e-6 and 7.1e-5,
    u 1.0e-6 and 5.0e-5, pi/(e+p) 5.2e-7 and 2.2e-5. At this event's freeze-out (1160 steps)
    the mixed path is further off than the stated tolerance in e and u (e 1.7e-3, u 5.0e-4,
    pi/(e+p) 3.4e-4); the last check bounds that drift so that a change that makes it worse
    is noticed."""
    w = workloads.CONFIG2
    prim = workloads.glauber_hotspots(w)
    prim.pop("_meta")
    kw = w.lattice_kwargs()
    M = gvh.Lattice(precision="mixed", **kw)
    D = gvh.Lattice(precision="fp64", **kw)
    M.set_primitive(prim)
    D.set_primitive(prim)
    t, n = w.tau0, 0
    for check, (et, ut, pt) in [(100, (E_TOL, U_TOL, PI_TOL)), (500, (E_TOL, U_TOL, PI_TOL)), (1160, (1e-2, 2e-3, 2e-3))]:
        while n < check:
            n += 1
            M.step(t, w.dtau)
            D.step(t, w.dtau)
            t = w.tau0 + n * w.dtau
        assert M.status() == 0
        err = mixed_errors(M, M.get_state(), D.get_state())
        assert err["e"] <= et and err["u"] <= ut and err["pi"] <= pt, (n, err)


def test_mixed_hotspot_event_stays_finite():
    """A 2+1D hotspot event of the serving mix (61x61, 0.2 fm) that ran away to NaN when the
    mixed path recovered face states in FP32; with FP64 recovery it stays finite and close
    to the FP64 path."""
    from gvh import serve
    rng = np.random.default_rng(2024)
    arr = serve.poisson_arrivals(4.0, 180, rng)
    r = [serve.make_request(i, a, rng) for i, a in enumerate(arr[:11])][10]
    lat = r.lattice
    kw = dict(nx=lat["nx"], ny=lat["ny"], nz=lat["nz"], dx=lat["dx"], dy=lat["dy"], dz=lat["dz"], dt=lat["dt"],
              etabar=lat["etabar"], theta=2.0, conformal=False, shear=True, bulk=True)
    M = gvh.Lattice(precision="mixed", **kw)
    D = gvh.Lattice(precision="fp64", **kw)
    M.set_primitive(r.prim)
    D.set_primitive(r.prim)
    t = r.tau0
    for n in range(1, 251):
        M.step(t, lat["dt"])
        D.step(t, lat["dt"])
        t = r.tau0 + n * lat["dt"]
    assert not M.status() & gvh.GVH_STATUS_NAN
    sm, sd = M.get_state(), D.get_state()
    e_m, e_d = M.interior(sm["e"]), D.interior(sd["e"])
    assert np.isfinite(e_m).all()
    assert float(np.max(np.abs(e_m - e_d)) / np.max(e_d)) <= 1e-3
