"""Known-answer physics tests of the scheme on the oracle (CPU): Bjorken flow and Gubser
flow (tests/analytic.py). The reference ships configurations for these flows but no expected
outputs; the answers here come from the equations of motion.

* Bjorken, conformal ideal, one cell (every stencil point is the cell itself, so only the
  Milne source acts): the lattice must follow the scheme's own Heun integration of
  de/dtau = -(e + p)/tau to rounding, and the analytic e0 (tau0/tau)^(4/3) to the Heun
  method's O(dtau^2) error (measured 8.7e-6 after 4000 steps).
* Bjorken, QCD EoS: against a fine RK4 integration of the same ODE; the primitive recovery's
  Newton stop test (|de| <= 1e-3 e) bounds the agreement (measured 4.2e-6).
* Gubser flow, 81x81 at 0.1 fm, tau 1 -> 1.5: L1 relative error of e 1.03e-2 and of u^x
  6.0e-3 (r < 2.5 fm; the limiter clips the ring-shaped maximum that forms near r = 1.2 fm),
  1.2e-3 at r < 0.5 fm.
"""
import numpy as np

import analytic
import oracle

HBARC = 0.197326938
E0 = 30 / HBARC


def _uniform(L, e0):
    ng = L.ng
    return dict(e=np.full(ng, e0), ut=np.ones(ng), ux=np.zeros(ng), uy=np.zeros(ng), un=np.zeros(ng))


def bjorken_run(cls, conformal, steps=4000, tau0=1.0, dtau=0.01, shape=(1, 1, 1)):
    kw = dict(nx=shape[0], ny=shape[1], nz=shape[2], dx=0.1, dy=0.1, dz=0.1, dt=dtau, etabar=0.2, theta=1.8,
              conformal=conformal, shear=False, bulk=False)
    L = cls(**kw)
    L.set_primitive(_uniform(L, E0))
    for n in range(steps):
        L.step(tau0 + n * dtau, dtau)
    return L, L.interior(L.get_state()["e"]).ravel()


def gubser_run(cls, nx, dx, dtau, tau1=1.5, tau0=1.0):
    kw = dict(nx=nx, ny=nx, nz=1, dx=dx, dy=dx, dz=0.1, dt=dtau, etabar=0.2, theta=1.8, conformal=True,
              shear=False, bulk=False)
    L = cls(**kw)
    x = (np.arange(nx + 4) - 2 - (nx - 1) / 2) * dx
    _, Y, X = np.meshgrid(np.zeros(5), x, x, indexing="ij")
    e, ut, ux, uy = analytic.gubser(tau0, X, Y)
    L.set_primitive(dict(e=e.ravel(), ut=ut.ravel(), ux=ux.ravel(), uy=uy.ravel(), un=np.zeros(e.size)))
    steps = int(round((tau1 - tau0) / dtau))
    for n in range(steps):
        L.step(tau0 + n * dtau, dtau)
    st = L.get_state()
    Xi, Yi = X[0, 2:-2, 2:-2], Y[0, 2:-2, 2:-2]
    ea, _, uxa, _ = analytic.gubser(tau0 + steps * dtau, Xi, Yi)
    r = np.sqrt(Xi ** 2 + Yi ** 2)
    eg, uxg = L.interior(st["e"])[0], L.interior(st["ux"])[0]
    m = r < 2.5
    c = r < 0.5
    return dict(l1_e=float(np.sum(np.abs(eg[m] - ea[m])) / np.sum(ea[m])),
                l1_ux=float(np.sum(np.abs(uxg[m] - uxa[m])) / np.sum(np.abs(uxa[m]))),
                centre_e=float(np.max(np.abs(eg[c] - ea[c]) / ea[c])), state=st)


def test_bjorken_conformal_on_oracle():
    _, e = bjorken_run(oracle.OracleLattice, True)
    heun = analytic.heun_bjorken(E0, 1.0, 0.01, 4000, lambda x: x / 3)
    exact = analytic.bjorken_conformal(E0, 1.0, 41.0)
    assert abs(e[0] - heun) <= 1e-13 * heun
    assert abs(e[0] - exact) <= 2e-5 * exact


def test_bjorken_qcd_on_oracle():
    L, e = bjorken_run(oracle.OracleLattice, False)
    ref = analytic.rk4_bjorken(E0, 1.0, 41.0, L.pressure, n=20000)
    assert abs(e[0] - ref) <= 1e-5 * ref


def test_gubser_flow_on_oracle():
    r = gubser_run(oracle.OracleLattice, 81, 0.1, 0.01)
    assert r["l1_e"] <= 1.5e-2 and r["l1_ux"] <= 1e-2 and r["centre_e"] <= 3e-3, r
