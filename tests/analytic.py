"""Analytic and semi-analytic solutions of relativistic hydrodynamics that the KT step must
reproduce (derived from the equations of motion, independent of the reference's code):

* Bjorken flow: a longitudinally boost-invariant, transversely uniform ideal fluid at rest in
  Milne coordinates obeys de/dtau = -(e + p(e)) / tau; for p = e/3, e = e0 (tau0/tau)^(4/3).
* Gubser flow (S. S. Gubser, Phys. Rev. D 82, 085027 (2010)): the boost-invariant,
  azimuthally symmetric ideal conformal flow with
      e(tau, r) = e_hat (2q)^(8/3) / (tau^(4/3) [1 + 2 q^2 (tau^2 + r^2) + q^4 (tau^2 - r^2)^2]^(4/3)),
      u^r / u^tau = 2 q^2 tau r / (1 + q^2 tau^2 + q^2 r^2).
"""
import numpy as np

HBARC = 0.197326938


def bjorken_conformal(e0, tau0, tau):
    return e0 * (tau0 / tau) ** (4.0 / 3.0)


def heun_bjorken(e0, tau0, dtau, steps, pressure):
    """The Bjorken ODE de/dtau = -(e + p(e))/tau integrated with the scheme's own time
    stepping (Heun: a predictor over dtau, a corrector from the predicted state, their
    mean), so that a uniform lattice must reproduce it to rounding."""
    e = e0
    t = tau0
    for n in range(steps):
        s1 = -(e + pressure(e)) / t
        e1 = e + dtau * s1
        t1 = t + dtau
        s2 = -(e1 + pressure(e1)) / t1
        e2 = e1 + dtau * s2
        e = (e + e2) / 2
        t = tau0 + (n + 1) * dtau
    return e


def rk4_bjorken(e0, tau0, tau1, pressure, n=200000):
    """A fine fourth-order integration of the same ODE (the exact solution to ~1e-12)."""
    h = (tau1 - tau0) / n
    e, t = e0, tau0
    f = lambda t_, e_: -(e_ + pressure(e_)) / t_
    for _ in range(n):
        k1 = f(t, e)
        k2 = f(t + h / 2, e + h / 2 * k1)
        k3 = f(t + h / 2, e + h / 2 * k2)
        k4 = f(t + h, e + h * k3)
        e += h / 6 * (k1 + 2 * k2 + 2 * k3 + k4)
        t += h
    return e


def gubser(tau, x, y, q=1.0, e_hat=30.0):
    """e, u^tau, u^x, u^y of ideal conformal Gubser flow at (tau, x, y)."""
    r2 = x * x + y * y
    r = np.sqrt(r2)
    e = e_hat * (2 * q) ** (8.0 / 3.0) / (tau ** (4.0 / 3.0) *
                                          (1 + 2 * q * q * (tau * tau + r2) + q ** 4 * (tau * tau - r2) ** 2)
                                          ** (4.0 / 3.0))
    v = 2 * q * q * tau * r / (1 + q * q * tau * tau + q * q * r2)
    ut = 1.0 / np.sqrt(1 - v * v)
    ur = ut * v
    with np.errstate(invalid="ignore", divide="ignore"):
        ux = np.where(r > 0, ur * x / np.where(r > 0, r, 1), 0.0)
        uy = np.where(r > 0, ur * y / np.where(r > 0, r, 1), 0.0)
    return e, ut, ux, uy
