"""Analytic and semi-analytic solutions of relativistic hydrodynamics that the KT step must
reproduce (derived from the equations of motion, independent of the reference's code):

* Bjorken flow: a longitudinally boost-invariant, transversely uniform ideal fluid at rest in
  Milne coordinates obeys de/dtau = -(e + p(e)) / tau; for p = e/3, e = e0 (tau0/tau)^(4/3).
* Gubser flow (S. S. Gubser, Phys. Rev. D 82, 085027 (2010)): the boost-invariant,
  azimuthally symmetric ideal conformal flow with
      e(tau, r) = e_hat (2q)^(8/3) / (tau^(4/3) [1 + 2 q^2 (tau^2 + r^2) + q^4 (tau^2 - r^2)^2]^(4/3)),
      u^r / u^tau = 2 q^2 tau r / (1 + q^2 tau^2 + q^2 r^2).
* The relativistic shock tube (Riemann problem) of a p = e/3 fluid in Cartesian coordinates,
  both sides at rest, e_L > e_R: a rarefaction moving left and a shock moving right around
  a uniform middle state (no contact wave: the fluid carries no conserved charge). Across
  the rarefaction the Riemann invariant y + c/(1 + c^2) ln e is constant (y the rapidity,
  c^2 = 1/3), and the fan is self-similar in xi = x/t with xi = (v - c)/(1 - v c). Across the
  shock, continuity of T^{tx} and T^{xx} in its rest frame gives the flow behind it,
  v^2 = (p - p_R)(e - e_R) / ((e_R + p)(e + p_R)), and its speed V = [T^{tx}] / [T^{tt}].
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


SOD_C = 1.0 / np.sqrt(3.0)           # sound speed of p = e/3
SOD_K = SOD_C / (1.0 + SOD_C ** 2)   # c / (1 + c^2) = sqrt(3)/4


def sod_shock_velocity(e, e_R):
    """Flow velocity behind a shock that runs into matter at rest with energy density e_R,
    when the matter behind it has e (p = e/3)."""
    p, p_R = e / 3.0, e_R / 3.0
    return np.sqrt((p - p_R) * (e - e_R) / ((e_R + p) * (e + p_R)))


def sod_rarefaction_velocity(e, e_L):
    """Flow velocity where a left-moving rarefaction from matter at rest at e_L has brought
    the energy density down to e."""
    return np.tanh(SOD_K * np.log(e_L / e))


def sod_middle_state(e_L, e_R):
    """(e*, v*, shock speed V) of the p = e/3 shock tube: e* where the rarefaction's and the
    shock's velocities meet (bisection to machine precision)."""
    lo, hi = e_R, e_L
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if sod_rarefaction_velocity(mid, e_L) > sod_shock_velocity(mid, e_R):
            lo = mid
        else:
            hi = mid
    e_s = 0.5 * (lo + hi)
    v_s = sod_shock_velocity(e_s, e_R)
    p_s = e_s / 3.0
    g2 = 1.0 / (1.0 - v_s * v_s)
    T_tt = (e_s + p_s) * g2 - p_s
    T_tx = (e_s + p_s) * g2 * v_s
    return e_s, v_s, T_tx / (T_tt - e_R)


def sod_conformal(x, t, e_L, e_R, x0=0.0):
    """e and v of the p = e/3 shock tube at time t after the discontinuity at x0 opened."""
    xi = (np.asarray(x, dtype=np.float64) - x0) / t
    e_s, v_s, V = sod_middle_state(e_L, e_R)
    c = SOD_C
    xi_tail = (v_s - c) / (1.0 - v_s * c)
    e = np.where(xi < -c, e_L, np.where(xi < xi_tail, 0.0, np.where(xi < V, e_s, e_R)))
    v = np.where(xi < -c, 0.0, np.where(xi < xi_tail, 0.0, np.where(xi < V, v_s, 0.0)))
    fan = (xi >= -c) & (xi < xi_tail)
    vf = (xi[fan] + c) / (1.0 + xi[fan] * c)
    e[fan] = e_L * np.exp(-np.arctanh(vf) / SOD_K)
    v[fan] = vf
    return e, v
