"""Seeded initial conditions for the benchmark and test workloads.

Every profile is produced the way the reference's type-10 reader would ingest it
(InitialConditions.cpp:98-489): values are rounded to float (the reader scans "%f" into a
float) and 1e-3 is added to e (InitialConditions.cpp:124). u^mu = (1,0,0,0) and
pi^{mu nu} = Pi = 0 (initializePimunuNavierStokes = 0). Energy densities are in fm^-4
(GeV/fm^3 divided by hbar*c, HydroPlugin.cpp:132).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

HBARC = 0.197326938


@dataclass
class Workload:
    name: str
    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dz: float
    tau0: float
    dtau: float
    conformal: bool
    shear: bool
    bulk: bool
    etabar: float
    theta: float
    T_fo_GeV: float = 0.150
    steps: int = 100
    seed: int = 0
    extra: dict = field(default_factory=dict)

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz

    def lattice_kwargs(self) -> dict:
        return dict(nx=self.nx, ny=self.ny, nz=self.nz, dx=self.dx, dy=self.dy, dz=self.dz, dt=self.dtau,
                    etabar=self.etabar, theta=self.theta, conformal=self.conformal, shear=self.shear, bulk=self.bulk)


# Config 1: small single event, conformal, shear on, bulk off, theta 1.8, 100 steps.
CONFIG1 = Workload("config1_33x33x17_conformal", 33, 33, 17, 0.2, 0.2, 0.2, 0.5, 0.02, True, True, False, 0.2, 1.8,
                   steps=100)
# Config 2: full event, QCD EoS, eta/s 0.16, bulk on. The limiter slope is the reference's
# shipped 2.0 (FluxLimiter.cu:15); the configuration names none.
CONFIG2 = Workload("config2_131x131x61_qcd_bulk", 131, 131, 61, 0.1, 0.1, 0.1, 0.6, 0.01, False, True, True, 0.16,
                   2.0, steps=0, seed=12345)


def coords(w: Workload):
    """Cell-centre coordinates on the ghosted lattice, x_i = (i - (n-1)/2) dx (centred grid)."""
    x = (np.arange(w.nx + 4) - 2 - (w.nx - 1) / 2) * w.dx
    y = (np.arange(w.ny + 4) - 2 - (w.ny - 1) / 2) * w.dy
    z = (np.arange(w.nz + 4) - 2 - (w.nz - 1) / 2) * w.dz
    return np.meshgrid(z, y, x, indexing="ij")  # (Z, Y, X), each (ncz, ncy, ncx)


def _as_file_values(e):
    """What the type-10 reader stores for an e value written to a file."""
    return e.astype(np.float32).astype(np.float64) + 1.0e-3


def gaussian_profile(w: Workload, e0_GeV=30.0, sigma_r=3.0, eta_flat=1.0, sigma_eta=0.5) -> dict:
    """e = e0 exp(-(x^2+y^2)/(2 sigma_r^2)) exp(-max(|eta|-eta_flat,0)^2/(2 sigma_eta^2))."""
    Z, Y, X = coords(w)
    e0 = e0_GeV / HBARC
    e = e0 * np.exp(-(X ** 2 + Y ** 2) / (2 * sigma_r ** 2)) * np.exp(
        -np.maximum(np.abs(Z) - eta_flat, 0) ** 2 / (2 * sigma_eta ** 2))
    return _primitive(w, _as_file_values(e))


def _primitive(w: Workload, e) -> dict:
    ng = e.size
    prim = dict(e=e.reshape(-1), ut=np.ones(ng), ux=np.zeros(ng), uy=np.zeros(ng), un=np.zeros(ng))
    return prim


def _sample_woods_saxon(rng, A, R, a):
    """A nucleon positions from a Woods-Saxon density by rejection sampling in r."""
    rmax = R + 10 * a
    out = []
    while len(out) < A:
        r = rmax * rng.random(4 * A) ** (1.0 / 3.0)  # uniform in the ball
        keep = rng.random(4 * A) < 1.0 / (1.0 + np.exp((r - R) / a))
        r = r[keep]
        n = min(len(r), A - len(out))
        r = r[:n]
        cth = rng.uniform(-1, 1, n)
        phi = rng.uniform(0, 2 * np.pi, n)
        sth = np.sqrt(1 - cth ** 2)
        out.extend(np.stack([r * sth * np.cos(phi), r * sth * np.sin(phi)], axis=1))
    return np.array(out[:A])


@dataclass
class Hotspots:
    """The sources of a Glauber-hotspot event: e(x, y, eta) = fz(eta) * scale *
    sum_p w_p exp(-((x - x_p)^2 + (y - y_p)^2) / s2) + background with
    fz = exp(-max(|eta| - eta_flat, 0)^2 / s2_eta), s2 = 2 sigma^2, s2_eta = 2 sigma_eta^2
    (energy densities in fm^-4)."""
    x: np.ndarray
    y: np.ndarray
    w: np.ndarray
    sigma: float
    scale: float
    eta_flat: float
    sigma_eta: float
    background: float
    meta: dict


def hotspot_sources(w: Workload, b=None, e0_GeV=40.0, A=197, R=6.4, a=0.54, sigma_nn=4.2, sigma_hot=0.4,
                    eta_flat=1.0, sigma_eta=0.6, b_max=10.0, background_GeV=0.05) -> Hotspots:
    """The Monte-Carlo part of glauber_hotspots (seeded): two Woods-Saxon nuclei at impact
    parameter b ~ U(0, b_max), their participants (a nucleon participates when it passes
    within sqrt(sigma_nn/pi) of a nucleon of the other nucleus), Gamma(k=1) weights, and the
    scale that makes the transverse profile's mean over the participant positions e0."""
    rng = np.random.default_rng(w.seed)
    if b is None:
        b = rng.uniform(0, b_max)
    nA = _sample_woods_saxon(rng, A, R, a) + np.array([b / 2, 0.0])
    nB = _sample_woods_saxon(rng, A, R, a) - np.array([b / 2, 0.0])
    d2 = sigma_nn / np.pi
    dist2 = ((nA[:, None, :] - nB[None, :, :]) ** 2).sum(-1)
    partA = (dist2 <= d2).any(1)
    partB = (dist2 <= d2).any(0)
    parts = np.concatenate([nA[partA], nB[partB]])
    if len(parts) == 0:
        parts = np.zeros((1, 2))
    weights = rng.gamma(1.0, 1.0, len(parts))
    at_parts = (weights[:, None] * np.exp(-((parts[None, :, :] - parts[:, None, :]) ** 2).sum(-1)
                                          / (2 * sigma_hot ** 2))).sum(0)
    scale = (e0_GeV / HBARC) / max(at_parts.mean(), 1e-30)
    return Hotspots(np.ascontiguousarray(parts[:, 0]), np.ascontiguousarray(parts[:, 1]), weights, sigma_hot, scale,
                    eta_flat, sigma_eta, background_GeV / HBARC,
                    dict(b=float(b), n_part=int(len(parts)), seed=w.seed))


def hotspot_field(w: Workload, hs: Hotspots) -> np.ndarray:
    """The ghosted energy density of the sources as the type-10 reader stores it (float,
    + 1e-3). The device fill (gvh_set_hotspot_state) follows the same operations."""
    Z, Y, X = coords(w)
    x = X[0, 0, :]
    y = Y[0, :, 0]
    s2 = 2 * hs.sigma ** 2
    T = np.zeros((len(y), len(x)))
    for p in range(len(hs.w)):  # sources in order: sum_p (w_p gy_p) gx_p
        gx = np.exp(-(x - hs.x[p]) ** 2 / s2)
        gy = np.exp(-(y - hs.y[p]) ** 2 / s2)
        T += (hs.w[p] * gy)[:, None] * gx[None, :]
    T = T * hs.scale
    z = Z[:, 0, 0]
    fz = np.exp(-np.maximum(np.abs(z) - hs.eta_flat, 0) ** 2 / (2 * hs.sigma_eta ** 2))
    e = fz[:, None, None] * T[None, :, :] + hs.background
    return _as_file_values(e)


def glauber_hotspots(w: Workload, b=None, e0_GeV=40.0, A=197, R=6.4, a=0.54, sigma_nn=4.2, sigma_hot=0.4,
                     eta_flat=1.0, sigma_eta=0.6, b_max=10.0, background_GeV=0.05) -> dict:
    """Fluctuating event: Gaussian hotspots (width sigma_hot) at the participants of two
    Woods-Saxon nuclei at impact parameter b ~ U(0, b_max), each with a Gamma(k=1) weight
    (hotspot_sources), filled into the lattice (hotspot_field). The transverse profile is
    scaled so that its mean over the participant positions is e0; the rapidity profile is
    flat for |eta| < eta_flat with Gaussian tails.

    background_GeV is a uniform energy density under the event (below e(T_fo) = 0.28
    GeV/fm^3, so it never delays freeze-out). The reference scheme, with its 1e-3 fm^-4 floor
    alone, runs away in the near-vacuum around steep hotspots: on a 61x61 lattice at 0.2 fm the
    oracle (bit-identical to the reference's CPU build) reaches NaN after ~44 steps; with
    0.05 GeV/fm^3 underneath it stays finite."""
    hs = hotspot_sources(w, b, e0_GeV, A, R, a, sigma_nn, sigma_hot, eta_flat, sigma_eta, b_max, background_GeV)
    prim = _primitive(w, hotspot_field(w, hs))
    prim["_meta"] = hs.meta
    return prim
