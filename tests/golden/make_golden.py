"""Generates the golden fixtures in this directory from the reference's own sources.

Run in a checkout that has the reference tree (it builds oracle/_ref first):
    python tests/golden/make_golden.py

Each case runs the reference's KT RK2 step, compiled for the CPU in FP64 (oracle/_ref,
built by oracle/build_ref.py from the reference's rhic/src files), on a seeded initial
state (tests/helpers.rich_state) and stores the interior of every field after
set-up and after the last step, plus scalar tables of the equation of state and of
primitive recovery. The reference has no stored outputs for this path, so these files
are the pinned answers the oracle and the CUDA path are checked against.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import oracle  # noqa: E402
from oracle import build_ref  # noqa: E402
from helpers import rich_state  # noqa: E402

HBARC = 0.197326938

# name: (lattice kwargs, steps, T_reg [fm^-1], state kwargs)
CASES = {
    "conf_shear": (dict(nx=8, ny=9, nz=6, dx=0.3, dy=0.3, dz=0.3, dt=0.02, etabar=0.2, theta=1.8, conformal=True,
                        shear=True, bulk=False), 4, 0.0, dict(seed=1)),
    "conf_ideal": (dict(nx=8, ny=9, nz=6, dx=0.3, dy=0.3, dz=0.3, dt=0.02, etabar=0.2, theta=1.8, conformal=True,
                        shear=False, bulk=False), 4, 0.0, dict(seed=2)),
    "qcd_bulk": (dict(nx=8, ny=9, nz=6, dx=0.3, dy=0.3, dz=0.3, dt=0.01, etabar=0.16, theta=2.0, conformal=False,
                      shear=True, bulk=True), 4, 0.0, dict(seed=3)),
    "qcd_shear_regulated": (dict(nx=7, ny=8, nz=5, dx=0.3, dy=0.3, dz=0.3, dt=0.01, etabar=0.16, theta=2.0,
                                 conformal=False, shear=True, bulk=False), 4, 0.5 / HBARC, dict(seed=4, pi=0.3)),
    "qcd_bulk_dilute_2d": (dict(nx=9, ny=8, nz=1, dx=0.3, dy=0.3, dz=0.3, dt=0.01, etabar=0.16, theta=2.0,
                                conformal=False, shear=True, bulk=True), 4, 0.0, dict(seed=5, emin=0.02, e0=3.0, spacing=1.5)),
    "conf_shear_line": (dict(nx=1, ny=1, nz=12, dx=0.3, dy=0.3, dz=0.3, dt=0.02, etabar=0.2, theta=1.8,
                             conformal=True, shear=True, bulk=False), 4, 0.0, dict(seed=6)),
    # USE_CARTESIAN_COORDINATES (SourceTerms.cu:738-743), the reference built with it defined
    "conf_shear_cart": (dict(nx=8, ny=9, nz=6, dx=0.3, dy=0.3, dz=0.3, dt=0.02, etabar=0.2, theta=1.8,
                             conformal=True, shear=True, bulk=False, cartesian=True), 4, 0.0, dict(seed=7)),
}

TAU0 = 0.5


def run_case(engine_cls, lat_kw, steps, T_reg, st_kw):
    L = engine_cls(**lat_kw)
    prim = rich_state(L, **st_kw)
    L.set_primitive(prim)
    s0 = L.get_state()
    t = TAU0
    for n in range(1, steps + 1):
        L.step(t, lat_kw["dt"], T_reg)
        t = TAU0 + n * lat_kw["dt"]
    s1 = L.get_state()
    return L, prim, s0, s1


def scalar_tables():
    out = {}
    e = np.array([1e-9, 1e-7, 1e-3, 0.05, 0.1, 0.3, 1.0, 2.5, 7.0, 20.0, 60.0, 150.0, 400.0, 1000.0])
    T = np.array([0.0, 0.1, 0.3, 0.5, 0.76, 0.9, 1.2, 1.6, 2.5])
    for conf in (True, False):
        tag = "conf" if conf else "qcd"
        kw = dict(nx=1, ny=1, nz=1, dx=0.1, dy=0.1, dz=0.1, dt=0.01, etabar=0.2, theta=2.0, conformal=conf,
                  shear=True, bulk=True)
        R = oracle.RefLattice(**kw)
        out[f"{tag}_e"] = e
        out[f"{tag}_p"] = np.array([R.pressure(x) for x in e])
        out[f"{tag}_T"] = np.array([R.temperature(x) for x in e])
        out[f"{tag}_Tgrid"] = T
        out[f"{tag}_eofT"] = np.array([R.energy_density(x) for x in T])
        rng = np.random.default_rng(7)
        qs, eps, res = [], [], []
        for n in range(40):
            ee = float(np.exp(rng.uniform(np.log(1e-4), np.log(300))))
            ux, uy, un = rng.normal(0, 0.4, 3)
            ut = np.sqrt(1 + ux * ux + uy * uy + 0.36 * un * un)
            p = R.pressure(ee)
            q = np.zeros(15)
            q[0] = (ee + p) * ut * ut - p
            q[1] = (ee + p) * ut * ux
            q[2] = (ee + p) * ut * uy
            q[3] = (ee + p) * ut * un
            q[4:14] = rng.normal(0, 0.02 * p, 10)
            q[14] = -0.05 * p
            e_prev = [0.05, ee, ee * 1.3, ee * 0.7][n % 4]
            qs.append(q)
            eps.append(e_prev)
            res.append(R.inferred(0.6, q, e_prev))
        out[f"{tag}_inf_q"] = np.array(qs)
        out[f"{tag}_inf_eprev"] = np.array(eps)
        out[f"{tag}_inf_out"] = np.array(res)
    return out


def main(names=None):
    build_ref.build()
    for name, (lat_kw, steps, T_reg, st_kw) in CASES.items():
        if names and name not in names:
            continue
        L, prim, s0, s1 = run_case(oracle.RefLattice, lat_kw, steps, T_reg, st_kw)
        data = {"steps": steps, "T_reg": T_reg, "tau0": TAU0}
        for k, v in s0.items():
            data["init_" + k] = L.interior(v)
        for k, v in s1.items():
            data["final_" + k] = L.interior(v)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **data)
        print("wrote", name)
    if not names or "scalars" in names:
        np.savez_compressed(os.path.join(HERE, "scalars.npz"), **scalar_tables())
        print("wrote scalars")


if __name__ == "__main__":
    # optional arguments: the case names to (re)write; none writes every case and the scalars
    main(sys.argv[1:] or None)
