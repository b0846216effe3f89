"""Freeze-out surface on the GPU (device marking + host cornelius) against the reference's own
freeze-out code (FreezeOut.cpp, cornelius.cpp and the loop of HydroPlugin.cpp:255-393 replayed
by oracle/ref_surface.cpp on the reference's CPU build).

1. Same states in, same surface.dat out: each iteration the library's lattice is given the
   reference's state, so the two surface finders see identical inputs and must write
   identical text (3+1D conformal and QCD, 2+1D).
2. The whole loop: gvh-run's surface.dat against the reference stepping on its own, within a
   tolerance set by the FP64 step parity.
3. The device marking: crossed hypercubes and copied points equal a numpy count.
"""
import os
import subprocess

import numpy as np
import pytest

import gvh
import oracle
from gvh import build as gbuild
from helpers import rich_state

pytestmark = pytest.mark.gpu

HBARC = 0.197326938


def e_freezeout(ref, T_GeV=0.150):
    return ref.energy_density(T_GeV / HBARC)


CASES = {
    "conformal_shear_3d": dict(nx=12, ny=11, nz=7, dx=0.3, dy=0.3, dz=0.3, dt=0.02, etabar=0.2, theta=1.8,
                               conformal=True, shear=True, bulk=False),
    "qcd_bulk_3d": dict(nx=12, ny=11, nz=7, dx=0.3, dy=0.3, dz=0.3, dt=0.02, etabar=0.16, theta=2.0,
                        conformal=False, shear=True, bulk=True),
    "qcd_bulk_2d": dict(nx=17, ny=15, nz=1, dx=0.3, dy=0.3, dz=0.3, dt=0.02, etabar=0.16, theta=2.0,
                        conformal=False, shear=True, bulk=True),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_same_states_same_surface_text(case, tmp_path):
    lat = CASES[case]
    t0, dt, iters = 0.5, lat["dt"], 31
    R = oracle.RefLattice(**lat)
    R.set_primitive(rich_state(R, seed=4, e0=25.0, emin=0.3, spacing=0.6))
    efo = e_freezeout(R)
    ref_path = tmp_path / "ref_surface.dat"
    R.surface_begin(t0, efo, ref_path)
    G = gvh.Lattice(**lat)
    S = gvh.Surface(G, efo, threads=4)
    ours, chunk = [], []
    t = t0
    for n in range(1, iters + 1):
        G.set_state(R.get_state())
        R.surface_iteration(n, t)
        if n == 1:
            S.set_lower()
        else:
            label, scale, flush = gvh.slab_labels(n - 2, t0, dt)
            S.find(label, scale)
            chunk.append(S.text())
            if flush == n:
                ours.extend(chunk)
                chunk = []
        R.step(t, dt)
        t = t0 + n * dt
    R.surface_end()
    ref_text = open(ref_path).read()
    our_text = "".join(ours)
    assert ref_text.count("\n") > 50, "the case must cross the surface"
    assert our_text == ref_text
    assert S.info()["errors_total"] == 0


@pytest.mark.parametrize("case", ["qcd_bulk_3d", "qcd_bulk_2d"])
def test_device_rows_equal_host_rows(case):
    """The rows made on the device (the default for the QCD EoS) are the host pool's rows to
    the last bit, slab by slab; the conformal EoS keeps the host form."""
    lat = CASES[case]
    t0, dt = 0.5, lat["dt"]
    G = gvh.Lattice(**lat)
    G.set_primitive(rich_state(G, seed=4, e0=25.0, emin=0.3, spacing=0.6))
    efo = gvh.energy_density_of_temperature(0.150)
    D = gvh.Surface(G, efo, threads=3)
    H = gvh.Surface(G, efo, threads=3)
    T = gvh.Surface(G, efo, threads=3)  # text only: the device sends text, rows only where needed
    H.set_device_rows(False)
    T.set_outputs(rows=False, text=True)
    D.set_lower()
    H.set_lower()
    T.set_lower()
    t, total = t0, 0
    for n in range(1, 25):
        G.step(t, dt)
        t = t0 + n * dt
        label, scale, _ = gvh.slab_labels(n - 1, t0, dt)
        nd, nh, nt = D.find(label, scale), H.find(label, scale), T.find(label, scale)
        assert nd == nh == nt
        rd, rh = D.rows(), H.rows()
        assert np.array_equal(rd.view(np.uint64), rh.view(np.uint64)), n
        assert D.text() == H.text() == T.text()
        total += nd
    assert total > 50
    assert D.info()["errors_total"] == H.info()["errors_total"] == 0
    C = gvh.Lattice(**CASES["conformal_shear_3d"])
    S = gvh.Surface(C, 1.0)
    with pytest.raises(gvh.GvhError):
        S.set_device_rows(True)
    S.set_device_rows(False)


@pytest.mark.parametrize("tiny_part", ["half", "all"])
def test_device_text_splices_host_formatted_rows(tiny_part):
    """A row with a number the device's fast %g leaves to the exact path (here bulk pressures
    of order 1e-28, outside its exponent range) is sent as values, formatted on the host and
    spliced into the device's text in order; with more such rows than their buffer holds
    ("all": every row of a slab of ~3.8 k crossed hypercubes) every row is sent and formatted
    on the host. Text-only, rows + text and the host pool's text agree. The time levels are
    set, not stepped (a step would relax the bulk pressure): the energy density falls by a
    fifth from level to level, so the surface is a shell crossing both halves."""
    lat = dict(CASES["qcd_bulk_3d"], nx=40, ny=40, nz=16)
    G = gvh.Lattice(**lat)
    prim = rich_state(G, seed=4, e0=25.0, emin=0.3, spacing=0.3)
    Pi = prim["Pi"].reshape(G.ncz, G.ncy, G.ncx).copy()
    if tiny_part == "half":
        Pi[:, :, : G.ncx // 2] *= 1e-27
    else:
        Pi *= 1e-27
    prim["Pi"] = Pi.reshape(-1)
    efo = gvh.energy_density_of_temperature(0.150)
    D, H, T = (gvh.Surface(G, efo, threads=3) for _ in range(3))
    H.set_device_rows(False)
    T.set_outputs(rows=False, text=True)
    G.set_primitive(prim)
    for S in (D, H, T):
        S.set_lower()
    tiny = plain = 0
    for n in range(1, 3):
        G.set_primitive(dict(prim, e=prim["e"] * 0.8 ** n))
        label, scale, _ = gvh.slab_labels(n - 1, 0.5, lat["dt"])
        assert D.find(label, scale) == H.find(label, scale) == T.find(label, scale)
        text = H.text()
        assert D.text() == text and T.text() == text, n
        rd, rh = D.rows(), H.rows()
        assert np.array_equal(rd.view(np.uint64), rh.view(np.uint64)), n
        for line in text.splitlines():
            ex = line.split()[-1].partition("e-")[2]
            if ex and int(ex) > 17:
                tiny += 1
            else:
                plain += 1
    if tiny_part == "half":
        assert tiny > 1000 and plain > 1000, (tiny, plain)
    else:
        assert tiny > 5000 and plain == 0, (tiny, plain)


def test_device_marking_counts():
    lat = CASES["qcd_bulk_3d"]
    R = oracle.RefLattice(**lat)
    R.set_primitive(rich_state(R, seed=4, e0=25.0, emin=0.3, spacing=0.6))
    efo = e_freezeout(R)
    G = gvh.Lattice(**lat)
    G.set_state(R.get_state())
    S = gvh.Surface(G, efo)
    S.set_lower()
    lo = G.interior(R.get_state()["e"]).copy()  # [k, j, i]
    R.step(0.5, lat["dt"])
    st = R.get_state()
    G.set_state(st)
    hi = G.interior(st["e"])
    S.find(0.5, 0.5)
    inf = S.info()
    # crossed: neither all 16 corners >= e_fo nor all below
    both = np.stack([lo, hi]) >= efo  # [t, k, j, i]
    cnt = np.zeros((lat["nz"] - 1, lat["ny"] - 1, lat["nx"] - 1), int)
    for t in (0, 1):
        for c in (0, 1):
            for b in (0, 1):
                for a in (0, 1):
                    cnt += both[t, c:c + lat["nz"] - 1, b:b + lat["ny"] - 1, a:a + lat["nx"] - 1]
    crossed = (cnt > 0) & (cnt < 16)
    assert inf["hypercubes_last"] == int(crossed.sum()) > 0
    need = np.zeros((lat["nz"], lat["ny"], lat["nx"]), bool)
    for c in (0, 1):
        for b in (0, 1):
            for a in (0, 1):
                need[c:c + lat["nz"] - 1, b:b + lat["ny"] - 1, a:a + lat["nx"] - 1] |= crossed
    assert inf["points_last"] == int(need.sum())
    assert inf["elements_last"] >= inf["hypercubes_last"]


def write_inputs(root, lat, prim, names):
    os.makedirs(os.path.join(root, "input"), exist_ok=True)
    nx, ny, nz = lat["nx"], lat["ny"], lat["nz"]
    for nm in names:
        g = np.asarray(prim[nm]).reshape(nz + 4, ny + 4, nx + 4)
        v = g[2:-2, 2:-2, 2:-2].transpose(2, 1, 0)
        if nm == "e":
            v = v - 1e-3
        lines = [f"0 0 0 {v[i, j, k]:.9e}" for i in range(nx) for j in range(ny) for k in range(nz)]
        with open(os.path.join(root, "input", f"{nm}.dat"), "w") as f:
            f.write("\n".join(lines) + "\n")


def test_gvh_run_surface_matches_reference_run(tmp_path):
    lat = dict(nx=13, ny=12, nz=7, dx=0.3, dy=0.3, dz=0.3, dt=0.02, etabar=0.2, theta=1.8, conformal=True,
               shear=True, bulk=False)
    nt = 40
    cfg = tmp_path / "conf"
    os.makedirs(cfg)
    open(cfg / "lattice.properties", "w").write(
        f"nx={lat['nx']}\nny={lat['ny']}\nnz={lat['nz']}\nnt={nt}\ndx={lat['dx']}\ndy={lat['dy']}\n"
        f"dz={lat['dz']}\ndt={lat['dt']}\n")
    open(cfg / "hydro.properties", "w").write("tau0=0.5\netas=0.2\nTfo=0.150\ninitPi=0\n")
    open(cfg / "ic.properties", "w").write("type=10\n")
    R = oracle.RefLattice(**lat)
    prim = rich_state(R, seed=9, e0=25.0, emin=0.3, spacing=0.6)
    for k in prim:
        prim[k] = np.asarray(prim[k], np.float32).astype(np.float64)
    names = ["e", "ut", "ux", "uy", "un", "pitt", "pitx", "pity", "pitn", "pixx", "pixy", "pixn", "piyy", "piyn",
             "pinn"]
    write_inputs(tmp_path, lat, prim, names)
    out = tmp_path / "out"
    os.makedirs(out)
    if gbuild.needs_rebuild():
        gbuild.build(verbose=False)
    r = subprocess.run([gbuild.EXE, "-c", str(cfg), "-o", str(out), "--conformal", "--no-bulk", "--theta", "1.8",
                        "--no-dump"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    # the reference: same file values, its own steps, its freeze-out loop
    ref = {}
    for nm in names:
        a = np.zeros(R.ng)
        g = a.reshape(R.ncz, R.ncy, R.ncx)
        src = np.loadtxt(tmp_path / "input" / f"{nm}.dat", usecols=3).astype(np.float32).astype(np.float64)
        g[2:-2, 2:-2, 2:-2] = src.reshape(lat["nx"], lat["ny"], lat["nz"]).transpose(2, 1, 0)
        if nm == "e":
            g[2:-2, 2:-2, 2:-2] += 1e-3
        ref[nm] = a
    R.set_primitive(ref)
    t0, dt = 0.5, lat["dt"]
    R.surface_begin(t0, e_freezeout(R), tmp_path / "ref_surface.dat")
    t = t0
    for n in range(1, nt + 2):
        R.surface_iteration(n, t)
        if n == nt + 1:
            break
        R.step(t, dt)
        t = t0 + n * dt
    R.surface_end()
    want = np.loadtxt(tmp_path / "ref_surface.dat")
    got = np.loadtxt(out / "surface.dat")
    assert want.shape[0] > 100
    assert got.shape == want.shape
    # 6 significant digits in the file; FP64 steps agree to ~1e-12: each value within 2e-5 of
    # itself or 1e-6 of its column's largest magnitude
    scale = np.abs(want).max(axis=0)
    err = np.abs(got - want)
    ok = err <= 2e-5 * np.abs(want) + 1e-6 * scale
    assert ok.all(), (np.argwhere(~ok)[:5], got[~ok][:5], want[~ok][:5])
