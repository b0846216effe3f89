"""The gvh-run executable (the reference's run() loop over libgvh) on a small event read
from type-10 input files, against the oracle driven with the same inputs."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from gvh import build as gbuild
from helpers import rich_state

pytestmark = pytest.mark.gpu


def write_inputs(root, lat, prim, names):
    os.makedirs(os.path.join(root, "input"), exist_ok=True)
    nx, ny, nz = lat["nx"], lat["ny"], lat["nz"]
    for nm in names:
        key = "Pi" if nm == "bulk" else nm
        g = np.asarray(prim[key]).reshape(nz + 4, ny + 4, nx + 4)
        v = g[2:-2, 2:-2, 2:-2].transpose(2, 1, 0)  # [i, j, k]
        if nm == "e":
            v = v - 1e-3  # the reader adds it back
        lines = [f"0 0 0 {v[i, j, k]:.9e}" for i in range(nx) for j in range(ny) for k in range(nz)]
        with open(os.path.join(root, "input", f"{nm}.dat"), "w") as f:
            f.write("\n".join(lines) + "\n")


def test_gvh_run_matches_oracle(tmp_path):
    lat = dict(nx=9, ny=8, nz=5, dx=0.3, dy=0.3, dz=0.3, dt=0.02, etabar=0.2, theta=1.8, conformal=True, shear=True,
               bulk=False)
    nt = 20
    cfg = tmp_path / "conf"
    os.makedirs(cfg)
    open(cfg / "lattice.properties", "w").write(
        f"nx={lat['nx']}\nny={lat['ny']}\nnz={lat['nz']}\nnt={nt}\ndx={lat['dx']}\ndy={lat['dy']}\n"
        f"dz={lat['dz']}\ndt={lat['dt']}\n")
    open(cfg / "hydro.properties", "w").write("tau0=0.5\netas=0.2\nTfo=0.150\ninitPi=0\n")
    open(cfg / "ic.properties", "w").write("type=10\n")
    O = oracle.OracleLattice(**lat)
    prim = rich_state(O, seed=9)
    # what the type-10 reader will see: %.9e text scanned as float, e + 1e-3
    for k in prim:
        prim[k] = np.asarray(prim[k], np.float32).astype(np.float64)
    write_inputs(tmp_path, lat, prim, ["e", "ut", "ux", "uy", "un", "pitt", "pitx", "pity", "pitn", "pixx", "pixy",
                                       "pixn", "piyy", "piyn", "pinn"])
    out = tmp_path / "out"
    os.makedirs(out)
    if gbuild.needs_rebuild():
        gbuild.build(verbose=False)
    r = subprocess.run([gbuild.EXE, "-c", str(cfg), "-o", str(out), "--conformal", "--no-bulk", "--theta", "1.8"],
                       cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Average time/step" in r.stdout
    # the oracle from the same file values
    ng = O.ng
    ref = {}
    for nm in ["e", "ut", "ux", "uy", "un", "pitt", "pitx", "pity", "pitn", "pixx", "pixy", "pixn", "piyy", "piyn",
               "pinn"]:
        a = np.zeros(ng)
        g = a.reshape(O.ncz, O.ncy, O.ncx)
        src = np.loadtxt(tmp_path / "input" / f"{nm}.dat", usecols=3).astype(np.float32).astype(np.float64)
        g[2:-2, 2:-2, 2:-2] = src.reshape(lat["nx"], lat["ny"], lat["nz"]).transpose(2, 1, 0)
        if nm == "e":
            g[2:-2, 2:-2, 2:-2] += 1e-3
        ref[nm] = a
    O.set_primitive(ref)
    t = 0.5
    for n in range(1, nt + 1):
        O.step(t, lat["dt"])
        t = 0.5 + n * lat["dt"]
    # gvh-run dumped the state after 20 steps at t = 0.9 (dump before step 21)
    so = O.get_state()
    for name in ("e", "ux", "pixx"):
        dump = np.loadtxt(out / f"{name}_0.900.dat")
        vals = dump[:, 3].reshape(lat["nz"], lat["ny"], lat["nx"])
        want = O.interior(so[name])
        np.testing.assert_allclose(vals, want, rtol=0, atol=1.5e-8 + 1e-12 * np.abs(want).max(), err_msg=name)


def test_gvh_run_type11_tmunu_file(tmp_path):
    """Initial-condition type 11 (one input/Tmunu.dat, p read from the file): gvh-run's dump
    after 10 steps against the reference build given the same values and pressure."""
    lat = dict(nx=8, ny=7, nz=5, dx=0.3, dy=0.3, dz=0.3, dt=0.02, etabar=0.16, theta=2.0, conformal=False,
               shear=True, bulk=True)
    nt = 10
    cfg = tmp_path / "conf"
    os.makedirs(cfg)
    open(cfg / "lattice.properties", "w").write(
        f"nx={lat['nx']}\nny={lat['ny']}\nnz={lat['nz']}\nnt={nt}\ndx={lat['dx']}\ndy={lat['dy']}\n"
        f"dz={lat['dz']}\ndt={lat['dt']}\n")
    open(cfg / "hydro.properties", "w").write("tau0=0.5\netas=0.16\nTfo=0.150\ninitPi=0\n")
    open(cfg / "ic.properties", "w").write("type=11\n")
    R = oracle.RefLattice(**lat)
    prim = rich_state(R, seed=17)
    cols = ["e", "p", "ut", "ux", "uy", "un", "pitt", "pitx", "pity", "pitn", "pixx", "pixy", "pixn", "piyy", "piyn",
            "pinn", "Pi"]
    grids = {}
    for c in cols:
        src = prim["e"] * 0.3 if c == "p" else prim[c]  # a pressure that is not p(e): the file's is used
        g = np.asarray(src, np.float64).reshape(R.ncz, R.ncy, R.ncx)[2:-2, 2:-2, 2:-2].transpose(2, 1, 0)
        grids[c] = np.asarray(g, np.float32)
    nx, ny, nz = lat["nx"], lat["ny"], lat["nz"]
    os.makedirs(tmp_path / "input")
    with open(tmp_path / "input" / "Tmunu.dat", "w") as f:
        for i in range(nx):
            for j in range(ny):
                for k in range(nz):
                    vals = [grids[c][i, j, k] - (1e-3 if c == "e" else 0.0) for c in cols]
                    f.write("0 0 0 " + " ".join(f"{v:.9e}" for v in vals) + "\n")
    out = tmp_path / "out"
    os.makedirs(out)
    if gbuild.needs_rebuild():
        gbuild.build(verbose=False)
    r = subprocess.run([gbuild.EXE, "-c", str(cfg), "-o", str(out), "--no-surface"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    # the reference from the values the reader sees (float scan, e + 1e-3, p from the file)
    data = np.loadtxt(tmp_path / "input" / "Tmunu.dat").astype(np.float32).astype(np.float64)
    ref, p = {}, np.zeros(R.ng)
    for n, c in enumerate(cols):
        a = np.zeros(R.ng)
        a.reshape(R.ncz, R.ncy, R.ncx)[2:-2, 2:-2, 2:-2] = data[:, 3 + n].reshape(nx, ny, nz).transpose(2, 1, 0)
        if c == "e":
            a.reshape(R.ncz, R.ncy, R.ncx)[2:-2, 2:-2, 2:-2] += 1e-3
        if c == "p":
            p = a
        else:
            ref[c] = a
    R.set_primitive(ref, p=p)
    t = 0.5
    for n in range(1, nt + 1):
        R.step(t, lat["dt"])
        t = 0.5 + n * lat["dt"]
    so = R.get_state()
    for name in ("e", "ux", "pixx", "Pi"):
        dump = np.loadtxt(out / f"{name}_{t:.3f}.dat")
        vals = dump[:, 3].reshape(nz, ny, nx)
        want = R.interior(so[name])
        np.testing.assert_allclose(vals, want, rtol=0, atol=1.5e-8 + 1e-9 * np.abs(want).max(), err_msg=name)
