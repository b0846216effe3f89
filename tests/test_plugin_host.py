"""Host-side readers of the plugin layer (no GPU): positional .properties files and the
type-10 initial-condition files, and the field-dump format."""
import ctypes
import os

import numpy as np
import pytest

import gvh
from gvh import build as gbuild


@pytest.fixture(scope="module")
def lib():
    if gbuild.needs_rebuild():
        gbuild.build(verbose=False)
    L = gvh.load()
    L.gvh_read_lattice_parameters.argtypes = [ctypes.c_char_p, ctypes.POINTER(gvh.LatticeParams)]
    L.gvh_read_hydro_parameters.argtypes = [ctypes.c_char_p, ctypes.POINTER(gvh.HydroParams)]
    L.gvh_read_ic_parameters.argtypes = [ctypes.c_char_p, ctypes.c_void_p]
    L.gvh_read_ic_files.argtypes = [ctypes.c_char_p, ctypes.POINTER(gvh.LatticeParams), ctypes.c_int, ctypes.c_int,
                                    ctypes.c_void_p, ctypes.c_int]
    L.gvh_write_field.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_double,
                                  ctypes.POINTER(gvh.LatticeParams), ctypes.c_void_p]
    L.gvh_plugin_last_error.restype = ctypes.c_char_p
    return L


class IcParams(ctypes.Structure):
    _fields_ = [("initialConditionType", ctypes.c_int), ("numberOfNucleonsPerNuclei", ctypes.c_int),
                ("numberOfSourceFiles", ctypes.c_int), ("initialEnergyDensity", ctypes.c_double),
                ("scatteringCrossSectionNN", ctypes.c_double), ("impactParameter", ctypes.c_double),
                ("fractionOfBinaryCollisions", ctypes.c_double), ("rapidityVariance", ctypes.c_double),
                ("rapidityMean", ctypes.c_double), ("sourceType", ctypes.c_int)]


def write(path, text):
    with open(path, "w") as f:
        f.write(text)


def test_properties_are_positional(lib, tmp_path):
    # keys are ignored (line n is field n), spaces are dropped, values follow '='
    write(tmp_path / "lattice.properties", "nx = 21\nwhatever=17\n numLatticePointsRapidity=5\nnt=300\n"
                                           "dx=0.25\ndy=0.3\ndeta=0.15\ndtau = 0.0125")
    L = gvh.LatticeParams()
    assert lib.gvh_read_lattice_parameters(str(tmp_path).encode(), ctypes.byref(L)) == 0
    assert (L.numLatticePointsX, L.numLatticePointsY, L.numLatticePointsRapidity, L.numProperTimePoints) == (21, 17,
                                                                                                               5, 300)
    assert (L.numComputationalLatticePointsX, L.numComputationalLatticePointsY,
            L.numComputationalLatticePointsRapidity) == (25, 21, 9)
    assert (L.latticeSpacingX, L.latticeSpacingY, L.latticeSpacingRapidity, L.latticeSpacingProperTime) == (
        0.25, 0.3, 0.15, 0.0125)
    # four-line hydro file: the regulation temperature stays 0
    write(tmp_path / "hydro.properties", "tau0=0.6\netas=0.16\nTfo=0.150\ninitPi=0")
    H = gvh.HydroParams()
    H.regulationTemperatureGeV = 9.0
    assert lib.gvh_read_hydro_parameters(str(tmp_path).encode(), ctypes.byref(H)) == 0
    assert (H.initialProperTimePoint, H.shearViscosityToEntropyDensity, H.freezeoutTemperatureGeV,
            H.initializePimunuNavierStokes, H.regulationTemperatureGeV) == (0.6, 0.16, 0.15, 0, 0.0)
    write(tmp_path / "ic.properties", "type=10\nnSource=3\nA=197\ne0=40.5\nsigma=4.2\nb=7\nfbin=0.5\nvar=0.36\n"
                                      "flat=2\nsrc=1\n")
    ic = IcParams()
    assert lib.gvh_read_ic_parameters(str(tmp_path).encode(), ctypes.byref(ic)) == 0
    assert (ic.initialConditionType, ic.numberOfSourceFiles, ic.numberOfNucleonsPerNuclei) == (10, 3, 197)
    assert (ic.initialEnergyDensity, ic.impactParameter, ic.rapidityMean, ic.sourceType) == (40.5, 7.0, 2.0, 1)


def test_missing_config_is_an_error(lib, tmp_path):
    L = gvh.LatticeParams()
    assert lib.gvh_read_lattice_parameters(str(tmp_path / "nope").encode(), ctypes.byref(L)) == -1
    assert b"lattice.properties" in lib.gvh_plugin_last_error()


def test_type10_reader(lib, tmp_path):
    nx, ny, nz = 3, 2, 4
    L = gvh.LatticeParams(nx, ny, nz, nx + 4, ny + 4, nz + 4, 10, 0.2, 0.2, 0.2, 0.02)
    os.makedirs(tmp_path / "input")
    rng = np.random.default_rng(0)
    names = ["e", "ut", "ux", "uy", "un", "pitt", "pitx", "pity", "pitn", "pixx", "pixy", "pixn", "piyy", "piyn",
             "pinn", "bulk"]
    vals = {}
    for nm in names:
        v = rng.uniform(0.1, 40.0, (nx, ny, nz))  # index [i, j, k]
        vals[nm] = v
        # i outermost, k innermost, as the reference reads them
        lines = [f"{0.1 * i:.3f} {0.1 * j:.3f} {0.1 * k:.3f} {v[i, j, k]:.6f}" for i in range(nx) for j in range(ny)
                 for k in range(nz)]
        write(tmp_path / "input" / f"{nm}.dat", "\n".join(lines) + "\n")
    ng = (nx + 4) * (ny + 4) * (nz + 4)
    arrs = [np.zeros(ng) for _ in names]
    ptrs = (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
    assert lib.gvh_read_ic_files(str(tmp_path).encode(), ctypes.byref(L), 1, 1, ptrs, len(arrs)) == 0
    for nm, a in zip(names, arrs):
        g = a.reshape(nz + 4, ny + 4, nx + 4)
        got = g[2:-2, 2:-2, 2:-2].transpose(2, 1, 0)  # -> [i, j, k]
        want = np.array([float(f"{x:.6f}") for x in vals[nm].ravel()]).reshape(vals[nm].shape)
        want = want.astype(np.float32).astype(np.float64)  # scanned as float
        if nm == "e":
            want = want + 1e-3
        np.testing.assert_array_equal(got, want, err_msg=nm)
        assert np.all(g[:2] == 0) and np.all(g[:, :, :2] == 0)  # ghosts untouched
    # a short file is reported, not read past
    write(tmp_path / "input" / "uy.dat", "0 0 0 1.0\n")
    assert lib.gvh_read_ic_files(str(tmp_path).encode(), ctypes.byref(L), 1, 1, ptrs, len(arrs)) == -1
    assert b"uy.dat" in lib.gvh_plugin_last_error()


def test_field_dump_format(lib, tmp_path):
    nx, ny, nz = 3, 2, 2
    L = gvh.LatticeParams(nx, ny, nz, nx + 4, ny + 4, nz + 4, 10, 0.5, 0.25, 0.1, 0.02)
    ng = (nx + 4) * (ny + 4) * (nz + 4)
    f = np.arange(ng, dtype=np.float64) / 7.0
    assert lib.gvh_write_field(str(tmp_path).encode(), b"e", 0.6, ctypes.byref(L), f.ctypes.data) == 0
    lines = open(tmp_path / "e_0.600.dat").read().splitlines()
    assert len(lines) == nx * ny * nz
    # k outermost, i innermost; coordinates centred
    x, y, z, v = lines[1].split("\t")
    assert (x, y, z) == ("0.000", "-0.125", "-0.050")
    s = 3 + (nx + 4) * (2 + (ny + 4) * 2)
    assert v == f"{f[s]:.8f}"
