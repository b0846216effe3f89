"""Oracle package: CPU checkers for the KT RK2 step. TEST INFRASTRUCTURE ONLY.

Two engines with one Python interface (ctypes, numpy arrays in the reference's ghosted
SoA layout):

* ``OracleLattice`` -- kt_oracle.c, this project's own C restatement of the reference
  algorithm (FP64 semantics), built into oracle/_build/.
* ``RefLattice`` -- the reference's own hot-path sources compiled for the CPU
  (oracle/build_ref.py -> oracle/_ref/), used to pin the restatement and as the
  benchmark's reference arm. Each variant library holds one lattice (the reference keeps
  its state in globals).
* ``RefGpuLattice`` -- the reference's own CUDA build (as shipped in FP32, and with the
  PRECISION double overlay) driven by oracle/ref_gpu_driver.cu: the reference's step timed
  on the same GPU, and its FP64 CUDA build as an oracle. Needs a GPU; one lattice per
  process and variant library.

Only tests/, the smoke check and the CPU-baseline/reference legs of bench.py use this
package; the product never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD_DIR = os.path.join(HERE, "_build")
ORACLE_LIB = os.path.join(BUILD_DIR, "libkt_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")

Q_NAMES = ["ttt", "ttx", "tty", "ttn", "pitt", "pitx", "pity", "pitn",
           "pixx", "pixy", "pixn", "piyy", "piyn", "pinn", "Pi"]
PRIM_NAMES = ["e", "p", "ut", "ux", "uy", "un", "utp", "uxp", "uyp", "unp"]


def q_names(shear: bool, bulk: bool) -> list[str]:
    names = Q_NAMES[:4]
    if shear:
        names += Q_NAMES[4:14]
    if bulk:
        names += ["Pi"]
    return names


def build_oracle(verbose: bool = True) -> str:
    """Compile kt_oracle.c (no FMA contraction, like the reference CPU build)."""
    os.makedirs(BUILD_DIR, exist_ok=True)
    src = os.path.join(HERE, "kt_oracle.c")
    cmd = ["gcc", "-std=c99", "-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-o", ORACLE_LIB, src, "-lm"]
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout)
    if verbose:
        print(f"[oracle] built {ORACLE_LIB}")
    return ORACLE_LIB


class KtParams(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
                ("dt", ctypes.c_double), ("etabar", ctypes.c_double), ("theta", ctypes.c_double),
                ("conformal", ctypes.c_int), ("shear", ctypes.c_int), ("bulk", ctypes.c_int),
                ("cartesian", ctypes.c_int)]


_oracle = None


def _load_oracle():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_LIB):
            build_oracle(verbose=False)
        L = ctypes.CDLL(ORACLE_LIB)
        L.kt_create.restype = ctypes.c_void_p
        L.kt_create.argtypes = [ctypes.POINTER(KtParams)]
        L.kt_destroy.argtypes = [ctypes.c_void_p]
        L.kt_nq.argtypes = [ctypes.POINTER(KtParams)]
        for fn in ("kt_set_state", "kt_get_state", "kt_set_primitive_state"):
            getattr(L, fn).argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.kt_rk2_step.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.kt_rk2_step.restype = None
        L.kt_max_propagation_speed.argtypes = [ctypes.c_void_p]
        L.kt_max_propagation_speed.restype = ctypes.c_double
        for fn in ("kt_equilibrium_pressure", "kt_speed_of_sound_squared", "kt_effective_temperature",
                   "kt_equilibrium_energy_density"):
            getattr(L, fn).argtypes = [ctypes.POINTER(KtParams), ctypes.c_double]
            getattr(L, fn).restype = ctypes.c_double
        L.kt_get_inferred_variables.argtypes = [ctypes.POINTER(KtParams), ctypes.c_double, ctypes.c_void_p,
                                                ctypes.c_double] + [ctypes.POINTER(ctypes.c_double)] * 6
        L.kt_get_inferred_variables.restype = None
        _oracle = L
    return _oracle


def _ptrs(arrays):
    return (ctypes.c_void_p * len(arrays))(*[None if a is None else a.ctypes.data for a in arrays])


class _Base:
    """Shared geometry and numpy plumbing."""

    def __init__(self, nx, ny, nz, dx, dy, dz, dt, etabar, theta, conformal, shear, bulk, cartesian=False):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.ncx, self.ncy, self.ncz = nx + 4, ny + 4, nz + 4
        self.ng = self.ncx * self.ncy * self.ncz
        self.conformal, self.shear, self.bulk = bool(conformal), bool(shear), bool(bulk)
        self.cartesian = bool(cartesian)
        self.params = dict(nx=nx, ny=ny, nz=nz, dx=dx, dy=dy, dz=dz, dt=dt, etabar=etabar, theta=theta,
                           conformal=int(conformal), shear=int(shear), bulk=int(bulk), cartesian=int(cartesian))
        self.qnames = q_names(shear, bulk)
        self.nq = len(self.qnames)
        self.field_names = self.qnames + PRIM_NAMES

    def _prim_list(self, prim: dict):
        order = ["e", "ut", "ux", "uy", "un"] + self.qnames[4:]
        out = []
        for k in order:
            a = prim.get(k)
            if a is None:
                a = np.zeros(self.ng)
            out.append(np.ascontiguousarray(np.broadcast_to(np.asarray(a, np.float64).reshape(-1), (self.ng,))))
        return out

    def _field_list(self, state: dict):
        out = []
        for k in self.field_names:
            a = state.get(k)
            out.append(None if a is None else np.ascontiguousarray(np.asarray(a, np.float64).reshape(-1)))
        return out

    def interior(self, a):
        return np.asarray(a).reshape(self.ncz, self.ncy, self.ncx)[2:-2, 2:-2, 2:-2]


class OracleLattice(_Base):
    """kt_oracle.c behind the shared interface."""

    def __init__(self, **kw):
        super().__init__(**kw)
        self._L = _load_oracle()
        self._p = KtParams(**self.params)
        self._h = self._L.kt_create(ctypes.byref(self._p))
        if not self._h:
            raise ValueError("kt_create rejected the parameters")

    def __del__(self):
        if getattr(self, "_h", None):
            self._L.kt_destroy(self._h)
            self._h = None

    def set_primitive(self, prim: dict):
        arrs = self._prim_list(prim)
        self._L.kt_set_primitive_state(self._h, _ptrs(arrs))

    def set_state(self, state: dict):
        arrs = self._field_list(state)
        self._L.kt_set_state(self._h, _ptrs(arrs))

    def get_state(self) -> dict:
        arrs = [np.zeros(self.ng) for _ in self.field_names]
        self._L.kt_get_state(self._h, _ptrs(arrs))
        return dict(zip(self.field_names, arrs))

    def step(self, t, dt, T_reg=0.0):
        self._L.kt_rk2_step(self._h, t, dt, T_reg)

    # scalar physics, for unit tests
    def max_propagation_speed(self) -> float:
        """Max of a / dx_axis over the predictor stages since the last call."""
        return self._L.kt_max_propagation_speed(self._h)

    def pressure(self, e):
        return self._L.kt_equilibrium_pressure(ctypes.byref(self._p), e)

    def temperature(self, e):
        return self._L.kt_effective_temperature(ctypes.byref(self._p), e)

    def energy_density(self, T):
        return self._L.kt_equilibrium_energy_density(ctypes.byref(self._p), T)

    def inferred(self, t, q, e_prev):
        qa = np.zeros(15)
        qa[:len(q)] = q
        outs = [ctypes.c_double() for _ in range(6)]
        self._L.kt_get_inferred_variables(ctypes.byref(self._p), t, qa.ctypes.data, e_prev, *outs)
        return [o.value for o in outs]


def ref_variant(precision: str, conformal: bool, shear: bool, bulk: bool, cartesian: bool = False) -> str:
    phys = "bulk" if bulk else ("shear" if shear else "ideal")
    return f"{precision}_{'conf' if conformal else 'qcd'}_{phys}" + ("_cart" if cartesian else "")


def ref_available(variant: str = "fp64_conf_shear") -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libref_{variant}.so"))


class RefLattice(_Base):
    """The reference's own sources built for the CPU (one lattice per variant library)."""

    def __init__(self, precision="fp64", threads=None, **kw):
        super().__init__(**kw)
        if self.bulk and not self.shear:
            raise ValueError("bulk without shear is not a valid reference build")
        self.variant = ref_variant(precision, self.conformal, self.shear, self.bulk, self.cartesian)
        path = os.path.join(REF_DIR, f"libref_{self.variant}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = ctypes.CDLL(path)
        L.gvh_ref_init.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 6
        L.gvh_ref_rk2_step.argtypes = [ctypes.c_double] * 3
        for fn in ("gvh_ref_set_state", "gvh_ref_get_state", "gvh_ref_set_primitive_state"):
            getattr(L, fn).argtypes = [ctypes.c_void_p]
        L.gvh_ref_set_primitive_state_p.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        for fn in ("gvh_ref_equilibrium_pressure", "gvh_ref_effective_temperature",
                   "gvh_ref_equilibrium_energy_density", "gvh_ref_speed_of_sound_squared"):
            getattr(L, fn).argtypes = [ctypes.c_double]
            getattr(L, fn).restype = ctypes.c_double
        L.gvh_ref_inferred.argtypes = [ctypes.c_double, ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p]
        L.gvh_ref_set_threads.argtypes = [ctypes.c_int]
        L.gvh_ref_get_validity.argtypes = [ctypes.c_void_p]
        L.gvh_ref_surface_begin.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 6 + [ctypes.c_char_p]
        L.gvh_ref_surface_begin.restype = ctypes.c_void_p
        L.gvh_ref_surface_iteration.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]
        L.gvh_ref_surface_iteration.restype = ctypes.c_longlong
        L.gvh_ref_surface_end.argtypes = [ctypes.c_void_p]
        L.gvh_ref_surface_end.restype = ctypes.c_longlong
        self._L = L
        if threads:
            L.gvh_ref_set_threads(int(threads))
        assert L.gvh_ref_nq() == self.nq, (L.gvh_ref_nq(), self.nq)
        p = self.params
        rc = L.gvh_ref_init(p["nx"], p["ny"], p["nz"], p["dx"], p["dy"], p["dz"], p["dt"], p["etabar"], p["theta"])
        if rc != 0:
            raise ValueError("gvh_ref_init failed")

    def max_threads(self) -> int:
        return int(self._L.gvh_ref_max_threads())

    def set_primitive(self, prim: dict, p=None):
        """p: a ghosted pressure array to use instead of p(e) (the type-11 reader)."""
        arrs = self._prim_list(prim)  # keep the arrays alive across the call
        if p is None:
            self._L.gvh_ref_set_primitive_state(_ptrs(arrs))
        else:
            pa = np.ascontiguousarray(p, dtype=np.float64)
            self._L.gvh_ref_set_primitive_state_p(_ptrs(arrs), pa.ctypes.data)

    def set_state(self, state: dict):
        arrs = self._field_list(state)
        self._L.gvh_ref_set_state(_ptrs(arrs))

    def get_state(self) -> dict:
        arrs = [np.zeros(self.ng) for _ in self.field_names]
        self._L.gvh_ref_get_state(_ptrs(arrs))
        return dict(zip(self.field_names, arrs))

    def step(self, t, dt, T_reg=0.0):
        self._L.gvh_ref_rk2_step(t, dt, T_reg)

    def pressure(self, e):
        return self._L.gvh_ref_equilibrium_pressure(e)

    VALIDITY_NAMES = ["regulations", "knudsenNumberTaupi", "knudsenNumberTauPi", "inverseReynoldsNumberPimunu",
                      "inverseReynoldsNumber2Pimunu", "inverseReynoldsNumberTilde2Pimunu", "inverseReynoldsNumberPi",
                      "inverseReynoldsNumber2Pi", "inverseReynoldsNumberTilde2Pi", "taupi", "dxux", "dyuy", "theta"]

    def get_validity(self) -> dict:
        """The reference's VALIDITY_DOMAIN arrays after the last step (ghosted)."""
        arrs = [np.zeros(self.ng) for _ in self.VALIDITY_NAMES]
        self._L.gvh_ref_get_validity(_ptrs(arrs))
        return dict(zip(self.VALIDITY_NAMES, arrs))

    # The freeze-out part of the reference's run loop (oracle/ref_surface.cpp).
    def surface_begin(self, t0, e_fo, path):
        p = self.params
        h = self._L.gvh_ref_surface_begin(p["nx"], p["ny"], p["nz"], t0, p["dt"], p["dx"], p["dy"], p["dz"], e_fo,
                                          str(path).encode())
        if not h:
            raise ValueError("the reference's surface finder needs nx, ny > 1")
        self._surface = h

    def surface_iteration(self, n, t):
        return int(self._L.gvh_ref_surface_iteration(self._surface, n, t))

    def surface_end(self):
        rows = int(self._L.gvh_ref_surface_end(self._surface))
        self._surface = None
        return rows

    def temperature(self, e):
        return self._L.gvh_ref_effective_temperature(e)

    def energy_density(self, T):
        return self._L.gvh_ref_equilibrium_energy_density(T)

    def inferred(self, t, q, e_prev):
        qa = np.zeros(15)
        qa[:len(q)] = q
        out = np.zeros(6)
        self._L.gvh_ref_inferred(t, qa.ctypes.data, e_prev, out.ctypes.data)
        return list(out)


def ref_gpu_variant(precision: str, conformal: bool, shear: bool, bulk: bool, theta: float) -> str:
    phys = "bulk" if bulk else ("shear" if shear else "ideal")
    return f"{precision}_{'conf' if conformal else 'qcd'}_{phys}_th{theta:.1f}"


def ref_gpu_available(variant: str, dropin: bool = False) -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libref_gpu_{'dropin_' if dropin else ''}{variant}.so"))


class RefGpuLattice(_Base):
    """The reference's own CUDA build (oracle/ref_gpu_driver.cu): its allocation, launch
    set-up, initial-state path and twoStepRungeKutta, on the current GPU. The reference keeps
    one lattice in globals, so a process holds at most one lattice per variant library (a
    second instance must have the same sizes and reuses the buffers)."""

    def __init__(self, precision="fp64", dropin=False, **kw):
        super().__init__(**kw)
        if self.cartesian:
            raise ValueError("the reference's CUDA builds here are Milne-coordinate builds")
        self.variant = ref_gpu_variant(precision, self.conformal, self.shear, self.bulk, kw["theta"])
        # dropin: the same program with gpu-vh_b200/dropin/twoStepRungeKutta_gvh.cu in place of
        # FullyDiscreteKurganovTadmorScheme.cu (libgvh's step behind the reference's loop)
        path = os.path.join(REF_DIR, f"libref_gpu_{'dropin_' if dropin else ''}{self.variant}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = ctypes.CDLL(path)
        L.gvh_ref_init.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 6
        L.gvh_ref_rk2_step.argtypes = [ctypes.c_double] * 3
        L.gvh_ref_time_steps.argtypes = [ctypes.c_int] + [ctypes.c_double] * 3 + [ctypes.POINTER(ctypes.c_double)]
        for fn in ("gvh_ref_set_state", "gvh_ref_get_state", "gvh_ref_set_primitive_state"):
            getattr(L, fn).argtypes = [ctypes.c_void_p]
        L.gvh_ref_set_primitive_state_p.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.gvh_ref_equilibrium_pressure.argtypes = [ctypes.c_double]
        L.gvh_ref_equilibrium_pressure.restype = ctypes.c_double
        self._L = L
        assert L.gvh_ref_nq() == self.nq, (L.gvh_ref_nq(), self.nq)
        assert L.gvh_ref_precision_bytes() == (8 if precision == "fp64" else 4)
        p = self.params
        if L.gvh_ref_init(p["nx"], p["ny"], p["nz"], p["dx"], p["dy"], p["dz"], p["dt"], p["etabar"], p["theta"]):
            raise ValueError("gvh_ref_init failed (sizes differ from this process's first lattice?)")

    def _ok(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"reference CUDA build: {what} failed ({rc})")

    def set_primitive(self, prim: dict, p=None):
        arrs = self._prim_list(prim)
        if p is None:
            self._ok(self._L.gvh_ref_set_primitive_state(_ptrs(arrs)), "set_primitive_state")
        else:
            pa = np.ascontiguousarray(p, dtype=np.float64)
            self._ok(self._L.gvh_ref_set_primitive_state_p(_ptrs(arrs), pa.ctypes.data), "set_primitive_state_p")

    def set_state(self, state: dict):
        arrs = self._field_list(state)
        self._ok(self._L.gvh_ref_set_state(_ptrs(arrs)), "set_state")

    def get_state(self) -> dict:
        arrs = [np.zeros(self.ng) for _ in self.field_names]
        self._ok(self._L.gvh_ref_get_state(_ptrs(arrs)), "get_state")
        return dict(zip(self.field_names, arrs))

    def step(self, t, dt, T_reg=0.0):
        self._ok(self._L.gvh_ref_rk2_step(t, dt, T_reg), "rk2_step")

    def time_steps(self, n, t0, dt, T_reg=0.0) -> float:
        """n steps of the reference's loop from t0; returns the CUDA-event time in ms."""
        ms = ctypes.c_double()
        self._ok(self._L.gvh_ref_time_steps(int(n), t0, dt, T_reg, ctypes.byref(ms)), "time_steps")
        return ms.value

    def pressure(self, e):
        return self._L.gvh_ref_equilibrium_pressure(e)
