"""Python host binding of libgvh.so, the B200 KT RK2 step of gpu-vh.

The binding mirrors the reference's interface for this path: the lattice/hydro parameter
structs (LatticeParameters.h:17-31, HydroParameters.h:15-22), the ghosted SoA state arrays
(DynamicalVariables.cu:32-35) and one call per Heun step (twoStepRungeKutta,
FullyDiscreteKurganovTadmorScheme.cu:109-139). All compute runs in the CUDA library; if
the library is missing this module raises instead of computing anything itself.
"""
from __future__ import annotations

import ctypes
import weakref
import os

import numpy as np

from . import build as _build

LIB_PATH = _build.LIB

GVH_EOS_QCD = 0
GVH_EOS_CONFORMAL = 1
GVH_PRECISION_FP64 = 0
GVH_PRECISION_MIXED = 1
GVH_COORDINATES_MILNE = 0
GVH_COORDINATES_CARTESIAN = 1
GVH_OK = 0
GVH_ERR_INVALID = -1
GVH_ERR_CUDA = -2
GVH_ERR_NUMERIC = -3
GVH_STATUS_NAN = 1
GVH_STATUS_NEWTON = 2
GVH_STATUS_DAMPED = 4       # informational (see include/gvh.h)
GVH_STATUS_BOUNDS = 8       # the bounds-checked build skipped a cell (see include/gvh.h)
GVH_STATUS_ERRORS = 9       # NaN or a bounds failure; a non-converged Newton solve is a
                            # warning, as in the reference

Q_NAMES = ["ttt", "ttx", "tty", "ttn", "pitt", "pitx", "pity", "pitn",
           "pixx", "pixy", "pixn", "piyy", "piyn", "pinn", "Pi"]
PRIM_NAMES = ["e", "p", "ut", "ux", "uy", "un", "utp", "uxp", "uyp", "unp"]
HBARC = 0.197326938  # GeV fm (HydroPlugin.cpp:132)


class GvhError(RuntimeError):
    pass


class LatticeParams(ctypes.Structure):
    """Layout-compatible with the reference's struct LatticeParameters."""
    _fields_ = [("numLatticePointsX", ctypes.c_int), ("numLatticePointsY", ctypes.c_int),
                ("numLatticePointsRapidity", ctypes.c_int), ("numComputationalLatticePointsX", ctypes.c_int),
                ("numComputationalLatticePointsY", ctypes.c_int),
                ("numComputationalLatticePointsRapidity", ctypes.c_int), ("numProperTimePoints", ctypes.c_int),
                ("latticeSpacingX", ctypes.c_double), ("latticeSpacingY", ctypes.c_double),
                ("latticeSpacingRapidity", ctypes.c_double), ("latticeSpacingProperTime", ctypes.c_double)]


class HydroParams(ctypes.Structure):
    """Layout-compatible with the reference's struct HydroParameters."""
    _fields_ = [("initialProperTimePoint", ctypes.c_double), ("shearViscosityToEntropyDensity", ctypes.c_double),
                ("freezeoutTemperatureGeV", ctypes.c_double), ("initializePimunuNavierStokes", ctypes.c_int),
                ("regulationTemperatureGeV", ctypes.c_double)]


class RunReport(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_longlong), ("tau_end", ctypes.c_double), ("average_ms_per_step", ctypes.c_double),
                ("frozen_out", ctypes.c_int), ("status", ctypes.c_uint),
                ("freezeout_energy_density", ctypes.c_double), ("surface_elements", ctypes.c_longlong),
                ("surface_seconds", ctypes.c_double), ("surface_hypercubes", ctypes.c_longlong),
                ("surface_bytes_to_host", ctypes.c_double), ("surface_host_seconds", ctypes.c_double)]


GVH_RUN_FIELDS = 1
GVH_RUN_SURFACE = 2


class Options(ctypes.Structure):
    _fields_ = [("eos", ctypes.c_int), ("shear", ctypes.c_int), ("bulk", ctypes.c_int),
                ("precision", ctypes.c_int), ("theta", ctypes.c_double), ("device", ctypes.c_int),
                ("coordinates", ctypes.c_int)]


_lib = None

EXPORTS = [
    "gvh_default_options", "gvh_create", "gvh_destroy", "gvh_num_conserved", "gvh_num_fields",
    "gvh_num_lattice_cells", "gvh_set_primitive_state", "gvh_set_state", "gvh_get_state", "gvh_rk2_step",
    "gvh_status", "gvh_clear_status", "gvh_synchronize", "gvh_launches_per_step", "gvh_last_error",
    "gvh_set_stream", "gvh_max_energy_density", "gvh_max_propagation_speed", "gvh_set_hotspot_state", "gvh_save_state", "gvh_load_state", "gvh_set_state_async", "gvh_get_state_async", "gvh_join_async",
]


def load(path: str | None = None):
    """Load libgvh.so (the CUDA implementation). Raises if it is not built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    # GVH_LIBRARY selects another build of the same library (the bounds-checked one)
    p = path or os.environ.get("GVH_LIBRARY") or LIB_PATH
    if not os.path.exists(p):
        raise GvhError(f"libgvh.so not found at {p}: build it with __graft_entry__.build()")
    L = ctypes.CDLL(p)
    vp, ip, dp = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    L.gvh_default_options.argtypes = [ctypes.POINTER(Options)]
    L.gvh_default_options.restype = None
    L.gvh_create.argtypes = [ctypes.POINTER(LatticeParams), ctypes.POINTER(HydroParams), ctypes.POINTER(Options),
                             ctypes.POINTER(vp)]
    L.gvh_destroy.argtypes = [vp]
    L.gvh_num_conserved.argtypes = [vp]
    L.gvh_num_fields.argtypes = [vp]
    L.gvh_num_lattice_cells.argtypes = [vp]
    L.gvh_num_lattice_cells.restype = ctypes.c_longlong
    L.gvh_set_primitive_state.argtypes = [vp, vp, ip]
    L.gvh_set_state.argtypes = [vp, vp, ip]
    L.gvh_get_state.argtypes = [vp, vp, ip]
    L.gvh_set_state_async.argtypes = [vp, vp, ip]
    L.gvh_get_state_async.argtypes = [vp, vp, ip]
    L.gvh_join_async.argtypes = [vp]
    L.gvh_rk2_step.argtypes = [vp, dp, dp, dp]
    L.gvh_status.argtypes = [vp, ctypes.POINTER(ctypes.c_uint)]
    L.gvh_clear_status.argtypes = [vp]
    L.gvh_synchronize.argtypes = [vp]
    L.gvh_launches_per_step.argtypes = [vp]
    L.gvh_set_stream.argtypes = [vp, vp]
    L.gvh_max_energy_density.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
    L.gvh_max_propagation_speed.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
    L.gvh_set_hotspot_state.argtypes = [vp, vp]
    L.gvh_save_state.argtypes = [vp, ctypes.c_char_p, dp, ctypes.c_longlong]
    L.gvh_load_state.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(dp), ctypes.POINTER(ctypes.c_longlong)]
    L.gvh_last_error.restype = ctypes.c_char_p
    if path is None:
        _lib = L
    return L


def _check(rc: int, what: str):
    if rc != 0:
        msg = load().gvh_last_error().decode(errors="replace")
        raise GvhError(f"{what} failed ({rc}): {msg}")


def _ptr_array(ptrs):
    return (ctypes.c_void_p * len(ptrs))(*ptrs)


def q_names(shear: bool, bulk: bool) -> list[str]:
    names = Q_NAMES[:4]
    if shear:
        names += Q_NAMES[4:14]
    if bulk:
        names += ["Pi"]
    return names


class Lattice:
    """One hydro lattice on the GPU (a libgvh handle)."""

    def __init__(self, nx, ny, nz, dx, dy, dz, dt, etabar, theta=2.0, conformal=False, shear=True, bulk=True,
                 precision="fp64", device=-1, tau0=0.5, T_fo_GeV=0.15, T_reg_GeV=0.0, cartesian=False):
        self._L = load()
        self.nx, self.ny, self.nz = nx, ny, nz
        self.ncx, self.ncy, self.ncz = nx + 4, ny + 4, nz + 4
        self.ng = self.ncx * self.ncy * self.ncz
        self.shear, self.bulk, self.conformal = bool(shear), bool(bulk), bool(conformal)
        self.qnames = q_names(self.shear, self.bulk)
        self.nq = len(self.qnames)
        self.field_names = self.qnames + PRIM_NAMES
        self.lattice = LatticeParams(nx, ny, nz, nx + 4, ny + 4, nz + 4, 0, dx, dy, dz, dt)
        self.hydro = HydroParams(tau0, etabar, T_fo_GeV, 0, T_reg_GeV)
        o = Options()
        self._L.gvh_default_options(ctypes.byref(o))
        o.eos = GVH_EOS_CONFORMAL if conformal else GVH_EOS_QCD
        o.shear, o.bulk, o.theta, o.device = int(shear), int(bulk), float(theta), int(device)
        o.precision = {"fp64": GVH_PRECISION_FP64, "mixed": GVH_PRECISION_MIXED}[precision]
        o.coordinates = GVH_COORDINATES_CARTESIAN if cartesian else GVH_COORDINATES_MILNE
        self.options = o
        h = ctypes.c_void_p()
        _check(self._L.gvh_create(ctypes.byref(self.lattice), ctypes.byref(self.hydro), ctypes.byref(o),
                                  ctypes.byref(h)), "gvh_create")
        self._h = h
        assert self._L.gvh_num_conserved(h) == self.nq
        assert self._L.gvh_num_lattice_cells(h) == self.ng

    def close(self):
        for dep in list(getattr(self, "_dependents", [])):  # surfaces bound to this lattice
            d = dep()
            if d is not None:
                d.close()
        if getattr(self, "_h", None):
            self._L.gvh_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- state ---------------------------------------------------------------------------
    def _as_ghosted(self, a):
        a = np.ascontiguousarray(np.broadcast_to(np.asarray(a, np.float64).reshape(-1), (self.ng,)))
        return a

    def set_primitive(self, prim: dict, p=None):
        """Initial state from primitives; p (ghosted) replaces p(e) of the EoS when given, as the
        type-11 reader does."""
        order = ["e", "ut", "ux", "uy", "un"] + self.qnames[4:]
        arrs = [self._as_ghosted(prim.get(k, 0.0)) for k in order]
        ptrs = _ptr_array([a.ctypes.data for a in arrs])
        if p is None:
            _check(self._L.gvh_set_primitive_state(self._h, ptrs, len(arrs)), "gvh_set_primitive_state")
        else:
            pa = self._as_ghosted(p)
            self._L.gvh_set_primitive_state_p.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                                          ctypes.c_void_p]
            _check(self._L.gvh_set_primitive_state_p(self._h, ptrs, len(arrs), pa.ctypes.data),
                   "gvh_set_primitive_state_p")

    def save(self, path, tau=0.0, step=0):
        """Binary snapshot of the state (with the caller's tau and step) to path."""
        _check(self._L.gvh_save_state(self._h, os.fsencode(path), float(tau), int(step)), "gvh_save_state")

    def load(self, path):
        """Restore a snapshot written by save(); returns (tau, step)."""
        t, n = ctypes.c_double(), ctypes.c_longlong()
        _check(self._L.gvh_load_state(self._h, os.fsencode(path), ctypes.byref(t), ctypes.byref(n)),
               "gvh_load_state")
        return t.value, n.value

    def set_hotspots(self, hs):
        """Initial state from hotspot sources (a workloads.Hotspots), filled on the device."""
        c, keep = _hotspots_c(hs)
        _check(self._L.gvh_set_hotspot_state(self._h, ctypes.byref(c)), "gvh_set_hotspot_state")

    def set_state(self, state: dict):
        arrs = [None if state.get(k) is None else self._as_ghosted(state[k]) for k in self.field_names]
        ptrs = [None if a is None else a.ctypes.data for a in arrs]
        _check(self._L.gvh_set_state(self._h, _ptr_array(ptrs), len(ptrs)), "gvh_set_state")

    def get_state(self, names=None) -> dict:
        want = set(names) if names else set(self.field_names)
        arrs = [np.empty(self.ng) if k in want else None for k in self.field_names]
        ptrs = [None if a is None else a.ctypes.data for a in arrs]
        _check(self._L.gvh_get_state(self._h, _ptr_array(ptrs), len(ptrs)), "gvh_get_state")
        return {k: a for k, a in zip(self.field_names, arrs) if a is not None}

    def set_state_ptrs(self, ptrs):
        _check(self._L.gvh_set_state(self._h, _ptr_array(list(ptrs)), len(ptrs)), "gvh_set_state")

    def get_state_ptrs(self, ptrs):
        _check(self._L.gvh_get_state(self._h, _ptr_array(list(ptrs)), len(ptrs)), "gvh_get_state")

    # Pipelined copies (gvh_set_state_async / gvh_get_state_async): queued on the handle's copy
    # streams and returned from at once; the host arrays (pinned, for overlap) must stay
    # untouched until synchronize(). join_async() orders the handle's stream and its copy
    # streams both ways: later stream work after every queued copy, later copies after every
    # queued stream work.
    def set_state_async_ptrs(self, ptrs):
        _check(self._L.gvh_set_state_async(self._h, _ptr_array(list(ptrs)), len(ptrs)), "gvh_set_state_async")

    def get_state_async_ptrs(self, ptrs):
        _check(self._L.gvh_get_state_async(self._h, _ptr_array(list(ptrs)), len(ptrs)), "gvh_get_state_async")

    def join_async(self):
        _check(self._L.gvh_join_async(self._h), "gvh_join_async")

    VALIDITY_NAMES = ["regulations", "knudsenNumberTaupi", "knudsenNumberTauPi", "inverseReynoldsNumberPimunu",
                      "inverseReynoldsNumber2Pimunu", "inverseReynoldsNumberTilde2Pimunu", "inverseReynoldsNumberPi",
                      "inverseReynoldsNumber2Pi", "inverseReynoldsNumberTilde2Pi", "taupi", "dxux", "dyuy", "theta"]

    def enable_validity(self, on=True):
        """Compute the validity diagnostics (checkValidity) with every step from now on."""
        self._L.gvh_enable_validity.argtypes = [ctypes.c_void_p, ctypes.c_int]
        _check(self._L.gvh_enable_validity(self._h, int(bool(on))), "gvh_enable_validity")

    def get_validity(self) -> dict:
        """The 13 VALIDITY_DOMAIN arrays of the last step (ghosted)."""
        arrs = [np.zeros(self.ng) for _ in self.VALIDITY_NAMES]
        self._L.gvh_get_validity.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        _check(self._L.gvh_get_validity(self._h, _ptr_array([a.ctypes.data for a in arrs]), len(arrs)),
               "gvh_get_validity")
        return dict(zip(self.VALIDITY_NAMES, arrs))

    def run_loop(self, nt, output_dir=None, fields=False, surface=True, tau0=None, T_fo_GeV=None,
                 T_reg_GeV=None) -> dict:
        """The reference's run loop (gvh_run_loop) from the current state: up to nt+1
        iterations, stop rule, field dumps and/or surface.dat in output_dir."""
        lat = LatticeParams.from_buffer_copy(self.lattice)
        lat.numProperTimePoints = int(nt)
        hyd = HydroParams.from_buffer_copy(self.hydro)
        if tau0 is not None:
            hyd.initialProperTimePoint = float(tau0)
        if T_fo_GeV is not None:
            hyd.freezeoutTemperatureGeV = float(T_fo_GeV)
        if T_reg_GeV is not None:
            hyd.regulationTemperatureGeV = float(T_reg_GeV)
        outputs = (GVH_RUN_FIELDS if fields else 0) | (GVH_RUN_SURFACE if surface else 0)
        rep = RunReport()
        L = self._L
        L.gvh_run_loop.argtypes = [ctypes.c_void_p, ctypes.POINTER(LatticeParams), ctypes.POINTER(HydroParams),
                                   ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(RunReport)]
        L.gvh_plugin_last_error.restype = ctypes.c_char_p
        rc = L.gvh_run_loop(self._h, ctypes.byref(lat), ctypes.byref(hyd),
                            None if output_dir is None else str(output_dir).encode(), outputs, ctypes.byref(rep))
        if rc != 0:
            raise GvhError(f"gvh_run_loop failed ({rc}): {L.gvh_plugin_last_error().decode()}")
        return {k: getattr(rep, k) for k, _ in RunReport._fields_}

    def interior(self, a):
        return np.asarray(a).reshape(self.ncz, self.ncy, self.ncx)[2:-2, 2:-2, 2:-2]

    # -- stepping ------------------------------------------------------------------------
    def step(self, t, dt, T_reg=0.0):
        _check(self._L.gvh_rk2_step(self._h, float(t), float(dt), float(T_reg)), "gvh_rk2_step")

    def max_energy_density(self) -> float:
        v = ctypes.c_double()
        _check(self._L.gvh_max_energy_density(self._h, ctypes.byref(v)), "gvh_max_energy_density")
        return v.value

    def max_propagation_speed(self) -> float:
        """Max of a / dx_axis (fm^-1) over the steps since the last call (the CFL bound)."""
        v = ctypes.c_double()
        _check(self._L.gvh_max_propagation_speed(self._h, ctypes.byref(v)), "gvh_max_propagation_speed")
        return v.value

    def set_stream(self, stream_ptr: int | None):
        """Queue this lattice's work on a caller-owned CUDA stream (raw cudaStream_t value)."""
        _check(self._L.gvh_set_stream(self._h, stream_ptr or None), "gvh_set_stream")

    def synchronize(self):
        _check(self._L.gvh_synchronize(self._h), "gvh_synchronize")

    def status(self) -> int:
        f = ctypes.c_uint(0)
        rc = self._L.gvh_status(self._h, ctypes.byref(f))
        if rc not in (0, -3):
            _check(rc, "gvh_status")
        return int(f.value)

    def clear_status(self):
        _check(self._L.gvh_clear_status(self._h), "gvh_clear_status")

    @property
    def launches_per_step(self) -> int:
        return int(self._L.gvh_launches_per_step(self._h))


# ---------------------------------------------------------------------------------------
# Batched events
# ---------------------------------------------------------------------------------------
class HotspotsC(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("x", ctypes.c_void_p), ("y", ctypes.c_void_p), ("w", ctypes.c_void_p),
                ("sigma", ctypes.c_double), ("scale", ctypes.c_double), ("eta_flat", ctypes.c_double),
                ("sigma_eta", ctypes.c_double), ("background", ctypes.c_double)]


def _hotspots_c(hs):
    """A gvh_hotspots over the arrays of a workloads.Hotspots (kept alive by the caller)."""
    x, y, w = (np.ascontiguousarray(a, dtype=np.float64) for a in (hs.x, hs.y, hs.w))
    c = HotspotsC(len(w), x.ctypes.data, y.ctypes.data, w.ctypes.data, float(hs.sigma), float(hs.scale),
                  float(hs.eta_flat), float(hs.sigma_eta), float(hs.background))
    return c, (x, y, w)


class EventInfo(ctypes.Structure):
    _fields_ = [("step", ctypes.c_longlong), ("tau", ctypes.c_double), ("max_energy_density", ctypes.c_double),
                ("freezeout_energy_density", ctypes.c_double), ("frozen_checks", ctypes.c_int),
                ("frozen_out", ctypes.c_int), ("status", ctypes.c_uint), ("cells", ctypes.c_longlong)]


BATCH_EXPORTS = [
    "gvh_batch_event_bytes", "gvh_batch_create", "gvh_batch_destroy", "gvh_batch_set_stream",
    "gvh_batch_add_event", "gvh_batch_remove_event", "gvh_batch_num_events", "gvh_batch_free_bytes",
    "gvh_batch_active_cells", "gvh_batch_step", "gvh_batch_synchronize", "gvh_batch_event_info",
    "gvh_batch_get_state", "gvh_batch_launch_config", "gvh_batch_set_grid", "gvh_batch_autotune",
    "gvh_batch_last_error", "gvh_batch_set_tile_shape", "gvh_batch_tile_shape", "gvh_batch_round",
    "gvh_batch_poll", "gvh_batch_add_event_hotspots",
]
EXPORTS += BATCH_EXPORTS


def _bind_batch(L):
    if getattr(L, "_batch_bound", False):
        return L
    vp, ip, ll = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong
    L.gvh_batch_event_bytes.argtypes = [ctypes.POINTER(LatticeParams), ctypes.POINTER(Options)]
    L.gvh_batch_event_bytes.restype = ll
    L.gvh_batch_create.argtypes = [ctypes.POINTER(Options), ll, ctypes.POINTER(vp)]
    L.gvh_batch_destroy.argtypes = [vp]
    L.gvh_batch_set_stream.argtypes = [vp, vp]
    L.gvh_batch_add_event.argtypes = [vp, ctypes.POINTER(LatticeParams), ctypes.POINTER(HydroParams), vp, ip,
                                      ctypes.POINTER(ip)]
    L.gvh_batch_remove_event.argtypes = [vp, ip]
    L.gvh_batch_add_event_hotspots.argtypes = [vp, ctypes.POINTER(LatticeParams), ctypes.POINTER(HydroParams), vp,
                                               ctypes.POINTER(ip)]
    L.gvh_batch_num_events.argtypes = [vp]
    L.gvh_batch_free_bytes.argtypes = [vp]
    L.gvh_batch_free_bytes.restype = ll
    L.gvh_batch_active_cells.argtypes = [vp]
    L.gvh_batch_active_cells.restype = ll
    L.gvh_batch_step.argtypes = [vp, ip]
    L.gvh_batch_synchronize.argtypes = [vp]
    L.gvh_batch_event_info.argtypes = [vp, ip, ctypes.POINTER(EventInfo)]
    L.gvh_batch_get_state.argtypes = [vp, ip, vp, ip]
    L.gvh_batch_launch_config.argtypes = [vp, ctypes.POINTER(ip), ctypes.POINTER(ip)]
    L.gvh_batch_set_grid.argtypes = [vp, ip]
    L.gvh_batch_autotune.argtypes = [vp, ip, ctypes.POINTER(ip)]
    L.gvh_batch_set_tile_shape.argtypes = [vp, ip]
    L.gvh_batch_tile_shape.argtypes = [vp, ctypes.POINTER(ip), ctypes.POINTER(ip)]
    L.gvh_batch_round.argtypes = [vp, ip, ctypes.POINTER(ll)]
    L.gvh_batch_poll.argtypes = [vp, ll, ip, ctypes.POINTER(ip), ctypes.POINTER(EventInfo), ctypes.POINTER(ip),
                                 ctypes.POINTER(ctypes.c_double)]
    L.gvh_batch_last_error.restype = ctypes.c_char_p
    L._batch_bound = True
    return L


def _bcheck(rc: int, what: str):
    if rc != 0:
        msg = load().gvh_batch_last_error().decode(errors="replace")
        raise GvhError(f"{what} failed ({rc}): {msg}")


GVH_ERR_NOMEM = -4


class Batch:
    """Many events in one HBM arena, advanced together by one persistent launch per stage
    and a CUDA graph per RK2 step. All events share the physics options."""

    def __init__(self, arena_bytes, conformal=False, shear=True, bulk=True, precision="fp64", theta=2.0, device=-1,
                 cartesian=False):
        self._L = _bind_batch(load())
        o = Options()
        self._L.gvh_default_options(ctypes.byref(o))
        o.eos = GVH_EOS_CONFORMAL if conformal else GVH_EOS_QCD
        o.shear, o.bulk, o.theta, o.device = int(shear), int(bulk), float(theta), int(device)
        o.precision = {"fp64": GVH_PRECISION_FP64, "mixed": GVH_PRECISION_MIXED}[precision]
        o.coordinates = GVH_COORDINATES_CARTESIAN if cartesian else GVH_COORDINATES_MILNE
        self.options = o
        self.shear, self.bulk = bool(shear), bool(bulk)
        self.qnames = q_names(self.shear, self.bulk)
        self.nq = len(self.qnames)
        self.field_names = self.qnames + PRIM_NAMES
        h = ctypes.c_void_p()
        _bcheck(self._L.gvh_batch_create(ctypes.byref(o), int(arena_bytes), ctypes.byref(h)), "gvh_batch_create")
        self._h = h
        self.events = {}

    def close(self):
        if getattr(self, "_h", None):
            self._L.gvh_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr):
        _bcheck(self._L.gvh_batch_set_stream(self._h, stream_ptr or None), "gvh_batch_set_stream")

    def event_bytes(self, nx, ny, nz) -> int:
        lat = LatticeParams(nx, ny, nz, nx + 4, ny + 4, nz + 4, 0, 1.0, 1.0, 1.0, 1.0)
        return int(self._L.gvh_batch_event_bytes(ctypes.byref(lat), ctypes.byref(self.options)))

    def add_event(self, nx, ny, nz, dx, dy, dz, dt, etabar, prim: dict, tau0=0.5, T_fo_GeV=0.15, T_reg_GeV=0.0):
        """Admit an event; returns its id, or None when the arena cannot hold it."""
        lat = LatticeParams(nx, ny, nz, nx + 4, ny + 4, nz + 4, 0, dx, dy, dz, dt)
        hyd = HydroParams(tau0, etabar, T_fo_GeV, 0, T_reg_GeV)
        ng = (nx + 4) * (ny + 4) * (nz + 4)
        order = ["e", "ut", "ux", "uy", "un"] + self.qnames[4:]
        arrs = [np.ascontiguousarray(np.broadcast_to(np.asarray(prim.get(k, 0.0), np.float64).reshape(-1), (ng,)))
                for k in order]
        eid = ctypes.c_int(-1)
        rc = self._L.gvh_batch_add_event(self._h, ctypes.byref(lat), ctypes.byref(hyd),
                                         _ptr_array([a.ctypes.data for a in arrs]), len(arrs), ctypes.byref(eid))
        if rc == GVH_ERR_NOMEM:
            return None
        _bcheck(rc, "gvh_batch_add_event")
        self.events[eid.value] = (nx, ny, nz)
        return eid.value

    def add_event_hotspots(self, nx, ny, nz, dx, dy, dz, dt, etabar, hs, tau0=0.5, T_fo_GeV=0.15, T_reg_GeV=0.0):
        """Admit an event whose initial state the device generates from hotspot sources (a
        workloads.Hotspots); returns its id, or None when the arena cannot hold it."""
        lat = LatticeParams(nx, ny, nz, nx + 4, ny + 4, nz + 4, 0, dx, dy, dz, dt)
        hyd = HydroParams(tau0, etabar, T_fo_GeV, 0, T_reg_GeV)
        c, keep = _hotspots_c(hs)
        eid = ctypes.c_int(-1)
        rc = self._L.gvh_batch_add_event_hotspots(self._h, ctypes.byref(lat), ctypes.byref(hyd), ctypes.byref(c),
                                                  ctypes.byref(eid))
        if rc == GVH_ERR_NOMEM:
            return None
        _bcheck(rc, "gvh_batch_add_event_hotspots")
        self.events[eid.value] = (nx, ny, nz)
        return eid.value

    def remove_event(self, eid):
        _bcheck(self._L.gvh_batch_remove_event(self._h, int(eid)), "gvh_batch_remove_event")
        self.events.pop(eid, None)

    def step(self, nsteps=1):
        _bcheck(self._L.gvh_batch_step(self._h, int(nsteps)), "gvh_batch_step")

    def synchronize(self):
        _bcheck(self._L.gvh_batch_synchronize(self._h), "gvh_batch_synchronize")

    def info(self, eid) -> EventInfo:
        inf = EventInfo()
        _bcheck(self._L.gvh_batch_event_info(self._h, int(eid), ctypes.byref(inf)), "gvh_batch_event_info")
        return inf

    def get_state(self, eid, names=None) -> dict:
        nx, ny, nz = self.events[eid]
        ng = (nx + 4) * (ny + 4) * (nz + 4)
        want = set(names) if names else set(self.field_names)
        arrs = [np.empty(ng) if k in want else None for k in self.field_names]
        ptrs = [None if a is None else a.ctypes.data for a in arrs]
        _bcheck(self._L.gvh_batch_get_state(self._h, int(eid), _ptr_array(ptrs), len(ptrs)), "gvh_batch_get_state")
        return {k: a for k, a in zip(self.field_names, arrs) if a is not None}

    @property
    def num_events(self) -> int:
        return int(self._L.gvh_batch_num_events(self._h))

    @property
    def free_bytes(self) -> int:
        return int(self._L.gvh_batch_free_bytes(self._h))

    @property
    def active_cells(self) -> int:
        return int(self._L.gvh_batch_active_cells(self._h))

    @property
    def grid(self) -> int:
        g, b = ctypes.c_int(), ctypes.c_int()
        self._L.gvh_batch_launch_config(self._h, ctypes.byref(g), ctypes.byref(b))
        return g.value

    def set_grid(self, g):
        _bcheck(self._L.gvh_batch_set_grid(self._h, int(g)), "gvh_batch_set_grid")

    def autotune(self, steps=2) -> int:
        g = ctypes.c_int()
        _bcheck(self._L.gvh_batch_autotune(self._h, int(steps), ctypes.byref(g)), "gvh_batch_autotune")
        return g.value

    def set_tile_shape(self, tile_x):
        _bcheck(self._L.gvh_batch_set_tile_shape(self._h, int(tile_x)), "gvh_batch_set_tile_shape")

    @property
    def tile_shape(self) -> tuple:
        x, y = ctypes.c_int(), ctypes.c_int()
        self._L.gvh_batch_tile_shape(self._h, ctypes.byref(x), ctypes.byref(y))
        return x.value, y.value

    def round(self, nsteps) -> int:
        """Queue nsteps steps of every event and a snapshot of their bookkeeping; returns a
        ticket for poll() (does not wait)."""
        t = ctypes.c_longlong()
        _bcheck(self._L.gvh_batch_round(self._h, int(nsteps), ctypes.byref(t)), "gvh_batch_round")
        return t.value

    def poll(self, ticket):
        """Wait for round `ticket`; returns ({event id: EventInfo at the round's end} for the
        events still admitted, the round's device time in ms)."""
        n = max(1, len(self.events))
        ids = (ctypes.c_int * n)()
        infos = (EventInfo * n)()
        cnt = ctypes.c_int()
        ms = ctypes.c_double()
        _bcheck(self._L.gvh_batch_poll(self._h, int(ticket), n, ids, infos, ctypes.byref(cnt), ctypes.byref(ms)),
                "gvh_batch_poll")
        return {ids[i]: infos[i] for i in range(cnt.value)}, ms.value


# ---- freeze-out hypersurface ------------------------------------------------------------

SURFACE_COLUMNS = 20
SURFACE_ROWS, SURFACE_TEXT = 1, 2  # gvh_surface_set_outputs
SURFACE_COLUMN_NAMES = ["tau", "x", "y", "eta", "dsigma_tau", "dsigma_x", "dsigma_y", "dsigma_eta", "ux", "uy",
                        "un", "e", "T", "p", "pixx", "pixy", "pixn", "piyy", "piyn", "Pi"]


class SurfaceInfo(ctypes.Structure):
    _fields_ = [("slabs", ctypes.c_longlong), ("hypercubes_last", ctypes.c_longlong),
                ("hypercubes_total", ctypes.c_longlong), ("points_last", ctypes.c_longlong),
                ("elements_last", ctypes.c_longlong), ("elements_total", ctypes.c_longlong),
                ("errors_total", ctypes.c_longlong), ("bytes_to_host_total", ctypes.c_double),
                ("device_seconds_total", ctypes.c_double), ("host_seconds_total", ctypes.c_double)]


def _bind_surface(L):
    if getattr(L, "_surface_bound", False):
        return L
    vp, dp, ll = ctypes.c_void_p, ctypes.c_double, ctypes.c_longlong
    L.gvh_surface_create.argtypes = [vp, dp, ctypes.POINTER(vp)]
    L.gvh_surface_destroy.argtypes = [vp]
    L.gvh_surface_set_threads.argtypes = [vp, ctypes.c_int]
    L.gvh_surface_set_device_rows.argtypes = [vp, ctypes.c_int]
    L.gvh_surface_set_outputs.argtypes = [vp, ctypes.c_int]
    L.gvh_surface_set_lower.argtypes = [vp]
    L.gvh_surface_find.argtypes = [vp, dp, dp, ctypes.POINTER(ll)]
    L.gvh_surface_get_rows.argtypes = [vp, ctypes.POINTER(dp), ll]
    L.gvh_surface_get_text.argtypes = [vp, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ll)]
    L.gvh_surface_get_info.argtypes = [vp, ctypes.POINTER(SurfaceInfo)]
    L.gvh_surface_last_error.restype = ctypes.c_char_p
    L.gvh_surface_slab_labels.argtypes = [ll, dp, dp, ctypes.POINTER(dp), ctypes.POINTER(dp), ctypes.POINTER(ll)]
    L.gvh_surface_slab_labels.restype = None
    L._surface_bound = True
    return L


def energy_density_of_temperature(T_GeV, conformal=False) -> float:
    """e(T) of the library's EoS in fm^-4 (the freeze-out threshold e(T_fo))."""
    L = load()
    L.gvh_energy_density_of_temperature.argtypes = [ctypes.c_int, ctypes.c_double]
    L.gvh_energy_density_of_temperature.restype = ctypes.c_double
    return float(L.gvh_energy_density_of_temperature(GVH_EOS_CONFORMAL if conformal else GVH_EOS_QCD, T_GeV))


def slab_labels(k, tau0, dtau):
    """(tau_label, tau_scale, flush_iteration) the reference gives the slab (k, k+1)."""
    L = _bind_surface(load())
    a, b, f = ctypes.c_double(), ctypes.c_double(), ctypes.c_longlong()
    L.gvh_surface_slab_labels(int(k), float(tau0), float(dtau), ctypes.byref(a), ctypes.byref(b), ctypes.byref(f))
    return a.value, b.value, f.value


class Surface:
    """Freeze-out hypersurface of a Lattice's evolution (gvh_surface_*): device marking of the
    crossed hypercubes, cornelius and the rows on the device (QCD EoS) or the host pool, rows
    in the reference's surface.dat layout."""

    def __init__(self, lattice, e_freezeout, threads=None):
        self._L = _bind_surface(load())
        self.lattice = lattice
        h = ctypes.c_void_p()
        rc = self._L.gvh_surface_create(lattice._h, float(e_freezeout), ctypes.byref(h))
        if rc != 0:
            raise GvhError(f"gvh_surface_create failed ({rc}): {self._L.gvh_surface_last_error().decode()}")
        self._h = h
        if not hasattr(lattice, "_dependents"):
            lattice._dependents = []
        lattice._dependents.append(weakref.ref(self))
        if threads:
            self._L.gvh_surface_set_threads(h, int(threads))

    def _check(self, rc, what):
        if rc != 0:
            raise GvhError(f"{what} failed ({rc}): {self._L.gvh_surface_last_error().decode()}")

    def close(self):
        if getattr(self, "_h", None):
            self._L.gvh_surface_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_lower(self):
        self._check(self._L.gvh_surface_set_lower(self._h), "gvh_surface_set_lower")

    def set_device_rows(self, on: bool):
        """Make the rows on the device (default for the QCD EoS) or with the host pool."""
        self._check(self._L.gvh_surface_set_device_rows(self._h, int(bool(on))), "gvh_surface_set_device_rows")

    def set_outputs(self, rows: bool = True, text: bool = True):
        """Keep the slab's rows, its surface.dat text, or both (the default)."""
        self._check(self._L.gvh_surface_set_outputs(self._h, (SURFACE_ROWS if rows else 0) |
                                                    (SURFACE_TEXT if text else 0)), "gvh_surface_set_outputs")

    def find(self, tau_label, tau_scale) -> int:
        n = ctypes.c_longlong()
        self._check(self._L.gvh_surface_find(self._h, float(tau_label), float(tau_scale), ctypes.byref(n)),
                    "gvh_surface_find")
        return n.value

    def rows(self) -> np.ndarray:
        n = self.info()["elements_last"]
        out = np.zeros((n, SURFACE_COLUMNS))
        self._check(self._L.gvh_surface_get_rows(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n),
                    "gvh_surface_get_rows")
        return out

    def text(self) -> str:
        p, n = ctypes.c_char_p(), ctypes.c_longlong()
        self._check(self._L.gvh_surface_get_text(self._h, ctypes.byref(p), ctypes.byref(n)), "gvh_surface_get_text")
        return ctypes.string_at(p, n.value).decode() if n.value else ""

    def info(self) -> dict:
        inf = SurfaceInfo()
        self._check(self._L.gvh_surface_get_info(self._h, ctypes.byref(inf)), "gvh_surface_get_info")
        return {k: getattr(inf, k) for k, _ in SurfaceInfo._fields_}
