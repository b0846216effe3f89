"""The drop-in twoStepRungeKutta run inside the reference's own program.

gpu-vh_b200/dropin/twoStepRungeKutta_gvh.cu is compiled into the reference's rhic/src in
place of FullyDiscreteKurganovTadmorScheme.cu and linked against libgvh.so
(oracle/build_ref.py, DROPIN_VARIANTS). oracle/ref_gpu_driver.cu then runs the reference's
own allocation, launch set-up, initial-state path and step loop (twoStepRungeKutta followed
by setCurrentConservedVariables, HydroPlugin.cpp:414-422), so every step goes through the
seam: the reference's device arrays gathered into libgvh, libgvh's fused step, the result
scattered back into d_Q, d_e, d_p, d_u with d_up = u^n and ghost cells filled.

Compared with the reference's unmodified FP64 CUDA build on the same inputs: per field, max
over interior cells |dropin - ref| / max |ref| <= 1e-12 on the conformal configuration
(33x33x17, theta 1.8) after its 100 steps, and <= 1e-9 on the 131x131x61 QCD + bulk event
(the Newton stop test, EnergyMomentumTensor.cu:39, as in test_ref_gpu.py). The ghost faces
the reference's setGhostCells writes (GhostCells.cu:15-144) are compared too.
"""
import numpy as np
import pytest

import oracle
from gvh import workloads
from helpers import rel_err

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12
QCD_TOL = 1e-9


def _need(variant):
    if not oracle.ref_gpu_available(variant):
        pytest.skip(f"reference CUDA build {variant} not built")
    if not oracle.ref_gpu_available(variant, dropin=True):
        pytest.skip(f"drop-in build {variant} not built")


def _faces(L, a):
    """The six ghost faces' interior-facing layers (not edges or corners, which the
    reference leaves as they were)."""
    g = np.asarray(a).reshape(L.ncz, L.ncy, L.ncx)
    return np.concatenate([g[2:-2, 2:-2, :2].ravel(), g[2:-2, 2:-2, -2:].ravel(), g[2:-2, :2, 2:-2].ravel(),
                           g[2:-2, -2:, 2:-2].ravel(), g[:2, 2:-2, 2:-2].ravel(), g[-2:, 2:-2, 2:-2].ravel()])


def _run(w, prim, steps, precision="fp64"):
    kw = w.lattice_kwargs()
    D = oracle.RefGpuLattice(precision=precision, dropin=True, **kw)
    R = oracle.RefGpuLattice(precision=precision, **kw)
    D.set_primitive(prim)
    R.set_primitive(prim)
    t = w.tau0
    for n in range(1, steps + 1):
        D.step(t, w.dtau)
        R.step(t, w.dtau)
        t = w.tau0 + n * w.dtau
    return D, D.get_state(), R.get_state()


def test_dropin_config1_100_steps_matches_reference_fp64():
    w = workloads.CONFIG1
    _need(oracle.ref_gpu_variant("fp64", w.conformal, w.shear, w.bulk, w.theta))
    D, sd, sr = _run(w, workloads.gaussian_profile(w), w.steps)
    for k in D.field_names:
        err = rel_err(D.interior(sd[k]), D.interior(sr[k]))
        assert err <= REL_TOL, f"{k}: {err:.3e}"
        assert rel_err(_faces(D, sd[k]), _faces(D, sr[k])) <= REL_TOL, k


def test_dropin_benchmark_event_matches_reference_fp64():
    w = workloads.CONFIG2
    _need(oracle.ref_gpu_variant("fp64", w.conformal, w.shear, w.bulk, w.theta))
    prim = workloads.glauber_hotspots(w)
    prim.pop("_meta")
    D, sd, sr = _run(w, prim, 5)
    for k in D.field_names:
        err = rel_err(D.interior(sd[k]), D.interior(sr[k]))
        assert err <= QCD_TOL, f"{k}: {err:.3e}"


def test_dropin_in_the_as_shipped_fp32_program():
    """The as-shipped FP32 program with the drop-in: libgvh steps in FP64 on the widened
    state and narrows the result, so it tracks the reference's FP32 step to single
    precision (e and u after 5 steps)."""
    w = workloads.CONFIG2
    _need(oracle.ref_gpu_variant("fp32", w.conformal, w.shear, w.bulk, w.theta))
    prim = workloads.glauber_hotspots(w)
    prim.pop("_meta")
    D, sd, sr = _run(w, prim, 5, precision="fp32")
    for k in ["e", "ut", "ux", "uy", "un"]:
        err = rel_err(D.interior(sd[k]), D.interior(sr[k]))
        assert err <= 1e-3, f"{k}: {err:.3e}"
