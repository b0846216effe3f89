"""The CUDA step against the reference's OWN CUDA build on the same GPU.

oracle/ref_gpu_driver.cu runs the reference's allocation, launch set-up, initial-state path
and twoStepRungeKutta (FullyDiscreteKurganovTadmorScheme.cu:109-139), compiled by nvcc
from its sources with the PRECISION double overlay (and as shipped, in FP32). Tolerances as
in test_parity_gpu.py: per field, max over cells |cuda - ref| / max over cells |ref|, 1e-12
on the conformal configuration after 100 steps and 1e-9 with the QCD equation of state (the
Newton stop test of EnergyMomentumTensor.cu:39). The FP32 build agrees only to single
precision; it is checked loosely (FP32_TOL) so that its timing in the benchmark's reference
arm stands for a build that computes the same event.

Each variant library keeps one lattice in globals (as the reference does), so each is used
at one size per process.
"""
import dataclasses

import numpy as np
import pytest

import gvh
import oracle
from gvh import workloads
from helpers import rel_err

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12
QCD_TOL = 1e-9
FP32_TOL = 1e-3


def _need(variant):
    if not oracle.ref_gpu_available(variant):
        pytest.skip(f"reference CUDA build {variant} not built (oracle/build_ref.py needs the reference tree)")


def _run_both(w, prim, steps, precision="fp64"):
    kw = w.lattice_kwargs()
    G = gvh.Lattice(**kw)
    R = oracle.RefGpuLattice(precision=precision, **kw)
    G.set_primitive(prim)
    R.set_primitive(prim)
    t = w.tau0
    for n in range(1, steps + 1):
        G.step(t, w.dtau)
        R.step(t, w.dtau)
        t = w.tau0 + n * w.dtau
    assert G.status() == 0
    return G, G.get_state(), R.get_state()


def test_config1_100_steps_matches_reference_cuda_fp64():
    """33x33x17, conformal, shear, theta 1.8, 100 steps: the plain FP64 path against the
    reference's own FP64 CUDA build."""
    w = workloads.CONFIG1
    _need(oracle.ref_gpu_variant("fp64", w.conformal, w.shear, w.bulk, w.theta))
    G, sg, sr = _run_both(w, workloads.gaussian_profile(w), w.steps)
    for k in G.field_names:
        err = rel_err(G.interior(sg[k]), G.interior(sr[k]))
        assert err <= REL_TOL, f"{k}: {err:.3e}"


def test_benchmark_event_matches_reference_cuda_fp64():
    """The 131x131x61 QCD + bulk hotspot event of the benchmark, 5 steps, against the
    reference's own FP64 CUDA build."""
    w = workloads.CONFIG2
    _need(oracle.ref_gpu_variant("fp64", w.conformal, w.shear, w.bulk, w.theta))
    prim = workloads.glauber_hotspots(w)
    prim.pop("_meta")
    G, sg, sr = _run_both(w, prim, 5)
    for k in G.field_names:
        err = rel_err(G.interior(sg[k]), G.interior(sr[k]))
        assert err <= QCD_TOL, f"{k}: {err:.3e}"


@pytest.mark.parametrize("which", ["config1", "config2"])
def test_reference_cuda_fp32_build_tracks_the_event(which):
    """The as-shipped FP32 build computes the same event to single precision (e and u after
    5 steps)."""
    w = workloads.CONFIG1 if which == "config1" else workloads.CONFIG2
    _need(oracle.ref_gpu_variant("fp32", w.conformal, w.shear, w.bulk, w.theta))
    if which == "config1":
        prim = workloads.gaussian_profile(w)
    else:
        prim = workloads.glauber_hotspots(w)
        prim.pop("_meta")
    G, sg, sr = _run_both(w, prim, 5, precision="fp32")
    for k in ["e", "ut", "ux", "uy", "un"]:
        err = rel_err(G.interior(sg[k]), G.interior(sr[k]))
        assert err <= FP32_TOL, f"{k}: {err:.3e}"
