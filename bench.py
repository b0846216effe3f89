"""Benchmark of the KT RK2 step (gpu-vh's hot path) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step" = one Heun RK2 step over the whole lattice): the full single event of
the benchmark configuration -- 131x131x61 cells, dx = dy = deta = 0.1, tau0 = 0.6,
dtau = 0.01, QCD equation of state, eta/s = 0.16, shear + bulk, plain FP64, on a seeded
Glauber-hotspot initial state (synthetic, see gvh/workloads.py). Metric: cell-updates/s
(one interior cell advanced by one full RK2 step). With N GPUs each rank advances its own
event (different seed): independent events, no collective in the step (weak scaling).

Timing: W untimed warm-up steps, then K steps bracketed by barrier + synchronize, timed
with CUDA events on the stream the kernels run on; the job time is the max over ranks.
The lattice state (~380 MB) is larger than L2 (126 MB), so no flush is needed between
steps. `e2e` times the same step through the C ABI with host buffers: each step copies the
full state from pinned host memory to the device (gvh_set_state_async), steps, and copies
it back (gvh_get_state_async); the copies run on the handle's two copy streams, so the
next state's copy in and the last state's copy out overlap the step. The blocking
gvh_set_state / gvh_get_state loop is reported beside it (`serial_ms_per_step`).

--impl reference times the reference's own KT step (its rhic/src sources compiled for the
CPU by oracle/build_ref.py, OpenMP over the launch grid) on the host cores; beside it
(`reference_gpu`) the reference's own CUDA build, as shipped in FP32 and in FP64, on the
full event on this GPU.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "gpu-vh_b200"))

import numpy as np  # noqa: E402

from gvh import workloads  # noqa: E402

METRIC = "cell-updates/s"
HBM_FALLBACK_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serving-sweep", default="1,16,50",
                    help="offered request rates (req/s) of the serving sweep; empty to skip")
    ap.add_argument("--serving-sweep-seconds", type=float, default=20.0)
    ap.add_argument("--no-surface", dest="surface", action="store_false",
                    help="skip the freeze-out surface extras (event to freeze-out with surface.dat, "
                         "mixed-vs-FP64 report)")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the mixed-precision, event-to-freeze-out and serving measurements")
    ap.add_argument("--serving-seconds", type=float, default=45.0)
    ap.add_argument("--serving-rate", type=float, default=4.0)
    ap.add_argument("--batch64-seconds", type=float, default=120.0,
                    help="time limit of the 64-event batched run (0 skips it)")
    ap.add_argument("--stage-case", default="", choices=["", "fp64", "mixed", "config1"],
                    help="only --warmup + --steps RK2 steps of the 131x131x61 event in this precision, "
                         "or of the 33x33x17 configuration (config1, FP64: the split stage kernel's "
                         "case), for profiling the stage kernels; prints one JSON line")
    ap.add_argument("--surface-slabs", type=int, default=0,
                    help="only the freeze-out surface of N slabs of the 131x131x61 event after "
                         "300 steps (text only, as the run loop keeps it); for profiling its kernels")
    return ap.parse_args()


def dist_info():
    from gvh import dist as gdist

    return gdist.rank_info()


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return HBM_FALLBACK_GBS, "fallback"


def bytes_per_cell_update(nq: int) -> int:
    """Algorithmic bytes of one cell-update (both stages), FP64: stage 1 reads q^n (nq), e,
    u^n (4), u^{n-1} (4) and writes q* (nq), e*, u* (4); stage 2 reads q* (nq), e*, u* (4),
    u^n (4), q^n (nq) and writes q^{n+1} (nq), e, u (4): 5 nq + 28 values. Pressure is a
    function of e and is not counted."""
    return (5 * nq + 28) * 8


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.dev)], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_event(w, rank):
    import dataclasses

    from gvh import dist as gdist

    w = dataclasses.replace(w, seed=gdist.event_seed(w.seed, rank))
    prim = workloads.glauber_hotspots(w)
    meta = prim.pop("_meta")
    return w, prim, meta


def central_planes(w, prim, nz_s):
    """The nz_s rapidity planes around eta = 0 of a ghosted event, as a ghosted sub-lattice."""
    k0 = (w.nz - nz_s) // 2
    ncx, ncy = w.nx + 4, w.ny + 4
    return {key: np.asarray(v).reshape(w.nz + 4, ncy, ncx)[k0: k0 + nz_s + 4].reshape(-1) if np.ndim(v) else v
            for key, v in prim.items()}


def cpu_baseline(w, prim, budget_s=20.0):
    """The oracle (this project's C restatement, OpenMP) timed on the host cores on a bounded
    sample of the workload: the first nz_s rapidity planes of the same event, sized so the
    timed steps take about budget_s."""
    import oracle

    threads = os.cpu_count() or 1
    kw = w.lattice_kwargs()

    def run(nz_s, steps):
        k = dict(kw, nz=nz_s)
        L = oracle.OracleLattice(**k)
        ncx, ncy = w.nx + 4, w.ny + 4
        L.set_primitive(central_planes(w, prim, nz_s))
        t0 = time.perf_counter()
        t = w.tau0
        for n in range(steps):
            L.step(t, w.dtau)
            t = w.tau0 + (n + 1) * w.dtau
        return time.perf_counter() - t0

    probe_nz = 2
    dt_probe = run(probe_nz, 1)
    per_cell = dt_probe / (w.nx * w.ny * probe_nz)
    nz_s = int(max(2, min(w.nz, budget_s / 2 / max(per_cell * w.nx * w.ny, 1e-9))))
    steps = 2
    el = run(nz_s, steps)
    cells = w.nx * w.ny * nz_s
    return {"value": cells * steps / el, "unit": METRIC, "cores": threads, "kind": "port",
            "sample": f"oracle (kt_oracle.c, OpenMP {threads} threads): {steps} RK2 steps of the first {nz_s} of "
                      f"{w.nz} rapidity planes of the same event ({cells} cells), {el:.1f} s"}


def run_reference(args):
    """Reference arm: the reference's own KT step built for the CPU, all host threads."""
    rank, world, local = dist_info()
    if rank != 0:
        return 0
    w = workloads.CONFIG2
    import oracle

    if not oracle.ref_available("fp64_qcd_bulk"):
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU build oracle/_ref/libref_fp64_qcd_bulk.so "
                                                              "missing (build needs the reference tree)"}))
        return 0
    w, prim, meta = make_event(w, 0)
    threads = os.cpu_count() or 1
    kw = w.lattice_kwargs()
    ncx, ncy = w.nx + 4, w.ny + 4
    # size the per-step sample so the whole run (warm-up + steps) ends within ~3 minutes
    total_budget = 180.0
    n_calls = args.warmup + args.steps

    def make(nz_s):
        R = oracle.RefLattice(threads=threads, **dict(kw, nz=nz_s))
        R.set_primitive(central_planes(w, prim, nz_s))
        return R

    R = make(2)
    t0 = time.perf_counter()
    R.step(w.tau0, w.dtau)
    per_cell = (time.perf_counter() - t0) / (w.nx * w.ny * 2)
    nz_s = int(max(2, min(w.nz, total_budget / max(n_calls, 1) / max(per_cell * w.nx * w.ny, 1e-9))))
    R = make(nz_s)
    t = w.tau0
    for n in range(args.warmup):
        R.step(t, w.dtau)
        t += w.dtau
    t0 = time.perf_counter()
    for n in range(args.steps):
        R.step(t, w.dtau)
        t += w.dtau
    el = time.perf_counter() - t0
    cells = w.nx * w.ny * nz_s
    value = cells * args.steps / el
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": w.name, "lattice": [w.nx, w.ny, w.nz], "sample_lattice": [w.nx, w.ny, nz_s],
                   "eos": "qcd", "shear": True, "bulk": True, "theta": w.theta, "impact_b_fm": meta["b"]},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "reference",
                         "sample": f"reference rhic/src KT step built for the CPU (g++ -O2, OpenMP {threads} threads) "
                                   f"on the central {nz_s} of {w.nz} rapidity planes of the event"},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    gpu = reference_gpu_timings(args, w, prim)
    if gpu:
        line["reference_gpu"] = gpu
    # the 33x33x17 conformal configuration: its 100 steps, on the host cores and on this GPU
    w1 = workloads.CONFIG1
    prim1 = workloads.gaussian_profile(w1)
    if oracle.ref_available("fp64_conf_shear"):
        R1 = oracle.RefLattice(threads=threads, **w1.lattice_kwargs())
        R1.set_primitive(prim1)
        t0 = time.perf_counter()
        t = w1.tau0
        for n in range(w1.steps):
            R1.step(t, w1.dtau)
            t = w1.tau0 + (n + 1) * w1.dtau
        el1 = time.perf_counter() - t0
        c1 = w1.nx * w1.ny * w1.nz
        line["config1"] = {"workload": w1.name, "steps": w1.steps,
                           "cpu": {"ms_per_step": el1 / w1.steps * 1e3, "cell_updates_per_s": c1 * w1.steps / el1,
                                   "cores": threads},
                           "gpu": reference_gpu_timings(argparse.Namespace(steps=w1.steps, warmup=5), w1, prim1)}
    print(json.dumps(line))
    return 0


def reference_gpu_timings(args, w, prim):
    """The reference's own CUDA build (oracle/ref_gpu_driver.cu: its allocation, set-up and
    twoStepRungeKutta, compiled with nvcc for sm_100a) on the full event on this GPU, as
    shipped (FP32) and with the PRECISION double overlay: W warm-up steps, then K steps timed
    with CUDA events. Reported beside the CPU arm; {} without a GPU or the builds."""
    import oracle

    try:
        import torch

        if not torch.cuda.is_available():
            return {}
    except ImportError:
        return {}
    out = {}
    kw = w.lattice_kwargs()
    cells = w.nx * w.ny * w.nz
    for prec in ("fp32", "fp64"):
        variant = oracle.ref_gpu_variant(prec, w.conformal, w.shear, w.bulk, w.theta)
        if not oracle.ref_gpu_available(variant):
            continue
        R = oracle.RefGpuLattice(precision=prec, **kw)
        R.set_primitive(prim)
        if args.warmup:
            R.time_steps(args.warmup, w.tau0, w.dtau)
        ms = R.time_steps(args.steps, w.tau0 + args.warmup * w.dtau, w.dtau)
        out[prec] = {"ms_per_step": ms / args.steps, "cell_updates_per_s": cells * args.steps / (ms / 1e3),
                     "build": f"reference rhic/src, nvcc sm_100a, PRECISION {'double' if prec == 'fp64' else 'float'}",
                     "timing": "CUDA events around the reference's own twoStepRungeKutta loop (legacy stream)"}
    return out


def dropin_seam_timings(args, w, prim):
    """The drop-in twoStepRungeKutta (gpu-vh_b200/dropin/twoStepRungeKutta_gvh.cu) built into
    the reference's own program in place of FullyDiscreteKurganovTadmorScheme.cu and driven
    by the reference's own loop (oracle/ref_gpu_driver.cu): per step one gather of its device
    arrays into libgvh, the two stage launches, one scatter back and the reference's closing
    cudaDeviceSynchronize. W warm-up steps, then K steps timed with CUDA events on the legacy
    stream; both the FP64 build and the as-shipped FP32 build. {} without the builds."""
    import oracle

    out = {}
    kw = w.lattice_kwargs()
    cells = w.nx * w.ny * w.nz
    for prec in ("fp64", "fp32"):
        variant = oracle.ref_gpu_variant(prec, w.conformal, w.shear, w.bulk, w.theta)
        if not oracle.ref_gpu_available(variant, dropin=True):
            continue
        D = oracle.RefGpuLattice(precision=prec, dropin=True, **kw)
        D.set_primitive(prim)
        if args.warmup:
            D.time_steps(args.warmup, w.tau0, w.dtau)
        ms = D.time_steps(args.steps, w.tau0 + args.warmup * w.dtau, w.dtau)
        out[prec] = {"ms_per_step": ms / args.steps, "cell_updates_per_s": cells * args.steps / (ms / 1e3),
                     "build": f"reference rhic/src with the drop-in twoStepRungeKutta, PRECISION "
                              f"{'double' if prec == 'fp64' else 'float'}",
                     "timing": "CUDA events around the reference's own step loop (legacy stream)"}
    return out


def time_steps(L, w, steps, warmup, stream):
    """ms per RK2 step of lattice L (CUDA events on its stream)."""
    import torch

    t = w.tau0
    for n in range(warmup):
        L.step(t, w.dtau)
        t += w.dtau
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for n in range(steps):
        L.step(t, w.dtau)
        t += w.dtau
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def event_to_freezeout(w, prim, precision, device, max_steps=6000, surface_dir=None):
    """One event on the single-lattice path, run the way the reference's loop runs it:
    before every step test max e against e(T_fo) (device reduction), stop after 11 all-frozen
    checks (HydroPlugin.cpp:396-413). With surface_dir, the library's own run loop
    (gvh_run_loop) also finds the freeze-out surface of every slab (device marking, host
    cornelius) and writes surface.dat there in the reference's chunks of 10 steps.
    Returns steps, seconds, status (and the surface's figures)."""
    import gvh

    L = gvh.Lattice(device=device, precision=precision, tau0=w.tau0, T_fo_GeV=w.T_fo_GeV, **w.lattice_kwargs())
    L.set_primitive(prim)
    L.synchronize()
    if surface_dir:
        t0 = time.perf_counter()
        rep = L.run_loop(max_steps, output_dir=surface_dir, surface=True)
        el = time.perf_counter() - t0
        ng = (w.nx + 4) * (w.ny + 4) * (w.nz + 4)
        slabs = max(1, rep["steps"])
        out = {"steps": rep["steps"], "seconds": el, "frozen_out": bool(rep["frozen_out"]), "status": rep["status"],
               "tau_end": rep["tau_end"],
               "surface": {"elements_written": rep["surface_elements"],
                           "hypercubes_crossed_per_slab_mean": rep["surface_hypercubes"] / slabs,
                           "finder_seconds": rep["surface_seconds"],
                           "host_cornelius_seconds": rep["surface_host_seconds"],
                           "bytes_to_host_per_step": rep["surface_bytes_to_host"] / slabs,
                           # copyDeviceToHostMemory: 30 ghosted arrays every step
                           # (HydroPlugin.cpp:264, DynamicalVariables.cu)
                           "reference_bytes_to_host_per_step": 30 * ng * 8,
                           "file_bytes": os.path.getsize(os.path.join(surface_dir, "surface.dat")),
                           "host_threads": os.cpu_count()}}
        L.close()
        return out
    e_fo = gvh.energy_density_of_temperature(w.T_fo_GeV, conformal=w.conformal)
    t0 = time.perf_counter()
    frozen, n, t = 0, 0, w.tau0
    while n < max_steps:
        if L.max_energy_density() <= e_fo:
            frozen += 1
        if frozen >= 11:
            break
        L.step(t, w.dtau)
        n += 1
        t = w.tau0 + n * w.dtau
    L.synchronize()
    el = time.perf_counter() - t0
    st = L.status()
    L.close()
    return {"steps": n, "seconds": el, "frozen_out": frozen >= 11, "status": st, "tau_end": t}


def precision_report(device):
    """Mixed precision against FP64 on the config-1 event (33x33x17, conformal, shear): the
    L2 and Linf relative errors of e, u^mu and pi^{mu nu}/(e+p) at steps 100, 500 and at
    freeze-out, and the total freeze-out sum of tau*dsigma_mu (surface.dat columns 5-8) of each
    run. The FP64 path is the reference's FP64 build to 1e-12 (tests/test_parity_gpu.py)."""
    import gvh

    w = workloads.CONFIG1
    prim = workloads.gaussian_profile(w)
    e_fo = gvh.energy_density_of_temperature(w.T_fo_GeV, conformal=w.conformal)
    runs = {}
    for prec in ("fp64", "mixed"):
        L = gvh.Lattice(device=device, precision=prec, **w.lattice_kwargs())
        L.set_primitive(prim)
        S = gvh.Surface(L, e_fo)
        S.set_lower()
        runs[prec] = {"L": L, "S": S, "dsigma": np.zeros(4), "frozen": 0, "done": False, "steps": 0}
    snaps = {}
    t, n = w.tau0, 0
    pin = ["pixx", "pixy", "pixn", "piyy", "piyn", "pitt", "pitx", "pity", "pitn", "pinn"]

    def snapshot(tag):
        snaps[tag] = {}
        for prec, r in runs.items():
            st = r["L"].get_state()
            g = {k: r["L"].interior(st[k]) for k in ["e", "p", "ut", "ux", "uy", "un"] + pin}
            snaps[tag][prec] = g

    while n < 3000 and not all(r["done"] for r in runs.values()):
        it = n + 1
        for r in runs.values():
            if r["done"]:
                continue
            if it >= 2:
                label, scale, flush = gvh.slab_labels(it - 2, w.tau0, w.dtau)
                r["S"].find(label, scale)
                rows = r["S"].rows()
                r.setdefault("pending", []).append(rows[:, 4:8].sum(axis=0) if len(rows) else np.zeros(4))
                if flush == it:
                    r["dsigma"] += np.sum(r["pending"], axis=0)
                    r["pending"] = []
            if r["L"].max_energy_density() <= e_fo:
                r["frozen"] += 1
            if r["frozen"] >= 11:
                r["done"], r["steps"] = True, n
        if n in (100, 500):
            snapshot(f"step_{n}")
        if runs["fp64"]["done"] and "freezeout" not in snaps:
            snapshot("freezeout")
        for r in runs.values():
            if not r["done"]:
                r["L"].step(t, w.dtau)
        n += 1
        t = w.tau0 + n * w.dtau

    def errs(a, b):
        d = (a - b).ravel()
        return {"l2": float(np.linalg.norm(d) / max(np.linalg.norm(b.ravel()), 1e-300)),
                "linf": float(np.max(np.abs(d)) / max(np.max(np.abs(b)), 1e-300))}

    report = {"workload": w.name, "fp64_freezeout_step": runs["fp64"]["steps"],
              "mixed_freezeout_step": runs["mixed"]["steps"]}
    for tag, sn in snaps.items():
        a, b = sn["mixed"], sn["fp64"]
        u_a = np.stack([a[k] for k in ("ut", "ux", "uy", "un")])
        u_b = np.stack([b[k] for k in ("ut", "ux", "uy", "un")])
        pa = np.stack([a[k] / (a["e"] + a["p"]) for k in pin])
        pb = np.stack([b[k] / (b["e"] + b["p"]) for k in pin])
        report[tag] = {"e": errs(a["e"], b["e"]), "u": errs(u_a, u_b), "pi_over_e_plus_p": errs(pa, pb)}
    d64, dmx = runs["fp64"]["dsigma"], runs["mixed"]["dsigma"]
    report["total_dsigma_fp64"] = d64.tolist()
    report["total_dsigma_mixed"] = dmx.tolist()
    report["total_dsigma_rel_err"] = float(np.max(np.abs(dmx - d64)) / max(np.max(np.abs(d64)), 1e-300))
    for r in runs.values():
        r["S"].close()
        r["L"].close()
    return report


def serving_mix_requests(n, seed=64):
    """n seeded requests of the serving mix, all offered at time 0, initial states not yet
    generated (the path that runs them generates each inside its own timing)."""
    from gvh import serve

    rng = np.random.default_rng(seed)
    return [serve.make_request(i, 0.0, rng, materialize=False) for i in range(n)]


def fp64_single_path_requests(reqs, device, max_steps=6000):
    """The plain FP64 single-event path on the given requests, one after another: generate
    the initial state (the sources on the host, the lattice fill on the device, as the serving
    path does), run the event alone on a gvh.Lattice the way the reference's loop runs it (max
    e against e(T_fo) before every step, stop after 11 all-frozen checks,
    HydroPlugin.cpp:396-413), or until a NaN status bit retires it. events_per_hour counts
    the events that reached freeze-out over the total time."""
    import gvh

    runs = []
    total = 0.0
    for r in reqs:
        t0 = time.perf_counter()
        lat = r.lattice
        L = gvh.Lattice(device=device, precision="fp64", nx=lat["nx"], ny=lat["ny"], nz=lat["nz"], dx=lat["dx"],
                        dy=lat["dy"], dz=lat["dz"], dt=lat["dt"], etabar=lat["etabar"], theta=2.0, conformal=False,
                        shear=True, bulk=True, tau0=r.tau0, T_fo_GeV=r.T_fo_GeV)
        L.set_hotspots(r.hotspots())
        e_fo = gvh.energy_density_of_temperature(r.T_fo_GeV, conformal=False)
        frozen, n, t, st = 0, 0, r.tau0, 0
        while n < max_steps:
            if L.max_energy_density() <= e_fo:
                frozen += 1
            if frozen >= 11:
                break
            if n % 10 == 0:
                st = L.status()
                if st & gvh.GVH_STATUS_ERRORS:
                    break
            L.step(t, lat["dt"])
            n += 1
            t = r.tau0 + n * lat["dt"]
        st = L.status()
        L.close()
        el = time.perf_counter() - t0
        total += el
        runs.append({"grid": [lat["nx"], lat["ny"], lat["nz"]], "steps": n, "seconds": el, "frozen_out": frozen >= 11,
                     "status": st})
    frozen_n = sum(x["frozen_out"] for x in runs)
    return {"events": len(runs), "frozen_out": frozen_n, "seconds": total,
            "events_per_hour": 3600.0 * frozen_n / total if total > 0 else None,
            "completed_per_hour": 3600.0 * len(runs) / total if total > 0 else None,
            "statuses": sorted(set(x["status"] for x in runs)),
            "per_grid_mean_seconds": {f"{g[0]}x{g[1]}x{g[2]}": float(np.mean([x["seconds"] for x in runs
                                                                              if tuple(x["grid"]) == g]))
                                      for g in sorted(set(tuple(x["grid"]) for x in runs))},
            "path": "gvh.Lattice, plain FP64, one event at a time, initial state generated inside the timing "
                    "(sources on the host, lattice fill on the device)"}


def serving_run(args, device, rate=None, seconds=None):
    from gvh import serve

    rate = args.serving_rate if rate is None else rate
    seconds = args.serving_seconds if seconds is None else seconds
    rng = np.random.default_rng(2024)
    n_req = max(8, int(rate * seconds))
    arrivals = serve.poisson_arrivals(rate, n_req, rng)
    reqs = [serve.make_request(i, a, rng, materialize=False) for i, a in enumerate(arrivals)]
    srv = serve.Server(int(60 * (1 << 30)), precision="mixed", steps_per_round=10, device=device)
    out = srv.run(reqs, time_limit=seconds)
    out.pop("steps", None)
    out.update({"rate_per_s": rate, "requests_offered": n_req, "precision": "mixed",
                "mix": "grids {61x61x1 @0.2 fm, 101x101x31 @0.15, 131x131x61 @0.1}, b~U(0,12), eta/s~U(0.08,0.24)"})
    return out


def batch64_run(args, device, fp64_same):
    """The batched configuration: 64 seeded events of the serving mix (grids
    {61x61x1, 101x101x31, 131x131x61}, b ~ U(0, 12) fm, eta/s ~ U(0.08, 0.24), QCD, shear +
    bulk, mixed precision) all offered at once to one batch (CUDA graph per step, tiles
    autotuned), run until every event has frozen out, initial states generated at admission.
    Beside it, the plain FP64 single-event path run on the same 64 events (fp64_same, from
    fp64_single_path_requests)."""
    from gvh import serve

    reqs = serving_mix_requests(64)
    srv = serve.Server(int(60 * (1 << 30)), precision="mixed", steps_per_round=10, device=device, autotune=True)
    out = srv.run(reqs, time_limit=args.batch64_seconds)
    out.pop("steps", None)
    out["events"] = len(reqs)
    grids = sorted(set((r.lattice["nx"], r.lattice["ny"], r.lattice["nz"]) for r in reqs))
    out["grids"] = {f"{g[0]}x{g[1]}x{g[2]}": sum(1 for r in reqs if (r.lattice["nx"], r.lattice["ny"],
                                                                     r.lattice["nz"]) == g) for g in grids}
    if fp64_same and fp64_same.get("events") == len(reqs):
        out["fp64_single_path_seconds_same_events"] = fp64_same["seconds"]
        out["fp64_single_path_events_per_hour"] = fp64_same["events_per_hour"]
        if out.get("events_per_hour") and fp64_same.get("events_per_hour"):
            out["events_per_hour_vs_fp64_single_path"] = out["events_per_hour"] / fp64_same["events_per_hour"]
    return out


def run_ours(args):
    import torch

    import gvh

    rank, world, local = dist_info()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    w, prim, meta = make_event(workloads.CONFIG2, rank)
    L = gvh.Lattice(device=local, **w.lattice_kwargs())
    L.set_primitive(prim)
    stream = torch.cuda.Stream(device=local)
    L.set_stream(stream.cuda_stream)
    t = w.tau0
    n_done = 0

    def step():
        nonlocal t, n_done
        L.step(t, w.dtau)
        n_done += 1
        t = w.tau0 + n_done * w.dtau

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        with torch.cuda.stream(stream):
            ev0.record(stream)
            for _ in range(args.steps):
                step()
            ev1.record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    flags = L.status()
    if flags & gvh.GVH_STATUS_ERRORS:
        raise RuntimeError(f"status flags {flags} raised during the timed steps")
    from gvh import dist as gdist

    ms_max = gdist.max_over_ranks(ms, dist, device=torch.device("cuda", local))
    cells = w.cells
    value = gdist.job_value(cells, args.steps, world, ms_max)
    launches = L.launches_per_step * args.steps

    # end to end through the C ABI with pinned host buffers
    e2e = None
    n_fields = len(L.field_names)
    host_in = torch.empty((n_fields, L.ng), dtype=torch.float64, pin_memory=True)
    host_out = torch.empty((n_fields, L.ng), dtype=torch.float64, pin_memory=True)
    st = L.get_state()
    for f, k in enumerate(L.field_names):
        host_in[f].copy_(torch.from_numpy(st[k]))
    ptr_in = [host_in[f].data_ptr() for f in range(n_fields)]
    ptr_out = [host_out[f].data_ptr() for f in range(n_fields)]
    L.set_stream(None)
    L.set_stream(stream.cuda_stream)

    def e2e_loop(pipelined: bool, n: int) -> float:
        """n steps, each: the state in from pinned host memory, one RK2 step, the state out.
        Pipelined: gvh_set_state_async / gvh_get_state_async, so that the next state's copy
        in, this step and the last state's copy out overlap; otherwise the blocking calls."""
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        if pipelined:
            L.join_async()
            for _ in range(n):
                L.set_state_async_ptrs(ptr_in)
                step()
                L.get_state_async_ptrs(ptr_out)
            L.join_async()
        else:
            for _ in range(n):
                L.set_state_ptrs(ptr_in)
                step()
                L.get_state_ptrs(ptr_out)
        e1.record(stream)
        L.synchronize()
        torch.cuda.synchronize()
        return gdist.max_over_ranks(e0.elapsed_time(e1), dist, device=torch.device("cuda", local))

    e2e_loop(True, 3)
    e2e_loop(False, 3)
    ms_e2e = e2e_loop(True, args.e2e_steps)
    ms_serial = e2e_loop(False, args.e2e_steps)
    bytes_io = n_fields * L.ng * 8
    e2e = {"value": gdist.job_value(cells, args.e2e_steps, world, ms_e2e), "unit": METRIC,
           "h2d_bytes_per_step": bytes_io, "d2h_bytes_per_step": bytes_io,
           "ms_per_step": ms_e2e / args.e2e_steps, "steps": args.e2e_steps,
           "calls": "gvh_set_state_async + gvh_rk2_step + gvh_get_state_async (pipelined)",
           "serial_ms_per_step": ms_serial / args.e2e_steps}

    peak, peak_kind = measured_peaks()
    b_cell = bytes_per_cell_update(L.nq)
    achieved = cells * b_cell / (ms / args.steps / 1e3) / 1e9
    traffic = None
    fp64_pipe = None
    tp = os.path.join(ROOT, "profiles", "kt_stage_traffic.json")
    if os.path.exists(tp):
        try:
            prof = json.load(open(tp))
            traffic = prof.get("bytes_per_step")
            fp64_pipe = prof.get("fp64_pipe_active_pct")
        except Exception:
            traffic = None
    # One step is the kernel's two launches (stage 1 + stage 2): achieved, traffic and the
    # algorithmic bytes are all per step. The kernel's real limit is FP64 issue, so the FP64
    # pipe's busy fraction from the same capture is given beside the HBM roofline.
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "peak_source": peak_kind,
                "algorithmic_bytes_per_step": cells * b_cell,
                "per": "step (2 launches of kt_stage_kernel)",
                "fp64_pipe_active_pct": fp64_pipe,
                "kernel": "kt_stage_kernel (stage 1 + stage 2 per step)"}

    extras = {}
    if rank == 0 and world == 1 and not args.no_extras:
        import gvh as _g

        Lm = _g.Lattice(device=local, precision="mixed", **w.lattice_kwargs())
        Lm.set_primitive(prim)
        Lm.set_stream(stream.cuda_stream)
        ms_mixed = time_steps(Lm, w, max(5, args.steps // 2), 3, stream)
        Lm.close()
        extras["mixed_cell_updates_per_s"] = cells / (ms_mixed / 1e3)
        extras["mixed_ms_per_step"] = ms_mixed
        # the same FP64 step with the validity diagnostics on (the reference's checkValidity,
        # which its step runs every time; opt-in here, one kernel after stage 2)
        Lv = _g.Lattice(device=local, **w.lattice_kwargs())
        Lv.set_primitive(prim)
        Lv.set_stream(stream.cuda_stream)
        Lv.enable_validity(True)
        ms_val = time_steps(Lv, w, max(5, args.steps // 2), 3, stream)
        Lv.close()
        extras["fp64_with_validity"] = {"ms_per_step": ms_val, "cell_updates_per_s": cells / (ms_val / 1e3),
                                        "validity_ms_per_step": ms_val - ms_max / args.steps}
        # the 33x33x17 conformal configuration (its 100 steps, after 5 warm-up steps)
        w1 = workloads.CONFIG1
        L1 = _g.Lattice(device=local, **w1.lattice_kwargs())
        L1.set_primitive(workloads.gaussian_profile(w1))
        L1.set_stream(stream.cuda_stream)
        ms1 = time_steps(L1, w1, w1.steps, 5, stream)
        L1.close()
        extras["config1_fp64"] = {"workload": w1.name, "ms_per_step": ms1,
                                  "cell_updates_per_s": w1.nx * w1.ny * w1.nz / (ms1 / 1e3), "steps": w1.steps}
        if rank == 0 and world == 1:
            try:
                extras["dropin_seam"] = dropin_seam_timings(args, w, prim)
            except Exception as ex:  # reported beside the arm, never required
                extras["dropin_seam"] = {"error": str(ex)}
        ev = event_to_freezeout(w, prim, "fp64", local)
        ev["events_per_hour"] = 3600.0 / ev["seconds"] if ev["seconds"] > 0 else None
        extras["fp64_single_event_to_freezeout"] = ev
        if args.surface:
            import tempfile

            with tempfile.TemporaryDirectory() as td:
                evs = event_to_freezeout(w, prim, "fp64", local, surface_dir=td)
            evs["events_per_hour"] = 3600.0 / evs["seconds"] if evs["seconds"] > 0 else None
            extras["fp64_single_event_to_freezeout_with_surface"] = evs
            extras["mixed_vs_fp64_config1"] = precision_report(local)
        if args.serving_seconds > 0:
            # the plain FP64 single-event path on the serving mix: the 64 seeded events of the
            # batched configuration (16 when that run is skipped), each run alone to freeze-out
            fp64_mix = fp64_single_path_requests(serving_mix_requests(64 if args.batch64_seconds > 0 else 16), local)
            extras["fp64_single_event_path_on_serving_mix"] = fp64_mix
            sv = serving_run(args, local)
            if fp64_mix.get("events_per_hour"):
                sv["events_per_hour_vs_fp64_single_path"] = sv["events_per_hour"] / fp64_mix["events_per_hour"]
            extras["batched_mixed_serving"] = sv
            if args.batch64_seconds > 0:
                extras["batched_64_events"] = batch64_run(args, local, fp64_mix)
            # the offered-rate sweep of the serving configuration (1-50 req/s), shorter windows
            sweep = []
            for rate in [float(r) for r in args.serving_sweep.split(",") if r.strip()]:
                r = serving_run(args, local, rate=rate, seconds=args.serving_sweep_seconds)
                sweep.append({k: r.get(k) for k in ("rate_per_s", "requests_offered", "completed", "frozen_out",
                                                    "elapsed_s", "events_per_hour", "p50_latency_s",
                                                    "p99_latency_s", "cell_updates_per_s", "gpu_busy_fraction")})
            if sweep:
                extras["serving_rate_sweep"] = sweep

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(w, prim)
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"value": None, "unit": METRIC, "cores": os.cpu_count(), "kind": "port", "sample": f"failed: {ex}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": w.name, "lattice": [w.nx, w.ny, w.nz], "spacing_fm": [w.dx, w.dy, w.dz],
                       "tau0": w.tau0, "dtau": w.dtau, "eos": "qcd", "eta_over_s": w.etabar, "shear": True,
                       "bulk": True, "theta": w.theta, "precision": "fp64", "events": world,
                       "impact_b_fm": meta["b"], "n_part": meta["n_part"],
                       "l2_policy": "state (~%.0f MB) larger than L2; no flush" % (L.ng * (2 * L.nq + 15) * 8 / 1e6),
                       "parallelism": f"events x{world}"},
            "e2e": e2e, "gpu_launches": launches, "roofline": roofline, "cpu_baseline": cpu,
            "clocks": clocks.summary(),
            "extras": extras,
        }
        print(json.dumps(line))
    L.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def stage_case(precision, steps, warmup):
    """W + K steps of the benchmark event on one lattice in the given precision, timed with
    CUDA events over the K steps (the profiling case of the stage kernel)."""
    import torch

    import gvh

    if precision == "config1":
        # the 33x33x17 conformal configuration in FP64 (the split kernel's case)
        w, prim = workloads.CONFIG1, workloads.gaussian_profile(workloads.CONFIG1)
        L = gvh.Lattice(device=0, precision="fp64", **w.lattice_kwargs())
    else:
        w, prim, _ = make_event(workloads.CONFIG2, 0)
        L = gvh.Lattice(device=0, precision=precision, **w.lattice_kwargs())
    L.set_primitive(prim)
    stream = torch.cuda.Stream()
    L.set_stream(stream.cuda_stream)
    ms = time_steps(L, w, steps, warmup, stream)
    print(json.dumps({"stage_case": precision, "steps": steps, "warmup": warmup, "ms_per_step": ms,
                      "status": L.status()}))
    L.close()
    return 0


def surface_slabs(n_slabs, warm_steps=300):
    """The surface of n_slabs consecutive slabs of the benchmark event, taken after
    warm_steps steps (where the surface is about 47 k crossed hypercubes a slab): step, then
    find the slab, as the run loop does; one JSON line with the slabs' wall time."""
    import gvh

    w, prim, _ = make_event(workloads.CONFIG2, 0)
    L = gvh.Lattice(device=0, precision="fp64", tau0=w.tau0, T_fo_GeV=w.T_fo_GeV, **w.lattice_kwargs())
    L.set_primitive(prim)
    t = w.tau0
    for _ in range(warm_steps):
        L.step(t, w.dtau)
        t += w.dtau
    S = gvh.Surface(L, gvh.energy_density_of_temperature(w.T_fo_GeV))
    S.set_outputs(rows=False, text=True)
    S.set_lower()
    L.synchronize()
    t0 = time.perf_counter()
    elements = 0
    for k in range(n_slabs):
        L.step(t, w.dtau)
        t += w.dtau
        label, scale, _ = gvh.slab_labels(warm_steps + k, w.tau0, w.dtau)
        elements += S.find(label, scale)
    S.text()
    el = time.perf_counter() - t0
    info = S.info()
    print(json.dumps({"surface_slabs": n_slabs, "seconds": el, "elements": elements,
                      "hypercubes_per_slab": info["hypercubes_total"] / max(1, n_slabs),
                      "bytes_to_host_per_slab": info["bytes_to_host_total"] / max(1, n_slabs)}))
    S.close()
    L.close()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.surface_slabs > 0:
        return surface_slabs(args.surface_slabs)
    if args.stage_case:
        return stage_case(args.stage_case, args.steps, args.warmup)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
