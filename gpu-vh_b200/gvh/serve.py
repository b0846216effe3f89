"""Continuous-batching server for event-by-event hydro runs on one GPU.

Requests arrive over time (a Poisson stream in the benchmark). The server keeps one
`Batch` (an HBM arena on the device) and loops:

  1. admit waiting requests in arrival order while their lattice fits in the arena
     (admission by HBM footprint; a request that does not fit waits for memory to free)
     and the resident cells stay within a compute budget (beyond the cells that saturate
     the GPU, more residents only slow every event down);
  2. advance every resident event by `steps_per_round` RK2 steps (CUDA-graph replays of the
     batched step -- events admitted mid-run join the next replay, nothing restarts);
  3. read each event's bookkeeping (a few bytes per event) and retire the ones that have
     frozen out by the reference's stop rule (or hit the request's step cap), freeing
     their memory for the next admissions.

Latency of a request = completion time - arrival time. A request carries the recipe of
its initial condition (grid, impact parameter, eta/s, seed); the server generates the
initial state when it admits the request, so that generation is part of the server's time
and of the request's latency: the sources (nucleon participants) on the host, the lattice
fill on the device (gvh_batch_add_event_hotspots). The report gives events/hour
(events that reached freeze-out; events retired by a status bit or a step cap are
reported beside it as `completed`), p50/p99 latency and cell-updates/s.
"""
from __future__ import annotations

import argparse
import collections
import json
import math
import os
import sys
import time
from dataclasses import dataclass, field, replace

import numpy as np

from . import GVH_STATUS_ERRORS, Batch
from . import workloads

GRIDS = [(61, 61, 1, 0.2), (101, 101, 31, 0.15), (131, 131, 61, 0.1)]  # nx, ny, neta, dx = dy


@dataclass
class Request:
    rid: int
    arrival: float                     # seconds after the start of the run
    lattice: dict                      # nx ny nz dx dy dz dt etabar
    prim: dict | None                  # the initial state, or None: generated from `ic`
    tau0: float = 0.6
    T_fo_GeV: float = 0.150
    max_steps: int = 100000
    meta: dict = field(default_factory=dict)
    ic: tuple | None = None            # (workload, impact parameter): the generator's inputs

    def hotspots(self):
        """The request's hotspot sources (host Monte Carlo; the device fills the lattice)."""
        w, b = self.ic
        hs = workloads.hotspot_sources(w, b=b)
        self.meta = hs.meta
        return hs

    def initial_state(self) -> dict:
        """The primitive initial state, generated on first use (seeded, so the same request
        always gives the same state)."""
        if self.prim is None:
            w, b = self.ic
            prim = workloads.glauber_hotspots(w, b=b)
            self.meta = prim.pop("_meta")
            self.prim = prim
        return self.prim


@dataclass
class Completed:
    rid: int
    arrival: float
    admitted: float
    finished: float
    steps: int
    cells: int
    frozen_out: bool
    status: int

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def make_request(rid: int, arrival: float, rng: np.random.Generator, max_steps: int = 100000,
                 grids=GRIDS, eta_over_s=(0.08, 0.24), b_max=12.0, materialize: bool = True) -> Request:
    """One event of the serving mix: grid drawn from `grids`, b ~ U(0, b_max),
    eta/s ~ U(eta_over_s), Glauber-hotspot initial state, dtau = dx/10. materialize=False
    leaves the initial state to be generated at admission (Request.initial_state)."""
    nx, ny, nz, dx = grids[int(rng.integers(len(grids)))]
    etabar = float(rng.uniform(*eta_over_s))
    w = replace(workloads.CONFIG2, name=f"serve_{nx}x{ny}x{nz}", nx=nx, ny=ny, nz=nz, dx=dx, dy=dx, dz=0.1,
                dtau=dx / 10, etabar=etabar, seed=int(rng.integers(1 << 30)))
    b = float(rng.uniform(0, b_max))
    lat = dict(nx=nx, ny=ny, nz=nz, dx=dx, dy=dx, dz=0.1, dt=dx / 10, etabar=etabar)
    r = Request(rid, arrival, lat, None, tau0=w.tau0, max_steps=max_steps, ic=(w, b))
    if materialize:
        r.initial_state()
    return r


def poisson_arrivals(rate: float, n: int, rng: np.random.Generator) -> list[float]:
    return list(np.cumsum(rng.exponential(1.0 / rate, n)))


class Server:
    """The serving loop. Rounds of `steps_per_round` steps are queued `depth` ahead
    (gvh_batch_round): while the device runs round k+1 the host reads round k's bookkeeping
    from mapped memory (gvh_batch_poll), retires frozen-out events and admits new ones, whose
    set-up is queued behind the rounds in flight. Nothing on the host waits for more than the
    round it reads."""

    def __init__(self, arena_bytes: int, precision: str = "mixed", steps_per_round: int = 10, theta: float = 2.0,
                 device: int = -1, autotune: bool = False, batch=None, max_resident_cells: int = 8_000_000,
                 depth: int = 2):
        self.batch = batch if batch is not None else Batch(arena_bytes, conformal=False, shear=True, bulk=True,
                                                           precision=precision, theta=theta, device=device)
        self.steps_per_round = steps_per_round
        # Compute budget: admitting more cells than the GPU needs to be saturated only makes
        # every resident event slower (processor sharing) and raises latency for all.
        self.max_resident_cells = max_resident_cells
        self.autotune = autotune
        self.tuned = False
        self.depth = max(1, min(2, depth))  # a round's snapshot lives until two rounds later

    def run(self, requests: list[Request], time_limit: float | None = None) -> dict:
        B = self.batch
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        waiting: collections.deque[Request] = collections.deque()
        resident: dict[int, tuple[Request, float, int]] = {}  # id -> (request, admitted at, last step seen)
        in_flight: collections.deque[int] = collections.deque()
        done: list[Completed] = []
        cell_updates = 0
        t0 = time.perf_counter()
        busy = 0.0
        ic_seconds = 0.0
        while pending or waiting or resident or in_flight:
            now = time.perf_counter() - t0
            if time_limit is not None and now > time_limit:
                break
            while pending and pending[0].arrival <= now:
                waiting.append(pending.popleft())
            while waiting:
                r = waiting[0]
                need = B.event_bytes(r.lattice["nx"], r.lattice["ny"], r.lattice["nz"])
                cells = r.lattice["nx"] * r.lattice["ny"] * r.lattice["nz"]
                if need > B.free_bytes:
                    break
                if resident and B.active_cells + cells > self.max_resident_cells:
                    break
                # the initial state is generated here, inside the request's latency: its
                # sources on the host, the lattice fill on the device where the batch can
                tg = time.perf_counter()
                if r.prim is None and r.ic is not None and hasattr(B, "add_event_hotspots"):
                    eid = B.add_event_hotspots(**r.lattice, hs=r.hotspots(), tau0=r.tau0, T_fo_GeV=r.T_fo_GeV)
                else:
                    eid = B.add_event(**r.lattice, prim=r.initial_state(), tau0=r.tau0, T_fo_GeV=r.T_fo_GeV)
                ic_seconds += time.perf_counter() - tg
                if eid is None:
                    break
                waiting.popleft()
                resident[eid] = (r, time.perf_counter() - t0, 0)
            if self.autotune and not self.tuned and len(resident) > 1 and not in_flight:
                B.autotune(steps=1)
                self.tuned = True
                for eid, (r, t_adm, _) in list(resident.items()):
                    resident[eid] = (r, t_adm, int(B.info(eid).step))
            while resident and len(in_flight) < self.depth:
                in_flight.append(B.round(self.steps_per_round))
            if not in_flight:
                if pending:
                    time.sleep(max(0.0, min(pending[0].arrival - now, 0.05)))
                continue
            infos, ms = B.poll(in_flight.popleft())
            busy += ms / 1e3
            now = time.perf_counter() - t0
            for eid, inf in infos.items():
                if eid not in resident:
                    continue
                r, t_adm, last = resident[eid]
                cell_updates += (int(inf.step) - last) * int(inf.cells)
                resident[eid] = (r, t_adm, int(inf.step))
                if inf.frozen_out or inf.step >= r.max_steps or (inf.status & GVH_STATUS_ERRORS):
                    done.append(Completed(r.rid, r.arrival, t_adm, now, int(inf.step), int(inf.cells),
                                          bool(inf.frozen_out), int(inf.status)))
                    B.remove_event(eid)
                    del resident[eid]
        B.synchronize()
        elapsed = time.perf_counter() - t0
        out = summarize(done, elapsed, cell_updates, busy)
        out["initial_state_seconds"] = ic_seconds
        out["rounds_in_flight"] = self.depth
        return out


def summarize(done: list[Completed], elapsed: float, cell_updates: int, busy: float) -> dict:
    """events_per_hour counts the events that reached freeze-out; `completed` also counts
    those retired by a status bit (NaN) or by the request's step cap."""
    lat = np.array([c.latency for c in done]) if done else np.array([float("nan")])
    frozen = sum(c.frozen_out for c in done)
    return {
        "completed": len(done),
        "frozen_out": frozen,
        "elapsed_s": elapsed,
        "events_per_hour": frozen / elapsed * 3600.0 if elapsed > 0 else 0.0,
        "completed_per_hour": len(done) / elapsed * 3600.0 if elapsed > 0 else 0.0,
        "p50_latency_s": float(np.percentile(lat, 50)),
        "p99_latency_s": float(np.percentile(lat, 99)),
        "cell_updates_per_s": cell_updates / elapsed if elapsed > 0 else 0.0,
        "gpu_busy_fraction": busy / elapsed if elapsed > 0 else 0.0,
        "steps": [c.steps for c in done],
        "statuses": sorted(set(c.status for c in done)),
    }


def main(argv=None):
    ap = argparse.ArgumentParser(description="continuous-batching hydro server on a Poisson request stream")
    ap.add_argument("--rate", type=float, default=2.0, help="requests per second")
    ap.add_argument("--requests", type=int, default=16)
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--arena-gb", type=float, default=40.0)
    ap.add_argument("--steps-per-round", type=int, default=10)
    ap.add_argument("--max-steps", type=int, default=100000)
    ap.add_argument("--time-limit", type=float, default=None)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--autotune", action="store_true")
    ap.add_argument("--max-resident-cells", type=int, default=8_000_000)
    args = ap.parse_args(argv)
    rng = np.random.default_rng(args.seed)
    arrivals = poisson_arrivals(args.rate, args.requests, rng)
    reqs = [make_request(i, a, rng, args.max_steps, materialize=False) for i, a in enumerate(arrivals)]
    srv = Server(int(args.arena_gb * (1 << 30)), precision=args.precision, steps_per_round=args.steps_per_round,
                 autotune=args.autotune, max_resident_cells=args.max_resident_cells)
    out = srv.run(reqs, time_limit=args.time_limit)
    out.update({"rate": args.rate, "requests": args.requests, "precision": args.precision, "seed": args.seed})
    out.pop("steps", None)
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
