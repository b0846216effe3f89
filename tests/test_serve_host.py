"""Host logic of the continuous-batching server, against a fake batch (no GPU): FIFO
admission by HBM footprint, events joining a running batch, retirement at freeze-out or at
the step cap, latency bookkeeping."""
import time

import numpy as np

from gvh import serve


class FakeInfo:
    def __init__(self, step, frozen_out, cells, status=0):
        self.step, self.frozen_out, self.cells, self.status = step, frozen_out, cells, status


class FakeBatch:
    """Stands in for gvh.Batch: an arena of `capacity` bytes; an event needs
    cells * 100 bytes and freezes out after `life` steps (then stops advancing, as the
    batch's events do). Rounds run in queue order when a poll needs them, each over the
    events admitted when it was queued, as the device runs them in stream order."""

    def __init__(self, capacity, step_seconds=0.0):
        self.capacity = capacity
        self.step_seconds = step_seconds
        self.events = {}      # admitted now
        self.state = {}       # every event ever admitted (rounds in flight may still step it)
        self.next_id = 0
        self.log = []
        self.rounds = []      # [ticket, nsteps, members, snapshot or None]
        self.max_in_flight = 0

    def event_bytes(self, nx, ny, nz):
        return nx * ny * nz * 100

    @property
    def free_bytes(self):
        return self.capacity - sum(e["bytes"] for e in self.events.values())

    @property
    def active_cells(self):
        return sum(e["cells"] for e in self.events.values())

    def add_event(self, nx, ny, nz, dx, dy, dz, dt, etabar, prim, tau0, T_fo_GeV):
        need = self.event_bytes(nx, ny, nz)
        if need > self.free_bytes:
            return None
        eid = self.next_id
        self.next_id += 1
        st = dict(bytes=need, cells=nx * ny * nz, step=0, life=int(prim["life"]))
        self.events[eid] = st
        self.state[eid] = st
        self.log.append(("add", eid))
        return eid

    def remove_event(self, eid):
        self.log.append(("remove", eid))
        del self.events[eid]

    def _run(self, rnd):
        time.sleep(self.step_seconds)
        for eid in rnd[2]:
            e = self.state[eid]
            e["step"] = min(e["step"] + rnd[1], max(e["step"], e["life"]))  # frozen events stop
        rnd[3] = {eid: FakeInfo(self.state[eid]["step"], self.state[eid]["step"] >= self.state[eid]["life"],
                                self.state[eid]["cells"]) for eid in rnd[2]}

    def round(self, n):
        t = len(self.rounds)
        self.rounds.append([t, n, list(self.events), None])
        self.max_in_flight = max(self.max_in_flight, sum(1 for r in self.rounds if r[3] is None))
        return t

    def poll(self, ticket):
        for rnd in self.rounds[:ticket + 1]:
            if rnd[3] is None:
                self._run(rnd)
        snap = self.rounds[ticket][3]
        return {eid: inf for eid, inf in snap.items() if eid in self.events}, 1.0

    def synchronize(self):
        for rnd in self.rounds:
            if rnd[3] is None:
                self._run(rnd)

    def info(self, eid):
        e = self.events[eid]
        return FakeInfo(e["step"], e["step"] >= e["life"], e["cells"])

    def autotune(self, steps=1):
        return 1


def req(rid, arrival, cells_side, life, max_steps=10 ** 6):
    lat = dict(nx=cells_side, ny=cells_side, nz=1, dx=0.1, dy=0.1, dz=0.1, dt=0.01, etabar=0.2)
    return serve.Request(rid, arrival, lat, {"life": life}, max_steps=max_steps)


def test_admission_fifo_by_footprint_and_retirement():
    fb = FakeBatch(capacity=2 * 100 * 100 * 100)   # room for two 100x100 events
    reqs = [req(0, 0.0, 100, 20), req(1, 0.0, 100, 40), req(2, 0.0, 100, 10), req(3, 0.0, 10, 10)]
    srv = serve.Server(0, steps_per_round=10, batch=fb)
    out = srv.run(reqs)
    assert out["completed"] == 4 and out["frozen_out"] == 4
    assert fb.max_in_flight == 2  # the next round is queued before the host reads the last
    adds = [e for op, e in fb.log if op == "add"]
    # FIFO: request 2 waits for memory although the small request 3 would fit -- no overtaking
    first_remove = fb.log.index(("remove", 0))
    assert fb.log[:2] == [("add", 0), ("add", 1)]
    assert fb.log[first_remove + 1] == ("add", 2)
    assert len(adds) == 4
    assert out["p99_latency_s"] >= out["p50_latency_s"] >= 0


def test_step_cap_retires_event():
    fb = FakeBatch(capacity=10 ** 9)
    srv = serve.Server(0, steps_per_round=5, batch=fb)
    out = srv.run([req(0, 0.0, 10, life=10 ** 9, max_steps=25)])
    assert out["completed"] == 1 and out["frozen_out"] == 0 and out["steps"] == [25]


def test_events_join_a_running_batch():
    fb = FakeBatch(capacity=10 ** 9, step_seconds=0.01)   # event 0 runs ~0.2 s
    srv = serve.Server(0, steps_per_round=10, batch=fb)
    out = srv.run([req(0, 0.0, 10, life=200), req(1, 0.05, 10, life=20)])
    assert out["completed"] == 2
    # event 1 arrived while event 0 was resident and finished first
    removes = [e for op, e in fb.log if op == "remove"]
    assert removes == [1, 0]


def test_a_retired_slot_reused_by_a_new_event_is_not_misread():
    """A round queued before a retirement still reports the old event; the new event that
    takes its place joins later rounds and is retired by its own bookkeeping only."""
    fb = FakeBatch(capacity=100 * 10 * 10)  # room for one 10x10 event at a time
    srv = serve.Server(0, steps_per_round=10, batch=fb)
    out = srv.run([req(0, 0.0, 10, life=20), req(1, 0.0, 10, life=50)])
    assert out["completed"] == 2 and out["frozen_out"] == 2
    assert sorted(out["steps"]) == [20, 50]


def test_poisson_arrivals_rate():
    rng = np.random.default_rng(0)
    a = serve.poisson_arrivals(5.0, 4000, rng)
    assert np.all(np.diff(a) >= 0)
    assert abs(len(a) / a[-1] - 5.0) < 0.3
