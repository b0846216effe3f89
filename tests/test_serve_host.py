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
    cells * 100 bytes and freezes out after `life` steps."""

    def __init__(self, capacity, step_seconds=0.0):
        self.capacity = capacity
        self.step_seconds = step_seconds
        self.events = {}
        self.next_id = 0
        self.log = []

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
        self.events[eid] = dict(bytes=need, cells=nx * ny * nz, step=0, life=int(prim["life"]))
        self.log.append(("add", eid))
        return eid

    def remove_event(self, eid):
        self.log.append(("remove", eid))
        del self.events[eid]

    def step(self, n):
        time.sleep(self.step_seconds)
        for e in self.events.values():
            e["step"] += n

    def synchronize(self):
        pass

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


def test_poisson_arrivals_rate():
    rng = np.random.default_rng(0)
    a = serve.poisson_arrivals(5.0, 4000, rng)
    assert np.all(np.diff(a) >= 0)
    assert abs(len(a) / a[-1] - 5.0) < 0.3
