"""Batched engine (many events, one persistent launch per stage, a CUDA graph per step):
each event advances as it would alone, freeze-out follows the reference's stop rule, and
admission/removal keep the other events intact."""
import numpy as np
import pytest

import gvh
from helpers import rich_state

pytestmark = pytest.mark.gpu

SHAPES = [(9, 8, 5), (40, 17, 1), (6, 11, 9)]


class _Geo:
    def __init__(self, nx, ny, nz, shear=True, bulk=True):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.ncx, self.ncy, self.ncz = nx + 4, ny + 4, nz + 4
        self.shear, self.bulk = shear, bulk


def interior(shape, a):
    nx, ny, nz = shape
    return np.asarray(a).reshape(nz + 4, ny + 4, nx + 4)[2:-2, 2:-2, 2:-2]


def make_events(conformal, shear, bulk):
    evs = []
    for n, (nx, ny, nz) in enumerate(SHAPES):
        prim = rich_state(_Geo(nx, ny, nz, shear, bulk), seed=20 + n)
        kw = dict(nx=nx, ny=ny, nz=nz, dx=0.3, dy=0.25, dz=0.3, dt=0.01 + 0.005 * n, etabar=0.12 + 0.04 * n)
        evs.append((kw, prim, 0.5 + 0.1 * n))
    return evs


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("conformal,shear,bulk", [(False, True, True), (True, True, False), (True, False, False)])
def test_event_same_alone_and_in_batch(precision, conformal, shear, bulk):
    evs = make_events(conformal, shear, bulk)
    B = gvh.Batch(1 << 26, conformal=conformal, shear=shear, bulk=bulk, precision=precision)
    ids = [B.add_event(**kw, prim=prim, tau0=t0) for kw, prim, t0 in evs]
    steps = 6
    B.step(steps)
    for eid, (kw, prim, t0) in zip(ids, evs):
        L = gvh.Lattice(conformal=conformal, shear=shear, bulk=bulk, precision=precision, **kw)
        L.set_primitive(prim)
        t = t0
        for n in range(1, steps + 1):
            L.step(t, kw["dt"])
            t = t0 + n * kw["dt"]
        alone = L.get_state()
        inb = B.get_state(eid)
        info = B.info(eid)
        assert info.step == steps and info.status == 0
        assert abs(info.tau - (t0 + steps * kw["dt"])) < 1e-12
        shape = (kw["nx"], kw["ny"], kw["nz"])
        for k in L.field_names:
            a, b = interior(shape, alone[k]), interior(shape, inb[k])
            # Same code on the same inputs, compiled into two kernels whose multiply-add
            # contraction may differ: FP64 agrees to 1e-12, the mixed path to FP32 rounding
            # (1e-6, far inside its 1e-4 accuracy bar against the FP64 oracle).
            tol = 1e-12 if precision == "fp64" else 1e-6
            scale = max(np.abs(a).max(), 1e-300)
            assert np.abs(a - b).max() / scale <= tol, (k, np.abs(a - b).max() / scale)
        assert np.isclose(info.max_energy_density, interior(shape, inb["e"]).max(), rtol=1e-15)


def test_cartesian_event_same_alone_and_in_batch():
    """A batch in Cartesian coordinates (the reference's USE_CARTESIAN_COORDINATES) advances
    each event as a Cartesian single lattice does, and differently from Milne."""
    evs = make_events(True, True, False)
    B = gvh.Batch(1 << 26, conformal=True, shear=True, bulk=False, cartesian=True)
    ids = [B.add_event(**kw, prim=prim, tau0=t0) for kw, prim, t0 in evs]
    B.step(4)
    for eid, (kw, prim, t0) in zip(ids, evs):
        out = {}
        for cart in (True, False):
            L = gvh.Lattice(conformal=True, shear=True, bulk=False, cartesian=cart, **kw)
            L.set_primitive(prim)
            for n in range(4):
                L.step(t0 + n * kw["dt"], kw["dt"])
            out[cart] = L.get_state()
        inb = B.get_state(eid)
        shape = (kw["nx"], kw["ny"], kw["nz"])
        for k in ("ttt", "ttx", "pixx", "e"):
            a, b, m = (interior(shape, out[True][k]), interior(shape, inb[k]), interior(shape, out[False][k]))
            scale = np.abs(a).max()
            assert np.abs(a - b).max() <= 1e-12 * scale, k
        assert np.abs(interior(shape, out[True]["ttt"]) - interior(shape, out[False]["ttt"])).max() > 1e-3


def test_freezeout_stop_rule():
    """Below e(T_fo) from the start: the initial check counts, then one per step; the event
    is frozen out after 11 checks (FOFREQ+1), as the reference's run loop stops."""
    geo = _Geo(7, 7, 3, True, False)
    prim = rich_state(geo, seed=3, e0=0.05, emin=0.01)
    B = gvh.Batch(1 << 24, conformal=True, shear=True, bulk=False)
    eid = B.add_event(7, 7, 3, 0.3, 0.3, 0.3, 0.01, 0.2, prim, tau0=0.6, T_fo_GeV=0.15)
    inf = B.info(eid)
    assert inf.frozen_checks == 1 and not inf.frozen_out
    B.step(9)
    assert B.info(eid).frozen_checks == 10 and not B.info(eid).frozen_out
    B.step(1)
    assert B.info(eid).frozen_out
    # a frozen-out event is not advanced further (the reference's loop ends there)
    frozen = B.get_state(eid)
    B.step(4)
    assert B.info(eid).step == 10
    after = B.get_state(eid)
    for k in frozen:
        np.testing.assert_array_equal(frozen[k], after[k])


def test_hot_event_is_not_frozen():
    geo = _Geo(7, 7, 3, True, False)
    B = gvh.Batch(1 << 24, conformal=True, shear=True, bulk=False)
    eid = B.add_event(7, 7, 3, 0.3, 0.3, 0.3, 0.01, 0.2, rich_state(geo, seed=3), tau0=0.6)
    B.step(3)
    inf = B.info(eid)
    assert inf.frozen_checks == 0 and inf.max_energy_density > inf.freezeout_energy_density


def test_admission_by_footprint_and_removal():
    evs = make_events(False, True, True)
    B = gvh.Batch(1 << 26, precision="mixed")
    need = [B.event_bytes(kw["nx"], kw["ny"], kw["nz"]) for kw, _, _ in evs]
    small = gvh.Batch(need[0] + need[2] + 1024, precision="mixed")
    ids = [small.add_event(**kw, prim=prim, tau0=t0) for kw, prim, t0 in evs]
    assert ids[0] is not None and ids[1] is None and ids[2] is not None  # event 1 did not fit
    small.step(3)
    ref = small.get_state(ids[2])
    small.remove_event(ids[0])
    again = small.add_event(**evs[0][0], prim=evs[0][1], tau0=evs[0][2])
    assert again is not None and small.num_events == 2
    # the event that stayed is untouched by the removal and re-admission
    after = small.get_state(ids[2])
    for k in ref:
        np.testing.assert_array_equal(ref[k], after[k])
    small.step(2)
    assert small.info(ids[2]).step == 5 and small.info(again).step == 2


def test_autotune_does_not_change_results():
    evs = make_events(False, True, True)
    A = gvh.Batch(1 << 26, precision="mixed")
    B = gvh.Batch(1 << 26, precision="mixed")
    ida = [A.add_event(**kw, prim=prim, tau0=t0) for kw, prim, t0 in evs]
    idb = [B.add_event(**kw, prim=prim, tau0=t0) for kw, prim, t0 in evs]
    g = B.autotune(steps=1)  # advances B by (candidates + 1) x 1 steps
    assert g >= 0  # 0 = one block per tile
    nb = B.info(idb[0]).step
    A.step(nb)
    for ea, eb in zip(ida, idb):
        sa, sb = A.get_state(ea), B.get_state(eb)
        for k in sa:
            np.testing.assert_array_equal(sa[k], sb[k])


def _alone(kw, prim, t0, steps, precision, conformal=False, shear=True, bulk=True):
    L = gvh.Lattice(conformal=conformal, shear=shear, bulk=bulk, precision=precision, **kw)
    L.set_primitive(prim)
    t = t0
    for n in range(1, steps + 1):
        L.step(t, kw["dt"])
        t = t0 + n * kw["dt"]
    return L.get_state()


def _close(shape, alone, inb, names, tol):
    for k in names:
        a, b = interior(shape, alone[k]), interior(shape, inb[k])
        scale = max(np.abs(a).max(), 1e-300)
        assert np.abs(a - b).max() / scale <= tol, (k, np.abs(a - b).max() / scale)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_event_admitted_mid_flight_is_the_same_as_alone(precision):
    """Serving: event 0 runs for a while; event 1 is admitted while rounds are in flight (its
    set-up queued behind them), event 2 after event 0 has been retired and its memory reused.
    Each event's result equals the same event run alone on a gvh.Lattice for the same number
    of steps (1e-12 FP64, 1e-6 mixed: the same per-cell code in two kernels)."""
    evs = make_events(False, True, True)
    B = gvh.Batch(1 << 26, precision=precision)
    tol = 1e-12 if precision == "fp64" else 1e-6
    e0 = B.add_event(**evs[0][0], prim=evs[0][1], tau0=evs[0][2])
    t_a = B.round(3)
    t_b = B.round(3)
    e1 = B.add_event(**evs[1][0], prim=evs[1][1], tau0=evs[1][2])  # while two rounds are in flight
    infos, ms = B.poll(t_a)
    assert set(infos) == {e0} and infos[e0].step == 3 and ms > 0
    t_c = B.round(4)
    infos, _ = B.poll(t_b)
    assert set(infos) == {e0} and infos[e0].step == 6
    infos, _ = B.poll(t_c)
    assert infos[e0].step == 10 and infos[e1].step == 4
    st0 = B.get_state(e0)
    B.remove_event(e0)
    e2 = B.add_event(**evs[2][0], prim=evs[2][1], tau0=evs[2][2])
    t_d = B.round(5)
    infos, _ = B.poll(t_d)
    assert infos[e1].step == 9 and infos[e2].step == 5
    for eid, (kw, prim, t0), steps, state in [(e0, evs[0], 10, st0), (e1, evs[1], 9, None),
                                              (e2, evs[2], 5, None)]:
        alone = _alone(kw, prim, t0, steps, precision)
        _close((kw["nx"], kw["ny"], kw["nz"]), alone, state if state is not None else B.get_state(eid),
               B.field_names, tol)


def test_poll_does_not_report_a_slot_refilled_after_its_round():
    evs = make_events(False, True, True)
    B = gvh.Batch(1 << 26, precision="fp64")
    x = B.add_event(**evs[0][0], prim=evs[0][1], tau0=evs[0][2])
    t = B.round(2)
    B.remove_event(x)
    y = B.add_event(**evs[2][0], prim=evs[2][1], tau0=evs[2][2])
    assert y == x  # the slot is reused at once (the round in flight runs before the new set-up)
    infos, _ = B.poll(t)
    assert infos == {}
    t2 = B.round(3)
    infos, _ = B.poll(t2)
    assert list(infos) == [y] and infos[y].step == 3
    kw, prim, t0 = evs[2]
    _close((kw["nx"], kw["ny"], kw["nz"]), _alone(kw, prim, t0, 3, "fp64"), B.get_state(y), B.field_names, 1e-12)
    # a snapshot two rounds old is gone
    t3, t4 = B.round(1), B.round(1)
    with pytest.raises(gvh.GvhError):
        B.poll(t2)
    B.poll(t3)
    B.poll(t4)


@pytest.mark.parametrize("tile_x", [32, 16, 8])
def test_tile_shapes_compute_the_same_values(tile_x):
    evs = make_events(False, True, True)
    A = gvh.Batch(1 << 26, precision="fp64")
    B = gvh.Batch(1 << 26, precision="fp64")
    B.set_tile_shape(tile_x)
    assert B.tile_shape == (tile_x, 128 // tile_x)
    ida = [A.add_event(**kw, prim=prim, tau0=t0) for kw, prim, t0 in evs]
    idb = [B.add_event(**kw, prim=prim, tau0=t0) for kw, prim, t0 in evs]
    A.step(4)
    B.step(4)
    for ea, eb in zip(ida, idb):
        sa, sb = A.get_state(ea), B.get_state(eb)
        for k in sa:
            np.testing.assert_array_equal(sa[k], sb[k])


def test_empty_batch_and_bad_ids():
    """A batch with no events steps and serves rounds as no-ops; ids that were never admitted
    or were removed are refused; the last event removed leaves an empty batch that admits
    again."""
    B = gvh.Batch(1 << 26, precision="fp64")
    assert B.num_events == 0
    B.step(3)
    t0 = B.round(2)
    t1 = B.round(2)
    infos, ms = B.poll(t0)
    assert infos == {} and ms >= 0
    infos, _ = B.poll(t1)
    assert infos == {}
    for bad in (-1, 0, 7):
        with pytest.raises(gvh.GvhError):
            B.remove_event(bad)
    kw, prim, t0_ev = make_events(False, True, True)[0]
    eid = B.add_event(**kw, prim=prim, tau0=t0_ev)
    assert eid is not None and B.num_events == 1
    B.step(1)
    B.remove_event(eid)
    with pytest.raises(gvh.GvhError):
        B.remove_event(eid)
    assert B.num_events == 0
    B.step(2)
    again = B.add_event(**kw, prim=prim, tau0=t0_ev)
    B.step(1)
    assert B.info(again).step == 1
