"""Host logic of the freeze-out surface: which slab the reference writes when, with which
labels (HydroPlugin.cpp:262-314), restated here as the reference's own slot bookkeeping."""
import gvh

FOFREQ = 10


def reference_schedule(n_last, t0, dt):
    """Simulate the reference's slots: iteration n stores level n-1 (slot nFO+1, or slots 0/1
    after a swap when nFO == 0) and, when nFO == FOFREQ-1, writes hypercubes between slots it
    and it+1 for it in [start, FOFREQ). Returns {lower level: (cell_tau, t, n)}."""
    slot = [None] * (FOFREQ + 1)
    out = {}
    for n in range(1, n_last + 1):
        nfo = n % FOFREQ
        if nfo == 0:
            slot[0] = slot[FOFREQ]
            slot[1] = n - 1
        else:
            slot[nfo + 1] = n - 1
        start = 2 if n <= FOFREQ else 0
        t = t0 + (n - 1) * dt
        if nfo == FOFREQ - 1:
            for it in range(start, FOFREQ):
                lo, hi = slot[it], slot[it + 1]
                assert hi == lo + 1
                if n <= FOFREQ:
                    cell_tau = t0 + float(n - FOFREQ + (it - 1)) * dt
                else:
                    cell_tau = t0 + float(n - FOFREQ + it) * dt
                assert lo not in out
                out[lo] = (cell_tau, t, n)
    return out


def test_slab_labels_follow_the_reference_loop():
    t0, dt = 0.6, 0.01
    ref = reference_schedule(400, t0, dt)
    assert sorted(ref) == list(range(len(ref)))  # every slab is written exactly once
    for k, (cell_tau, t, n) in ref.items():
        label, scale, flush = gvh.slab_labels(k, t0, dt)
        assert flush == n, k
        assert label == cell_tau, k
        assert scale == t, k


def test_first_chunk_labels_lower_level_later_chunks_upper():
    t0, dt = 0.5, 0.02
    assert gvh.slab_labels(0, t0, dt)[0] == t0
    assert gvh.slab_labels(7, t0, dt)[:2] == (t0 + 7 * dt, t0 + 8 * dt)
    assert gvh.slab_labels(8, t0, dt)[0] == t0 + 9 * dt  # the reference's label is the upper level's time
    assert gvh.slab_labels(8, t0, dt)[2] == 19
