"""Checkpoint and resume (gvh_save_state / gvh_load_state): a run that is saved, restored
into a fresh handle and continued gives the original run's values bit for bit; a snapshot of
another lattice, a corrupted snapshot and a truncated one are refused before the handle's
state changes."""
import numpy as np
import pytest

import gvh
from helpers import rich_state

pytestmark = pytest.mark.gpu

KW = dict(nx=12, ny=10, nz=6, dx=0.3, dy=0.3, dz=0.3, dt=0.01, etabar=0.16, theta=2.0, conformal=False, shear=True,
          bulk=True)


def _steps(L, t0, n, first):
    for k in range(first, first + n):
        L.step(t0 + k * KW["dt"], KW["dt"])


def test_resume_reproduces_the_run(tmp_path):
    path = str(tmp_path / "state.gvh")
    A = gvh.Lattice(**KW)
    A.set_primitive(rich_state(A, seed=41))
    _steps(A, 0.6, 3, 0)
    A.save(path, tau=0.6 + 3 * KW["dt"], step=3)
    _steps(A, 0.6, 4, 3)
    B = gvh.Lattice(**KW)
    tau, step = B.load(path)
    assert step == 3 and tau == 0.6 + 3 * KW["dt"]
    _steps(B, 0.6, 4, 3)
    sa, sb = A.get_state(), B.get_state()
    for k in A.field_names:
        assert np.array_equal(sa[k], sb[k]), k


def test_bad_snapshots_are_refused(tmp_path):
    path = str(tmp_path / "state.gvh")
    A = gvh.Lattice(**KW)
    A.set_primitive(rich_state(A, seed=42))
    A.save(path)
    before = A.get_state()
    other = gvh.Lattice(**dict(KW, nx=11))
    with pytest.raises(gvh.GvhError):
        other.load(path)
    raw = bytearray(open(path, "rb").read())
    raw[len(raw) // 2] ^= 0x40
    bad = str(tmp_path / "corrupt.gvh")
    open(bad, "wb").write(bytes(raw))
    with pytest.raises(gvh.GvhError):
        A.load(bad)
    short = str(tmp_path / "short.gvh")
    open(short, "wb").write(bytes(raw[: len(raw) // 3]))
    with pytest.raises(gvh.GvhError):
        A.load(short)
    after = A.get_state()
    for k in A.field_names:
        assert np.array_equal(before[k], after[k]), k
