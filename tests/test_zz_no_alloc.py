"""The allocation-free RK2 step (gvh_rk2_step_noalloc) against the handle path.

gvh_rk2_step_noalloc is for callers that own all their device memory and cannot let the
library allocate at step time (a fixed memory plan, a pool allocator that forbids foreign
cudaMalloc, a region where allocating would synchronise the device). It takes the state in
caller-owned device arrays and keeps its intermediate RK stage in a fixed-size array
compiled into the library. Here the caller's arrays are torch CUDA tensors allocated by
the test, and two consecutive steps must agree with gvh_rk2_step on the same state within
the FP64 parity tolerance of the other GPU tests (1e-12 relative).

This file is collected last on purpose (test_zz_*): if it fails, a run that stops at the
first failure has already run every other test. It must also pass alone in a fresh
process, where its first call performs the library's one-time device set-up.
"""
import ctypes

import numpy as np
import pytest

import gvh
from helpers import rich_state

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12
# The handle runs small lattices on its split stage kernel (four warps per 32 cells), the
# allocation-free step on the one-thread-per-cell kernel: the same code compiled into two
# kernels, whose multiply-add contraction of the mixed path's FP32 arithmetic may differ. The
# mixed path's bar, as between a batched event and the same event alone (far inside its 1e-4
# accuracy against the FP64 oracle).
MIXED_TOL = 1e-6


def bound():
    L = gvh.load()
    vp, dp = ctypes.c_void_p, ctypes.c_double
    L.gvh_rk2_step_noalloc.argtypes = [ctypes.POINTER(gvh.LatticeParams), ctypes.POINTER(gvh.HydroParams),
                                       ctypes.POINTER(gvh.Options), dp, dp, dp, vp, vp, vp, vp, vp, vp,
                                       ctypes.POINTER(ctypes.c_uint), vp]
    L.gvh_rk2_step_noalloc_max_bytes.restype = ctypes.c_longlong
    L.gvh_noalloc_last_error.restype = ctypes.c_char_p
    return L


def stack(G, state, names):
    """Interior-only, component-stacked copy (cell s = i + nx*(j + ny*k))."""
    return np.stack([G.interior(state[k]).reshape(-1) for k in names])


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


HBARC = 0.197326938

# (eos, shear, bulk, T_reg [fm^-1], state kwargs[, Cartesian coordinates]): the scratch holds
# nq + 5 values per cell, so each component count (4, 14, 15) lays it out differently;
# T_reg > 0 on a state with large pi regulates cells (the regulation branch of the stage
# kernel); the last case takes the options' Cartesian coordinates through the same call.
CASES = {
    "qcd_shear_bulk": (False, True, True, 0.0, dict(seed=31)),
    "qcd_shear": (False, True, False, 0.0, dict(seed=32)),
    "conformal_ideal": (True, False, False, 0.0, dict(seed=33)),
    "conformal_shear": (True, True, False, 0.0, dict(seed=34)),
    "qcd_shear_regulated": (False, True, False, 0.5 / HBARC, dict(seed=35, pi=0.3)),
    "conformal_shear_cartesian": (True, True, False, 0.0, dict(seed=36), True),
}


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", list(CASES))
def test_noalloc_step_matches_handle_on_two_calls(case, precision):
    import torch

    conformal, shear, bulk, T_reg, st_kw, *cart = CASES[case]
    L = bound()
    kw = dict(nx=12, ny=10, nz=7, dx=0.3, dy=0.3, dz=0.3, dt=0.01, etabar=0.16, theta=2.0, conformal=conformal,
              shear=shear, bulk=bulk, cartesian=bool(cart and cart[0]))
    G = gvh.Lattice(precision=precision, **kw)
    G.set_primitive(rich_state(G, **st_kw))
    s = G.get_state()
    dev = torch.device("cuda", torch.cuda.current_device())
    q = torch.tensor(stack(G, s, G.qnames), device=dev).contiguous()
    e = torch.tensor(G.interior(s["e"]).reshape(-1), device=dev).contiguous()
    p = torch.tensor(G.interior(s["p"]).reshape(-1), device=dev).contiguous()
    u_prev = torch.tensor(stack(G, s, ["utp", "uxp", "uyp", "unp"]), device=dev).contiguous()
    u = torch.tensor(stack(G, s, ["ut", "ux", "uy", "un"]), device=dev).contiguous()
    u_next = torch.empty_like(u)
    stream = torch.cuda.current_stream(dev).cuda_stream
    opts = gvh.Options()
    ctypes.memmove(ctypes.byref(opts), ctypes.byref(G.options), ctypes.sizeof(opts))
    opts.device = dev.index  # an explicit device: the call must leave the caller's current
    t = 0.5
    for call in range(2):
        status = ctypes.c_uint(123)
        before = torch.cuda.current_device()
        rc = L.gvh_rk2_step_noalloc(ctypes.byref(G.lattice), ctypes.byref(G.hydro), ctypes.byref(opts), t,
                                    kw["dt"], T_reg, q.data_ptr(), e.data_ptr(), p.data_ptr(), u_prev.data_ptr(),
                                    u.data_ptr(), u_next.data_ptr(), ctypes.byref(status), stream)
        assert rc == 0, L.gvh_noalloc_last_error()
        assert torch.cuda.current_device() == before
        G.clear_status()
        G.step(t, kw["dt"], T_reg)
        assert status.value == G.status(), (call, status.value, G.status())
        ref = G.get_state()
        torch.cuda.synchronize()
        tol = REL_TOL if precision == "fp64" else MIXED_TOL
        for n, name in enumerate(G.qnames):
            assert rel(q[n].cpu().numpy(), G.interior(ref[name]).reshape(-1)) <= tol, (call, name)
        assert rel(e.cpu().numpy(), G.interior(ref["e"]).reshape(-1)) <= tol
        assert rel(p.cpu().numpy(), G.interior(ref["p"]).reshape(-1)) <= tol
        for m, name in enumerate(["ut", "ux", "uy", "un"]):
            assert rel(u_next[m].cpu().numpy(), G.interior(ref[name]).reshape(-1)) <= tol, (call, name)
        # next step: u^n becomes the previous level, u^{n+1} the current one
        u_prev, u, u_next = u, u_next, u_prev
        t = 0.5 + (call + 1) * kw["dt"]
    if T_reg > 0 and shear:
        # the case is meant to regulate: the regulated run differs from an unregulated one
        H = gvh.Lattice(precision=precision, **kw)
        H.set_primitive(rich_state(H, **st_kw))
        H.step(0.5, kw["dt"])
        H.step(0.5 + kw["dt"], kw["dt"])
        free = H.get_state()
        assert rel(q[8].cpu().numpy(), H.interior(free["pixx"]).reshape(-1)) > 1e-6


def test_noalloc_rejects_lattices_beyond_its_scratch():
    import torch

    L = bound()
    limit = L.gvh_rk2_step_noalloc_max_bytes()
    assert limit == 32 << 20
    nx = ny = 131
    nz = 61  # ~1e6 cells x 20 values: far beyond 32 MiB
    lat = gvh.LatticeParams(nx, ny, nz, nx + 4, ny + 4, nz + 4, 0, 0.1, 0.1, 0.1, 0.01)
    hyd = gvh.HydroParams(0.6, 0.16, 0.15, 0, 0.0)
    o = gvh.Options()
    L.gvh_default_options(ctypes.byref(o))
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    ptr = dummy.data_ptr()
    rc = L.gvh_rk2_step_noalloc(ctypes.byref(lat), ctypes.byref(hyd), ctypes.byref(o), 0.6, 0.01, 0.0, ptr,
                                ptr + 8, ptr + 16, ptr + 24, ptr + 32, ptr + 40, None, None)
    assert rc == -1  # GVH_ERR_INVALID
    msg = L.gvh_noalloc_last_error()
    assert b"static scratch" in msg and b"131x131x61" in msg
