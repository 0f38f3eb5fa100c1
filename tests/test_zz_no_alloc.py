"""fvb_step_noalloc: SSP-RK3 steps for callers that cannot allocate device
memory (their device memory belongs to their own pool, or is fixed at
start-up).  Its stage buffers live in a fixed __device__ array of the library
instead of cudaMalloc'd memory; the result must be the one the allocating
path (fvb_create + fvb_step) gives, on two calls in a row (the second call
starts from what the first left in that shared array).

Kept in a file of its own that pytest collects last.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import fvstuff_b200 as F
from fvstuff_b200 import _lib as L
from cases import pad, rel_linf, smooth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
TOL64 = 1e-12


def _noalloc(Qd, n, h, cfl, bc, nsteps, t0, np_=None):
    st = L.Stats()
    np_ = n + 8 if np_ is None else np_
    code = F.lib().fvb_step_noalloc(Qd.data_ptr(), n, np_, h, cfl, 1.4, bc, bc, nsteps, t0, 1e300, None,
                                    C.byref(st))
    L.check(code, "fvb_step_noalloc")
    return st


def _conserved_sums(U, n, g=4):
    r, u, v, p = (U[q, g:g + n, g:g + n] for q in range(4))
    return np.array([r.sum(), (r * u).sum(), (r * v).sum(), (p / 0.4 + 0.5 * r * (u * u + v * v)).sum()])


@pytest.mark.parametrize("n,bc", [(96, "periodic"), (37, "reflect")])
def test_noalloc_matches_allocating_path_twice(n, bc):
    h, cfl, k = 1.0 / n, 0.45, 6
    w = smooth(n, seed=11)
    U = pad(w, 4)
    s = F.Solver(n, bc=bc, cfl=cfl)
    s.set_state(U)
    Qd = torch.from_numpy(U.copy()).cuda()
    # first call
    s.step(k)
    ref1, st_ref1 = s.get_state(), s.sync()
    st1 = _noalloc(Qd, n, h, cfl, F.BC[bc], k, 0.0)
    torch.cuda.synchronize()
    assert st1.status == 0 and st1.steps == k
    assert abs(st1.t - st_ref1.t) <= 1e-13 * st_ref1.t
    assert rel_linf(Qd.cpu().numpy(), ref1) <= TOL64
    # second call, continuing from the first
    s.step(k)
    ref2, st_ref2 = s.get_state(), s.sync()
    st2 = _noalloc(Qd, n, h, cfl, F.BC[bc], k, st1.t)
    torch.cuda.synchronize()
    assert st2.status == 0 and st2.steps == k
    assert abs(st2.t - st_ref2.t) <= 1e-13 * st_ref2.t
    assert rel_linf(Qd.cpu().numpy(), ref2) <= TOL64


def test_noalloc_wider_unaligned_pitch():
    # the caller's rows may be longer than n + 8 and need not be 16-byte
    # aligned: n = 37 in rows of 51 doubles; the columns past the ghost ring
    # hold a sentinel that must survive
    n, np_, k = 37, 51, 5
    h, cfl = 1.0 / n, 0.45
    U = pad(smooth(n, seed=5), 4)
    s = F.Solver(n, bc="periodic", cfl=cfl)
    s.set_state(U)
    s.step(k)
    ref = s.get_state()
    wide = np.full((4, np_, np_), -7.25)
    wide[:, :n + 8, :n + 8] = U
    Qd = torch.from_numpy(wide).cuda()
    st = _noalloc(Qd, n, h, cfl, F.BC["periodic"], k, 0.0, np_=np_)
    torch.cuda.synchronize()
    got = Qd.cpu().numpy()
    assert st.status == 0 and st.steps == k
    assert rel_linf(got[:, :n + 8, :n + 8], ref) <= TOL64
    assert np.all(got[:, n + 8:, :] == -7.25) and np.all(got[:, :, n + 8:] == -7.25)


def test_noalloc_largest_grid_conserves():
    # n = 512 in rows of 520: the largest grid the fixed scratch holds
    n, k = 512, 4
    U = pad(smooth(n, seed=9), 4)
    Qd = torch.from_numpy(U.copy()).cuda()
    st = _noalloc(Qd, n, 1.0 / n, 0.45, F.BC["periodic"], k, 0.0)
    torch.cuda.synchronize()
    got = Qd.cpu().numpy()
    assert st.status == 0 and st.steps == k and st.t > 0
    assert np.all(np.isfinite(got))
    s0, s1 = _conserved_sums(U, n), _conserved_sums(got, n)
    assert np.all(np.abs(s1 - s0) <= 1e-13 * n * n), (s0, s1)


def test_noalloc_allocates_no_device_memory():
    # what the entry point is for: after a first call (which may load the
    # library's kernels), further calls leave the device's free memory as it was
    n, k = 64, 3
    Qd = torch.from_numpy(pad(smooth(n, seed=3), 4)).cuda()
    _noalloc(Qd, n, 1.0 / n, 0.45, F.BC["periodic"], 1, 0.0)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    t = 0.0
    for _ in range(5):
        t = _noalloc(Qd, n, 1.0 / n, 0.45, F.BC["periodic"], k, t).t
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_noalloc_rejects_grids_beyond_its_scratch():
    Qd = torch.zeros((4, 521, 521), dtype=torch.float64, device="cuda")
    st = L.Stats()
    code = F.lib().fvb_step_noalloc(Qd.data_ptr(), 513, 521, 1.0 / 513, 0.4, 1.4, 0, 0, 1, 0.0, 1.0, None,
                                    C.byref(st))
    assert code == L.ERR_INVALID
    assert b"512" in F.lib().fvb_last_error()
