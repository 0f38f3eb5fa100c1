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


def _noalloc(Qd, n, h, cfl, bc, nsteps, t0):
    st = L.Stats()
    code = F.lib().fvb_step_noalloc(Qd.data_ptr(), n, n + 8, h, cfl, 1.4, bc, bc, nsteps, t0, 1e300, None,
                                    C.byref(st))
    L.check(code, "fvb_step_noalloc")
    return st


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


def test_noalloc_rejects_grids_beyond_its_scratch():
    Qd = torch.zeros((4, 521, 521), dtype=torch.float64, device="cuda")
    st = L.Stats()
    code = F.lib().fvb_step_noalloc(Qd.data_ptr(), 513, 521, 1.0 / 513, 0.4, 1.4, 0, 0, 1, 0.0, 1.0, None,
                                    C.byref(st))
    assert code == L.ERR_INVALID
    assert b"512" in F.lib().fvb_last_error()
