"""GPU parity of the rec3 family (fv_rec3_2d.cu: unlimited rec3
reconstruction of the conserved variables, face Zhang-Shu scaling, HLLC,
2x2-block Zhang-Shu positivity limiter after every stage; FP64, periodic,
N even) against the oracle, which is bit-identical to fv_rec3's own kernels
run serially on the host.  The device path gathers each cell's face terms
in that serial scatter's order and is compiled without multiply-add
contraction, so the bar is bit-exact where the oracle and the device run
the same operations; it is held at 1e-13 to leave room for the last bit of
the initial-state transcendentals."""
from __future__ import annotations

import numpy as np
import pytest

import fvstuff_b200 as F
import oracle as O
from cases import rel_linf

pytestmark = pytest.mark.gpu


def _solver(n, length=1.0, cfl=0.4):
    return F.Solver(n, flux="rec3", bc="periodic", length=length, cfl=cfl)


def _prep(case, n):
    L = 10.0 if case == "pv" else 1.0
    p0 = O.rec3_p0(0.1) if case == "lmv" else 0.0
    U = O.rec3_ic(n, L / n, case, p0)
    O.rec3_limit(U, n)
    O.bc(U, n, 2, 1)
    return U, L


@pytest.mark.parametrize("case,n,steps", [("sod", 32, 25), ("pv", 24, 15), ("lmv", 20, 15), ("sod", 66, 12)])
def test_rec3_matches_oracle(case, n, steps):
    U, L = _prep(case, n)
    s = _solver(n, L)
    s.set_state(U, layout="cons")
    s.step(steps)
    st = s.sync()
    ref = U.copy()
    status, t, k, lmax, dt, brutal = O.rec3_run(ref, n, L / n, 0.4, steps)
    assert status == 0 and st.status == 0 and st.steps == k == steps
    got = s.get_state(layout="cons")
    err = rel_linf(got[:, 2:-2, 2:-2], ref[:, 2:-2, 2:-2])
    exact = np.array_equal(got[:, 2:-2, 2:-2], ref[:, 2:-2, 2:-2])
    print("rec3 %s %d^2 x %d: rel L-inf %.2e, bit-exact %s, t %.17g / %.17g" % (case, n, steps, err, exact, st.t, t))
    assert err <= 1e-13
    assert abs(st.t - t) <= 1e-14 * t


def test_rec3_limiters_engage_like_the_oracle():
    """two strong rarefactions: the face scaling and the block limiter act
    every stage; compare a run that stays short of the breakdown"""
    n = 32
    h = 1.0 / n
    x = (np.arange(n) + 0.5) * h
    X, Y = np.meshgrid(x, x)
    rho = np.where(np.abs(X - 0.5) < 0.25, 1.0, 0.5)
    u = np.where(X < 0.5, -1.5, 1.5)
    v = 0.3 * np.sin(2 * np.pi * Y)
    p = np.full_like(rho, 0.05)
    U = np.zeros((4, n + 4, n + 4))
    U[:, 2:-2, 2:-2] = np.stack([rho, rho * u, rho * v, p / 0.4 + 0.5 * rho * (u * u + v * v)])
    O.rec3_limit(U, n)
    O.bc(U, n, 2, 1)
    ref = U.copy()
    status, t, k, lmax, dt, brutal = O.rec3_run(ref, n, h, 0.4, 10)
    s = _solver(n)
    s.set_state(U, layout="cons")
    s.step(10)
    st = s.sync()
    assert st.status == status and st.steps == k
    got = s.get_state(layout="cons")
    assert rel_linf(got[:, 2:-2, 2:-2], ref[:, 2:-2, 2:-2]) <= 1e-13
    r = got[0, 2:-2, 2:-2]
    pr = 0.4 * (got[3, 2:-2, 2:-2] - 0.5 * (got[1, 2:-2, 2:-2] ** 2 + got[2, 2:-2, 2:-2] ** 2) / r)
    assert r.min() >= 1e-12 and pr.min() >= 0.0


@pytest.mark.parametrize("kind,case", [("rec3_sod", "sod"), ("paper_vortex", "pv"), ("gresho", "lmv")])
def test_rec3_device_initial_states(kind, case):
    n = 40
    U, L = _prep(case, n)
    s = _solver(n, L)
    s.init_case(kind)
    got = s.get_state(layout="cons")
    assert rel_linf(got[:, 2:-2, 2:-2], U[:, 2:-2, 2:-2]) <= 1e-14


def test_rec3_conserves_and_reports_l2_errors():
    n, L = 48, 10.0
    s = _solver(n, L)
    s.init_case("paper_vortex")
    a = s.stats().sums
    st = s.advance(0.5)
    b = s.stats().sums
    for q in (0, 1, 2, 3):
        assert abs(b[q] - a[q]) <= 1e-12 * max(abs(a[q]), 1.0)
    e_dev = O.rec3_err(np.ascontiguousarray(s.get_state(layout="cons")), n, L / n, "pv")
    U, _ = _prep("pv", n)
    O.rec3_run(U, n, L / n, 0.4, 10 ** 6, t_stop=0.5)
    e_ref = O.rec3_err(U, n, L / n, "pv")
    assert st.t == pytest.approx(0.5, abs=1e-14)
    assert e_dev[0] == pytest.approx(e_ref[0], rel=1e-10) and e_dev[1] == pytest.approx(e_ref[1], rel=1e-10)


def test_rec3_rejects_what_the_reference_does_not_run():
    for kw in (dict(bc="reflect"), dict(precision="f32c")):
        with pytest.raises(F.FvbError):
            F.Solver(32, flux="rec3", **{"bc": "periodic", **kw})
    with pytest.raises(F.FvbError):
        F.Solver(33, flux="rec3", bc="periodic")


@pytest.mark.skipif(not O.have_ref_gpu_rec3(), reason="GPU build of fv_rec3 absent")
def test_rec3_faster_than_reference_gpu_kernels():
    """fv_rec3_2d.cu's own kernels (FP64 build, its loop: memset + atomicAdd
    scatter of the face fluxes, rk_stage, the block limiter, apply_bc,
    gpu_max per stage) on its paper vortex at 512^2, against the fused rec3
    stage kernel.  Prints both times and the difference (the reference's
    GPU scatter adds in a run-dependent order, so its results carry
    last-bit noise); asserts the fused path is faster."""
    import torch
    n, steps = 512, 20
    U, L = _prep("pv", n)
    V = U.copy()
    st, t, k, lmax, dt, ms_ref = O.refg_rec3_run(V, n, L / n, 0.4, steps)
    assert st == 0 and k == steps
    ts = torch.cuda.Stream()
    s = F.Solver(n, flux="rec3", bc="periodic", length=L, cfl=0.4, stream=ts.cuda_stream)
    s.set_state(U, layout="cons")
    s.step(2)  # warm-up (the step graph is recorded here), then the same start again
    s.sync()
    s.set_state(U, layout="cons")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(ts)
    s.step(steps)
    e1.record(ts)
    torch.cuda.synchronize()
    st2 = s.sync()
    ms = e0.elapsed_time(e1)
    err = rel_linf(s.get_state(layout="cons")[:, 2:-2, 2:-2], V[:, 2:-2, 2:-2])
    print("rec3 pv %d^2 x %d: reference kernels %.2f ms (%.2f G cell-stages/s), fused %.2f ms (%.2f G/s, %.1fx); "
          "rel L-inf difference %.1e" % (n, steps, ms_ref, 3.0 * n * n * steps / ms_ref / 1e6, ms,
                                          3.0 * n * n * steps / ms / 1e6, ms_ref / ms, err))
    assert st2.status == 0 and st2.steps == steps
    assert ms < ms_ref
