"""GPU parity of the plain FP64 path (and the FP32 drop-in mode) against the
oracle and against the reference's own CUDA kernels (oracle/_ref GPU build),
through the C ABI.

Bar (the plain method): <= 1e-12 relative L-inf on the conserved variables
(max over variables of max|a-b| / max|b|) after a fixed number of steps.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import fvstuff_b200 as F
import oracle as O
from cases import kh, pad, prim_to_cons, rel_linf, riemann4, smooth, sod, vortex

pytestmark = pytest.mark.gpu
TOL64 = 1e-12

torch = pytest.importorskip("torch")


def _padded(w, bc, g=4):
    U = pad(np.ascontiguousarray(w), g)
    O.bc(U, w.shape[-1], g, bc)
    return U


def _cons(U, g=4):
    n = U.shape[-1] - 2 * g
    return prim_to_cons(U[:, g:g + n, g:g + n].astype(np.float64))


BCS = {"reflect": 0, "periodic": 1, "transmissive": 2}


# --- kernel-level contract -------------------------------------------------

@pytest.mark.parametrize("n", [8, 17, 40, 67])
@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-13), (np.float32, 2e-5)])
def test_up_rhs_matches_oracle(n, dtype, tol):
    # smooth states keep the comparison well conditioned; a reconstruction
    # floored to 1e-14 next to a strong jump gives c ~ 1e7 and a star flux
    # that cancels to the last bits in any two builds
    U = _padded(smooth(n, seed=n).astype(dtype), 0)
    h = 1.0 / n
    Qd = torch.from_numpy(U).cuda()
    rhs = torch.empty((4, n, n), dtype=Qd.dtype, device="cuda")
    lam = torch.empty((n, n), dtype=Qd.dtype, device="cuda")
    F.up_rhs(Qd, rhs, lam, n, n + 8, h)
    torch.cuda.synchronize()
    R, l = O.up_rhs(U, n, h)
    assert rel_linf(rhs.cpu().numpy(), R) <= tol
    assert rel_linf(lam.cpu().numpy()[None], l[None]) <= tol


@pytest.mark.parametrize("order", [3, 5, 9])
@pytest.mark.parametrize("n", [9, 40])
def test_up_rhs_orders_match_oracle(order, n):
    """The other UP orders of fv_up7_ducros_2d.cu:149-186 (FP64), UP9 with
    its published weights."""
    g = (order + 1) // 2
    U = _padded(smooth(n, seed=n), 0, g)
    h = 1.0 / n
    Qd = torch.from_numpy(U).cuda()
    rhs = torch.empty((4, n, n), dtype=Qd.dtype, device="cuda")
    lam = torch.empty((n, n), dtype=Qd.dtype, device="cuda")
    F.up_rhs(Qd, rhs, lam, n, n + 2 * g, h, order=order)
    torch.cuda.synchronize()
    R, l = O.up_rhs(U, n, h, order=order)
    assert rel_linf(rhs.cpu().numpy(), R) <= 1e-13
    assert rel_linf(lam.cpu().numpy()[None], l[None]) <= 1e-13


@pytest.mark.skipif(not O.have_ref_gpu(), reason="reference GPU build absent")
@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-13), (np.float32, 2e-5)])
def test_up_rhs_matches_reference_kernel(dtype, tol):
    n = 96
    U = O.ref_up_ic_sod(n, 1.0 / n, dtype)
    O.ref_up_bc(U, n, 0)
    Rr, lr = O.refg_up_rhs(U, n, 1.0 / n)
    Qd = torch.from_numpy(U).cuda()
    rhs = torch.empty((4, n, n), dtype=Qd.dtype, device="cuda")
    lam = torch.empty((n, n), dtype=Qd.dtype, device="cuda")
    F.up_rhs(Qd, rhs, lam, n, n + 8, 1.0 / n)
    torch.cuda.synchronize()
    assert rel_linf(rhs.cpu().numpy(), Rr) <= tol
    assert rel_linf(lam.cpu().numpy()[None], lr[None]) <= tol


@pytest.mark.parametrize("bcx,bcy", [(0, 0), (1, 1), (2, 2), (1, 0), (2, 1)])
@pytest.mark.parametrize("n", [8, 13])
def test_apply_bc_matches_oracle(bcx, bcy, n):
    w = riemann4(n, seed=3)
    U = pad(w, 4)
    Ud = torch.from_numpy(U).cuda()
    names = {v: k for k, v in BCS.items()}
    F.apply_bc(Ud, n, n + 8, names[bcx], names[bcy])
    torch.cuda.synchronize()
    got = Ud.cpu().numpy()
    if bcx == bcy:
        ref = U.copy()
        O.bc(ref, n, 4, bcx)
        assert np.array_equal(got, ref)
    else:
        # per-axis rule: x-ghost columns follow bcx, y-ghost rows follow bcy
        ref_x = U.copy(); O.bc(ref_x, n, 4, bcx)
        ref_y = U.copy(); O.bc(ref_y, n, 4, bcy)
        assert np.array_equal(got[:, 4:4 + n, :], ref_x[:, 4:4 + n, :])
        assert np.array_equal(got[:, :, 4:4 + n], ref_y[:, :, 4:4 + n])


@pytest.mark.parametrize("stage", [1, 2, 3])
def test_rk3_stage_matches_oracle(stage):
    n = 19
    U0 = _padded(riemann4(n, seed=1), 1)
    Uk = _padded(riemann4(n, seed=2), 1)
    L = np.random.default_rng(stage).uniform(-1, 1, (4, n, n))
    ref = U0.copy()
    O.rk3(stage, ref, U0, Uk, L, 0.01, n, 4)
    out = torch.from_numpy(U0.copy()).cuda()
    F.rk3_stage(stage, out, torch.from_numpy(U0).cuda(), torch.from_numpy(Uk).cuda(), torch.from_numpy(L).cuda(),
                0.01, n, n + 8)
    torch.cuda.synchronize()
    assert rel_linf(out.cpu().numpy(), ref) <= 1e-15


def test_device_max_skips_nan():
    x = torch.tensor([0.5, float("nan"), 3.25, 1.0], dtype=torch.float64, device="cuda")
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    F.device_max(x, out)
    assert out.item() == 3.25


# --- fused step against the oracle ----------------------------------------

CASES = {
    "smooth": lambda n: smooth(n, seed=7 + n),
    "riemann4": lambda n: riemann4(n, seed=2),
    "vortex": lambda n: vortex(n),
    "sod": lambda n: sod(n),
}


@pytest.mark.parametrize("bc", ["reflect", "periodic", "transmissive"])
@pytest.mark.parametrize("n", [8, 9, 17, 37, 64])
@pytest.mark.parametrize("case", ["smooth", "riemann4", "vortex", "sod"])
def test_step_f64_matches_oracle(bc, n, case):
    if case == "riemann4" and bc == "periodic":
        # wrapping a four-quadrant state puts unsmoothed jumps on the domain
        # edge; floored reconstructions there make any two builds differ at
        # ~1e-11 (the same conditioning the sharp-jump cases showed)
        pytest.skip("periodic wrap of a four-quadrant state is not smooth")
    _step_against_oracle(bc, n, case, 7)


def _step_against_oracle(bc, n, case, order):
    g = (order + 1) // 2
    w = CASES[case](n)
    length = 10.0 if case == "vortex" else 1.0
    U = _padded(w, BCS[bc], g)
    s = F.Solver(n, order=order, bc=bc, length=length, x0=-5.0 if case == "vortex" else 0.0,
                 y0=-5.0 if case == "vortex" else 0.0, cfl=0.45)
    s.set_state(U)
    # UP9's published weights scale every reconstructed state by 4217/2520,
    # and the scheme doubles a perturbation about every step: on the 37^2
    # vortex the oracle against itself with a 1-ulp change of the initial
    # state differs by 1.7e-14 after 3 steps, 5.1e-13 after 6 and 7.3e-12
    # after 12 (UP7: 1.9e-15 after 12), so UP9 is compared after 4 steps
    steps = 4 if order == 9 else 12
    s.step(steps)
    st = s.sync()
    got = s.get_state()
    ref = U.copy()
    status, t, k, lmax, dt = O.up_run(ref, n, length / n, 0.45, BCS[bc], steps, order=order)
    # the same stop, at the same step, when the scheme itself breaks down
    assert st.status == {0: 0, 1: F._lib.ERR_BLOWUP, 2: F._lib.ERR_DT_UNDERFLOW}[status]
    assert st.steps == k
    if status:
        return
    err = rel_linf(_cons(got, g), _cons(ref, g))
    print("UP%d %s %s %d^2 x %d: rel L-inf %.2e, t rel %.2e" % (order, case, bc, n, steps, err, abs(st.t - t) / t))
    assert abs(st.t - t) <= 1e-13 * t
    assert err <= TOL64
    # the ghost ring is the boundary rule applied to the new interior
    assert rel_linf(got, ref) <= TOL64


@pytest.mark.parametrize("order", [3, 5, 9])
@pytest.mark.parametrize("bc", ["reflect", "periodic", "transmissive"])
@pytest.mark.parametrize("n,case", [(17, "smooth"), (37, "vortex"), (40, "sod")])
def test_orders_step_f64_matches_oracle(order, bc, n, case):
    """Whole steps at the other UP orders (FP64; the reference selects the
    order with its ORDER macro, fv_up7_ducros_2d.cu:30-37), UP9 with its
    published weights."""
    _step_against_oracle(bc, n, case, order)


@pytest.mark.parametrize("tile", [0, 1, 2, 3, 4, 5, 6])
def test_tile_variants_agree(tile):
    n = 70
    U = _padded(riemann4(n, seed=5), 1)
    s = F.Solver(n, bc="periodic", tile=tile)
    s.set_state(U)
    s.step(6)
    got = s.get_state()
    ref = U.copy()
    O.up_run(ref, n, 1.0 / n, 0.4, 1, 6)
    assert rel_linf(_cons(got), _cons(ref)) <= TOL64


@pytest.mark.skipif(not O.have_ref_gpu(), reason="reference GPU build absent")
def test_vortex_256_matches_reference_cuda_kernels():
    """The plain-method parity case: periodic isentropic vortex on [-5,5]^2,
    256^2, UP7 + Ducros HLLC, SSP-RK3 at CFL 0.5, 100 steps, against the
    reference's own kernels retyped to FP64 and run on this GPU."""
    n, steps = 256, 100
    U = _padded(vortex(n), 1)
    ref = U.copy()
    status, t, k, lmax, dt, ms = O.refg_up_run(ref, n, 10.0 / n, 0.5, 1, steps)
    s = F.Solver(n, bc="periodic", x0=-5, y0=-5, length=10.0, cfl=0.5)
    s.set_state(U)
    s.step(steps)
    st = s.sync()
    assert st.steps == k == steps and abs(st.t - t) <= 1e-13
    err = rel_linf(_cons(s.get_state()), _cons(ref))
    print("vortex 256^2 x 100 steps: rel L-inf vs reference kernels = %.3e" % err)
    assert err <= TOL64


@pytest.mark.skipif(not O.have_ref_gpu(), reason="reference GPU build absent")
def test_vortex_256_full_period_against_reference_and_exact():
    """The whole configuration-1 run: one period (t = 10, about 2200 steps)
    on the plain FP64 path and on the reference's own FP64 kernels, both
    landing on t = 10; prints their difference (which grows from the
    last-bit level of the first steps) and both errors against the exact
    solution (the initial vortex)."""
    n = 256
    w0 = vortex(n)
    U = _padded(w0, 1)
    ref = U.copy()
    status, t, k, lmax, dt, ms = O.refg_up_run(ref, n, 10.0 / n, 0.5, 1, 10 ** 6, t_stop=10.0)
    assert status == 0 and abs(t - 10.0) < 1e-12
    s = F.Solver(n, bc="periodic", x0=-5, y0=-5, length=10.0, cfl=0.5)
    s.set_state(U)
    st = s.advance(10.0)
    assert st.status == 0 and st.steps == k and abs(st.t - 10.0) < 1e-12
    got = s.get_state()
    err = rel_linf(_cons(got), _cons(ref))
    got, want = got[:, 4:-4, 4:-4], ref[:, 4:-4, 4:-4]
    l2 = lambda w: float(np.sqrt(np.mean((w[0] - w0[0]) ** 2)))
    print("vortex 256^2, one period (%d steps): rel L-inf vs reference kernels %.3e; L2(rho) vs exact "
          "%.4e (fvb) / %.4e (reference)" % (k, err, l2(got), l2(want)))
    assert err <= TOL64
    assert abs(l2(got) - l2(want)) <= 1e-6 * l2(want)


@pytest.mark.skipif(not O.have_ref_gpu(), reason="reference GPU build absent")
def test_f32_mode_matches_shipped_fp32_kernels():
    """FVB_PREC_F32 reproduces the solver as shipped (float state, double
    reconstruction arithmetic) against its own FP32 kernels."""
    n, steps = 64, 20
    U = O.ref_up_ic_sod(n, 1.0 / n, np.float32)
    O.ref_up_bc(U, n, 0)
    ref = U.copy()
    O.refg_up_run(ref, n, np.float32(1.0 / n), np.float32(0.4), 0, steps)
    s = F.Solver(n, precision="f32")
    s.set_state(U)
    s.step(steps)
    got = s.get_state(dtype=np.float32)
    err = rel_linf(_cons(got.astype(np.float64)), _cons(ref.astype(np.float64)))
    print("fp32 mode vs shipped kernels: %.3e" % err)
    assert err <= 1e-5


# --- step control ------------------------------------------------------------

def test_advance_lands_on_t_stop_like_reference_loop():
    n = 32
    U = _padded(vortex(n), 1)
    s = F.Solver(n, bc="periodic", x0=-5, y0=-5, length=10.0, cfl=0.5)
    s.set_state(U)
    st = s.advance(0.7)
    ref = U.copy()
    status, t, k, lmax, dt = O.up_run(ref, n, 10.0 / n, 0.5, 1, 10 ** 6, t_stop=0.7)
    assert st.t == t == 0.7 and st.steps == k
    assert rel_linf(_cons(s.get_state()), _cons(ref)) <= TOL64
    # further steps at t >= t_stop do nothing
    s.step(5, t_stop=0.7)
    assert s.sync().steps == k


def test_graph_and_direct_launches_agree_bitwise():
    n = 48
    U = _padded(riemann4(n, seed=9), 2)
    a = F.Solver(n, bc="transmissive")
    b = F.Solver(n, bc="transmissive")
    b.set_graph(False)
    for s in (a, b):
        s.set_state(U)
        s.step(7)
    assert np.array_equal(a.get_state(), b.get_state())


def test_posted_stats_match_sync():
    """fvb_stats_post / fvb_stats_wait give each step's control as fvb_sync
    does, read while later steps are enqueued"""
    n = 64
    a = F.Solver(n, bc="periodic", cfl=0.5)
    b = F.Solver(n, bc="periodic", cfl=0.5)
    for s in (a, b):
        s.set_state(riemann4(n, seed=8), interior=True)
    posted = []
    for k in range(12):
        a.step(1)
        a.post_stats(k % 3)
        if k >= 2:
            posted.append(a.wait_stats((k - 2) % 3))
    posted += [a.wait_stats(10 % 3), a.wait_stats(11 % 3)]
    for k in range(12):
        b.step(1)
        want = b.sync()
        got = posted[k]
        assert (got.t, got.dt, got.lam_max, got.steps, got.status) == \
            (want.t, want.dt, want.lam_max, want.steps, want.status), k
    with pytest.raises(F.FvbError):
        F.Solver(n).wait_stats(0)  # nothing posted


def test_blowup_reported_not_fatal():
    n = 16
    s = F.Solver(n, bc="periodic")
    bad = np.full((4, n, n), np.nan)
    s.set_state(bad, interior=True)
    with pytest.raises(F.FvbError) as e:
        s.advance(1.0)
    assert e.value.status == F._lib.ERR_BLOWUP
    # the solver stays usable
    s.set_state(np.stack([np.ones((n, n)), np.zeros((n, n)), np.zeros((n, n)), np.ones((n, n))]), interior=True)
    st = s.advance(0.01)
    assert st.status == 0 and st.t == 0.01


def test_conservation_periodic_f64():
    n = 64
    s = F.Solver(n, bc="periodic", x0=-5, y0=-5, length=10.0, cfl=0.5)
    s.set_state(vortex(n), interior=True)
    a = s.stats().sums
    s.step(50)
    b = s.stats().sums
    for q in (0, 1, 2, 3):
        assert abs(b[q] - a[q]) <= 1e-12 * max(abs(a[q]), 1.0)


def test_state_roundtrip_layouts():
    n = 20
    w = riemann4(n, seed=4)
    s = F.Solver(n, bc="reflect")
    s.set_state(w, interior=True)
    assert np.array_equal(s.get_state(interior=True), w)
    c = s.get_state(layout="cons", interior=True)
    assert rel_linf(c, prim_to_cons(w)) <= 1e-15
    s.set_state(c, layout="cons", interior=True)
    assert rel_linf(s.get_state(interior=True), w) <= 1e-14
    f = s.get_state(dtype=np.float32, interior=True)
    assert np.array_equal(f, w.astype(np.float32))
    # device tensors in and out
    d = torch.from_numpy(w).cuda()
    s.set_state(d, interior=True)
    out = torch.empty_like(d)
    s.get_state(interior=True, out=out)
    torch.cuda.synchronize()
    assert torch.equal(out, d)


@pytest.mark.parametrize("kind", ["vortex", "kh", "riemann4", "sod"])
def test_device_initial_states(kind):
    n = 48
    if kind == "vortex":
        s = F.Solver(n, bc="periodic", x0=-5, y0=-5, length=10.0)
        s.init_case("vortex")
        ref = vortex(n)
    elif kind == "kh":
        s = F.Solver(n, bc="periodic")
        s.init_case("kh", seed=99)
        ref = kh(n, seed=99)
    elif kind == "riemann4":
        s = F.Solver(n, bc="transmissive")
        s.init_case("riemann4", seed=31)
        ref = riemann4(n, seed=31)
    else:
        s = F.Solver(n)
        s.init_case("sod")
        ref = sod(n)
    got = s.get_state(interior=True)
    assert rel_linf(got, ref) <= 1e-13
    assert s.sync().t == 0.0


# --- carb_fv's Riemann solvers behind the same kernel ------------------------

@pytest.mark.parametrize("riemann", ["hll", "roe"])
@pytest.mark.parametrize("bc", ["reflect", "periodic", "transmissive"])
@pytest.mark.parametrize("n,case", [(37, "vortex"), (64, "smooth"), (41, "riemann4")])
def test_riemann_variants_match_oracle(riemann, bc, n, case):
    """UP7 + Ducros with carb_fv_2d.cu's HLL or Roe (Harten-Hyman fix) on the
    reconstructed states, FP64, against the oracle (itself bit-identical to
    carb_fv's own functions) at the plain method's 1e-12 bar."""
    if case == "riemann4" and bc == "periodic":
        pytest.skip("periodic wrap of a four-quadrant state is not smooth")
    w = CASES[case](n)
    length = 10.0 if case == "vortex" else 1.0
    org = -5.0 if case == "vortex" else 0.0
    U = _padded(w, BCS[bc])
    s = F.Solver(n, bc=bc, length=length, x0=org, y0=org, cfl=0.45, flux="up_ducros_" + riemann)
    s.set_state(U)
    s.step(10)
    st = s.sync()
    ref = U.copy()
    status, t, k, lmax, dt = O.up_run(ref, n, length / n, 0.45, BCS[bc], 10, riemann=riemann)
    assert status == 0 and st.status == 0 and st.steps == k == 10
    assert abs(st.t - t) <= 1e-13 * t
    assert rel_linf(_cons(s.get_state()), _cons(ref)) <= TOL64


def test_riemann_variant_rejects_other_forms():
    with pytest.raises(F.FvbError):
        F.Solver(64, flux="up_ducros_roe", precision="f32c")


# --- guard bands: nothing is written outside the caller's arrays ----------------

SENTINEL = 12345.678


def _guarded(count, dtype, guard=4096):
    """a device array of `count` elements between two sentinel-filled guards"""
    big = torch.full((guard + count + guard,), SENTINEL, dtype=dtype, device="cuda")
    return big, big[guard:guard + count]


def _guards_intact(big, count, guard=4096):
    torch.cuda.synchronize()
    g = torch.cat([big[:guard], big[guard + count:]])
    return bool(torch.all(g == SENTINEL).item())


@pytest.mark.parametrize("n", [8, 13, 37])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_kernel_contract_writes_stay_in_bounds(n, dtype):
    """the kernel-level entry points on ragged sizes write only inside their
    output arrays (guard bands of a sentinel value on both sides), and
    apply_bc / rk3_stage leave the parts they do not own untouched"""
    npd = n + 8
    U = torch.from_numpy(_padded(smooth(n, seed=n), 1)).to(dtype).cuda().contiguous()
    big_r, rhs = _guarded(4 * n * n, dtype)
    big_l, lam = _guarded(n * n, dtype)
    F.up_rhs(U, rhs.view(4, n, n), lam.view(n, n), n, npd, 1.0 / n)
    assert _guards_intact(big_r, 4 * n * n) and _guards_intact(big_l, n * n)
    # apply_bc on a guarded copy: the interior is not touched
    big_q, Q = _guarded(4 * npd * npd, dtype)
    Q.copy_(U.reshape(-1))
    F.apply_bc(Q.view(4, npd, npd), n, npd, "periodic")
    assert _guards_intact(big_q, 4 * npd * npd)
    assert torch.equal(Q.view(4, npd, npd)[:, 4:-4, 4:-4], U[:, 4:-4, 4:-4])
    # rk3_stage writes the interior of Uo only
    big_o, Uo = _guarded(4 * npd * npd, dtype)
    Uo.fill_(-7.0)
    F.rk3_stage(2, Uo.view(4, npd, npd), U, U, rhs.view(4, n, n), 1e-3, n, npd)
    assert _guards_intact(big_o, 4 * npd * npd)
    V = Uo.view(4, npd, npd)
    ring = torch.ones((npd, npd), dtype=torch.bool, device="cuda")
    ring[4:-4, 4:-4] = False
    assert bool(torch.all(V[:, ring] == -7.0).item())
    # the solver's state export to a device array
    s = F.Solver(n, bc="periodic")
    s.set_state(U.cpu().numpy())
    s.step(3)
    big_s, out = _guarded(4 * n * n, torch.float64)
    s.get_state(interior=True, out=out.view(4, n, n))
    assert _guards_intact(big_s, 4 * n * n)
