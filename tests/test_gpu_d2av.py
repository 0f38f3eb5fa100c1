"""GPU parity of the scheme kept in fv_up7_ducros_2d.cu.bak (UP-order
reconstruction of the conserved variables, HLLC, D2 artificial viscosity
gated by a Ducros weight from the 6th-order velocity divergence; FP64)
against the oracle, which is bit-identical to the .bak's own kernels built
for the host.  The device kernel keeps the reference's association order
and is compiled without multiply-add contraction, so the bar is bit-exact;
the assertion leaves 1e-13 for the record and prints whether it was exact.
"""
from __future__ import annotations

import numpy as np
import pytest

import fvstuff_b200 as F
import oracle as O
from cases import rel_linf

pytestmark = pytest.mark.gpu

BC = {"reflect": 0, "periodic": 1, "transmissive": 2}


def _sod_state(n, order):
    U = O.d2av_ic_sod(n, 1.0 / n, order)
    return U


def _moving_state(n, order, seed):
    """the .bak's Sod plus a seeded smooth velocity field (every term active)"""
    U = O.d2av_ic_sod(n, 1.0 / n, order)
    g = O.d2av_ghost(order)
    x = (np.arange(n) + 0.5) / n
    X, Y = np.meshgrid(x, x)
    rng = np.random.default_rng(seed)
    a, b = rng.uniform(0.2, 0.6, 2)
    u = a * np.sin(2 * np.pi * Y) + 0.01 * rng.uniform(-1, 1, (n, n))
    v = b * np.cos(2 * np.pi * X) + 0.01 * rng.uniform(-1, 1, (n, n))
    r = U[0, g:-g, g:-g]
    U[1, g:-g, g:-g] = r * u
    U[2, g:-g, g:-g] = r * v
    U[3, g:-g, g:-g] += 0.5 * r * (u * u + v * v)
    return U


def _run_both(U, n, order, bc, steps, c2=0.5, cg=0.0, sc=0.05, cfl=0.4):
    g = O.d2av_ghost(order)
    O.bc(U, n, g, BC[bc])
    s = F.Solver(n, order=order, flux="up_hllc_d2av", bc=bc, cfl=cfl)
    assert s.g == g
    if (c2, cg, sc) != (0.5, 0.0, 0.05):
        s.set_d2av(c2, cg, sc)
    s.set_state(U[:, g:-g, g:-g].copy(), layout="cons", interior=True)
    s.step(steps)
    st = s.sync()
    ref = U.copy()
    info = O.d2av_run(ref, n, 1.0 / n, cfl, BC[bc], steps, 1e30, order, c2, cg, sc)
    got = s.get_state(layout="cons", interior=True)
    want = ref[:, g:-g, g:-g]
    err = rel_linf(got, want)
    exact = np.array_equal(got, want)
    return s, st, info, err, exact


@pytest.mark.parametrize("order,n,steps", [(3, 64, 20), (5, 64, 20), (7, 64, 20), (9, 64, 20), (5, 100, 8),
                                           (9, 100, 8)])
def test_d2av_sod_matches_oracle(order, n, steps):
    """the .bak's own configuration: circular Sod, reflecting walls, C2 0.5,
    Cg 0, sc 0.05, CFL 0.4 (n = 100: partial tiles in x and y)"""
    s, st, info, err, exact = _run_both(_sod_state(n, order), n, order, "reflect", steps)
    print("d2av UP%d sod %d^2 x %d: rel L-inf %.2e, bit-exact %s" % (order, n, steps, err, exact))
    assert st.status == 0 and info[0] == 0 and st.steps == info[2] == steps
    assert err <= 1e-13
    assert abs(st.t - info[1]) <= 1e-14 * info[1]
    assert abs(st.lam_max - info[3]) <= 1e-13 * info[3]


@pytest.mark.parametrize("bc,order,cg", [("periodic", 5, 0.02), ("transmissive", 7, 0.01), ("reflect", 3, 0.05),
                                         ("periodic", 9, 0.01)])
def test_d2av_boundaries_and_global_viscosity(bc, order, cg):
    n = 72
    s, st, info, err, exact = _run_both(_moving_state(n, order, 3), n, order, bc, 12, c2=0.8, cg=cg, sc=0.1)
    print("d2av UP%d %s Cg %.2f: rel L-inf %.2e, bit-exact %s" % (order, bc, cg, err, exact))
    assert st.status == 0 and info[0] == 0 and st.steps == 12
    assert err <= 1e-13


def test_d2av_init_case_and_frame_sensor():
    """fvb_init_case('sod', rho_in = 10) is the .bak's initial state (up to
    the last bit of tanh); the frame's sensor panel is the .bak's S_D"""
    n, order = 96, 5
    g = O.d2av_ghost(order)
    s = F.Solver(n, order=order, flux="up_hllc_d2av")
    s.init_case("sod", rho_in=10.0)
    got = s.get_state(layout="cons", interior=True)
    want = O.d2av_ic_sod(n, 1.0 / n, order)[:, g:-g, g:-g]
    assert rel_linf(got, want) <= 1e-14
    s.step(10)
    s.frame_begin()
    fr = s.frame_end()
    Q = O.padded(n, g)
    Q[:, g:-g, g:-g] = s.get_state(layout="cons", interior=True)
    O.bc(Q, n, g, 0)
    sd = O.d2av_sensor(Q, n, 1.0 / n, order, 0.05)
    assert sd.max() > 0.1  # the expanding shock is seen
    assert np.abs(fr["ducros"] - sd).max() <= 1e-6
    assert np.abs(fr["rho"] - Q[0, g:-g, g:-g]).max() <= 1e-5 * Q[0].max()


def test_d2av_rejects_what_the_reference_lacks():
    with pytest.raises(F.FvbError):
        F.Solver(64, order=7, flux="up_hllc_d2av", precision="f32c")
    # orders 3, 5, 7 and 9 only (fv_up7_ducros_2d.cu.bak:746-751)
    with pytest.raises(F.FvbError):
        F.Solver(64, order=11, flux="up_hllc_d2av")
    s = F.Solver(64, order=7)
    with pytest.raises(F.FvbError):
        s.set_d2av(0.5, 0.0, 0.05)


@pytest.mark.skipif(not O.have_ref_gpu_bak(), reason="GPU build of the .bak absent")
def test_d2av_against_reference_gpu_kernels():
    """the .bak's own kernels on the same GPU: same result (they contract
    multiply-adds, so to 1e-12), and the fused kernel is faster"""
    import torch
    n, order, steps = 512, 5, 30
    U = O.d2av_ic_sod(n, 1.0 / n, order)
    g = O.d2av_ghost(order)
    V = np.ascontiguousarray(U[:, g:-g, g:-g])
    st, t, k, lmax, dt, ms_ref = O.refg_bak_run(V, n, 1.0 / n, 0.4, steps, 1e30, order)
    assert st == 0 and k == steps
    # on a torch stream of its own (not the legacy default stream, which the
    # library would replace by a private one), so that its events bracket the steps
    ts = torch.cuda.Stream()
    s = F.Solver(n, order=order, flux="up_hllc_d2av", stream=ts.cuda_stream)
    s.set_state(U[:, g:-g, g:-g].copy(), layout="cons", interior=True)
    s.step(2)
    s.sync()
    s.set_state(U[:, g:-g, g:-g].copy(), layout="cons", interior=True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(ts)
    s.step(steps)
    e1.record(ts)
    st2 = s.sync()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    got = s.get_state(layout="cons", interior=True)
    err = rel_linf(got, V)
    print("d2av UP%d %d^2 x %d: reference kernels %.2f ms, fused %.2f ms (%.1fx); rel L-inf %.2e"
          % (order, n, steps, ms_ref, ms, ms_ref / ms, err))
    assert st2.steps == steps and err <= 1e-10
    assert ms < ms_ref
