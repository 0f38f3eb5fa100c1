"""The oracle restatement (oracle/fvb_oracle.c) pinned to the reference.

* against golden fixtures produced by the reference's own kernels
  (tests/golden/make_golden.py): always run;
* against the reference's kernels compiled for the host (oracle/_ref), on
  seeded states of ragged sizes and every boundary condition: run where
  that build exists.

Both sides are compiled without FMA contraction, so the bar is bit-exact.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import oracle as O
from cases import pad, riemann4, vortex

GOLD = Path(__file__).resolve().parent / "golden"


@pytest.mark.parametrize("sfx,dtype", [("f64", np.float64), ("f32", np.float32)])
def test_faces_golden(sfx, dtype):
    z = np.load(GOLD / ("faces_%s.npz" % sfx))
    for k in range(len(z["WL"])):
        wl, wr = z["WL"][k], z["WR"][k]
        # x-normal: (rho, u, v, p) is already (rho, un, ut, p)
        assert np.array_equal(O.hllc(wl, wr, dtype), z["hllc_x"][k])
        assert np.array_equal(O.hlle(wl, wr, dtype), z["hlle_x"][k])
        # y-normal: relabel (u, v) -> (ut, un) and swap the momentum fluxes back
        sw = [0, 2, 1, 3]
        fy = O.hllc(wl[sw], wr[sw], dtype)[sw]
        assert np.array_equal(fy, z["hllc_y"][k]), k
        fy = O.hlle(wl[sw], wr[sw], dtype)[sw]
        assert np.array_equal(fy, z["hlle_y"][k]), k
        vl, vr = O.upface(7, z["stencil"][k], dtype)
        assert (vl, vr) == tuple(z["up7"][k])


@pytest.mark.parametrize("sfx,dtype", [("f64", np.float64), ("f32", np.float32)])
def test_sod16_golden(sfx, dtype):
    z = np.load(GOLD / ("up7_sod16_%s.npz" % sfx))
    N, h = 16, 1.0 / 16
    U = O.ic_sod(N, h, dtype)
    O.bc(U, N, 4, 0)
    assert np.array_equal(U, z["U0"])
    R, lam = O.up_rhs(U, N, h)
    assert np.array_equal(R, z["rhs"]) and np.array_equal(lam, z["lam"])
    info = O.up_run(U, N, h, 0.4, 0, 5)
    assert np.array_equal(U, z["U5"])
    assert np.allclose(info, z["info"], rtol=0, atol=0)


@pytest.mark.parametrize("tag,bc", [("periodic", 1), ("transmissive", 2)])
def test_vortex16_golden(tag, bc):
    z = np.load(GOLD / ("up7_vortex16_%s_f64.npz" % tag))
    U = z["U0"].copy()
    O.up_run(U, 16, 10.0 / 16, 0.5, bc, 5)
    assert np.array_equal(U, z["U5"])


@pytest.mark.parametrize("tag,lmv", [("sod", False), ("lmv", True)])
def test_keep_golden(tag, lmv):
    z = np.load(GOLD / ("keep_%s16.npz" % tag))
    n, h = 16, 1.0 / 16
    U = O.keep_ic(n, h, lmv)
    O.bc(U, n, 2, 1)
    assert np.array_equal(U, z["U0"])
    R, lam, edm = O.keep_rhs(U, n, h)
    assert edm == float(z["edmax"])
    assert np.array_equal(R, z["rhs"]) and np.array_equal(lam, z["lam"])
    O.keep_run(U, n, h, 0.2, 5)
    assert np.array_equal(U, z["U5"])


needs_ref = pytest.mark.skipif(not O.have_ref_host(), reason="oracle/_ref host build absent")


@needs_ref
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("bc", [0, 1, 2])
@pytest.mark.parametrize("n", [8, 9, 17, 23])
def test_oracle_matches_reference_host(dtype, bc, n):
    w = riemann4(n, seed=100 + n + bc).astype(dtype)
    U = pad(w, 4)
    O.bc(U, n, 4, bc)
    V = U.copy()
    O.ref_up_bc(V, n, bc)
    assert np.array_equal(U, V)
    h = 1.0 / n
    a = O.up_rhs(U, n, h)
    b = O.ref_up_rhs(V, n, h)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    ia = O.up_run(U, n, h, 0.45, bc, 8)
    ib = O.ref_up_run(V, n, h, 0.45, bc, 8)
    assert ia == ib
    assert np.array_equal(U, V)


@needs_ref
def test_oracle_matches_reference_host_t_stop():
    # the frame-clamped dt (fv_up7_ducros_2d.cu:999-1001) lands on t_stop
    n = 24
    U = pad(vortex(n), 4)
    O.bc(U, n, 4, 1)
    V = U.copy()
    ia = O.up_run(U, n, 10.0 / n, 0.5, 1, 1000, t_stop=0.3)
    ib = O.ref_up_run(V, n, 10.0 / n, 0.5, 1, 1000, t_stop=0.3)
    assert ia == ib and ia[1] == 0.3
    assert np.array_equal(U, V)


def test_keep_reference_scheme_loses_energy_on_sod():
    """A property of the reference scheme the GPU path reproduces: on the
    circular Sod case the rk_stage floor E >= 1e-14 (keep_fv_euler_2d.cu:
    390-391) clips energies the scheme drives negative, so total energy
    drifts while mass and momentum stay conserved."""
    n, h = 48, 1.0 / 48
    U = O.keep_ic(n, h, False)
    O.bc(U, n, 2, 1)
    sums = lambda V: [V[q, 2:2 + n, 2:2 + n].sum() * h * h for q in range(4)]
    a = sums(U)
    O.keep_run(U, n, h, 0.2, 5)
    b = sums(U)
    assert abs(b[0] - a[0]) < 1e-14 and abs(b[1] - a[1]) < 1e-14 and abs(b[2] - a[2]) < 1e-14
    assert b[3] - a[3] > 1e-6


@needs_ref
def test_keep_oracle_matches_reference_host():
    n = 20
    for lmv in (False, True):
        U = O.keep_ic(n, 1.0 / n, lmv)
        V = O.ref_keep_ic(n, 1.0 / n, lmv)
        assert np.array_equal(U, V)
        O.bc(U, n, 2, 1)
        O.bc(V, n, 2, 1)
        assert O.keep_run(U, n, 1.0 / n, 0.2, 6) == O.ref_keep_run(V, n, 1.0 / n, 0.2, 6)
        assert np.array_equal(U, V)


def test_carb_riemann_golden():
    """HLL and Roe (carb_fv_2d.cu:116-211) in the normal frame against the
    fixture frozen from carb_fv's own functions, x and y normals."""
    z = np.load(GOLD / "faces_carb_f64.npz")
    sw = [0, 2, 1, 3]
    for k in range(len(z["WL"])):
        wl, wr = z["WL"][k], z["WR"][k]
        for name in ("hll", "roe"):
            f = getattr(O, name)
            assert np.array_equal(f(wl, wr), z[name + "_x"][k]), (name, k)
            assert np.array_equal(f(wl[sw], wr[sw])[sw], z[name + "_y"][k]), (name, k)


@pytest.mark.skipif(not O.have_ref_carb(), reason="carb_fv host build absent")
def test_carb_riemann_matches_reference_host():
    rng = np.random.default_rng(3)
    sw = [0, 2, 1, 3]
    for _ in range(500):
        wl = np.array([rng.uniform(1e-3, 5), rng.uniform(-4, 4), rng.uniform(-4, 4), rng.uniform(1e-3, 5)])
        wr = np.array([rng.uniform(1e-3, 5), rng.uniform(-4, 4), rng.uniform(-4, 4), rng.uniform(1e-3, 5)])
        for name in ("hll", "roe"):
            f = getattr(O, name)
            assert np.array_equal(f(wl, wr), O.ref_carb_flux(name, wl, wr, 1.0, 0.0))
            assert np.array_equal(f(wl[sw], wr[sw])[sw], O.ref_carb_flux(name, wl, wr, 0.0, 1.0))


@pytest.mark.parametrize("riemann", ["hll", "roe"])
def test_riemann_variants_step_conserves_and_differs(riemann):
    """The UP7 + Ducros scheme with carb_fv's solvers on the reconstructed
    states: a periodic vortex conserves mass and energy to round-off and
    differs from the HLLC scheme at the discretisation-error level."""
    from cases import prim_to_cons
    n = 32
    U = pad(vortex(n), 4)
    O.bc(U, n, 4, 1)
    V = U.copy()
    a = prim_to_cons(U[:, 4:-4, 4:-4]).sum(axis=(1, 2))
    O.up_run(U, n, 10.0 / n, 0.5, 1, 10, riemann=riemann)
    O.up_run(V, n, 10.0 / n, 0.5, 1, 10)
    b = prim_to_cons(U[:, 4:-4, 4:-4]).sum(axis=(1, 2))
    assert abs(b[0] - a[0]) <= 1e-12 * abs(a[0]) and abs(b[3] - a[3]) <= 1e-12 * abs(a[3])
    d = np.abs(U - V).max()
    assert 1e-8 < d < 1e-1


# --- fv_rec3_2d.cu: rec3 + HLLC + 2x2-block Zhang-Shu -------------------------

def _rec3_case(case, N):
    L = 10.0 if case == "pv" else 1.0
    p0 = O.rec3_p0(0.1) if case == "lmv" else 0.0
    return L / N, p0


@pytest.mark.parametrize("case", ["sod", "pv", "lmv"])
def test_rec3_golden(case):
    z = np.load(GOLD / "rec3_16.npz")
    N = 16
    h, p0 = _rec3_case(case, N)
    U = O.rec3_ic(N, h, case, p0)
    O.rec3_limit(U, N)
    O.bc(U, N, 2, 1)
    assert np.array_equal(U, z[case + "_U0"])
    R, lam = O.rec3_rhs(U, N, h)
    assert np.array_equal(R, z[case + "_rhs"]) and np.array_equal(lam, z[case + "_lam"])
    info = O.rec3_run(U, N, h, 0.4, 8)
    assert np.array_equal(U, z[case + "_U8"])
    assert np.array_equal(np.array(info), z[case + "_info"])


def _rec3_stress(N):
    """two strong rarefactions: near-vacuum that drives both positivity
    limiters, the brutal mean fix and finally the dt-underflow guard"""
    h = 1.0 / N
    x = (np.arange(N) + 0.5) * h
    X, Y = np.meshgrid(x, x)
    rho = np.where(np.abs(X - 0.5) < 0.25, 1.0, 0.5)
    u = np.where(X < 0.5, -3.0, 3.0)
    v = 0.5 * np.sin(2 * np.pi * Y)
    p = np.full_like(rho, 0.05)
    U = np.zeros((4, N + 4, N + 4))
    c = (slice(None), slice(2, -2), slice(2, -2))
    U[c] = np.stack([rho, rho * u, rho * v, p / 0.4 + 0.5 * rho * (u * u + v * v)])
    return U


needs_rec3 = pytest.mark.skipif(not O.have_ref_rec3(), reason="fv_rec3 host build absent")


@needs_rec3
@pytest.mark.parametrize("case,N", [("sod", 32), ("pv", 24), ("lmv", 20), ("stress", 32)])
def test_rec3_oracle_matches_reference_host(case, N):
    O.ref_set_threads(1)
    if case == "stress":
        h, p0 = 1.0 / N, 0.0
        U = _rec3_stress(N)
        V = U.copy()
    else:
        h, p0 = _rec3_case(case, N)
        U = O.rec3_ic(N, h, case, p0)
        V = O.ref_rec3_ic(N, h, case, p0)
        assert np.array_equal(U, V)
    assert O.rec3_limit(U, N) == O.ref_rec3_limit(V, N)
    O.bc(U, N, 2, 1)
    O.ref_rec3_bc(V, N)
    assert np.array_equal(U, V)
    ia = O.rec3_run(U, N, h, 0.4, 40)
    ib = O.ref_rec3_run(V, N, h, 0.4, 40)
    assert ia == ib
    assert np.array_equal(U, V)
    if case == "stress":
        assert ia[0] == 2 and ia[5] > 0   # the reference scheme breaks down, with brutal fixes


@needs_rec3
def test_rec3_face_scaling_and_hllc_match_reference():
    rng = np.random.default_rng(9)
    sw = [0, 2, 1, 3]
    for _ in range(300):
        Ub = np.array([rng.uniform(0.1, 2), rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(1, 3)])
        U = Ub + rng.normal(0, 1.5, 4)   # often inadmissible
        a = O.rec3_scale(Ub, U)
        b = U.copy()
        O.ref_rec3("scale")(O._ptr(Ub), O._ptr(b))
        assert np.array_equal(a, b)
        wl = np.array([rng.uniform(0.1, 3), rng.uniform(-2, 2), rng.uniform(-2, 2), rng.uniform(0.1, 3)])
        wr = np.array([rng.uniform(0.1, 3), rng.uniform(-2, 2), rng.uniform(-2, 2), rng.uniform(0.1, 3)])
        for nx, ny, perm in ((1.0, 0.0, [0, 1, 2, 3]), (0.0, 1.0, sw)):
            F = np.empty(4)
            O.ref_rec3("hllc")(O._ptr(wl), O._ptr(wr), O.C.c_double(nx), O.C.c_double(ny), O._ptr(F))
            assert np.array_equal(O.rec3_hllc(wl[perm], wr[perm])[perm], F)


# --- fv_up7_ducros_2d.cu.bak: UP + HLLC + Ducros-gated D2 viscosity -----------
def _bak_padded(U, N, order, bc=0):
    g = O.d2av_ghost(order)
    Q = O.padded(N, g)
    Q[:, g:g + N, g:g + N] = U
    O.bc(Q, N, g, bc)
    return Q, g


@pytest.mark.parametrize("order", [3, 5, 7])
def test_bak_golden(order):
    z = np.load(GOLD / "bak_16.npz")
    N = 16
    h = 1.0 / N
    g = O.d2av_ghost(order)
    assert np.array_equal(O.d2av_ic_sod(N, h, order)[:, g:-g, g:-g], z["ic"])
    Q, g = _bak_padded(z["o%d_U" % order], N, order)
    R, lam = O.d2av_rhs(Q, N, h, order, 0.5, 0.02, 0.05)
    assert np.array_equal(R, z["o%d_rhs" % order])
    assert np.array_equal(lam, z["o%d_lam" % order])
    assert np.array_equal(O.d2av_sensor(Q, N, h, order, 0.05), z["o%d_sd" % order])
    Q, g = _bak_padded(z["ic"], N, order)
    info = O.d2av_run(Q, N, h, 0.4, 0, 6, 1e30, order, 0.5, 0.02, 0.05)
    assert np.array_equal(np.array(info), z["o%d_info" % order])
    assert np.array_equal(Q[:, g:-g, g:-g], z["o%d_U6" % order])


needs_bak = pytest.mark.skipif(not O.have_ref_bak(), reason="fv_up7_ducros_2d.cu.bak host build absent")


@needs_bak
@pytest.mark.parametrize("order,N,cg", [(3, 20, 0.0), (5, 33, 0.01), (7, 41, 0.0), (9, 24, 0.0)])
def test_bak_oracle_matches_reference_host(order, N, cg):
    """Ragged sizes, every order the .bak takes (UP9 with its published
    weights), both viscosity terms, 12 steps through the reference's loop."""
    O.ref_set_threads(1)
    from golden.make_golden import bak_state
    h = 1.0 / N
    U = bak_state(N, 100 + order)
    Q, g = _bak_padded(U, N, order)
    R, lam = O.d2av_rhs(Q, N, h, order, 0.5, cg, 0.05)
    Rr, lamr = O.ref_bak_rhs(U, N, h, order, 0.5, cg, 0.05)
    assert np.array_equal(R, Rr) and np.array_equal(lam, lamr)
    assert np.array_equal(O.d2av_sensor(Q, N, h, order, 0.05), O.ref_bak_sensor(U, N, h, 0.05))
    V = O.ref_bak_ic(N, h)
    Q, g = _bak_padded(V, N, order)
    ia = O.d2av_run(Q, N, h, 0.4, 0, 12, 1e30, order, 0.5, cg, 0.05)
    ib = O.ref_bak_run(V, N, h, 0.4, 12, 1e30, order, 0.5, cg, 0.05)
    assert ia == ib and ia[0] == 0 and ia[2] == 12
    assert np.array_equal(Q[:, g:-g, g:-g], V)


@needs_bak
def test_bak_hllc_matches_reference():
    rng = np.random.default_rng(21)
    sw = [0, 2, 1, 3]
    f = O.ref_host("bak").ref_bak_hllc
    for _ in range(400):
        U = []
        for _side in range(2):
            r = rng.uniform(0.1, 3)
            u, v, p = rng.uniform(-3, 3), rng.uniform(-3, 3), rng.uniform(0.1, 5)
            U.append(np.array([r, r * u, r * v, p / 0.4 + 0.5 * r * (u * u + v * v)]))
        for yface, perm in ((0, [0, 1, 2, 3]), (1, sw)):
            F = np.empty(4)
            f(O._ptr(U[0]), O._ptr(U[1]), O.C.c_int(yface), O._ptr(F))
            assert np.array_equal(O.d2av_hllc(U[0][perm], U[1][perm])[perm], F)
