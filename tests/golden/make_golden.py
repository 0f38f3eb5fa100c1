"""Generate the golden fixtures in tests/golden/ from the reference's own
kernels, compiled for the host by oracle/build.py (oracle/_ref/).

The reference has no test suite and no golden vectors of its own; these
fixtures are outputs of its kernels (fv_up7_ducros_2d.cu as shipped and
retyped to FP64, keep_fv_euler_2d.cu) on small seeded inputs, frozen so the
oracle restatement stays pinned where the reference checkout is absent.

    python tests/golden/make_golden.py          # every fixture
    python tests/golden/make_golden.py carb     # carb_fv's HLL / Roe faces only
    python tests/golden/make_golden.py rec3     # those and fv_rec3's cases
    python tests/golden/make_golden.py bak      # those and the .bak scheme's cases
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))
sys.path.insert(0, str(HERE.parent))

import oracle as O  # noqa: E402
from cases import pad, vortex  # noqa: E402


def _faces(dtype, seed=7, count=64):
    """random face states, with supersonic and subsonic, left- and right-
    moving contacts, through the reference's hllc_n / hlle_n with x and y
    normals, and the UP7 face values of random stencils"""
    rng = np.random.default_rng(seed)
    sfx = "f64" if dtype == np.float64 else "f32"
    L = O.ref_host("up7_" + sfx)
    real = C.c_double if dtype == np.float64 else C.c_float
    WL = np.empty((count, 4), dtype)
    WR = np.empty((count, 4), dtype)
    WL[:, 0] = rng.uniform(0.1, 3, count); WR[:, 0] = rng.uniform(0.1, 3, count)
    WL[:, 3] = rng.uniform(0.1, 5, count); WR[:, 3] = rng.uniform(0.1, 5, count)
    WL[:, 1:3] = rng.uniform(-3, 3, (count, 2)); WR[:, 1:3] = rng.uniform(-3, 3, (count, 2))
    out = {"WL": WL, "WR": WR}
    for name in ("hllc", "hlle"):
        for tag, (nx, ny) in (("x", (1, 0)), ("y", (0, 1))):
            F = np.empty((count, 4), dtype)
            fn = getattr(L, "ref_up7_%s_%s" % (name, sfx))
            for k in range(count):
                a, b, f = WL[k].copy(), WR[k].copy(), np.empty(4, dtype)
                fn(O._ptr(a), O._ptr(b), real(nx), real(ny), O._ptr(f))
                F[k] = f
            out["%s_%s" % (name, tag)] = F
    S = rng.uniform(-2, 2, (count, 8)).astype(dtype)
    up = np.empty((count, 2), dtype)
    for k in range(count):
        s = S[k].copy(); vl = np.empty(1, dtype); vr = np.empty(1, dtype)
        getattr(L, "ref_up7_up7_" + sfx)(O._ptr(s), O._ptr(vl), O._ptr(vr))
        up[k] = vl[0], vr[0]
    out["stencil"] = S
    out["up7"] = up
    return out


def _faces_carb(seed=11, count=64):
    """random face states through carb_fv_2d.cu's own hll_n and roe_n (FP64),
    x and y normals"""
    rng = np.random.default_rng(seed)
    WL = np.empty((count, 4)); WR = np.empty((count, 4))
    WL[:, 0] = rng.uniform(0.1, 3, count); WR[:, 0] = rng.uniform(0.1, 3, count)
    WL[:, 3] = rng.uniform(0.1, 5, count); WR[:, 3] = rng.uniform(0.1, 5, count)
    WL[:, 1:3] = rng.uniform(-3, 3, (count, 2)); WR[:, 1:3] = rng.uniform(-3, 3, (count, 2))
    out = {"WL": WL, "WR": WR}
    for name in ("hll", "roe"):
        for tag, (nx, ny) in (("x", (1.0, 0.0)), ("y", (0.0, 1.0))):
            out["%s_%s" % (name, tag)] = np.array([O.ref_carb_flux(name, WL[k], WR[k], nx, ny)
                                                   for k in range(count)])
    return out


def _rec3():
    """fv_rec3_2d.cu's own kernels (FP64, one host thread): initial states of
    the Sod, paper-vortex and Gresho cases after the limiter and ghost fill,
    their residuals, and 8 steps of each"""
    out = {}
    for case, N, L in (("sod", 16, 1.0), ("pv", 16, 10.0), ("lmv", 16, 1.0)):
        h = L / N
        p0 = O.rec3_p0(0.1) if case == "lmv" else 0.0
        U = O.ref_rec3_ic(N, h, case, p0)
        O.ref_rec3_limit(U, N)
        O.ref_rec3_bc(U, N)
        R, lam = O.ref_rec3_rhs(U, N, h)
        U8 = U.copy()
        info = O.ref_rec3_run(U8, N, h, 0.4, 8)
        out.update({case + "_U0": U, case + "_rhs": R, case + "_lam": lam, case + "_U8": U8,
                    case + "_info": np.array(info)})
    return out


def bak_state(N, seed):
    """The .bak's circular Sod with a seeded velocity field and the kinetic
    energy added (so every term of the scheme is exercised), unpadded."""
    U = O.ref_bak_ic(N, 1.0 / N)
    rng = np.random.default_rng(seed)
    U[1] = U[0] * rng.uniform(-0.5, 0.5, (N, N))
    U[2] = U[0] * rng.uniform(-0.5, 0.5, (N, N))
    U[3] += 0.5 * (U[1] ** 2 + U[2] ** 2) / U[0]
    return U


def _bak():
    """fv_up7_ducros_2d.cu.bak's own kernels (FP64): its circular Sod, the
    residual, lam and sensor of a seeded state for orders 3/5/7 with both
    viscosity terms on, and 6 steps of each from the Sod state"""
    out = {}
    N = 16
    h = 1.0 / N
    out["ic"] = O.ref_bak_ic(N, h)
    for order in (3, 5, 7):
        U = bak_state(N, order)
        R, lam = O.ref_bak_rhs(U, N, h, order, 0.5, 0.02, 0.05)
        out.update({"o%d_U" % order: U, "o%d_rhs" % order: R, "o%d_lam" % order: lam,
                    "o%d_sd" % order: O.ref_bak_sensor(U, N, h, 0.05)})
        U6 = out["ic"].copy()
        info = O.ref_bak_run(U6, N, h, 0.4, 6, 1e30, order, 0.5, 0.02, 0.05)
        out.update({"o%d_U6" % order: U6, "o%d_info" % order: np.array(info)})
    return out


def main() -> None:
    if not O.have_ref_host():
        raise SystemExit("oracle/_ref is not built (python oracle/build.py)")
    O.ref_set_threads(1)  # scatter kernels add in work-item order
    if O.have_ref_carb():
        np.savez_compressed(HERE / "faces_carb_f64.npz", **_faces_carb())
    if O.have_ref_rec3():
        np.savez_compressed(HERE / "rec3_16.npz", **_rec3())
    if O.have_ref_bak():
        np.savez_compressed(HERE / "bak_16.npz", **_bak())
    if sys.argv[1:] in (["carb"], ["rec3"], ["bak"]):
        return
    N = 16
    for dtype, sfx in ((np.float64, "f64"), (np.float32, "f32")):
        np.savez_compressed(HERE / ("faces_%s.npz" % sfx), **_faces(dtype))
        h = 1.0 / N
        U = O.ref_up_ic_sod(N, h, dtype)
        O.ref_up_bc(U, N, 0)
        R, lam = O.ref_up_rhs(U, N, h)
        U5 = U.copy()
        info = O.ref_up_run(U5, N, h, 0.4, 0, 5)
        np.savez_compressed(HERE / ("up7_sod16_%s.npz" % sfx), U0=U, rhs=R, lam=lam, U5=U5, info=np.array(info[:5]))
    # periodic and transmissive harness compositions on a vortex / random state
    for bc, tag in ((1, "periodic"), (2, "transmissive")):
        n = 16
        w = vortex(n, x0=-5, y0=-5, length=10.0)
        U = pad(w, 4)
        O.ref_up_bc(U, n, bc)
        U5 = U.copy()
        info = O.ref_up_run(U5, n, 10.0 / n, 0.5, bc, 5)
        np.savez_compressed(HERE / ("up7_vortex16_%s_f64.npz" % tag), U0=U, U5=U5, info=np.array(info[:5]))
    # KEEP
    n = 16
    for lmv, tag in ((False, "sod"), (True, "lmv")):
        U = O.ref_keep_ic(n, 1.0 / n, lmv)
        O.ref_host("keep").ref_keep_bc(O._ptr(U), C.c_int(n), C.c_int(n + 4))
        R, lam, edm = O.ref_keep_rhs(U, n, 1.0 / n)
        U5 = U.copy()
        info = O.ref_keep_run(U5, n, 1.0 / n, 0.2, 5)
        np.savez_compressed(HERE / ("keep_%s16.npz" % tag), U0=U, rhs=R, lam=lam, edmax=np.array(edm), U5=U5,
                            info=np.array(info[:5]))
    print("wrote", sorted(p.name for p in HERE.glob("*.npz")))


if __name__ == "__main__":
    main()
