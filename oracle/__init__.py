"""The oracle -- TEST INFRASTRUCTURE ONLY.

ctypes access to
  * ``liboracle.so``: the plain-C restatement of fvStuff's finite-volume step
    (fvb_oracle.c), and
  * ``_ref/*.so``: the reference's own kernels compiled for the host and for
    the GPU (built by oracle/build.py from the reference checkout).

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py
use this package, and only as the checker or the timed CPU baseline; the
product library (fvstuff_b200) never imports it.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF = HERE / "_ref"

_D = C.POINTER(C.c_double)
_F = C.POINTER(C.c_float)
_libs: dict[str, C.CDLL] = {}


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_D if a.dtype == np.float64 else _F)


def _load(path: Path) -> C.CDLL:
    key = str(path)
    if key not in _libs:
        if not path.exists():
            raise FileNotFoundError("%s is not built (run oracle/build.py)" % path)
        _libs[key] = C.CDLL(key)
    return _libs[key]


def lib() -> C.CDLL:
    p = HERE / "liboracle.so"
    if not p.exists():
        from . import build as _b
        _b.build_oracle()
    return _load(p)


def have_ref_host() -> bool:
    return (REF / "libref_host_up7_f64.so").exists()


def have_ref_gpu() -> bool:
    return (REF / "libref_gpu_up7_f64.so").exists()


def ref_host(kind: str) -> C.CDLL:
    """kind: 'up7_f32', 'up7_f64' or 'keep'."""
    return _load(REF / ("libref_host_%s.so" % kind))


def ref_gpu(kind: str) -> C.CDLL:
    return _load(REF / ("libref_gpu_%s.so" % kind))


def _sfx(dtype) -> str:
    return "f64" if np.dtype(dtype) == np.float64 else "f32"


def _real(dtype):
    return C.c_double if np.dtype(dtype) == np.float64 else C.c_float


def ghost_width(order: int = 7) -> int:
    return (order + 1) // 2


def padded(N: int, g: int, dtype=np.float64) -> np.ndarray:
    return np.zeros((4, N + 2 * g, N + 2 * g), dtype=dtype)


# ---------------------------------------------------------------------------
# restatement (liboracle.so)
# ---------------------------------------------------------------------------
RIEMANN = {"hllc": 0, "hll": 1, "roe": 2}


def up_rhs(Q: np.ndarray, N: int, h: float, order: int = 7, riemann: str = "hllc"):
    """Residual (4,N,N) and lam (N,N) of a padded primitive state; `riemann`
    picks the solver on the reconstructed states (fv_up7's HLLC, or carb_fv's
    HLL / Roe)."""
    g = ghost_width(order)
    assert Q.shape == (4, N + 2 * g, N + 2 * g) and Q.flags.c_contiguous
    s = _sfx(Q.dtype)
    R = np.empty((4, N, N), Q.dtype)
    lam = np.empty((N, N), Q.dtype)
    getattr(lib(), "orc_up_rhs_" + s)(_ptr(Q), _ptr(R), _ptr(lam), C.c_int(N), C.c_int(g),
                                      C.c_int(order + 100 * RIEMANN[riemann]), _real(Q.dtype)(h))
    return R, lam


def bc(Q: np.ndarray, N: int, g: int, kind: int) -> None:
    getattr(lib(), "orc_bc_" + _sfx(Q.dtype))(_ptr(Q), C.c_int(N), C.c_int(g), C.c_int(kind))


def rk3(stage, Uo, U0, Uk, L, dt, N, g) -> None:
    getattr(lib(), "orc_rk3_" + _sfx(Uo.dtype))(C.c_int(stage), _ptr(Uo), _ptr(U0), _ptr(Uk), _ptr(L),
                                                _real(Uo.dtype)(dt), C.c_int(N), C.c_int(g))


def up_run(U: np.ndarray, N: int, h: float, cfl: float, bc_kind: int, max_steps: int,
           t_stop: float = 1e30, order: int = 7, riemann: str = "hllc"):
    """Advance U (padded primitives, ghosts filled) in place; returns
    (status, t, steps, lam_max, last_dt)."""
    g = ghost_width(order)
    info = np.zeros(4)
    st = getattr(lib(), "orc_up_run_" + _sfx(U.dtype))(
        _ptr(U), C.c_int(N), C.c_int(g), C.c_int(order + 100 * RIEMANN[riemann]), C.c_int(bc_kind),
        _real(U.dtype)(h),
        _real(U.dtype)(cfl), C.c_int(max_steps), C.c_double(t_stop), _ptr(info))
    return int(st), float(info[0]), int(info[1]), float(info[2]), float(info[3])


def ic_sod(N: int, h: float, dtype=np.float64, order: int = 7) -> np.ndarray:
    g = ghost_width(order)
    U = padded(N, g, dtype)
    getattr(lib(), "orc_ic_sod_" + _sfx(dtype))(_ptr(U), C.c_int(N), C.c_int(g), _real(dtype)(h))
    return U


def hllc(L, R, dtype=np.float64):
    L = np.ascontiguousarray(L, dtype); R = np.ascontiguousarray(R, dtype); F = np.empty(4, dtype)
    getattr(lib(), "orc_hllc_" + _sfx(dtype))(_ptr(L), _ptr(R), _ptr(F))
    return F


def hll(L, R):
    """carb_fv's HLL flux, FP64, normal frame."""
    L, R = np.ascontiguousarray(L, np.float64), np.ascontiguousarray(R, np.float64)
    F = np.empty(4)
    lib().orc_hll_f64(_ptr(L), _ptr(R), _ptr(F))
    return F


def roe(L, R):
    """carb_fv's Roe flux with the Harten-Hyman fix, FP64, normal frame."""
    L, R = np.ascontiguousarray(L, np.float64), np.ascontiguousarray(R, np.float64)
    F = np.empty(4)
    lib().orc_roe_f64(_ptr(L), _ptr(R), _ptr(F))
    return F


def have_ref_carb() -> bool:
    return (REF / "libref_host_carb.so").exists()


def ref_carb_flux(kind: str, WL, WR, nx: float, ny: float):
    """carb_fv_2d.cu's own hll_n / roe_n / hllc_n, compiled for the host."""
    WL, WR = np.ascontiguousarray(WL, np.float64), np.ascontiguousarray(WR, np.float64)
    F = np.empty(4)
    getattr(ref_host("carb"), "ref_carb_" + kind)(_ptr(WL), _ptr(WR), C.c_double(nx), C.c_double(ny), _ptr(F))
    return F


# ---- fv_rec3_2d.cu (FP64, periodic, g = 2, N even) --------------------------
REC3_CASES = {"sod": 0, "pv": 1, "lmv": 2}


def rec3_p0(eps: float = 0.1) -> float:
    """Gresho background pressure 1/(gamma eps^2) - 1/2 (fv_rec3_2d.cu:518)."""
    return 1.0 / (1.4 * eps * eps) - 0.5


def rec3_ic(N: int, h: float, case: str = "sod", p0: float = 0.0) -> np.ndarray:
    U = np.zeros((4, N + 4, N + 4))
    lib().orc_rec3_ic(_ptr(U), C.c_int(N), C.c_double(h), C.c_int(REC3_CASES[case]), C.c_double(p0))
    return U


def rec3_limit(U: np.ndarray, N: int) -> int:
    return int(lib().orc_rec3_limit(_ptr(U), C.c_int(N)))


def rec3_rhs(U: np.ndarray, N: int, h: float):
    R = np.empty((4, N, N)); lam = np.empty((N, N))
    lib().orc_rec3_rhs(_ptr(U), _ptr(R), _ptr(lam), C.c_int(N), C.c_double(h))
    return R, lam


def rec3_run(U: np.ndarray, N: int, h: float, cfl: float, max_steps: int, t_stop: float = 1e30):
    """(status, t, steps, lam_max, last dt, brutal fixes); U advanced in place."""
    info = np.zeros(5)
    st = lib().orc_rec3_run(_ptr(U), C.c_int(N), C.c_double(h), C.c_double(cfl), C.c_int(max_steps),
                            C.c_double(t_stop), _ptr(info))
    return int(st), float(info[0]), int(info[1]), float(info[2]), float(info[3]), int(info[4])


def rec3_err(U: np.ndarray, N: int, h: float, case: str, p0: float = 0.0):
    out = np.zeros(2)
    lib().orc_rec3_err(_ptr(U), C.c_int(N), C.c_double(h), C.c_int(REC3_CASES[case]), C.c_double(p0), _ptr(out))
    return float(out[0]), float(out[1])


def rec3_hllc(L, R):
    L, R = np.ascontiguousarray(L, np.float64), np.ascontiguousarray(R, np.float64)
    F = np.empty(4)
    lib().orc_rec3_hllc(_ptr(L), _ptr(R), _ptr(F))
    return F


def rec3_scale(Ub, U):
    Ub, U = np.ascontiguousarray(Ub, np.float64), np.array(U, np.float64)
    lib().orc_rec3_scale(_ptr(Ub), _ptr(U))
    return U


def have_ref_rec3() -> bool:
    return (REF / "libref_host_rec3.so").exists()


def ref_rec3(name: str):
    f = getattr(ref_host("rec3"), "ref_rec3_" + name)
    if name in ("limit", "run"):
        f.restype = C.c_int
    return f


def ref_rec3_ic(N, h, case="sod", p0=0.0):
    U = np.zeros((4, N + 4, N + 4))
    ref_rec3("ic")(_ptr(U), C.c_int(N), C.c_int(N + 4), C.c_double(h), C.c_int(REC3_CASES[case]), C.c_double(p0))
    return U


def ref_rec3_rhs(U, N, h):
    R = np.empty((4, N, N)); lam = np.empty((N, N))
    ref_rec3("rhs")(_ptr(U), _ptr(R), _ptr(lam), C.c_int(N), C.c_int(N + 4), C.c_double(h))
    return R, lam


def ref_rec3_limit(U, N):
    return int(ref_rec3("limit")(_ptr(U), C.c_int(N), C.c_int(N + 4)))


def ref_rec3_bc(U, N):
    ref_rec3("bc")(_ptr(U), C.c_int(N), C.c_int(N + 4))


def ref_rec3_run(U, N, h, cfl, max_steps, t_stop=1e30):
    info = np.zeros(5)
    st = ref_rec3("run")(_ptr(U), C.c_int(N), C.c_double(h), C.c_double(cfl), C.c_int(max_steps),
                         C.c_double(t_stop), _ptr(info))
    return int(st), float(info[0]), int(info[1]), float(info[2]), float(info[3]), int(info[4])


# ---- fv_up7_ducros_2d.cu.bak: UP + HLLC + Ducros-gated D2 viscosity (FP64) -
def d2av_ghost(order: int = 5) -> int:
    return max((order + 1) // 2, 3)


def d2av_ic_sod(N: int, h: float, order: int = 5) -> np.ndarray:
    """The .bak's circular Sod, conserved, padded (ghosts not filled)."""
    g = d2av_ghost(order)
    U = padded(N, g)
    lib().orc_d2av_ic_sod(_ptr(U), C.c_int(N), C.c_double(h), C.c_int(g))
    return U


def d2av_rhs(Q: np.ndarray, N: int, h: float, order: int = 5, c2: float = 0.5, cg: float = 0.0,
             sc: float = 0.05):
    """Residual (4,N,N) and lam (N,N) of a padded conserved state with its ghosts filled."""
    g = d2av_ghost(order)
    assert Q.shape == (4, N + 2 * g, N + 2 * g) and Q.flags.c_contiguous and Q.dtype == np.float64
    R = np.empty((4, N, N)); lam = np.empty((N, N))
    lib().orc_d2av_rhs(_ptr(Q), _ptr(R), _ptr(lam), C.c_int(N), C.c_int(order), C.c_double(h), C.c_double(c2),
                       C.c_double(cg), C.c_double(sc))
    return R, lam


def d2av_sensor(Q: np.ndarray, N: int, h: float, order: int = 5, sc: float = 0.05) -> np.ndarray:
    SD = np.empty((N, N))
    lib().orc_d2av_sensor(_ptr(Q), _ptr(SD), C.c_int(N), C.c_int(order), C.c_double(h), C.c_double(sc))
    return SD


def d2av_run(U: np.ndarray, N: int, h: float, cfl: float, bc_kind: int, max_steps: int, t_stop: float = 1e30,
             order: int = 5, c2: float = 0.5, cg: float = 0.0, sc: float = 0.05):
    """Advance U (padded conserved, ghosts filled) in place; returns
    (status, t, steps, lam_max, last_dt)."""
    info = np.zeros(4)
    st = lib().orc_d2av_run(_ptr(U), C.c_int(N), C.c_int(order), C.c_int(bc_kind), C.c_double(h),
                            C.c_double(cfl), C.c_double(c2), C.c_double(cg), C.c_double(sc), C.c_int(max_steps),
                            C.c_double(t_stop), _ptr(info))
    return int(st), float(info[0]), int(info[1]), float(info[2]), float(info[3])


def d2av_hllc(UL, UR):
    """The .bak's HLLC on conserved states, normal frame (rho, m_n, m_t, E)."""
    UL, UR = np.ascontiguousarray(UL, np.float64), np.ascontiguousarray(UR, np.float64)
    F = np.empty(4)
    lib().orc_d2av_hllc(_ptr(UL), _ptr(UR), _ptr(F))
    return F


def have_ref_bak() -> bool:
    return (REF / "libref_host_bak.so").exists()


def ref_bak_rhs(U: np.ndarray, N: int, h: float, order: int = 5, c2: float = 0.5, cg: float = 0.0,
                sc: float = 0.05):
    """The .bak's own compute_rhs (host build) on an unpadded (4,N,N) conserved state."""
    U = np.ascontiguousarray(U, np.float64)
    R = np.empty((4, N, N)); lam = np.empty((N, N))
    ref_host("bak").ref_bak_rhs(_ptr(U), _ptr(R), _ptr(lam), C.c_int(N), C.c_double(h), C.c_double(c2),
                                C.c_double(cg), C.c_double(sc), C.c_int(order))
    return R, lam


def ref_bak_sensor(U: np.ndarray, N: int, h: float, sc: float = 0.05) -> np.ndarray:
    U = np.ascontiguousarray(U, np.float64)
    SD = np.empty((N, N))
    ref_host("bak").ref_bak_sensor(_ptr(U), _ptr(SD), C.c_int(N), C.c_double(h), C.c_double(sc))
    return SD


def ref_bak_ic(N: int, h: float) -> np.ndarray:
    U = np.zeros((4, N, N))
    ref_host("bak").ref_bak_ic(_ptr(U), C.c_int(N), C.c_double(h))
    return U


def ref_bak_run(U: np.ndarray, N: int, h: float, cfl: float, max_steps: int, t_stop: float = 1e30,
                order: int = 5, c2: float = 0.5, cg: float = 0.0, sc: float = 0.05):
    """The .bak's kernels in its time loop (reflecting walls), unpadded U in place."""
    info = np.zeros(4)
    f = ref_host("bak").ref_bak_run
    f.restype = C.c_int
    st = f(_ptr(U), C.c_int(N), C.c_double(h), C.c_double(cfl), C.c_double(c2), C.c_double(cg), C.c_double(sc),
           C.c_int(order), C.c_int(max_steps), C.c_double(t_stop), _ptr(info))
    return int(st), float(info[0]), int(info[1]), float(info[2]), float(info[3])


def hlle(L, R, dtype=np.float64):
    L = np.ascontiguousarray(L, dtype); R = np.ascontiguousarray(R, dtype); F = np.empty(4, dtype)
    getattr(lib(), "orc_hlle_" + _sfx(dtype))(_ptr(L), _ptr(R), _ptr(F))
    return F


def upface(order, s, dtype=np.float64):
    s = np.ascontiguousarray(s, dtype)
    vL = np.empty(1, dtype); vR = np.empty(1, dtype)
    getattr(lib(), "orc_upface_" + _sfx(dtype))(C.c_int(order), _ptr(s), _ptr(vL), _ptr(vR))
    return float(vL[0]), float(vR[0])


# KEEP family ---------------------------------------------------------------
def keep_rhs(Q: np.ndarray, N: int, h: float):
    R = np.empty((4, N, N)); lam = np.empty((N, N)); ed = np.empty((N, N))
    lib().orc_keep_ed(_ptr(Q), _ptr(ed), C.c_int(N))
    edmax = float(max(0.0, np.nanmax(ed))) if ed.size else 0.0
    lib().orc_keep_rhs(_ptr(Q), _ptr(R), _ptr(lam), C.c_int(N), C.c_double(h), C.c_double(edmax))
    return R, lam, edmax


def keep_run(U: np.ndarray, N: int, h: float, cfl: float, max_steps: int, t_stop: float = 1e30):
    info = np.zeros(4)
    st = lib().orc_keep_run(_ptr(U), C.c_int(N), C.c_double(h), C.c_double(cfl), C.c_int(max_steps),
                            C.c_double(t_stop), _ptr(info))
    return int(st), float(info[0]), int(info[1]), float(info[2]), float(info[3])


def keep_ic(N: int, h: float, lmv: bool = False, eps: float = 0.1) -> np.ndarray:
    U = padded(N, 2)
    if lmv:
        lib().orc_keep_ic_lmv(_ptr(U), C.c_int(N), C.c_double(h), C.c_double(eps))
    else:
        lib().orc_keep_ic_sod(_ptr(U), C.c_int(N), C.c_double(h))
    return U


def keep_err_lmv(U: np.ndarray, N: int, h: float, eps: float = 0.1):
    out = np.zeros(2)
    lib().orc_keep_err_lmv(_ptr(U), C.c_int(N), C.c_double(h), C.c_double(eps), _ptr(out))
    return float(out[0]), float(out[1])


# ---------------------------------------------------------------------------
# the reference's own kernels, host build (oracle/_ref/libref_host_*.so)
# ---------------------------------------------------------------------------
def ref_set_threads(n: int) -> None:
    for k in ("up7_f32", "up7_f64", "keep", "carb", "rec3", "bak"):
        try:
            ref_host(k).ref_set_threads(C.c_int(n))
        except FileNotFoundError:
            pass


def ref_up_rhs(Q: np.ndarray, N: int, h: float):
    s = _sfx(Q.dtype)
    L = ref_host("up7_" + s)
    Np = Q.shape[-1]
    R = np.empty((4, N, N), Q.dtype); lam = np.empty((N, N), Q.dtype)
    getattr(L, "ref_up7_rhs_" + s)(_ptr(Q), _ptr(R), _ptr(lam), C.c_int(N), C.c_int(Np), _real(Q.dtype)(h))
    return R, lam


def ref_up_bc(Q: np.ndarray, N: int, kind: int) -> None:
    s = _sfx(Q.dtype)
    getattr(ref_host("up7_" + s), "ref_up7_bc_" + s)(_ptr(Q), C.c_int(N), C.c_int(Q.shape[-1]), C.c_int(kind))


def ref_up_ic_sod(N: int, h: float, dtype=np.float64) -> np.ndarray:
    s = _sfx(dtype)
    U = padded(N, 4, dtype)
    getattr(ref_host("up7_" + s), "ref_up7_ic_sod_" + s)(_ptr(U), C.c_int(N), C.c_int(N + 8), _real(dtype)(h))
    return U


def ref_native() -> C.CDLL | None:
    """The reference's FP64 kernels built for speed on this machine
    (``-O3 -march=native``, contraction allowed; oracle/build.py
    ``build_timing``): the timed CPU baseline, never a checker.  None when the
    extracted reference source is absent or the compiler fails."""
    from . import build as _b
    try:
        p = _b.build_timing()
    except (RuntimeError, OSError):
        return None
    return _load(p) if p is not None else None


def ref_up_run(U: np.ndarray, N: int, h: float, cfl: float, bc_kind: int, max_steps: int,
               t_stop: float = 1e30, lib: C.CDLL | None = None):
    """The reference's own SSP-RK3 loop on the host (U in place); `lib` picks
    another build of the same kernels (ref_native)."""
    s = _sfx(U.dtype)
    info = np.zeros(4)
    st = getattr(lib if lib is not None else ref_host("up7_" + s), "ref_up7_run_" + s)(
        _ptr(U), C.c_int(N), _real(U.dtype)(h), _real(U.dtype)(cfl), C.c_int(bc_kind), C.c_int(max_steps),
        C.c_double(t_stop), _ptr(info))
    return int(st), float(info[0]), int(info[1]), float(info[2]), float(info[3])


def ref_keep_rhs(Q: np.ndarray, N: int, h: float):
    L = ref_host("keep")
    Np = Q.shape[-1]
    R = np.empty((4, N, N)); lam = np.empty((N, N)); ed = np.empty((N, N))
    L.ref_keep_ed(_ptr(Q), _ptr(ed), C.c_int(N), C.c_int(Np))
    edmax = float(max(0.0, np.nanmax(ed)))
    L.ref_keep_rhs(_ptr(Q), _ptr(R), _ptr(lam), C.c_int(N), C.c_int(Np), C.c_double(h), C.c_double(edmax))
    return R, lam, edmax


def ref_keep_ic(N: int, h: float, lmv: bool = False, eps: float = 0.1) -> np.ndarray:
    U = padded(N, 2)
    ref_host("keep").ref_keep_ic(_ptr(U), C.c_int(N), C.c_int(N + 4), C.c_double(h), C.c_int(int(lmv)),
                                 C.c_double(eps))
    return U


def ref_keep_run(U: np.ndarray, N: int, h: float, cfl: float, max_steps: int, t_stop: float = 1e30):
    info = np.zeros(4)
    st = ref_host("keep").ref_keep_run(_ptr(U), C.c_int(N), C.c_double(h), C.c_double(cfl), C.c_int(max_steps),
                                       C.c_double(t_stop), _ptr(info))
    return int(st), float(info[0]), int(info[1]), float(info[2]), float(info[3])


# ---------------------------------------------------------------------------
# the reference's own kernels on the GPU (oracle/_ref/libref_gpu_*.so)
# ---------------------------------------------------------------------------
def refg_up_rhs(Q: np.ndarray, N: int, h: float):
    s = _sfx(Q.dtype)
    R = np.empty((4, N, N), Q.dtype); lam = np.empty((N, N), Q.dtype)
    e = getattr(ref_gpu("up7_" + s), "refg_up7_rhs_" + s)(_ptr(Q), _ptr(R), _ptr(lam), C.c_int(N),
                                                          C.c_int(Q.shape[-1]), _real(Q.dtype)(h))
    if e:
        raise RuntimeError("reference GPU rhs failed: cuda error %d" % e)
    return R, lam


def refg_up_run(U: np.ndarray, N: int, h: float, cfl: float, bc_kind: int, max_steps: int,
                t_stop: float = 1e30):
    """Returns (status, t, steps, lam_max, last_dt, ms of the stepping loop)."""
    s = _sfx(U.dtype)
    info = np.zeros(4)
    ms = C.c_float(0)
    st = getattr(ref_gpu("up7_" + s), "refg_up7_run_" + s)(
        _ptr(U), C.c_int(N), _real(U.dtype)(h), _real(U.dtype)(cfl), C.c_int(bc_kind), C.c_int(max_steps),
        C.c_double(t_stop), _ptr(info), C.byref(ms))
    if st > 0:
        raise RuntimeError("reference GPU run failed: cuda error %d" % st)
    return -int(st), float(info[0]), int(info[1]), float(info[2]), float(info[3]), float(ms.value)


def refg_keep_run(U: np.ndarray, N: int, h: float, cfl: float, max_steps: int, t_stop: float = 1e30):
    info = np.zeros(4)
    ms = C.c_float(0)
    st = ref_gpu("keep").refg_keep_run(_ptr(U), C.c_int(N), C.c_double(h), C.c_double(cfl), C.c_int(max_steps),
                                       C.c_double(t_stop), _ptr(info), C.byref(ms))
    if st > 0:
        raise RuntimeError("reference GPU run failed: cuda error %d" % st)
    return -int(st), float(info[0]), int(info[1]), float(info[2]), float(info[3]), float(ms.value)


def have_ref_gpu_bak() -> bool:
    return (REF / "libref_gpu_bak.so").exists()


def refg_bak_run(U: np.ndarray, N: int, h: float, cfl: float, max_steps: int, t_stop: float = 1e30,
                 order: int = 5, c2: float = 0.5, cg: float = 0.0, sc: float = 0.05):
    """The .bak's kernels and loop on the GPU (unpadded U in place);
    (status, t, steps, lam_max, last_dt, ms of the stepping loop)."""
    info = np.zeros(4)
    ms = C.c_float(0)
    st = ref_gpu("bak").refg_bak_run(_ptr(U), C.c_int(N), C.c_double(h), C.c_double(cfl), C.c_double(c2),
                                     C.c_double(cg), C.c_double(sc), C.c_int(order), C.c_int(max_steps),
                                     C.c_double(t_stop), _ptr(info), C.byref(ms))
    if st > 0:
        raise RuntimeError("reference GPU run failed: cuda error %d" % st)
    return -int(st), float(info[0]), int(info[1]), float(info[2]), float(info[3]), float(ms.value)


def have_ref_gpu_rec3() -> bool:
    return (REF / "libref_gpu_rec3.so").exists()


def refg_rec3_run(U: np.ndarray, N: int, h: float, cfl: float, max_steps: int, t_stop: float = 1e30):
    """fv_rec3_2d.cu's kernels and loop on the GPU (FP64; padded U after its
    limiter pass and ghost fill, in place); (status, t, steps, lam_max,
    last_dt, ms of the stepping loop)."""
    info = np.zeros(4)
    ms = C.c_float(0)
    st = ref_gpu("rec3").refg_rec3_run(_ptr(U), C.c_int(N), C.c_double(h), C.c_double(cfl), C.c_int(max_steps),
                                       C.c_double(t_stop), _ptr(info), C.byref(ms))
    if st > 0:
        raise RuntimeError("reference GPU run failed: cuda error %d" % st)
    return -int(st), float(info[0]), int(info[1]), float(info[2]), float(info[3]), float(ms.value)


def refg_up7_frame(Q: np.ndarray, N: int, h: float, fn: str) -> None:
    """The reference's frame pipeline (its sensor and derived-field kernels,
    colour ranges and 2x2 composite writer) on the padded primitive state Q
    (float32 as shipped, or float64 with the retype), written to `fn`."""
    s = _sfx(Q.dtype)
    st = getattr(ref_gpu("up7_" + s), "refg_up7_frame_" + s)(_ptr(np.ascontiguousarray(Q)), C.c_int(N),
                                                             _real(Q.dtype)(h), str(fn).encode())
    if st != 0:
        raise RuntimeError("reference frame failed: cuda error %d" % st)


def refg_program(kind: str, args: list[str]) -> list[str]:
    """Command line that runs the reference program itself -- its main(),
    unchanged, from the GPU build of `kind` ('up7_f32', 'keep', ...) -- with
    `args`, in a process of its own (it writes its files into the current
    directory and its report to stdout)."""
    import sys
    lib_path = str(REF / ("libref_gpu_%s.so" % kind))
    code = ("import ctypes, sys\n"
            "L = ctypes.CDLL(sys.argv[1])\n"
            "argv = [b'ref'] + [a.encode() for a in sys.argv[2:]]\n"
            "arr = (ctypes.c_char_p * len(argv))(*argv)\n"
            "r = L.refg_main(len(argv), arr)\n"
            "ctypes.CDLL(None).fflush(None)\n"
            "sys.exit(r)\n")
    return [sys.executable, "-c", code, lib_path, *args]


def refg_up7_frame(Q: np.ndarray, N: int, h: float, fn: str) -> None:
    """The reference's frame pipeline (its sensor and derived-field kernels,
    colour ranges and 2x2 composite writer) on the padded primitive state Q
    (float32 as shipped, or float64 with the retype), written to `fn`."""
    s = _sfx(Q.dtype)
    st = getattr(ref_gpu("up7_" + s), "refg_up7_frame_" + s)(_ptr(np.ascontiguousarray(Q)), C.c_int(N),
                                                             _real(Q.dtype)(h), str(fn).encode())
    if st != 0:
        raise RuntimeError("reference frame failed: cuda error %d" % st)


def refg_program(kind: str, args: list[str]) -> list[str]:
    """Command line that runs the reference program itself -- its main(),
    unchanged, from the GPU build of `kind` ('up7_f32', 'keep', ...) -- with
    `args`, in a process of its own (it writes its files into the current
    directory and its report to stdout)."""
    import sys
    lib_path = str(REF / ("libref_gpu_%s.so" % kind))
    code = ("import ctypes, sys\n"
            "L = ctypes.CDLL(sys.argv[1])\n"
            "argv = [b'ref'] + [a.encode() for a in sys.argv[2:]]\n"
            "arr = (ctypes.c_char_p * len(argv))(*argv)\n"
            "r = L.refg_main(len(argv), arr)\n"
            "ctypes.CDLL(None).fflush(None)\n"
            "sys.exit(r)\n")
    return [sys.executable, "-c", code, lib_path, *args]


def refg_keep_frame(Q: np.ndarray, N: int, lmv: bool, fn: str) -> None:
    """The reference's KEEP frame pipeline (its extract_fields kernel, colour
    ranges and 2-panel PNG writer) on the padded conserved state Q (g = 2)."""
    st = ref_gpu("keep").refg_keep_frame(_ptr(np.ascontiguousarray(Q, dtype=np.float64)), C.c_int(N),
                                         C.c_int(int(lmv)), str(fn).encode())
    if st != 0:
        raise RuntimeError("reference frame failed: cuda error %d" % st)
