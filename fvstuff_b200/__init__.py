"""fvstuff_b200 -- B200-native finite-volume Euler time step.

Host-side Python mirror of the C ABI (include/fvb.h).  The solver mirrors the
reference solver's knobs (fv_up7_ducros_2d.cu:886-902: N, CFL, final time,
test case; gamma and order were compile-time constants there) and its padded
SoA state layout ``Q[q, jp, ip]`` with ``Np = N + 2g``.

All computation happens in libfvb.so on the GPU; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from ._lib import BC, CASE, DTYPE, FLUX, LAYOUT, PREC, FvbError, check, lib

__all__ = ["Solver", "Stats", "FvbError", "case_params", "up_rhs", "apply_bc", "rk3_stage", "device_max",
           "ghost_width", "BC", "CASE", "PREC", "FLUX", "Batch", "serve_run"]


def ghost_width(order: int = 7, flux: str = "up_ducros") -> int:
    if flux in ("keep", "rec3"):
        return 2
    if flux == "up_hllc_d2av":  # the velocity-divergence sensor reaches 3 cells
        return max((order + 1) // 2, 3)
    return (order + 1) // 2


@dataclass
class Stats:
    t: float
    dt: float
    lam_max: float
    t_stop: float
    steps: int
    status: int
    nonfinite: int = 0
    sums: tuple = (0.0, 0.0, 0.0, 0.0)

    @classmethod
    def from_c(cls, s: L.Stats) -> "Stats":
        return cls(s.t, s.dt, s.lam_max, s.t_stop, int(s.steps), int(s.status), int(s.nonfinite), tuple(s.sums))


def case_params(kind: str, x0: float = 0.0, y0: float = 0.0, length: float = 1.0, seed: int | None = None,
                **overrides) -> L.Case:
    """fvb_case with the library defaults for `kind`, then `overrides`
    given as param0..param7 or by the names below."""
    c = L.Case()
    lib().fvb_case_default(C.byref(c), CASE[kind], x0, y0, length)
    names = {
        "sod": ["xc", "yc", "radius", "rho_out", "rho_in", "p_out", "p_in"],
        "vortex": ["beta", "u0", "v0", "xc", "yc"],
        "kh": ["yc", "half_width", "rho_in", "rho_out", "u_in", "u_out", "p", "noise"],
        "riemann4": ["xm", "ym"],
        "lmv": ["eps"],
        "gresho": ["eps"],
        "uniform": ["rho", "u", "v", "p"],
    }.get(kind, [])
    for k, v in overrides.items():
        idx = int(k[5:]) if k.startswith("param") else names.index(k)
        c.param[idx] = float(v)
    if seed is not None:
        c.seed = int(seed)
    return c


def _ptr(x):
    """Device or host address of a numpy array, a torch tensor or an int."""
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    return int(x)


def _is_device(x) -> bool:
    return hasattr(x, "is_cuda") and bool(x.is_cuda)


def _dtype_code(x) -> int:
    s = str(x.dtype)
    if "float64" in s:
        return DTYPE["f64"]
    if "float32" in s:
        return DTYPE["f32"]
    raise TypeError("state arrays must be float32 or float64, got %s" % s)


class Solver:
    """One N x N grid advanced by the fused SSP-RK3 stage kernels.

    Parameters mirror fvb_config: ``n`` cells per side on
    ``[x0, x0+length] x [y0, y0+length]``, ``order`` (3/5/7/9), ``flux``
    ('up_ducros' | 'up_ducros_hll' | 'up_ducros_roe' | 'keep' | 'rec3' |
    'up_hllc_d2av'), ``precision`` ('f64' | 'f32' | 'f32c'),
    ``bc`` / ``bc_y`` ('reflect' | 'periodic' | 'transmissive'), ``gamma``,
    ``cfl``.  Defaults are those of fv_up7_ducros_2d.cu (UP7, reflecting
    walls, unit square, CFL 0.4) with FP64 arithmetic.
    """

    def __init__(self, n: int, order: int = 7, flux: str = "up_ducros", precision: str = "f64",
                 bc: str = "reflect", bc_y: str | None = None, x0: float = 0.0, y0: float = 0.0,
                 length: float = 1.0, gamma: float = 1.4, cfl: float = 0.4, device: int = 0, tile: int = -1,
                 stream: int | None = None):
        cfg = L.Config()
        lib().fvb_config_default(C.byref(cfg), int(n))
        cfg.order, cfg.flux, cfg.precision = int(order), FLUX[flux], PREC[precision]
        cfg.bc_x, cfg.bc_y = BC[bc], BC[bc_y or bc]
        cfg.x0, cfg.y0, cfg.length, cfg.gamma, cfg.cfl = x0, y0, length, gamma, cfl
        cfg.device, cfg.tile = device, tile
        cfg.stream = stream
        h = C.c_void_p()
        check(lib().fvb_create(C.byref(cfg), C.byref(h)), "fvb_create")
        self._h = h
        self.n, self.order, self.flux, self.precision = int(n), int(order), flux, precision
        self.g = lib().fvb_ghost_width(h)
        self.np = self.n + 2 * self.g
        self.x0, self.y0, self.length, self.gamma, self.cfl = x0, y0, length, gamma, cfl
        self.h = length / n

    # lifetime -------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().fvb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # state ------------------------------------------------------------------
    def init_case(self, kind: str | L.Case, seed: int | None = None, **params) -> "Solver":
        c = kind if isinstance(kind, L.Case) else case_params(kind, self.x0, self.y0, self.length, seed, **params)
        check(lib().fvb_init_case(self._h, C.byref(c)), "fvb_init_case")
        return self

    def set_state(self, arr, layout: str = "prim", interior: bool | None = None) -> None:
        """Load a (4, Np, Np) padded or (4, N, N) interior array (numpy on the
        host or a torch CUDA tensor); ghosts are refilled, t reset to 0."""
        shape = tuple(arr.shape)
        if interior is None:
            interior = shape[-1] == self.n
        want = (4, self.n, self.n) if interior else (4, self.np, self.np)
        if shape != want:
            raise ValueError("state shape %s, expected %s" % (shape, want))
        if isinstance(arr, np.ndarray):
            arr = np.ascontiguousarray(arr)
        elif not arr.is_contiguous():
            raise ValueError("device tensor must be contiguous")
        check(lib().fvb_set_state(self._h, _ptr(arr), LAYOUT[layout], _dtype_code(arr), int(_is_device(arr)),
                                  int(interior)), "fvb_set_state")

    def get_state(self, layout: str = "prim", dtype=np.float64, interior: bool = False, out=None):
        """Copy the state out as a numpy array (or into `out`, numpy or a torch
        CUDA tensor), padded (4, Np, Np) or interior (4, N, N)."""
        side = self.n if interior else self.np
        if out is None:
            out = np.empty((4, side, side), dtype=dtype)
        check(lib().fvb_get_state(self._h, _ptr(out), LAYOUT[layout], _dtype_code(out), int(_is_device(out)),
                                  int(interior)), "fvb_get_state")
        return out

    def get_state_hilo(self):
        hi = np.empty((4, self.n, self.n), np.float32)
        lo = np.empty((4, self.n, self.n), np.float32)
        check(lib().fvb_get_state_hilo(self._h, hi.ctypes.data, lo.ctypes.data), "fvb_get_state_hilo")
        return hi, lo

    def debug_drop_load(self) -> None:
        """Failure injection: the next stage launch loses its first halo-box
        load; its bounded wait runs out and the status becomes
        FVB_ERR_TIMEOUT (see fvb_debug_drop_load)."""
        check(lib().fvb_debug_drop_load(self._h), "fvb_debug_drop_load")

    def limiter_fixes(self) -> int:
        """rec3 family: blocks whose mean needed the floor fix since the
        state was set (see fvb_limiter_fixes); 0 for the other families."""
        v = C.c_int64(0)
        check(lib().fvb_limiter_fixes(self._h, C.byref(v)), "fvb_limiter_fixes")
        return int(v.value)

    def set_d2av(self, c2: float = 0.5, cg: float = 0.0, sc: float = 0.05) -> None:
        """Coefficients of the 'up_hllc_d2av' viscosity (the .bak solver's
        C2, Cg and sc arguments; see fvb_set_d2av)."""
        check(lib().fvb_set_d2av(self._h, c2, cg, sc), "fvb_set_d2av")

    # frames ------------------------------------------------------------------
    FRAME_FIELDS = ("rho", "vorticity", "ducros", "speed", "p")

    def frame_begin(self) -> None:
        """Start extracting fv_up7's frame fields from the current state (on
        the device; copied to host on a second stream).  Steps enqueued after
        this call overlap the copy."""
        check(lib().fvb_frame_begin(self._h), "fvb_frame_begin")

    def frame_end(self) -> dict:
        """Wait for the frame begun last; {field: (n, n) float32 array}."""
        out = np.empty((5, self.n, self.n), np.float32)
        check(lib().fvb_frame_end(self._h, out.ctypes.data), "fvb_frame_end")
        return dict(zip(self.FRAME_FIELDS, out))

    # stepping ----------------------------------------------------------------
    def step(self, nsteps: int = 1, t_stop: float = math.inf) -> None:
        """Enqueue up to `nsteps` steps (asynchronous)."""
        check(lib().fvb_step(self._h, int(nsteps), float(min(t_stop, 1e300))), "fvb_step")

    def advance(self, t_stop: float, max_steps: int = 2 ** 62, chunk: int = 0) -> Stats:
        check(lib().fvb_advance(self._h, float(t_stop), int(max_steps), int(chunk)), "fvb_advance")
        return self.sync()

    def sync(self) -> Stats:
        s = L.Stats()
        check(lib().fvb_sync(self._h, C.byref(s)), "fvb_sync")
        return Stats.from_c(s)

    def post_stats(self, slot: int = 0) -> None:
        """Enqueue a read of the step control behind the steps enqueued so far."""
        check(lib().fvb_stats_post(self._h, int(slot)), "fvb_stats_post")

    def wait_stats(self, slot: int = 0) -> Stats:
        """Wait for the read posted to `slot` (not for later steps)."""
        s = L.Stats()
        check(lib().fvb_stats_wait(self._h, int(slot), C.byref(s)), "fvb_stats_wait")
        return Stats.from_c(s)

    def stats(self) -> Stats:
        s = L.Stats()
        check(lib().fvb_stats_sums(self._h, C.byref(s)), "fvb_stats_sums")
        return Stats.from_c(s)

    def save(self, path) -> None:
        """Exact checkpoint (state, time, steps, next-dt wave speed)."""
        check(lib().fvb_save(self._h, str(path).encode()), "fvb_save")

    def load(self, path) -> None:
        check(lib().fvb_load(self._h, str(path).encode()), "fvb_load")

    def set_graph(self, enable: bool) -> None:
        check(lib().fvb_set_graph(self._h, int(bool(enable))), "fvb_set_graph")


# ---- the reference's kernel-level contract (device buffers, IDX_P layout) --

def up_rhs(Qp, rhs, lam, n: int, np_: int, h: float, order: int = 7, gamma: float = 1.4, stream: int = 0) -> None:
    """compute_rhs of fv_up7_ducros_2d.cu:370 on torch CUDA tensors."""
    check(lib().fvb_up_rhs(_ptr(Qp), _ptr(rhs), _ptr(lam), n, np_, order, h, gamma, _dtype_code(Qp), stream),
          "fvb_up_rhs")


def apply_bc(Qp, n: int, np_: int, bc: str = "reflect", bc_y: str | None = None, layout: str = "prim",
             stream: int = 0) -> None:
    check(lib().fvb_apply_bc(_ptr(Qp), n, np_, BC[bc], BC[bc_y or bc], LAYOUT[layout], _dtype_code(Qp), stream),
          "fvb_apply_bc")


def rk3_stage(stage: int, Uo, U0, Uk, Lr, dt: float, n: int, np_: int, gamma: float = 1.4, stream: int = 0) -> None:
    check(lib().fvb_rk3_stage(stage, _ptr(Uo), _ptr(U0), _ptr(Uk) if Uk is not None else 0, _ptr(Lr), dt, n, np_,
                              gamma, _dtype_code(Uo), stream), "fvb_rk3_stage")


def device_max(x, out, stream: int = 0) -> None:
    check(lib().fvb_max(_ptr(x), x.numel(), _ptr(out), _dtype_code(x), stream), "fvb_max")


from .batch import Batch, serve_run  # noqa: E402
