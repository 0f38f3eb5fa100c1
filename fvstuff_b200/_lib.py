"""ctypes declarations of the C ABI in include/fvb.h.

The shared library must exist (built by ``fvstuff_b200.build``); there is no
fallback: importing the bindings without it raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import os

# the in-tree build; FVB_LIBRARY may name another build of the same sources
LIB_PATH = Path(os.environ.get("FVB_LIBRARY", Path(__file__).resolve().parent / "libfvb.so"))

# enums (include/fvb.h)
OK, ERR_INVALID, ERR_CUDA, ERR_NOMEM, ERR_BLOWUP, ERR_DT_UNDERFLOW, ERR_NOT_FOUND, ERR_TIMEOUT = range(8)
FLUX = {"up_ducros": 0, "keep": 1, "up_ducros_hll": 2, "up_ducros_roe": 3, "rec3": 4, "up_hllc_d2av": 5}
PREC = {"f64": 0, "f32": 1, "f32c": 2}
BC = {"reflect": 0, "periodic": 1, "transmissive": 2}
LAYOUT = {"prim": 0, "cons": 1}
DTYPE = {"f32": 0, "f64": 1}
CASE = {"sod": 0, "vortex": 1, "kh": 2, "riemann4": 3, "keep_sod": 4, "lmv": 5, "uniform": 6, "rec3_sod": 7,
        "paper_vortex": 8, "gresho": 9}


class Config(C.Structure):
    _fields_ = [("n", C.c_int), ("order", C.c_int), ("flux", C.c_int), ("precision", C.c_int),
                ("bc_x", C.c_int), ("bc_y", C.c_int), ("x0", C.c_double), ("y0", C.c_double),
                ("length", C.c_double), ("gamma", C.c_double), ("cfl", C.c_double), ("device", C.c_int),
                ("stream", C.c_void_p), ("tile", C.c_int)]


class Case(C.Structure):
    _fields_ = [("kind", C.c_int), ("seed", C.c_uint64), ("param", C.c_double * 8)]


class Stats(C.Structure):
    _fields_ = [("t", C.c_double), ("dt", C.c_double), ("lam_max", C.c_double), ("t_stop", C.c_double),
                ("steps", C.c_int64), ("status", C.c_int), ("nonfinite", C.c_int), ("sums", C.c_double * 4)]


class BatchConfig(C.Structure):
    _fields_ = [("precision", C.c_int), ("order", C.c_int), ("device", C.c_int), ("stream", C.c_void_p),
                ("hbm_budget", C.c_size_t), ("max_instances", C.c_int), ("use_graph", C.c_int), ("tile", C.c_int)]


class InstanceDesc(C.Structure):
    _fields_ = [("n", C.c_int), ("bc_x", C.c_int), ("bc_y", C.c_int), ("x0", C.c_double), ("y0", C.c_double),
                ("length", C.c_double), ("gamma", C.c_double), ("cfl", C.c_double), ("t_end", C.c_double),
                ("ic", Case)]


class Request(C.Structure):
    _fields_ = [("arrival", C.c_double), ("desc", InstanceDesc), ("out", C.c_void_p), ("out_layout", C.c_int),
                ("out_dtype", C.c_int)]


class RequestResult(C.Structure):
    _fields_ = [("admitted", C.c_double), ("finished", C.c_double), ("status", C.c_int), ("steps", C.c_int64),
                ("t", C.c_double)]


class ServeConfig(C.Structure):
    _fields_ = [("batch", BatchConfig), ("steps_per_round", C.c_int), ("policy", C.c_int), ("max_cells", C.c_double),
                ("max_seconds", C.c_double)]


SERVE_POLICY = {"fifo": 0, "shortest": 1}


_P = C.c_void_p
_SIG = {
    "fvb_version": (C.c_char_p, []),
    "fvb_device_name": (C.c_char_p, [C.c_int]),
    "fvb_last_error": (C.c_char_p, []),
    "fvb_config_default": (None, [C.POINTER(Config), C.c_int]),
    "fvb_case_default": (None, [C.POINTER(Case), C.c_int, C.c_double, C.c_double, C.c_double]),
    "fvb_create": (C.c_int, [C.POINTER(Config), C.POINTER(_P)]),
    "fvb_destroy": (None, [_P]),
    "fvb_ghost_width": (C.c_int, [_P]),
    "fvb_init_case": (C.c_int, [_P, C.POINTER(Case)]),
    "fvb_set_state": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_int, C.c_int]),
    "fvb_get_state": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_int, C.c_int]),
    "fvb_get_state_hilo": (C.c_int, [_P, _P, _P]),
    "fvb_frame_begin": (C.c_int, [_P]),
    "fvb_debug_drop_load": (C.c_int, [_P]),
    "fvb_set_d2av": (C.c_int, [_P, C.c_double, C.c_double, C.c_double]),
    "fvb_limiter_fixes": (C.c_int, [_P, C.POINTER(C.c_int64)]),
    "fvb_frame_end": (C.c_int, [_P, _P]),
    "fvb_save": (C.c_int, [_P, C.c_char_p]),
    "fvb_load": (C.c_int, [_P, C.c_char_p]),
    "fvb_step": (C.c_int, [_P, C.c_int, C.c_double]),
    "fvb_advance": (C.c_int, [_P, C.c_double, C.c_int64, C.c_int]),
    "fvb_sync": (C.c_int, [_P, C.POINTER(Stats)]),
    "fvb_stats_post": (C.c_int, [_P, C.c_int]),
    "fvb_stats_wait": (C.c_int, [_P, C.c_int, C.POINTER(Stats)]),
    "fvb_stats_sums": (C.c_int, [_P, C.POINTER(Stats)]),
    "fvb_set_graph": (C.c_int, [_P, C.c_int]),
    "fvb_up_rhs": (C.c_int, [_P, _P, _P, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, _P]),
    "fvb_apply_bc": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _P]),
    "fvb_rk3_stage": (C.c_int, [C.c_int, _P, _P, _P, _P, C.c_double, C.c_int, C.c_int, C.c_double, C.c_int, _P]),
    "fvb_max": (C.c_int, [_P, C.c_size_t, _P, C.c_int, _P]),
    "fvb_step_noalloc": (C.c_int, [_P, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
                                   C.c_int, C.c_double, C.c_double, _P, C.POINTER(Stats)]),
    "fvb_batch_create": (C.c_int, [C.POINTER(BatchConfig), C.POINTER(_P)]),
    "fvb_batch_destroy": (None, [_P]),
    "fvb_batch_instance_bytes": (C.c_size_t, [_P, C.c_int]),
    "fvb_batch_add": (C.c_int, [_P, C.POINTER(InstanceDesc), C.POINTER(C.c_int)]),
    "fvb_batch_run": (C.c_int, [_P, C.c_int]),
    "fvb_batch_poll": (C.c_int, [_P, C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_int)]),
    "fvb_batch_get_state": (C.c_int, [_P, C.c_int, _P, C.c_int, C.c_int, C.c_int]),
    "fvb_batch_instance_stats": (C.c_int, [_P, C.c_int, C.POINTER(Stats)]),
    "fvb_batch_instance_sums": (C.c_int, [_P, C.c_int, C.POINTER(Stats)]),
    "fvb_batch_remove": (C.c_int, [_P, C.c_int]),
    "fvb_batch_active": (C.c_int, [_P]),
    "fvb_batch_bytes_in_use": (C.c_size_t, [_P]),
    "fvb_serve_run": (C.c_int, [C.POINTER(ServeConfig), C.POINTER(Request), C.c_int, C.POINTER(RequestResult),
                                C.POINTER(C.c_double)]),
}

_lib = None


def lib() -> C.CDLL:
    """The loaded libfvb.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError("libfvb.so is not built: run `python -m fvstuff_b200.build` "
                              "(there is no CPU fallback)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIG.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def declared_symbols() -> list[str]:
    return list(_SIG)


class FvbError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = lib().fvb_last_error().decode(errors="replace")
        super().__init__("%s failed (status %d): %s" % (where, status, msg))
        self.status = status


def check(status: int, where: str) -> None:
    if status != OK:
        raise FvbError(status, where)
