"""Batched and served forms: many grids of different sizes advanced together
by one persistent launch per RK stage (fvb_batch_*), and a continuous-
batching serving loop over a request stream (fvb_serve_run)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from ._lib import BC, LAYOUT, PREC, check, lib


class Batch:
    def __init__(self, precision: str = "f32c", device: int = 0, hbm_budget: int = 0, max_instances: int = 0,
                 use_graph: bool = True, tile: int = -1, order: int = 7):
        cfg = L.BatchConfig()
        cfg.precision, cfg.order, cfg.device = PREC[precision], order, device
        cfg.hbm_budget, cfg.max_instances, cfg.use_graph, cfg.tile = hbm_budget, max_instances, int(use_graph), tile
        h = C.c_void_p()
        check(lib().fvb_batch_create(C.byref(cfg), C.byref(h)), "fvb_batch_create")
        self._h = h
        self.precision = precision

    def close(self):
        if getattr(self, "_h", None):
            lib().fvb_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def desc(n: int, case: L.Case, t_end: float, bc: str = "transmissive", bc_y: str | None = None,
             x0: float = 0.0, y0: float = 0.0, length: float = 1.0, gamma: float = 1.4, cfl: float = 0.5):
        d = L.InstanceDesc()
        d.n, d.bc_x, d.bc_y = n, BC[bc], BC[bc_y or bc]
        d.x0, d.y0, d.length, d.gamma, d.cfl, d.t_end = x0, y0, length, gamma, cfl, t_end
        d.ic = case
        return d

    def add(self, d: L.InstanceDesc) -> int:
        i = C.c_int()
        check(lib().fvb_batch_add(self._h, C.byref(d), C.byref(i)), "fvb_batch_add")
        return i.value

    def instance_bytes(self, n: int) -> int:
        return int(lib().fvb_batch_instance_bytes(self._h, n))

    def run(self, nsteps: int) -> None:
        check(lib().fvb_batch_run(self._h, nsteps), "fvb_batch_run")

    def poll(self, cap: int = 4096) -> list[int]:
        ids = (C.c_int * cap)()
        nd = C.c_int()
        check(lib().fvb_batch_poll(self._h, ids, cap, C.byref(nd)), "fvb_batch_poll")
        return list(ids[: nd.value])

    def get_state(self, iid: int, n: int, layout: str = "prim", dtype=np.float64, interior: bool = True):
        side = n if interior else n + 8
        out = np.empty((4, side, side), dtype)
        check(lib().fvb_batch_get_state(self._h, iid, out.ctypes.data, LAYOUT[layout],
                                        1 if out.dtype == np.float64 else 0, int(interior)), "fvb_batch_get_state")
        return out

    def stats(self, iid: int, sums: bool = False):
        """The instance's step control; with `sums`, also its FP64 conserved
        sums and non-finite flag."""
        from . import Stats
        s = L.Stats()
        if sums:
            check(lib().fvb_batch_instance_sums(self._h, iid, C.byref(s)), "fvb_batch_instance_sums")
        else:
            check(lib().fvb_batch_instance_stats(self._h, iid, C.byref(s)), "fvb_batch_instance_stats")
        return Stats.from_c(s)

    def remove(self, iid: int) -> None:
        check(lib().fvb_batch_remove(self._h, iid), "fvb_batch_remove")

    def active(self) -> int:
        return int(lib().fvb_batch_active(self._h))

    def bytes_in_use(self) -> int:
        return int(lib().fvb_batch_bytes_in_use(self._h))


def serve_run(requests, precision: str = "f32c", hbm_budget: int = 0, steps_per_round: int = 8,
              max_instances: int = 0, max_seconds: float = 0.0, device: int = 0, policy: str = "fifo",
              max_cells: float = 0.0, keep_results: bool = False, layout: str = "prim", dtype=np.float64):
    """Play a list of (arrival_seconds, InstanceDesc) through fvb_serve_run;
    returns (results as a list of dicts, wall seconds).  `policy` "fifo"
    admits in arrival order, "shortest" least estimated work (n^3 t_end)
    first; `max_cells` caps the interior cells of the live instances (0: HBM
    budget and slots only).  With `keep_results` each result carries the
    final interior state ("state", 4 x n x n in `layout` / `dtype`)."""
    n = len(requests)
    reqs = (L.Request * n)()
    states = []
    for i, (t, d) in enumerate(requests):
        reqs[i].arrival = t
        reqs[i].desc = d
        if keep_results:
            a = np.empty((4, d.n, d.n), dtype)
            states.append(a)
            reqs[i].out = a.ctypes.data
            reqs[i].out_layout = LAYOUT[layout]
            reqs[i].out_dtype = 1 if a.dtype == np.float64 else 0
    res = (L.RequestResult * n)()
    cfg = L.ServeConfig()
    cfg.batch.precision, cfg.batch.order, cfg.batch.device = PREC[precision], 7, device
    cfg.batch.hbm_budget, cfg.batch.max_instances, cfg.batch.use_graph, cfg.batch.tile = hbm_budget, max_instances, 1, -1
    cfg.steps_per_round, cfg.max_seconds = steps_per_round, max_seconds
    cfg.policy, cfg.max_cells = L.SERVE_POLICY[policy], float(max_cells)
    wall = C.c_double()
    check(lib().fvb_serve_run(C.byref(cfg), reqs, n, res, C.byref(wall)), "fvb_serve_run")
    out = [dict(arrival=requests[i][0], admitted=r.admitted, finished=r.finished, status=r.status,
                steps=int(r.steps), t=r.t) for i, r in enumerate(res)]
    if keep_results:
        for o, a in zip(out, states):
            o["state"] = a
    return out, wall.value
