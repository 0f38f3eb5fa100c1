#!/usr/bin/env python
"""Throughput of the finite-volume Euler step on B200: cell-stage updates/s.

Workload (one grid per GPU): Kelvin-Helmholtz double shear layer, periodic
[0,1]^2, 2048 x 2048 cells, gamma 1.4, UP7 + Ducros-blended HLLC/HLLE,
SSP-RK3 at CFL 0.5 -- the FP32-compensated-vs-FP64 configuration.  A bench
"step" is one SSP-RK3 time step (three stages) over the whole grid; the unit
of work is one cell-stage update (one interior cell through one stage).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]
                    [--precision f64|f32c] [--n 2048]

Under torchrun each rank advances its own replica (weak scaling, no
data-path collective); the time is the max over ranks.  `--impl reference`
times the reference's own kernels compiled for the host CPU (oracle/_ref),
with every host thread, on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from fvstuff_b200 import ranks as R  # noqa: E402  (no torch / CUDA at import)

BYTES_PER_CELL_STAGE = {"f64": 256.0 / 3.0, "f32": 128.0 / 3.0, "f32c": 160.0 / 3.0}
METRIC = "cell-stage updates/s on 1 B200 (plain vs batched/served); p50/p99 solve latency"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=None, help="timed steps (plain 400, large 2000)")
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", default="fvb", choices=["fvb", "reference"])
    p.add_argument("--precision", default="f64", choices=["f64", "f32c", "f32"])
    p.add_argument("--n", type=int, default=None, help="grid side (plain 2048, large 8192)")
    p.add_argument("--no-forms", action="store_true", help="skip the extra FP32c measurement")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--mode", default="plain",
                   choices=["plain", "batched", "serve", "large", "families", "precision", "aux"],
                   help="plain: the headline line; batched / serve / large: the other configurations; "
                        "families: the other flux families on their own cases; precision: FP32c against "
                        "FP64 over a whole run; aux: the auxiliary kernels' bandwidth")
    p.add_argument("--t-end", type=float, default=1.0, help="precision: final time of the KH run")
    p.add_argument("--families", default="up_ducros_hll,up_ducros_roe,keep,rec3,up_hllc_d2av",
                   help="families: which ones")
    p.add_argument("--instances", type=int, default=512, help="batched: number of grids")
    p.add_argument("--plain-sample", type=int, default=0,
                   help="batched: how many of the grids (evenly spaced) the plain FP64 path runs (0: all)")
    p.add_argument("--riemann-width", type=float, default=0.0,
                   help="batched: quadrant interfaces smoothed over this many cells (0: sharp)")
    p.add_argument("--requests", type=int, default=48, help="serve: requests in the stream")
    p.add_argument("--rate", type=float, default=200.0, help="serve: mean arrivals per second")
    p.add_argument("--max-n", type=int, default=2048, help="serve: largest grid side")
    p.add_argument("--steps-per-round", type=int, default=16, help="serve: batch steps between admissions")
    p.add_argument("--policy", default="shortest", choices=["fifo", "shortest"],
                   help="serve: admission order (arrival, or least estimated work first)")
    p.add_argument("--max-cells", type=float, default=16e6,
                   help="serve: cap on the live instances' interior cells (0: none)")
    p.add_argument("--no-sequential", action="store_true", help="serve: skip the one-at-a-time FP64 comparison")
    p.add_argument("--rates", default="1,2,4,6,10",
                   help="serve: offered loads (requests/s) of the latency sweep, '' for none")
    p.add_argument("--span", type=float, default=10.0, help="serve: seconds of arrivals per sweep stream")
    a = p.parse_args()
    large = a.mode == "large"
    if a.n is None:
        a.n = 8192 if large else 2048
    if a.steps is None:
        a.steps = 2000 if large else 50 if a.mode == "families" else 20 if a.mode == "aux" else 400
    return a


def workload(n):
    return {"workload": "kelvin-helmholtz %dx%d periodic [0,1]^2, UP7+Ducros HLLC, SSP-RK3, CFL 0.5" % (n, n),
            "n": n, "case": "kh", "cfl": 0.5, "gamma": 1.4, "order": 7,
            "l2": "inputs larger than L2 (state buffers %.0f MB each)" % (4 * (n + 8) ** 2 * 8 / 1e6)}


class ClockSampler:
    """SM clock and throttle reasons sampled through NVML during a region."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown", 0x4: "sw_power_cap",
               0x80: "hw_power_brake_slowdown"}

    def __init__(self, device_index: int):
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self._stop = threading.Event()
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nv = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self._nv = None

    def _run(self):
        nv = self._nv
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                for bit, name in self.REASONS.items():
                    if r & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.005)

    def __enter__(self):
        if self._nv:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        if self._nv:
            self._stop.set()
            self._t.join()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons), "samples": 0}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _profile_value(precision: str, n: int, key: str):
    """A number from the committed ncu summary of the stage kernel, if any."""
    kernel = "stage32c_kernel" if precision == "f32c" else "stage_kernel"
    f = ROOT / "profiles" / ("%s_kh%d_%s.txt" % (kernel, n, precision))
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith(key):
            try:
                return float(line[len(key):].lstrip(": ").split()[0])
            except (IndexError, ValueError):
                return None
    return None


def traffic_from_profiles(precision: str, n: int):
    """dram bytes per stage launch from the committed ncu summary, if any."""
    return _profile_value(precision, n, "traffic_bytes_per_launch_full_size:")


# ---------------------------------------------------------------------------
# CPU: the reference's own kernels compiled for the host (oracle/_ref)
# ---------------------------------------------------------------------------
def cpu_reference_rate(sample_n: int, steps: int, warmup: int, threads: int | None = None):
    """cell-stage updates/s of the reference's own FP64 kernels and host loop
    (fv_up7_ducros_2d.cu retyped, oracle/_ref) on the KH case at sample_n^2.
    The build timed is the speed build (-O3 -march=native, contraction
    allowed, compiled on this machine); without it the bit-exact pin build,
    and without either the oracle's C restatement ("port")."""
    import oracle as O
    sys.path.insert(0, str(ROOT / "tests"))
    from cases import kh, pad
    threads = threads or os.cpu_count() or 1
    lib, build = None, "port"
    if O.have_ref_host():
        lib = O.ref_native()
        build = "g++ -O3 -march=native -fopenmp" if lib is not None else "g++ -O3 -march=x86-64-v3 " \
                                                                         "-ffp-contract=off -fopenmp"
        (lib or O.ref_host("up7_f64")).ref_set_threads(threads)
    kind = "reference" if O.have_ref_host() else "port"
    U = pad(kh(sample_n), 4)
    O.bc(U, sample_n, 4, 1)
    if kind == "reference":
        run = lambda U, n, h, c, b, k: O.ref_up_run(U, n, h, c, b, k, lib=lib)
    else:
        run = lambda U, n, h, c, b, k: O.up_run(U, n, h, c, b, k)
    if warmup:
        run(U, sample_n, 1.0 / sample_n, 0.5, 1, warmup)
    t0 = time.perf_counter()
    run(U, sample_n, 1.0 / sample_n, 0.5, 1, 1)  # prologue residual + 1 step
    t1 = time.perf_counter()
    run(U, sample_n, 1.0 / sample_n, 0.5, 1, 1 + steps)
    t2 = time.perf_counter()
    sec = (t2 - t1) - (t1 - t0)  # `steps` steps without the prologue
    sec = max(sec, 1e-9)
    rate = 3.0 * sample_n * sample_n * steps / sec
    return rate, kind, threads, sec, build


def run_reference(args):
    """The reference arm: the reference's own kernels and loop on the host
    cores, on the GPU line's configuration (the same n, case, CFL and dt
    rule), with every host thread.  Under torchrun only rank 0 runs."""
    rank, world, _ = R.env()
    if rank != 0:
        return
    n = args.n
    # timed steps bounded so the arm ends within a few minutes at 2048^2
    steps = max(1, min(args.steps, 20))
    rate, kind, threads, sec, build = cpu_reference_rate(n, steps, min(args.warmup, 2))
    # the same kernels on one host thread, on a smaller grid
    rate1, _, _, sec1, _ = cpu_reference_rate(256, 4, 1, threads=1)
    cfg = dict(workload(n), parallelism="replicas%d" % world if world > 1 else "single")
    line = {"metric": METRIC, "value": rate, "unit": "cell-stage updates/s", "n_gpus": args.gpus,
            "steps": steps, "warmup": args.warmup, "ms_per_step": sec / steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": cfg, "impl": "reference",
            "cpu_baseline": {"value": rate, "unit": "cell-stage updates/s", "cores": threads, "kind": kind,
                             "build": build,
                             "sample": "%d SSP-RK3 steps of the KH case on the full %dx%d grid (FP64 retype of "
                                       "fv_up7_ducros_2d.cu's kernels and loop, OpenMP over all host threads)"
                                       % (steps, n, n),
                             "single_thread": {"value": rate1, "cores": 1,
                                               "sample": "4 steps on a 256x256 grid"}},
            "e2e": {"value": rate, "unit": "cell-stage updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
def measure_form(F, torch, stream, precision, n, steps, warmup, dist):
    s = F.Solver(n, bc="periodic", cfl=0.5, precision=precision, stream=stream.cuda_stream)
    s.init_case("kh", seed=12345)
    s.step(warmup)
    s.sync()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    s.step(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    st = s.sync()
    if st.status != 0 or st.steps != warmup + steps:
        raise RuntimeError("run stopped early: %s" % (st,))
    return s, ms


def e2e_run(F, torch, stream, precision, n, steps, dist):
    """Through the public API with host buffers: upload the initial state from
    pinned host memory, then per step one fvb_step and the D2H read of that
    step's t, dt and lam_max (fvb_stats_post behind the step, fvb_stats_wait
    for it while the next step runs; the last one is waited for before the
    download), then download the final state."""
    sys.path.insert(0, str(ROOT / "tests"))
    from cases import kh
    host_in = torch.from_numpy(kh(n)).pin_memory()
    host_out = torch.empty((4, n, n), dtype=torch.float64).pin_memory()
    s = F.Solver(n, bc="periodic", cfl=0.5, precision=precision, stream=stream.cuda_stream)
    # warm-up of the whole path: the staging buffers, and one download into
    # the pinned output buffer (its first transfer pays a one-time set-up)
    s.set_state(host_in.numpy(), interior=True)
    s.step(2)
    s.sync()
    s.get_state(interior=True, out=host_out.numpy())
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s.set_state(host_in.numpy(), interior=True)
    ta = time.perf_counter()
    for k in range(steps):
        s.step(1)
        s.post_stats(k % 2)
        if k:
            st = s.wait_stats((k - 1) % 2)
            if st.status:
                raise RuntimeError("step %d stopped with status %d" % (k, st.status))
    s.wait_stats((steps - 1) % 2)
    tb = time.perf_counter()
    s.get_state(interior=True, out=host_out.numpy())
    t1 = time.perf_counter()
    breakdown = {"upload_ms": (ta - t0) * 1e3, "steps_ms": (tb - ta) * 1e3, "download_ms": (t1 - tb) * 1e3}
    sec = R.max_over_ranks(t1 - t0, dist)
    # the two state transfers alone (upload with its layout conversion,
    # download with its conversion), best of three: with the device time of
    # the steps they bound what any end-to-end run of this length can reach
    up, down = [], []
    for _ in range(3):
        torch.cuda.synchronize()
        a = time.perf_counter()
        s.set_state(host_in.numpy(), interior=True)
        s.sync()
        b = time.perf_counter()
        s.get_state(interior=True, out=host_out.numpy())
        c = time.perf_counter()
        up.append(b - a)
        down.append(c - b)
    s.close()
    state_bytes = 4 * n * n * 8
    return sec, state_bytes / steps + 8, state_bytes / steps + 80, min(up), min(down), state_bytes, breakdown


def small_forms(F, torch, plain_value):
    """The batched, served and precision forms at sizes that take about a
    minute together: configuration 3 on 128 of its grids, configuration 4 as
    a 16-request stream, and the configuration-1 vortex over one period in
    FP32c against FP64."""
    out = {}
    with ClockSampler(0) as clk:
        insts = riemann_instances(128)
        b = batched_vs_plain(F, insts, 0.25)
        b["workload"] = "128 of configuration 3's four-quadrant Riemann grids (sharp interfaces, N 64..512, t=0.25)"
        b["vs_plain_f64_kh2048"] = b["value"] / plain_value
        out["batched"] = b
    out["batched"]["clocks"] = clk.summary()
    with ClockSampler(0) as clk:
        out["serve"] = serve_form(F, torch, 16, 200.0, 2048)
    out["serve"]["clocks"] = clk.summary()
    with ClockSampler(0) as clk:
        sys.path.insert(0, str(ROOT / "tests"))
        from cases import vortex
        m = 256
        w0 = vortex(m)
        res = {}
        for prec in ("f64", "f32c"):
            s = F.Solver(m, bc="periodic", x0=-5.0, y0=-5.0, length=10.0, cfl=0.5, precision=prec)
            s.set_state(w0, layout="prim", interior=True)
            st = s.advance(10.0)
            res[prec] = (s.get_state(layout="cons", interior=True), st)
            s.close()
        l1, linf = _density_errors(res["f32c"][0][0], res["f64"][0][0])
        out["precision"] = {"workload": "isentropic vortex 256^2 periodic, one period (t=10), FP32c vs FP64",
                            "l1_rel_density": l1, "linf_rel_density": linf, "bar_l1": 1e-6,
                            "conserved_l1_rel": {name: _density_errors(res["f32c"][0][q], res["f64"][0][q])[0]
                                                 for q, name in enumerate(("rho", "rho_u", "rho_v", "E"))},
                            "steps_f64": res["f64"][1].steps, "steps_f32c": res["f32c"][1].steps}
    out["precision"]["clocks"] = clk.summary()
    return out


def run_gpu(args):
    import torch

    import fvstuff_b200 as F

    rank, world, local = R.env()
    torch.cuda.set_device(local)
    dist = R.init("nccl")
    stream = torch.cuda.Stream()
    n, K, W = args.n, args.steps, args.warmup
    hbm, peak_kind = peaks()

    with ClockSampler(local) as clk:
        s, ms = measure_form(F, torch, stream, args.precision, n, K, W, dist)
    ms = R.max_over_ranks(ms, dist)
    s.close()
    units = 3.0 * n * n * K
    value = world * units / (ms / 1e3)
    launch_ms = ms / (3 * K)
    bpl = BYTES_PER_CELL_STAGE[args.precision] * n * n
    achieved = bpl / (launch_ms / 1e3) / 1e9
    line = {"metric": METRIC, "value": value, "unit": "cell-stage updates/s", "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": args.precision, "data": "synthetic",
            "config": dict(workload(n), parallelism="replicas%d" % world if world > 1 else "single"),
            "gpu_launches": 3 * K + 1,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": traffic_from_profiles(args.precision, n),
                         "peak_kind": peak_kind,
                         "bytes_per_cell_stage": BYTES_PER_CELL_STAGE[args.precision],
                         "kernel": "fvb::stage_kernel (one launch per RK stage)",
                         # what bounds it instead (ncu summary of the same kernel): the FP64
                         # pipe, busy this share of the time; at 100 % the stage would
                         # still move only ~45 % of the HBM peak
                         "fp64_pipe_pct_ncu": _profile_value(args.precision, n, "pipe_fp64_pct"),
                         "issue_active_pct_ncu": _profile_value(args.precision, n, "issue_active_pct")},
            "clocks": clk.summary()}

    if not args.no_forms and args.precision == "f64":
        with ClockSampler(local) as clk2:
            s2, ms2 = measure_form(F, torch, stream, "f32c", n, K, W, dist)
        s2.close()
        ms2 = R.max_over_ranks(ms2, dist)
        v2 = world * units / (ms2 / 1e3)
        a2 = BYTES_PER_CELL_STAGE["f32c"] * n * n / (ms2 / (3 * K) / 1e3) / 1e9
        line["forms"] = {"f32c": {"value": v2, "ms_per_step": ms2 / K, "vs_f64": v2 / value,
                                  "roofline_achieved_gbs": a2, "roofline_frac": a2 / hbm,
                                  "clocks": clk2.summary()}}
        if world == 1:
            # the other north-star forms on small instances of their
            # configurations, so the default line carries them
            line["forms"].update(small_forms(F, torch, value))

    if not args.no_e2e:
        sec, bi, bo, up_s, down_s, sbytes, brk = e2e_run(F, torch, stream, args.precision, n, K, dist)
        line["e2e"] = {"value": world * units / sec, "unit": "cell-stage updates/s",
                       "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo,
                       "state_upload_ms": up_s * 1e3, "state_download_ms": down_s * 1e3,
                       "timed_region_ms": brk,
                       "link_gbs": {"h2d": sbytes / up_s / 1e9, "d2h": sbytes / down_s / 1e9},
                       # the steps' device time plus the two transfers, unoverlapped:
                       # the state must be whole on the device before the first dt
                       # (a max over every cell) and whole after the last stage
                       "bound_value": world * units / (ms / 1e3 + up_s + down_s),
                       "how": "fvb_set_state from pinned host memory, then per step fvb_step + fvb_stats_post "
                              "(D2H of t/dt/lam_max, waited for while the next step runs), then fvb_get_state "
                              "to pinned host memory; wall clock"}

    if rank == 0 and not args.no_cpu:
        rate, kind, threads, sec, build = cpu_reference_rate(n, 2, 0)
        line["cpu_baseline"] = {"value": rate, "unit": "cell-stage updates/s", "cores": threads, "kind": kind,
                                "build": build,
                                "sample": "2 SSP-RK3 steps of the KH case on the full %dx%d grid" % (n, n)}
    R.finish(dist)
    if rank == 0:
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# the other configurations: batched (3), serving (4), large grid (5)
# ---------------------------------------------------------------------------
def riemann_instances(count, seed=2024, width=0.0):
    """`count` four-quadrant Riemann problems, N uniform in {64, 96, ..., 512},
    quadrant states from per-instance seeds, transmissive, t_end 0.25.  The
    quadrant interfaces are sharp (width 0, as the configuration states);
    width > 0 smooths them over that many cells."""
    import fvstuff_b200 as F
    rng = np.random.default_rng(seed)
    sizes = list(range(64, 513, 32))
    out = []
    for k in range(count):
        n = int(rng.choice(sizes))
        c = F.case_params("riemann4", 0.0, 0.0, 1.0, seed=int(rng.integers(1, 2 ** 62)), param2=width)
        out.append((n, c))
    return out


def advance_counted(s, t_end):
    """fvb_advance; a grid that trips the blow-up / dt-underflow guard (as the
    reference's own loop does, fv_up7_ducros_2d.cu:997-1007) stops there and
    still counts the steps it made."""
    import fvstuff_b200 as F
    try:
        s.advance(t_end)
    except F.FvbError as e:
        if e.status not in (F._lib.ERR_BLOWUP, F._lib.ERR_DT_UNDERFLOW):
            raise
    return s.sync()


def plain_f64_each(F, insts, t_end):
    """The plain FP64 path, one grid at a time: per grid (cell-stages,
    seconds, status).  Set-up (allocation, initial state) is not timed."""
    import torch
    out = []
    for n, c in insts:
        s = F.Solver(n, bc="transmissive", cfl=0.5, precision="f64")
        s.init_case(c)
        s.sync()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st = advance_counted(s, t_end)
        out.append((3.0 * n * n * st.steps, time.perf_counter() - t0, st.status))
        s.close()
    return out


def batch_f32c(F, insts, t_end):
    """All grids in one FP32c batch (one persistent launch per RK stage,
    graph-replayed), timed from the first step to the last completion;
    returns (seconds, per grid (cell-stages, status))."""
    import torch
    b = F.Batch(precision="f32c")
    ids = [b.add(F.Batch.desc(n, c, t_end, bc="transmissive", cfl=0.5)) for n, c in insts]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    done = set()
    while len(done) < len(ids):
        b.run(16)
        done.update(b.poll())
    sec = time.perf_counter() - t0
    per = []
    for iid, (n, _) in zip(ids, insts):
        st = b.stats(iid)
        per.append((3.0 * n * n * st.steps, st.status))
    b.close()
    return sec, per


def batched_vs_plain(F, insts, t_end, plain_sample=None):
    """Configuration 3 on one GPU: the FP32c batch and the plain FP64 path
    (each grid alone) on the same grids.  Failures (grids stopped by the
    reference scheme's blow-up / dt-underflow guard) are counted per form,
    and the speed-up is taken on the grids both forms finish: the batch is
    run again on exactly those, against the sum of their FP64 times."""
    sec, per = batch_f32c(F, insts, t_end)
    idx = list(range(len(insts)))
    if plain_sample:
        idx = idx[:: max(1, len(insts) // plain_sample)]
    plain = plain_f64_each(F, [insts[i] for i in idx], t_end)
    both = [i for i, (w, st, k) in zip(idx, plain) if k == 0 and per[i][1] == 0]
    sec_c, per_c = batch_f32c(F, [insts[i] for i in both], t_end) if both else (0.0, [])
    keep = set(both)
    plain_c = [p for i, p in zip(idx, plain) if i in keep]
    rate_b = sum(w for w, _ in per_c) / sec_c if both else None
    rate_p = sum(w for w, _, _ in plain_c) / sum(t for _, t, _ in plain_c) if both else None
    return {"value": sum(w for w, _ in per) / sec, "seconds": sec, "instances": len(insts),
            "failed_f32c": sum(st != 0 for _, st in per),
            "plain_f64_compared": len(idx), "failed_f64": sum(k != 0 for _, _, k in plain),
            "failed_f32c_of_compared": sum(per[i][1] != 0 for i in idx),
            "common_finishers": len(both),
            "batched_f32c_common": rate_b, "plain_f64_one_at_a_time_common": rate_p,
            "ratio_common": rate_b / rate_p if both else None,
            "failed_means": "stopped by the blow-up / dt-underflow guard of the reference scheme "
                            "(fv_up7_ducros_2d.cu:997-1007) before t_end"}


def run_batched(args):
    import torch

    import fvstuff_b200 as F
    rank, world, local = R.env()
    torch.cuda.set_device(local)
    dist = R.init("nccl")
    count = args.instances
    insts = riemann_instances(count, width=args.riemann_width)
    # N ranks split the instances by work (~N^3: cells x steps)
    mine = [insts[i] for i in R.shard_by_work([float(n) ** 3 for n, _ in insts], rank, world)]
    t_end = 0.25
    if dist:
        dist.barrier()
    sec, per = batch_f32c(F, mine, t_end)
    work, bad = sum(w for w, _ in per), sum(st != 0 for _, st in per)
    sec = R.max_over_ranks(sec, dist)
    work = R.sum_over_ranks(work, dist)
    bad = int(R.sum_over_ranks(bad, dist))
    # every form on the same grids (rank 0's share), failures per form
    cmp = batched_vs_plain(F, mine, t_end, plain_sample=args.plain_sample) if rank == 0 else None
    R.finish(dist)
    if rank != 0:
        return
    value = work / sec
    line = {"metric": METRIC, "value": value, "unit": "cell-stage updates/s", "n_gpus": world, "steps": None,
            "warmup": 0, "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32c",
            "data": "synthetic", "mode": "batched",
            "config": {"workload": "%d four-quadrant Riemann problems (%s interfaces), N in {64..512} step 32, "
                                   "transmissive, t=0.25, CFL 0.5, one persistent launch per RK stage "
                                   "(graph-replayed); timed from the first step to the last instance's "
                                   "completion, set-up excluded as for the plain path"
                                   % (count, "sharp" if args.riemann_width == 0 else
                                      "%g-cell tanh" % args.riemann_width),
                       "instances": count, "parallelism": "instances split by work over %d GPU(s)" % world,
                       "failed": bad},
            "seconds": sec, "cell_stages": work, "forms_same_grids": cmp}
    print(json.dumps(line), flush=True)


def serve_requests(F, count, rate, max_n, seed=7):
    """The seeded request stream: Poisson arrivals, half isentropic vortices
    (periodic [-5,5]^2), half four-quadrant Riemann problems with sharp
    quadrant interfaces (transmissive [0,1]^2), N log-uniform in [128,
    max_n], t_end uniform in [0.1, 1]."""
    rng = np.random.default_rng(seed)
    reqs, t = [], 0.0
    for k in range(count):
        t += rng.exponential(1.0 / rate)
        n = int(round(math.exp(rng.uniform(math.log(128), math.log(max_n)))))
        t_end = float(rng.uniform(0.1, 1.0))
        if rng.random() < 0.5:
            c = F.case_params("vortex", -5.0, -5.0, 10.0)
            d = F.Batch.desc(n, c, t_end, bc="periodic", x0=-5.0, y0=-5.0, length=10.0, cfl=0.5)
        else:
            c = F.case_params("riemann4", 0.0, 0.0, 1.0, seed=int(rng.integers(1, 2 ** 62)), param2=0.0)
            d = F.Batch.desc(n, c, t_end, bc="transmissive", cfl=0.5)
        reqs.append((t, d))
    return reqs


def _pct(v, q):
    v = sorted(v)
    return v[min(len(v) - 1, int(q * len(v)))] if v else None


def serve_form(F, torch, count, rate, max_n, policy="shortest", max_cells=16e6, steps_per_round=16,
               sequential=True, seed=7):
    """One served stream on this GPU: `count` requests arriving at `rate`
    per second, admitted against a 150 GB budget and a cap on live cells;
    p50 / p99 time to solution, throughput, and the same requests one after
    another on the plain FP64 path (arrival times respected)."""
    reqs = serve_requests(F, count, rate, max_n, seed=seed)
    torch.cuda.synchronize()
    res, wall = F.serve_run(reqs, precision="f32c", hbm_budget=150 << 30, steps_per_round=steps_per_round,
                            policy=policy, max_cells=max_cells)
    lat = [r["finished"] - r["arrival"] for r in res]
    work = sum(3.0 * d.n * d.n * r["steps"] for (_, d), r in zip(reqs, res))
    out = {"workload": "Poisson stream, %d requests at %g/s, vortex or seeded Riemann, N log-uniform in [128, %d], "
                       "t_end U[0.1, 1], 150 GB HBM budget" % (count, rate, max_n),
           "admission": policy, "max_cells": max_cells, "value": work / wall, "p50_s": _pct(lat, 0.5),
           "p99_s": _pct(lat, 0.99), "wall_s": wall, "arrival_span_s": reqs[-1][0] if reqs else 0.0,
           "failed": sum(r["status"] != 0 for r in res)}
    if sequential:
        t0 = time.perf_counter()
        seq_lat, clock = [], 0.0
        for (arr, d), r in zip(reqs, res):
            s = F.Solver(d.n, bc={0: "reflect", 1: "periodic", 2: "transmissive"}[d.bc_x], x0=d.x0, y0=d.y0,
                         length=d.length, cfl=d.cfl, precision="f64")
            s.init_case(d.ic)
            a = time.perf_counter()
            advance_counted(s, d.t_end)
            clock = max(clock, arr) + (time.perf_counter() - a)
            seq_lat.append(clock - arr)
            s.close()
        seq_wall = time.perf_counter() - t0
        out["sequential_plain_f64"] = {"value": work / seq_wall, "p50_s": _pct(seq_lat, 0.5),
                                       "p99_s": _pct(seq_lat, 0.99), "wall_s": seq_wall}
    return out


def run_serve(args):
    """Configuration 4.  One stream at --rate (with the sequential FP64
    comparison), then, unless --rates is empty, latency against offered
    load: a stream per rate, each sized so its arrivals span --span seconds."""
    import torch

    import fvstuff_b200 as F
    rank, world, local = R.env()
    torch.cuda.set_device(local)
    dist = R.init("nccl")
    reqs = serve_requests(F, args.requests, args.rate, args.max_n)
    # N ranks: request k goes to rank k mod N, each rank serves its own stream
    mine = reqs[rank::world]
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    res, wall = F.serve_run(mine, precision="f32c", hbm_budget=150 << 30, steps_per_round=args.steps_per_round,
                            policy=args.policy, max_cells=args.max_cells)
    lat = [r["finished"] - r["arrival"] for r in res]
    work = sum(3.0 * d.n * d.n * r["steps"] for (_, d), r in zip(mine, res))
    failed = sum(r["status"] != 0 for r in res)
    # the same requests one at a time on the plain FP64 path, back to back
    t0 = time.perf_counter()
    seq_lat, clock = [], 0.0
    for (arr, d), r in zip([] if args.no_sequential else mine, res):
        s = F.Solver(d.n, bc={0: "reflect", 1: "periodic", 2: "transmissive"}[d.bc_x], x0=d.x0, y0=d.y0,
                     length=d.length, cfl=d.cfl, precision="f64")
        s.init_case(d.ic)
        a = time.perf_counter()
        advance_counted(s, d.t_end)
        clock = max(clock, arr) + (time.perf_counter() - a)
        seq_lat.append(clock - arr)
        s.close()
    seq_wall = time.perf_counter() - t0
    lat = sorted(sum(R.gather(lat, dist), []))
    seq_lat = sorted(sum(R.gather(seq_lat, dist), []))
    wall = R.max_over_ranks(wall, dist)
    seq_wall = R.max_over_ranks(seq_wall, dist)
    work = R.sum_over_ranks(work, dist)
    failed = int(R.sum_over_ranks(failed, dist))
    # latency against offered load (each rank its own stream, rank 0 reports)
    sweep = []
    for lam in [float(x) for x in args.rates.split(",") if x.strip()]:
        count = max(4, int(round(lam * args.span)))
        sweep.append(dict(rate=lam, requests=count,
                          **serve_form(F, torch, count, lam, args.max_n, args.policy, args.max_cells,
                                       args.steps_per_round, sequential=False, seed=11 + rank)))
        print("rate %g/s: %d requests over %.1f s, p50 %.3f s, p99 %.3f s, %.2f G/s"
              % (lam, count, sweep[-1]["arrival_span_s"], sweep[-1]["p50_s"], sweep[-1]["p99_s"],
                 sweep[-1]["value"] / 1e9), file=sys.stderr, flush=True)
    R.finish(dist)
    if rank != 0:
        return
    line = {"metric": METRIC, "value": work / wall, "unit": "cell-stage updates/s", "n_gpus": world,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32c", "data": "synthetic",
            "mode": "serve",
            "config": {"workload": "Poisson stream, %d requests at %.0f/s, vortex or seeded Riemann, N log-uniform "
                                   "in [128, %d], t_end U[0.1, 1], 150 GB HBM budget" % (args.requests, args.rate,
                                                                                        args.max_n),
                       "admission": args.policy, "max_cells": args.max_cells,
                       "parallelism": "request k served by GPU k mod %d" % world},
            "p50_s": _pct(lat, 0.5), "p99_s": _pct(lat, 0.99), "wall_s": wall,
            "failed": failed, "latency_vs_offered_load": sweep}
    if seq_lat:
        line["sequential_plain_f64"] = {"value": work / seq_wall, "p50_s": _pct(seq_lat, 0.5),
                                        "p99_s": _pct(seq_lat, 0.99), "wall_s": seq_wall}
    print(json.dumps(line), flush=True)


def run_large(args):
    import torch

    import fvstuff_b200 as F
    n, K = args.n, args.steps
    out = {}
    for prec in ("f32c", "f64"):
        stream = torch.cuda.Stream()
        s = F.Solver(n, bc="periodic", cfl=0.5, precision=prec, stream=stream.cuda_stream)
        s.init_case("kh")
        a = s.stats().sums
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        with ClockSampler(0) as clk:
            e0.record(stream)
            s.step(K)
            e1.record(stream)
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        st = s.stats()
        drift = [(st.sums[q] - a[q]) / abs(a[q]) for q in (0, 3)]
        hbm, _ = peaks()
        gbs = BYTES_PER_CELL_STAGE[prec] * n * n * 3 * K / (ms / 1e3) / 1e9
        out[prec] = {"value": 3.0 * n * n * K / (ms / 1e3), "ms_per_step": ms / K, "t": st.t, "steps": st.steps,
                     "status": st.status, "mass_drift": drift[0], "energy_drift": drift[1],
                     "achieved_gbs": gbs, "roofline_frac": gbs / hbm, "clocks": clk.summary()}
        s.close()
    line = {"metric": METRIC, "value": out["f32c"]["value"], "unit": "cell-stage updates/s", "n_gpus": 1,
            "steps": K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32c",
            "data": "synthetic", "mode": "large",
            "config": {"workload": "kelvin-helmholtz %dx%d periodic, %d SSP-RK3 steps at CFL 0.5" % (n, n, K)},
            "forms": out}
    print(json.dumps(line), flush=True)


# flux family -> (solver options, initial state, its case options): each on
# the case its reference solver runs
FAMILY_CASES = {
    "up_ducros_hll": ({"order": 7, "bc": "periodic", "cfl": 0.5}, "kh", {}),
    "up_ducros_roe": ({"order": 7, "bc": "periodic", "cfl": 0.5}, "kh", {}),
    # keep_fv's low-Mach vortex (its Sod breaks down within ~25 steps in the
    # reference scheme itself at these sizes: dt underflow)
    "keep": ({"bc": "periodic", "cfl": 0.4}, "lmv", {}),
    "rec3": ({"bc": "periodic", "cfl": 0.4}, "rec3_sod", {}),
    "up_hllc_d2av": ({"order": 5, "bc": "reflect", "cfl": 0.4}, "sod", {"rho_in": 10.0}),
}


def run_families(args):
    """The other flux families, FP64, one grid each: cell-stage updates/s
    over `steps` steps after `warmup`, CUDA events on the solver's stream."""
    import torch

    import fvstuff_b200 as F
    n, K = args.n, args.steps
    out = {}
    for fam in args.families.split(","):
        opts, case, cparams = FAMILY_CASES[fam]
        stream = torch.cuda.Stream()
        s = F.Solver(n, flux=fam, stream=stream.cuda_stream, **opts)
        s.init_case(case, **cparams)
        s.step(max(3, args.warmup))
        k0 = s.sync().steps
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        with ClockSampler(0) as clk:
            e0.record(stream)
            s.step(K)
            e1.record(stream)
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        st = s.sync()
        done = st.steps - k0
        out[fam] = {"value": 3.0 * n * n * done / (ms / 1e3) if done else None,
                    "ms_per_step": ms / max(done, 1), "steps": done, "case": case, "options": opts,
                    "status": st.status,
                    "clocks": clk.summary()}
        s.close()
    line = {"metric": METRIC, "value": None, "unit": "cell-stage updates/s", "n_gpus": 1, "steps": K,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "mode": "families",
            "config": {"workload": "each flux family on its reference solver's case, %dx%d, %d steps" % (n, n, K)},
            "families": out}
    print(json.dumps(line), flush=True)


def _density_errors(a, b):
    """relative L1 and L-inf of a field a against b (interior arrays)"""
    d = np.abs(a - b)
    return float(d.sum() / np.abs(b).sum()), float(d.max() / np.abs(b).max())


def run_precision(args):
    """FP32c against the plain FP64 form (itself held to the oracle at 1e-12)
    over whole runs: Kelvin-Helmholtz n^2 to t_end with the error of density
    at every tenth of the run, and the periodic isentropic vortex 256^2 over
    one period (t = 10).  Both forms land exactly on each checkpoint time.
    Beside the KH curve, the same FP64 run started from a density one ulp
    away in every cell: how far the flow itself carries a last-bit change."""
    import torch

    import fvstuff_b200 as F
    n, t_end = args.n, args.t_end
    curve = []
    a = F.Solver(n, bc="periodic", cfl=0.5, precision="f64")
    b = F.Solver(n, bc="periodic", cfl=0.5, precision="f32c")
    c = F.Solver(n, bc="periodic", cfl=0.5, precision="f64")
    a.init_case("kh")
    b.init_case("kh")
    w = a.get_state(interior=True)
    w[0] = np.nextafter(w[0], np.inf)
    c.set_state(w, interior=True)
    for k in range(1, 11):
        t = t_end * k / 10
        sa, sb, sc = a.advance(t), b.advance(t), c.advance(t)
        ca = a.get_state(layout="cons", interior=True)
        cb = b.get_state(layout="cons", interior=True)
        ra = ca[0]
        l1, linf = _density_errors(cb[0], ra)
        p1, pinf = _density_errors(c.get_state(interior=True)[0], ra)
        # every conserved variable (rho, rho u, rho v, E): L1 and L-inf relative
        per_var = {name: dict(zip(("l1_rel", "linf_rel"), _density_errors(cb[q], ca[q])))
                   for q, name in enumerate(("rho", "rho_u", "rho_v", "E"))}
        curve.append({"t": t, "l1_rel": l1, "linf_rel": linf, "f64_1ulp_l1_rel": p1, "f64_1ulp_linf_rel": pinf,
                      "conserved": per_var,
                      "steps_f64": sa.steps, "steps_f32c": sb.steps, "status": [sa.status, sb.status, sc.status]})
        print("KH %d^2 t=%.2f: FP32c L1 %.3e Linf %.3e | FP64 1-ulp start L1 %.3e Linf %.3e (steps %d / %d)"
              % (n, t, l1, linf, p1, pinf, sa.steps, sb.steps), file=sys.stderr, flush=True)
    a.close()
    b.close()
    c.close()
    sys.path.insert(0, str(ROOT / "tests"))
    from cases import vortex
    m = 256
    w0 = vortex(m)
    res = {}
    for prec in ("f64", "f32c"):
        s = F.Solver(m, bc="periodic", x0=-5.0, y0=-5.0, length=10.0, cfl=0.5, precision=prec)
        s.set_state(w0, layout="prim", interior=True)
        st = s.advance(10.0)
        res[prec] = (s.get_state(interior=True)[0], st)
        s.close()
    torch.cuda.synchronize()
    vl1, vlinf = _density_errors(res["f32c"][0], res["f64"][0])
    # a sample of the batched bench's grids: FP32c in one batch against each
    # grid alone on the plain FP64 path, at t_end (instances stopped early by
    # the reference scheme's guard in either form are listed, not compared)
    inst = riemann_instances(args.instances, width=args.riemann_width)[:: max(1, args.instances // 32)]
    bt = F.Batch(precision="f32c")
    ids = [bt.add(F.Batch.desc(nn, c, 0.25, bc="transmissive", cfl=0.5)) for nn, c in inst]
    done = set()
    while len(done) < len(ids):
        bt.run(16)
        done.update(bt.poll())
    riem = []
    for iid, (nn, c) in zip(ids, inst):
        s = F.Solver(nn, bc="transmissive", cfl=0.5, precision="f64")
        s.init_case(c)
        sa = advance_counted(s, 0.25)
        sb = bt.stats(iid)
        if sa.status == 0 and sb.status == 0:
            l1, linf = _density_errors(bt.get_state(iid, nn)[0], s.get_state(interior=True)[0])
            riem.append({"n": nn, "l1_rel": l1, "linf_rel": linf})
        else:
            riem.append({"n": nn, "stopped": [sa.status, sb.status]})
        s.close()
    bt.close()
    ok = [r["l1_rel"] for r in riem if "l1_rel" in r]
    line = {"metric": METRIC, "value": curve[-1]["l1_rel"], "unit": "relative L1 density error, FP32c vs FP64",
            "n_gpus": 1, "higher_is_better": False, "dtype": "f32c", "data": "synthetic", "mode": "precision",
            "config": {"workload": "kelvin-helmholtz %dx%d periodic CFL 0.5 to t=%g, FP32c and FP64 side by side; "
                                   "isentropic vortex 256^2 periodic, one period" % (n, n, t_end)},
            "kh_curve": curve,
            "vortex_one_period": {"l1_rel": vl1, "linf_rel": vlinf, "steps_f64": res["f64"][1].steps,
                                  "steps_f32c": res["f32c"][1].steps},
            "riemann_batched_sample": {"instances": riem, "l1_rel_median": float(np.median(ok)) if ok else None,
                                       "l1_rel_max": max(ok) if ok else None}}
    print(json.dumps(line), flush=True)


def run_aux(args):
    """The library's kernels other than the stage kernels, FP64 at n^2 on
    one GPU: each entry point timed with CUDA events on its stream (median of
    --steps repetitions after --warmup), against the bytes it must move."""
    import torch

    import fvstuff_b200 as F
    n, K, W = args.n, max(1, args.steps), max(1, args.warmup)
    np_ = n + 8
    # one stream for the solver, the caller arrays and the events: a
    # library call on any other stream would leave the events around nothing
    st = torch.cuda.Stream()
    torch.cuda.set_stream(st)
    h = st.cuda_stream
    s = F.Solver(n, bc="periodic", cfl=0.5, precision="f64", stream=h)
    s.init_case("kh")
    dev = dict(dtype=torch.float64, device="cuda")
    Q = torch.empty((4, np_, np_), **dev)
    s.get_state(out=Q)
    U0, Uk, Uo = Q.clone(), Q.clone(), torch.empty_like(Q)
    rhs, lam, mx = torch.zeros((4, n, n), **dev), torch.zeros((n, n), **dev), torch.zeros(1, **dev)
    state, cells, ghost = 4 * np_ * np_ * 8, 4 * n * n * 8, 4 * (np_ * np_ - n * n) * 8
    items = [
        ("fvb_set_state (device IDX_P in: import, ghost ring, wave-speed max, step control)",
         lambda: s.set_state(Q), state + state + cells),
        ("fvb_get_state (device IDX_P out: export)", lambda: s.get_state(out=Q), state + state),
        ("fvb_apply_bc (ghost ring of a caller array, periodic)", lambda: F.apply_bc(Q, n, np_, "periodic", stream=h), 2 * ghost),
        ("fvb_up_rhs (residual and wave speeds of a caller array)",
         lambda: F.up_rhs(Q, rhs, lam, n, np_, 1.0 / n, stream=h), state + cells + n * n * 8),
        ("fvb_rk3_stage (stage 2 on caller arrays)",
         lambda: F.rk3_stage(2, Uo, U0, Uk, rhs, 1e-4, n, np_, stream=h), 3 * cells + cells),
        ("fvb_max (n^2 doubles)", lambda: F.device_max(lam, mx, stream=h), n * n * 8),
        ("fvb_stats_sums (conserved FP64 sums of the state)", lambda: s.stats(), cells),
        # (the device part on the solver's stream; the copy to the host runs
        # on a second stream and is collected outside the timed region)
        ("fvb_frame_begin (device part: FP32 export, frame fields)", s.frame_begin,
         cells + cells // 2 + cells // 2 + 5 * n * n * 4, s.frame_end),
    ]
    hbm, peak_kind = peaks()
    out = []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clk:
        for name, fn, nbytes, *post in items:
            after = post[0] if post else (lambda: None)
            for _ in range(W):
                fn()
                after()
            torch.cuda.synchronize()
            ts = []
            for _ in range(K):
                e0.record(st)
                fn()
                e1.record(st)
                e1.synchronize()
                after()
                ts.append(e0.elapsed_time(e1))
            ms = statistics.median(ts)
            out.append({"entry": name, "ms": ms, "algorithmic_bytes": nbytes, "achieved_gbs": nbytes / ms / 1e6,
                        "roofline_frac": nbytes / ms / 1e6 / hbm})
            print("%-80s %8.3f ms %8.1f GB/s" % (name, ms, nbytes / ms / 1e6), file=sys.stderr, flush=True)
    s.close()
    line = {"metric": METRIC, "value": None, "unit": "GB/s", "n_gpus": 1, "steps": K, "warmup": W,
            "higher_is_better": True, "dtype": "f64", "data": "synthetic", "mode": "aux",
            "config": {"workload": "the library's auxiliary kernels on a %dx%d FP64 state (KH), caller arrays in "
                                   "the reference's IDX_P layout; larger than L2" % (n, n)},
            "peak_gbs": hbm, "peak_kind": peak_kind, "kernels": out, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.mode == "batched":
        run_batched(args)
    elif args.mode == "serve":
        run_serve(args)
    elif args.mode == "large":
        run_large(args)
    elif args.mode == "families":
        run_families(args)
    elif args.mode == "precision":
        run_precision(args)
    elif args.mode == "aux":
        run_aux(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
