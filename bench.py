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

BYTES_PER_CELL_STAGE = {"f64": 256.0 / 3.0, "f32": 128.0 / 3.0, "f32c": 160.0 / 3.0}
METRIC = "cell-stage updates/s on 1 B200 (plain vs batched/served); p50/p99 solve latency"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=400)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", default="fvb", choices=["fvb", "reference"])
    p.add_argument("--precision", default="f64", choices=["f64", "f32c", "f32"])
    p.add_argument("--n", type=int, default=2048)
    p.add_argument("--no-forms", action="store_true", help="skip the extra FP32c measurement")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    p.add_argument("--no-e2e", action="store_true")
    return p.parse_args()


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


def traffic_from_profiles(precision: str, n: int):
    """dram bytes per stage launch from the committed ncu summary, if any."""
    f = ROOT / "profiles" / ("stage_kernel_kh%d_%s.txt" % (n, precision))
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith("traffic_bytes_per_launch_full_size:"):
            return float(line.split(":", 1)[1])
    return None


# ---------------------------------------------------------------------------
# CPU: the reference's own kernels compiled for the host (oracle/_ref)
# ---------------------------------------------------------------------------
def cpu_reference_rate(sample_n: int, steps: int, warmup: int):
    import oracle as O
    sys.path.insert(0, str(ROOT / "tests"))
    from cases import kh, pad
    threads = os.cpu_count() or 1
    O.ref_set_threads(threads)
    kind = "reference" if O.have_ref_host() else "port"
    U = pad(kh(sample_n), 4)
    O.bc(U, sample_n, 4, 1)
    run = O.ref_up_run if kind == "reference" else (lambda U, n, h, c, b, k: O.up_run(U, n, h, c, b, k))
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
    return rate, kind, threads, sec


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sample = min(args.n, 512)
    steps = max(1, min(args.steps, 20))
    rate, kind, threads, sec = cpu_reference_rate(sample, steps, min(args.warmup, 2))
    line = {"metric": METRIC, "value": rate, "unit": "cell-stage updates/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec / steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": workload(args.n), "impl": "reference",
            "cpu_baseline": {"value": rate, "unit": "cell-stage updates/s", "cores": threads, "kind": kind,
                             "sample": "%d steps of the same KH case on a %dx%d grid (FP64 retype of "
                                       "fv_up7_ducros_2d.cu kernels, OpenMP over all host threads)"
                                       % (steps, sample, sample)},
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


def max_over_ranks(torch, dist, x):
    if not dist:
        return x
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def e2e_run(F, torch, stream, precision, n, steps, dist):
    """Through the public API with host buffers: upload the initial state from
    pinned host memory, then per step one fvb_step and one fvb_sync (the D2H
    read of the step's t, dt and lam_max), then download the final state."""
    sys.path.insert(0, str(ROOT / "tests"))
    from cases import kh
    host_in = torch.from_numpy(kh(n)).pin_memory()
    host_out = torch.empty((4, n, n), dtype=torch.float64).pin_memory()
    s = F.Solver(n, bc="periodic", cfl=0.5, precision=precision, stream=stream.cuda_stream)
    s.set_state(host_in.numpy(), interior=True)  # warm the staging buffers
    s.step(2)
    s.sync()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s.set_state(host_in.numpy(), interior=True)
    for _ in range(steps):
        s.step(1)
        s.sync()
    s.get_state(interior=True, out=host_out.numpy())
    t1 = time.perf_counter()
    sec = max_over_ranks(torch, dist, t1 - t0)
    s.close()
    state_bytes = 4 * n * n * 8
    return sec, state_bytes / steps + 8, state_bytes / steps + 80


def run_gpu(args):
    import torch

    import fvstuff_b200 as F

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as D
        D.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = D
    stream = torch.cuda.Stream()
    n, K, W = args.n, args.steps, args.warmup
    hbm, peak_kind = peaks()

    with ClockSampler(local) as clk:
        s, ms = measure_form(F, torch, stream, args.precision, n, K, W, dist)
    ms = max_over_ranks(torch, dist, ms)
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
                         "kernel": "fvb::stage_kernel (one launch per RK stage)"},
            "clocks": clk.summary()}

    if not args.no_forms and args.precision == "f64":
        with ClockSampler(local):
            s2, ms2 = measure_form(F, torch, stream, "f32c", n, K, W, dist)
        s2.close()
        ms2 = max_over_ranks(torch, dist, ms2)
        v2 = world * units / (ms2 / 1e3)
        a2 = BYTES_PER_CELL_STAGE["f32c"] * n * n / (ms2 / (3 * K) / 1e3) / 1e9
        line["forms"] = {"f32c": {"value": v2, "ms_per_step": ms2 / K, "vs_f64": v2 / value,
                                  "roofline_achieved_gbs": a2, "roofline_frac": a2 / hbm}}

    if not args.no_e2e:
        sec, bi, bo = e2e_run(F, torch, stream, args.precision, n, K, dist)
        line["e2e"] = {"value": world * units / sec, "unit": "cell-stage updates/s",
                       "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo,
                       "how": "fvb_set_state from pinned host memory, then per step fvb_step + fvb_sync "
                              "(D2H of t/dt/lam_max), then fvb_get_state to pinned host memory; wall clock"}

    if rank == 0 and not args.no_cpu:
        rate, kind, threads, sec = cpu_reference_rate(min(n, 512), 4, 1)
        line["cpu_baseline"] = {"value": rate, "unit": "cell-stage updates/s", "cores": threads, "kind": kind,
                                "sample": "4 SSP-RK3 steps of the KH case on a %dx%d grid" % ((min(n, 512),) * 2)}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
