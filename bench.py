"""Benchmark of the PSBLAS single-GPU sparse hot path on B200.

Default workload (N = 1): FP64 SpMV y = A*x on the 27-point Poisson operator
of a 200^3 grid (8,000,000 rows, 213,847,192 entries) stored in HLL with
hack size 32 and int32 indices, x uniform in [-1,1] (seed 0).  One step is
one SpMV over the whole matrix.  The metric is the reference's own SpMV
bandwidth (test/cudakern/dpdegenmv.F90:930-941): algorithmic bytes
n*(2*8+4) + nnz*(8+4) per SpMV divided by the time.

Timed region: K SpMVs on the library's stream bracketed by CUDA events,
after W warm-up SpMVs; the inputs (2.74 GB per SpMV) are far larger than the
126 MB L2, so no flush is needed between steps.  Under torchrun every rank
runs its own replica on its own GPU (the SpMV of one matrix does not shard;
independent replicas), the time is the max over ranks and the value is the
sum of the ranks' bytes over that time.

``--impl reference`` times the reference's CPU path for the same workload:
the reference (Fortran) cannot be compiled in this image, so its restatement
in oracle/ (C, OpenMP over rows, the reference's per-row order) runs on all
host cores.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

GRID = 200


def algorithmic_bytes(n, nnz):
    return n * (2 * 8 + 4) + nnz * (8 + 4)


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic():
    """DRAM bytes per launch of the HLL SpMV kernel from the committed ncu
    summary (profiles/hll_spmv_27pt_200.txt), or None."""
    p = os.path.join(ROOT, "profiles", "hll_spmv_27pt_200.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("dram_bytes_per_launch:"):
            return float(line.split(":")[1].split()[0])
    return None


class ClockSampler:
    """SM clock and throttle reasons sampled through NVML every ~5 ms in a
    background thread during the timed region (the same counters nvidia-smi
    prints: clocks.sm, clocks.max.sm, clocks_event_reasons.*)."""

    def __init__(self, index, period=0.005):
        self.index, self.period = index, period
        self.samples, self.reasons, self.smax = [], set(), None
        self._stop = None

    def _run(self):
        import pynvml as N
        names = {"hw_slowdown": getattr(N, "nvmlClocksEventReasonHwSlowdown", 0x8),
                 "hw_thermal_slowdown": getattr(N, "nvmlClocksEventReasonHwThermalSlowdown", 0x40),
                 "sw_thermal_slowdown": getattr(N, "nvmlClocksEventReasonSwThermalSlowdown", 0x20),
                 "sw_power_cap": getattr(N, "nvmlClocksEventReasonSwPowerCap", 0x4)}
        h = N.nvmlDeviceGetHandleByIndex(self.index)
        self.smax = N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM)
        while not self._stop.is_set():
            self.samples.append(N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM))
            try:
                r = N.nvmlDeviceGetCurrentClocksEventReasons(h)
            except Exception:
                r = N.nvmlDeviceGetCurrentClocksThrottleReasons(h)
            for k, bit in names.items():
                if r & bit:
                    self.reasons.add(k)
            self._stop.wait(self.period)

    def __enter__(self):
        import threading
        try:
            import pynvml as N
            N.nvmlInit()
            # NVML indexes physical GPUs; map through CUDA_VISIBLE_DEVICES
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            if vis:
                ids = [v.strip() for v in vis.split(",")]
                if self.index < len(ids) and ids[self.index].isdigit():
                    self.index = int(ids[self.index])
            self._stop = threading.Event()
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        except Exception:
            self._stop = None
        return self

    def __exit__(self, *a):
        if self._stop is not None:
            self._stop.set()
            self._t.join(timeout=2)

    def summary(self):
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None, "sm_max_mhz": self.smax,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def dist_max(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_spmv_gbs(irp, ja, va, x, seconds=12.0, max_reps=30):
    """The oracle's row-parallel CSR csmv (the reference's row order) on all
    host cores over the full matrix; returns (GB/s, reps, threads)."""
    import oracle as O
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    n, nnz = len(irp) - 1, len(ja)
    y = np.zeros(n)
    L = O.lib()
    xi = np.ascontiguousarray(x)
    L.or_csr_csmv(b"N", n, n, irp, ja, va, 1.0, xi, 0.0, y)  # warm-up
    t0 = time.perf_counter()
    reps = 0
    while reps < max_reps and (time.perf_counter() - t0) < seconds:
        L.or_csr_csmv(b"N", n, n, irp, ja, va, 1.0, xi, 0.0, y)
        reps += 1
    dt = (time.perf_counter() - t0) / reps
    return algorithmic_bytes(n, nnz) / dt / 1e9, reps, threads


def base_line(args, world):
    return {"metric": "SpMV GB/s (27-point 200^3, FP64 HLL-32, reference byte count)", "unit": "GB/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)"}


def run_reference(args):
    # rank 0 alone times the CPU path; other ranks exit without work
    if int(os.environ.get("RANK", "0")) != 0:
        return
    from psblas3_b200 import gen
    irp, ja, va = gen.stencil27(args.grid)
    n = len(irp) - 1
    x = np.random.default_rng(0).uniform(-1, 1, n)
    vals = []
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_spmv_gbs(irp, ja, va, x, seconds=0.5, max_reps=1)
    for _ in range(args.steps):
        gbs, reps, threads = cpu_spmv_gbs(irp, ja, va, x, seconds=4.0, max_reps=10)
        vals.append(gbs)
    v = statistics.median(vals)
    line = base_line(args, 1)
    line.update({
        "impl": "reference", "value": v, "ms_per_step": algorithmic_bytes(n, len(ja)) / v / 1e6,
        "config": {"workload": f"C2a: FP64 SpMV, 27-point Poisson {args.grid}^3, CSR rows (reference CPU csmv order)",
                   "rows": n, "nnz": len(ja)},
        "cpu_baseline": {"value": v, "unit": "GB/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} steps x up to 10 full-matrix SpMVs (<= 4 s each)"},
        "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    })
    print(json.dumps(line), flush=True)


def run_ours(args):
    world, rank, local = dist_setup()
    import torch
    torch.cuda.set_device(local)
    from psblas3_b200 import gen, psb
    from psblas3_b200._lib import check, lib
    psb.init(local)

    # ---- matrix: generated on the host, built into HLL on the device
    irp, ja, va = gen.stencil27(args.grid)
    n, nnz = len(irp) - 1, len(ja)
    d_irp, d_ja, d_va = (torch.from_numpy(a).to(f"cuda:{local}") for a in (irp, ja, va))
    A = psb.HllMat.from_csr_device(n, n, nnz, d_irp.data_ptr(), d_ja.data_ptr(), d_va.data_ptr(), 32)
    del d_irp, d_ja, d_va
    torch.cuda.empty_cache()
    x_host = np.random.default_rng(0).uniform(-1, 1, n)
    X, Y = psb.DVect.bld(x_host), psb.DVect(n)
    stream = torch.cuda.ExternalStream(lib.psb_cudaGetStream(), device=f"cuda:{local}")
    bytes_alg = algorithmic_bytes(n, nnz)

    # ---- device-resident timing
    for _ in range(max(args.warmup, 3)):
        A.spmv(1.0, X, 0.0, Y)
    torch.cuda.synchronize()
    dist_barrier(world)
    torch.cuda.synchronize()
    l0 = psb.kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            A.spmv(1.0, X, 0.0, Y)
        e1.record(stream)
        torch.cuda.synchronize()
    dist_barrier(world)
    torch.cuda.synchronize()
    launches = psb.kernel_launches() - l0
    ms = e0.elapsed_time(e1) / args.steps
    ms_max = dist_max(ms, world)
    value = world * bytes_alg / (ms_max * 1e-3) / 1e9

    # ---- end to end through the C-ABI with host buffers (pinned)
    xh = torch.from_numpy(x_host).pin_memory()
    yh = torch.empty(n, dtype=torch.float64).pin_memory()
    xp, yp = C.c_void_p(xh.data_ptr()), C.c_void_p(yh.data_ptr())
    for _ in range(2):
        check(lib.writeMultiVecDeviceDouble(X.h, xp), "write")
        check(lib.spmvHllDeviceDouble(A.h, 1.0, X.h, 0.0, Y.h), "spmv")
        check(lib.readMultiVecDeviceDouble(Y.h, yp), "read")
    dist_barrier(world)
    torch.cuda.synchronize()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for _ in range(args.steps):
        check(lib.writeMultiVecDeviceDouble(X.h, xp), "write")
        check(lib.spmvHllDeviceDouble(A.h, 1.0, X.h, 0.0, Y.h), "spmv")
        check(lib.readMultiVecDeviceDouble(Y.h, yp), "read")
    s1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = dist_max(s0.elapsed_time(s1) / args.steps, world)
    e2e = world * bytes_alg / (e2e_ms * 1e-3) / 1e9

    if rank == 0:
        peak, peak_kind = measured_peak()
        achieved = bytes_alg / (ms * 1e-3) / 1e9
        line = base_line(args, world)
        line.update({
            "value": value, "ms_per_step": ms_max,
            "config": {"workload": f"C2a: FP64 SpMV, 27-point Poisson {args.grid}^3, HLL hack 32, int32 indices",
                       "rows": n, "nnz": nnz, "bytes_per_step": bytes_alg, "parallelism": f"replicas x{world}",
                       "l2": "inputs 2.74 GB per step > 126 MB L2, no flush"},
            "e2e": {"value": e2e, "unit": "GB/s", "h2d_bytes_per_step": n * 8, "d2h_bytes_per_step": n * 8,
                    "ms_per_step": e2e_ms},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": profile_traffic(), "peak_source": peak_kind},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
        })
        if not args.no_cpu_baseline:
            gbs, reps, threads = cpu_spmv_gbs(irp, ja, va, x_host)
            line["cpu_baseline"] = {"value": gbs, "unit": "GB/s", "cores": threads, "kind": "port",
                                    "sample": f"{reps} full-matrix SpMVs of the same operator (CSR, oracle csmv)"}
        print(json.dumps(line), flush=True)
    A.free()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--grid", type=int, default=GRID, help="grid side (profiling runs use a smaller case)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
