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
        self.samples, self.stamps, self.reasons, self.smax = [], [], set(), None
        self._stop = None
        self.t_start = self.t_stop = None

    def start(self):
        """Marks the start of the timed region (sampling runs before it)."""
        self.t_start = time.perf_counter()

    def stop(self):
        self.t_stop = time.perf_counter()

    def _run(self):
        import pynvml as N
        names = {"hw_slowdown": getattr(N, "nvmlClocksEventReasonHwSlowdown", 0x8),
                 "hw_thermal_slowdown": getattr(N, "nvmlClocksEventReasonHwThermalSlowdown", 0x40),
                 "sw_thermal_slowdown": getattr(N, "nvmlClocksEventReasonSwThermalSlowdown", 0x20),
                 "sw_power_cap": getattr(N, "nvmlClocksEventReasonSwPowerCap", 0x4)}
        h = N.nvmlDeviceGetHandleByIndex(self.index)
        self.smax = N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM)
        while not self._stop.is_set():
            self.stamps.append(time.perf_counter())
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
        inside = [c for c, t in zip(self.samples, self.stamps)
                  if self.t_start is None or (self.t_start <= t <= (self.t_stop or t))]
        return {"sm_mhz": statistics.median(inside) if inside else None, "sm_max_mhz": self.smax,
                "reasons": sorted(self.reasons), "samples": len(inside)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def local_device(local):
    """The GPU of a rank: its local rank, wrapped over the visible devices
    (ranks beyond the device count share GPUs, as in a one-GPU check of the
    sharded paths)."""
    import torch
    return local % max(1, torch.cuda.device_count())


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


def host_residual(irp, ja, va, x, b):
    """||b - A x|| / ||b|| on the host (scipy CSR product) for the spot
    checks of solver outputs; CSR arrays with base irp[0]."""
    import scipy.sparse as sp
    b0 = int(irp[0])
    n = len(irp) - 1
    A = sp.csr_matrix((va, np.asarray(ja) - b0, np.asarray(irp) - b0), shape=(n, n))
    return float(np.linalg.norm(b - A @ x) / np.linalg.norm(b))


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
    g = gpu_reference_kernel(irp, ja, va, x, steps=max(args.steps, 10))
    if g is not None:
        line["gpu_reference_kernel"] = g
        del irp, ja, va
        line["gpu_reference_cg_c3"] = gpu_reference_cg_c3()
    print(json.dumps(line), flush=True)


def gpu_reference_cg_c3():
    """C3's plain FP64 CG (7-point Poisson 256^3, b = A u*, DIAG, 1e-10) on
    the reference's own GPU kernels driven in psb_dcg's call sequence
    (oracle/ref_cg.c): one kernel per PSBLAS call, dots and norms read back
    to the host.  The matrix comes from the oracle's restatement of the
    reference's CPU converter."""
    import torch
    import oracle as O
    from psblas3_b200 import gen
    ref = O.ref_gpu()
    try:
        irp, ja, va = gen.poisson7(256)
        n, nnz = len(irp) - 1, len(ja)
        ia, _, _ = gen.csr_to_coo(irp, ja, va)
        h = O.hll_from_coo(n, ia, ja, va, 32)
        dinv = O.diag_prec_build(O.hll_get_diag(h, n))
        del ia
        dv = {k: torch.from_numpy(np.ascontiguousarray(h[k])).cuda() for k in ("val", "ja", "hkoffs", "irn")}
        del h
        ustar = np.random.default_rng(0).uniform(0, 1, n)
        d_b = torch.from_numpy(O.csr_csmv(irp, ja, va, 1.0, ustar, 0.0, np.zeros(n))).cuda()
        d_dinv = torch.from_numpy(dinv).cuda()
        d_x = torch.zeros(n, dtype=torch.float64, device="cuda")
        ptrs = (dv["val"].data_ptr(), dv["ja"].data_ptr(), dv["hkoffs"].data_ptr(), dv["irn"].data_ptr())
        ref.cg(n, *ptrs, -(-nnz // n), d_dinv.data_ptr(), d_b.data_ptr(), d_x.data_ptr(), 1e-10, 5)  # warm-up
        d_x.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        it, err = ref.cg(n, *ptrs, -(-nnz // n), d_dinv.data_ptr(), d_b.data_ptr(), d_x.data_ptr(), 1e-10, 20000)
        t = time.perf_counter() - t0
        xr = d_x.cpu().numpy()
        return {"solve_ms": t * 1e3, "solves_per_s": 1.0 / t, "iters": it, "err": err,
                "max_abs_err_vs_ustar": float(np.max(np.abs(xr - ustar))),
                "path": "psb_dcg call sequence over SPGPU hell/dot/nrm2/axpby/maxypbz built for sm_100a"}
    finally:
        ref.close()


def gpu_reference_kernel(irp, ja, va, x, steps=20):
    """The reference's own GPU HLL SpMV (SPGPU spgpuDhellspmv, compiled from
    the psblas3 sources for sm_100a into oracle/_ref/) on the same matrix,
    timed with CUDA events on its handle's stream; None when it is not built
    or no GPU is present.  The HLL arrays come from the oracle's restatement
    of the reference's CPU converter, so nothing of this library runs here."""
    try:
        import torch
        import oracle as O
    except ImportError:
        return None
    if not torch.cuda.is_available():
        return None
    ref = O.ref_gpu()
    if ref is None:
        return None
    try:
        n, nnz = len(irp) - 1, len(ja)
        from psblas3_b200 import gen
        ia, _, _ = gen.csr_to_coo(irp, ja, va)
        h = O.hll_from_coo(n, ia, ja, va, 32)
        dv = {k: torch.from_numpy(np.ascontiguousarray(h[k])).cuda() for k in ("val", "ja", "hkoffs", "irn")}
        del h, ia
        dx = torch.from_numpy(x).cuda()
        dy = torch.zeros(n, dtype=torch.float64, device="cuda")
        st = torch.cuda.ExternalStream(ref.stream)
        args = (dy.data_ptr(), dy.data_ptr(), 1.0, dv["val"].data_ptr(), dv["ja"].data_ptr(), 32,
                dv["hkoffs"].data_ptr(), dv["irn"].data_ptr(), -(-nnz // n), n, dx.data_ptr(), 0.0)
        torch.cuda.synchronize()
        for _ in range(3):
            ref.hll_spmv(*args)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(steps):
            ref.hll_spmv(*args)
        e1.record(st)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        return {"value": algorithmic_bytes(n, nnz) / ms / 1e6, "unit": "GB/s", "ms_per_spmv": ms, "steps": steps,
                "kernel": "spgpuDhellspmv (cuda/spgpu/kernels/hell_dspmv.cu) built for sm_100a, HLL hack 32"}
    finally:
        ref.close()


def _time_spmv(mat, X, Y, steps, stream):
    import torch
    for _ in range(3):
        mat.spmv(1.0, X, 0.0, Y)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        mat.spmv(1.0, X, 0.0, Y)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def _host_ell(irp, ja, va):
    """ELL arrays (nzm x n, column-major by row, padding = last column of the
    row, value 0) from 1-based CSR, as psi_d_convert_ell_from_coo lays them."""
    n = len(irp) - 1
    irn = np.diff(irp).astype(np.int32)
    nzm = int(irn.max())
    ia = np.repeat(np.arange(n), irn)
    pos = np.arange(len(ja)) - (irp[ia].astype(np.int64) - 1)
    last = ja[np.maximum(irp[1:].astype(np.int64) - 2, 0)]
    eja = np.repeat(last[None, :], nzm, axis=0).astype(np.int32)
    eva = np.zeros((nzm, n))
    eja[pos, ia] = ja
    eva[pos, ia] = va
    idiag = np.zeros(n, np.int32)
    d = ja == ia + 1
    idiag[ia[d]] = pos[d] + 1
    return nzm, irn, eja.ravel(), eva.ravel(), idiag


def _part(out, name, fn):
    """Runs one sub-benchmark; a failure is recorded, not fatal."""
    import torch
    t0 = time.perf_counter()
    try:
        out[name] = fn()
    except Exception as e:  # keep the other measurements
        out[name] = {"error": f"{type(e).__name__}: {e}"}
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    print(f"[bench] {name}: {time.perf_counter() - t0:.1f} s {json.dumps(out[name])[:300]}", file=sys.stderr,
          flush=True)


def secondary(args, psb, gen, irp, ja, va, x_host, y_ref, stream):
    """Other configurations of the workload set, timed the same way (CUDA
    events on the library stream): C2a in ELL and CSR, the C2b power-law
    matrix, the C1 BiCGSTAB solve (with the oracle's CPU time), the C3 CG
    solve in FP64 and in mixed precision, C4 batched and C5 serving."""
    import torch
    import oracle as O
    out = {}
    n, nnz = len(irp) - 1, len(ja)
    B = algorithmic_bytes(n, nnz)
    steps = max(10, min(args.steps, 50))

    def c2a_formats():
        X, Y = psb.DVect.bld(x_host), psb.DVect(n)
        res = {}
        nzm, irn, eja, eva, idiag = _host_ell(irp, ja, va)
        E = psb.EllMat.from_host_ell(n, nzm, irn, eja, eva, idiag, n, nnz=nnz)
        del eja, eva
        ms = _time_spmv(E, X, Y, steps, stream)
        res["ell"] = {"gb_s": B / ms / 1e6, "ms": ms, "bitexact_vs_hll": bool(np.array_equal(Y.get_vect(), y_ref))}
        E.free()
        Cm = psb.CsrMat(n, irp, ja, va)
        ms = _time_spmv(Cm, X, Y, steps, stream)
        res["csr"] = {"gb_s": B / ms / 1e6, "ms": ms, "bitexact_vs_hll": bool(np.array_equal(Y.get_vect(), y_ref))}
        Cm.free()
        # autotuned HLL layout (hack size and wide-hack threshold)
        d_irp, d_ja, d_va = (torch.from_numpy(a).cuda() for a in (irp, ja, va))
        T, info = psb.HllMat.autotune_from_csr_device(n, n, nnz, d_irp.data_ptr(), d_ja.data_ptr(), d_va.data_ptr())
        del d_irp, d_ja, d_va
        ms = _time_spmv(T, X, Y, steps, stream)
        res["hll_autotuned"] = dict(info, gb_s=B / ms / 1e6, ms=ms,
                                    bitexact_vs_hll=bool(np.array_equal(Y.get_vect(), y_ref)))
        T.free()
        return res

    def c1_bicgstab():
        ci, cj, cv = gen.pde3d(40, a=(1, 1, 1), b=(1 / np.sqrt(3),) * 3)
        n1 = len(ci) - 1
        d_irp, d_ja, d_va = (torch.from_numpy(a).cuda() for a in (ci, cj, cv))
        A1 = psb.HllMat.from_csr_device(n1, n1, len(cj), d_irp.data_ptr(), d_ja.data_ptr(), d_va.data_ptr(), 32)
        P1 = psb.DiagPrec("DIAG").build(A1)
        ones, B1 = psb.DVect.bld(np.ones(n1)), psb.DVect(n1)
        A1.spmv(1.0, ones, 0.0, B1)
        X1 = psb.DVect(n1)
        times = []
        for _ in range(6):
            X1.zero()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            its, err = psb.psb_krylov("BICGSTAB", A1, P1, B1, X1, eps=1e-9, itmax=1000)
            times.append(time.perf_counter() - t0)
        b_host = B1.get_vect()
        O.set_threads(os.cpu_count() or 1)
        rows1 = np.repeat(np.arange(n1), np.diff(ci))
        diag1 = np.zeros(n1)
        on_diag = cj == rows1 + 1
        diag1[rows1[on_diag]] = cv[on_diag]
        dinv = O.diag_prec_build(diag1)
        t0 = time.perf_counter()
        _, ito, erro = O.krylov("BICGSTAB", ci, cj, cv, b_host, dinv=dinv, eps=1e-9)
        tcpu = time.perf_counter() - t0
        A1.free()
        return {"gpu_ms": 1e3 * statistics.median(times[1:]), "iters": its, "err": err, "cpu_ms": 1e3 * tcpu,
                "cpu_iters": ito, "cpu_err": erro, "cpu_threads": os.cpu_count()}

    _part(out, "c2a_formats", c2a_formats)
    _part(out, "c2b_powerlaw", lambda: c2b_powerlaw(psb, gen, stream, steps))
    _part(out, "c1_bicgstab", c1_bicgstab)
    if not args.skip_c3:
        _part(out, "c3_cg", lambda: c3_cg(psb, gen))
    if not args.skip_c4:
        _part(out, "c4_batched", lambda: c4_batched(psb, gen))
    if not args.skip_c5:
        _part(out, "c5_serving", lambda: c5_serving(psb, gen))
    return out


def c3_cg(psb, gen):
    """C3: SPD 7-point Poisson 256^3, b = A u* (u* uniform [0, 1]); plain FP64
    device CG to 1e-10 beside the mixed-precision CG (FP32 iterations,
    FP64-accumulated dots, FP64 residual replacement) to the same FP64
    tolerance, and the same system through the batched engine."""
    import torch
    qi, qj, qv = gen.poisson7(256)
    n3 = len(qi) - 1
    d_irp, d_ja, d_va = (torch.from_numpy(a).cuda() for a in (qi, qj, qv))
    A3 = psb.HllMat.from_csr_device(n3, n3, len(qj), d_irp.data_ptr(), d_ja.data_ptr(), d_va.data_ptr(), 32)
    del d_irp, d_ja, d_va
    P3 = psb.DiagPrec("DIAG").build(A3)
    ustar = np.random.default_rng(0).uniform(0, 1, n3)
    U, B3, X3 = psb.DVect.bld(ustar), psb.DVect(n3), psb.DVect(n3)
    A3.spmv(1.0, U, 0.0, B3)
    times = []
    for _ in range(2):
        X3.zero()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        it3, err3 = psb.psb_krylov("CG", A3, P3, B3, X3, eps=1e-10, itmax=20000)
        times.append(time.perf_counter() - t0)
    x64 = X3.get_vect()
    res = {"rows": n3, "nnz": len(qj),
           "fp64": {"solve_ms": 1e3 * min(times), "solves_per_s": 1.0 / min(times), "iters": it3, "err": err3,
                    "max_abs_err_vs_ustar": float(np.max(np.abs(x64 - ustar)))}}
    # mixed precision, single-system solver: FP32 iterations (values, vectors),
    # FP64-accumulated dots, FP64 residual replacement and stop test
    A3.make_single()
    times = []
    for _ in range(2):
        X3.zero()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        itm, errm, nref = psb.psb_mixed_cg(A3, P3, B3, X3, eps=1e-10, itmax=20000, delta=0.1)
        times.append(time.perf_counter() - t0)
    xm = X3.get_vect()
    res["mixed"] = {"solver": "psbx_dmixed_cg", "solve_ms": 1e3 * min(times), "solves_per_s": 1.0 / min(times),
                    "inner_iters": itm, "residual_replacements": nref, "delta": 0.1, "err": errm,
                    "converged": errm <= 1e-10,
                    "max_abs_err_vs_ustar": float(np.max(np.abs(xm - ustar))),
                    "max_abs_diff_vs_fp64_solve": float(np.max(np.abs(xm - x64)))}
    res["mixed_speedup_vs_fp64"] = res["mixed"]["solves_per_s"] / res["fp64"]["solves_per_s"]
    # the same system through the batched engine (restarted inner CG per refinement)
    eng = psb.BatchSolver(1, n3, 1)
    dx = torch.zeros(n3, dtype=torch.float64, device="cuda")
    db = torch.from_numpy(B3.get_vect()).cuda()
    times = []
    for _ in range(2):
        dx.zero_()
        s = eng.add(A3, db, dx, P3.dv.data_ptr, eps=1e-10)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eng.run(replays_per_step=8)
        times.append(time.perf_counter() - t0)
        st, outer, its, err = eng.poll(s)
        eng.remove(s)
    xe = dx.cpu().numpy()
    res["mixed_batch_engine"] = {"solve_ms": 1e3 * min(times), "solves_per_s": 1.0 / min(times),
                                 "inner_iters": its[0], "outer": outer, "converged": st == 1, "err": err[0],
                                 "max_abs_err_vs_ustar": float(np.max(np.abs(xe - ustar)))}
    eng.free()
    A3.free()
    return res


def c4_batched(psb, gen, n_sys=512, k=8, seed=0, fp64_sample=32, world=1, rank=0):
    """C4: 512 SPD 2-D anisotropic systems -eps u_xx - u_yy on n x n grids
    (n uniform in [32, 256], eps log-uniform in [1e-2, 1]), 8 right-hand
    sides each (uniform [-1, 1]), solved to ||r|| <= 1e-10 ||b|| by the
    batched mixed-precision engine; beside it the same systems through the
    engine with FP64 inner iterations, and the plain FP64 device CG one
    solve at a time on a random sample of the same (system, rhs) pairs.
    Under torchrun the systems are split over the ranks by shard.assign
    (work ~ rows; nothing crosses ranks on the data path), each rank solves
    its share on its own GPU, and the times are the max over ranks."""
    import torch
    from psblas3_b200 import shard

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    rng = np.random.default_rng(seed)
    specs = [(int(rng.integers(32, 257)), float(np.exp(rng.uniform(np.log(1e-2), 0.0)))) for _ in range(n_sys)]
    mine = shard.assign([m * m for m, _ in specs], world)[rank]
    mats, total = [], 0
    for i in mine:
        m, eps = specs[i]
        irp, ja, va = gen.aniso2d(m, eps)
        n = len(irp) - 1
        rhs = np.random.default_rng((seed, i)).uniform(-1, 1, (n, k))
        d = [torch.from_numpy(a).cuda() for a in (irp, ja, va)]
        A = psb.HllMat.from_csr_device(n, n, len(ja), d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), 32)
        A.make_single()
        P = psb.DiagPrec("DIAG").build(A)
        db = torch.from_numpy(np.ascontiguousarray(rhs.reshape(-1))).cuda()
        dx = torch.zeros_like(db)
        mats.append((irp, ja, va, rhs, A, P, db, dx))
        total += n
    nm = len(mats)
    eng = psb.BatchSolver(nm, total, k)
    slots = [eng.add(A, db, dx, P.dv.data_ptr, eps=1e-10)
             for (_, _, _, _, A, P, db, dx) in mats]
    torch.cuda.synchronize()
    barrier()
    l0 = psb.kernel_launches()
    t0 = time.perf_counter()
    eng.run(replays_per_step=4)
    tb = time.perf_counter() - t0
    launches = psb.kernel_launches() - l0
    states, iters, worst = [], [], 0.0
    for s in slots:
        st, outer, its, err = eng.poll(s)
        states.append(st)
        iters.extend(its)
        worst = max(worst, max(err))
    # the same systems through the engine with FP64 inner iterations: the
    # batched FP64 solve (batching without the FP32 inner iterations)
    eng64 = psb.BatchSolver(nm, total, k, inner_fp64=True)
    xs64 = [torch.zeros_like(db) for (_, _, _, _, _, _, db, _) in mats]
    slots64 = [eng64.add(A, db, x64, P.dv.data_ptr, eps=1e-10)
               for (_, _, _, _, A, P, db, _), x64 in zip(mats, xs64)]
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    eng64.run(replays_per_step=4)
    tb64 = time.perf_counter() - t0
    states64, iters64 = [], []
    for s in slots64:
        st, outer, its, err = eng64.poll(s)
        states64.append(st)
        iters64.extend(its)
    eng64.free()
    del xs64
    # FP64 check of a few solutions on the host (scipy CSR product)
    checked = 0.0
    for i in rng.choice(nm, min(4, nm), replace=False):
        irp, ja, va, rhs, A, P, db, dx = mats[i]
        x = dx.cpu().numpy().reshape(-1, k)
        for j in range(k):
            checked = max(checked, host_residual(irp, ja, va, x[:, j], rhs[:, j]))
    eng.free()
    # plain FP64 GPU path, one solve at a time, on a sample (rank 0's systems)
    t64, it64, pairs = 0.0, [], []
    if rank == 0:
        pairs = [(int(i), int(j)) for i, j in zip(rng.integers(0, nm, fp64_sample), rng.integers(0, k, fp64_sample))]
    for i, j in pairs:
        irp, ja, va, rhs, A, P, db, dx = mats[i]
        B, X = psb.DVect.bld(rhs[:, j]), psb.DVect(len(irp) - 1)
        best = None
        for _ in range(2):  # best of two: the baseline at its fastest
            X.zero()
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            it, err = psb.psb_krylov("CG", A, P, B, X, eps=1e-10, itmax=100000)
            dt = time.perf_counter() - t1
            best = dt if best is None else min(best, dt)
        t64 += best
        it64.append(it)
    tb, tb64 = shard.max_over_ranks(tb, world), shard.max_over_ranks(tb64, world)
    conv = int(shard.sum_over_ranks(sum(1 for s in states if s == 1), world))
    conv64 = int(shard.sum_over_ranks(sum(1 for s in states64 if s == 1), world))
    worst = shard.max_over_ranks(worst, world)
    checked = shard.max_over_ranks(checked, world)
    launches = int(shard.sum_over_ranks(launches, world))
    total = int(shard.sum_over_ranks(total, world))
    got = shard.gather_to_root((iters, iters64), world, rank)
    if rank != 0:
        return None
    iters = [v for g in got for v in g[0]]
    iters64 = [v for g in got for v in g[1]]
    solves = n_sys * k
    return {"systems": n_sys, "rhs_per_system": k, "rows_total": total, "ranks": world, "batched_s": tb,
            "batched_solves_per_s": solves / tb, "converged": conv,
            "fp64_batched_s": tb64, "fp64_batched_solves_per_s": solves / tb64,
            "fp64_batched_converged": conv64,
            "fp64_batched_inner_iters_median": float(np.median(iters64)),
            "mixed_over_fp64_batched": tb64 / tb,
            "max_err": worst, "host_checked_max_relres": checked, "inner_iters_max": int(max(iters)),
            "inner_iters_median": float(np.median(iters)), "kernel_launches": launches,
            "fp64_one_at_a_time_solves_per_s": len(pairs) / t64, "fp64_sample": len(pairs),
            "fp64_iters_median": float(np.median(it64)),
            "speedup_vs_fp64_one_at_a_time": (solves / tb) / (len(pairs) / t64 * world)}


def c2b_powerlaw(psb, gen, stream, steps=10):
    """C2b: the power-law matrix (4M rows, alpha 2.1, rows up to 4,096
    entries) in CSR, in HLL-32 as stored, and in HLL-32 with the rows held in
    decreasing-length order through a row permutation: exact mode (stored
    order, compared bit for bit), tolerance mode (the default: wide hacks
    summed split across the SMs, within 1e-13 of |A||x| row by row), and
    autotuned (hack size, wide threshold, threads per row)."""
    import torch
    pi, pj, pv = gen.powerlaw(4_000_000, seed=0)
    n2, nnz2 = len(pi) - 1, len(pj)
    B2 = algorithmic_bytes(n2, nnz2)
    x2 = np.random.default_rng(0).uniform(-1, 1, n2)
    X2, Y2 = psb.DVect.bld(x2), psb.DVect(n2)
    Cm = psb.CsrMat(n2, pi, pj, pv)
    ms = _time_spmv(Cm, X2, Y2, steps, stream)
    lens = np.diff(pi)
    res = {"rows": n2, "nnz": nnz2, "max_row": int(lens.max()), "rows_over_2048": int((lens > 2048).sum()),
           "csr": {"gb_s": B2 / ms / 1e6, "ms": ms}}
    y_csr = Y2.get_vect()
    Cm.free()
    # the gather floor: the reads of x at this matrix's column indices alone
    # (one L2 sector request each, columns being random), no values, no sums
    import ctypes as C
    from psblas3_b200._lib import check, lib
    d_ja = torch.from_numpy(pj).cuda()
    d_out = torch.empty((nnz2 + 7) // 8, dtype=torch.float64, device="cuda")
    g_ms = C.c_double(0.0)
    check(lib.psbx_probe_gather(C.c_void_p(d_ja.data_ptr()), nnz2, int(pi[0]), C.c_void_p(X2.data_ptr),
                                C.c_void_p(d_out.data_ptr()), 10, C.byref(g_ms)), "psbx_probe_gather")
    del d_ja, d_out
    res["gather_floor"] = {"ms": g_ms.value, "gathers": nnz2, "g_per_s": nnz2 / g_ms.value / 1e6,
                           "gb_s_at_floor": B2 / g_ms.value / 1e6}
    d_irp, d_ja, d_va = (torch.from_numpy(a).cuda() for a in (pi, pj, pv))
    H = psb.HllMat.from_csr_device(n2, n2, nnz2, d_irp.data_ptr(), d_ja.data_ptr(), d_va.data_ptr(), 32)
    del d_irp, d_ja, d_va
    H.set_wide_split(False)  # exact mode: the CPU csmv's bits
    ms = _time_spmv(H, X2, Y2, max(3, steps // 5), stream)
    res["hll_unsorted"] = {"gb_s": B2 / ms / 1e6, "ms": ms, "stored_over_nnz": H.params()["allocsize"] / nnz2}
    yh = Y2.get_vect()
    short = lens <= 2048
    res["csr_equals_hll_on_short_rows"] = bool(np.array_equal(yh[short], y_csr[short]))
    H.free()
    # HLL holding the rows in decreasing-length order through a row
    # permutation (y comes back in the original order): hacks of similar
    # rows; the wide ones go through the wide-hack path
    order = np.argsort(-lens, kind="stable").astype(np.int32)
    d_irp, d_ja, d_va = (torch.from_numpy(a).cuda() for a in (pi, pj, pv))
    d_perm = torch.from_numpy(order).cuda()
    H = psb.HllMat.from_csr_device(n2, n2, nnz2, d_irp.data_ptr(), d_ja.data_ptr(), d_va.data_ptr(), 32,
                                   d_perm.data_ptr())
    del d_irp, d_ja, d_va, d_perm
    H.set_wide_split(False)
    ms = _time_spmv(H, X2, Y2, steps, stream)
    res["hll_row_sorted"] = {"gb_s": B2 / ms / 1e6, "ms": ms, "stored_over_nnz": H.params()["allocsize"] / nnz2,
                             "bitexact_vs_unsorted_hll": bool(np.array_equal(Y2.get_vect(), yh))}
    # tolerance mode (the default): each wide hack summed in 64-column chunks
    # by all the SMs, in the same launch as the other rows; every row within
    # 1e-13 * (|A| |x|)_i of the stored-order sum
    import scipy.sparse as sp
    b0 = int(pi[0])  # index base of the generated CSR
    scale = sp.csr_matrix((np.abs(pv), pj - b0, pi - b0), shape=(n2, n2)) @ np.abs(x2)
    H.set_wide_split(True)
    ms = _time_spmv(H, X2, Y2, steps, stream)
    ys = Y2.get_vect()
    res["hll_row_sorted_split"] = {"gb_s": B2 / ms / 1e6, "ms": ms,
                                   "max_err_over_scale": float(np.max(np.abs(ys - yh) / scale)),
                                   "within_1e-13": bool(np.all(np.abs(ys - yh) <= 1e-13 * scale))}
    H.free()
    d_irp, d_ja, d_va = (torch.from_numpy(a).cuda() for a in (pi, pj, pv))
    d_perm = torch.from_numpy(order).cuda()
    T, info = psb.HllMat.autotune_from_csr_device(n2, n2, nnz2, d_irp.data_ptr(), d_ja.data_ptr(),
                                                  d_va.data_ptr(), d_perm.data_ptr())
    del d_irp, d_ja, d_va, d_perm
    ms = _time_spmv(T, X2, Y2, steps, stream)
    yt = Y2.get_vect()
    res["hll_row_sorted_autotuned"] = dict(info, gb_s=B2 / ms / 1e6, ms=ms)
    res["hll_row_sorted_autotuned"]["within_1e-13"] = bool(np.all(np.abs(yt - yh) <= 1e-13 * scale))
    for k in ("csr", "hll_row_sorted", "hll_row_sorted_split", "hll_row_sorted_autotuned"):
        res[k]["frac_of_gather_floor"] = res["gather_floor"]["ms"] / res[k]["ms"]
    T.set_wide_split(False)
    T.spmv(1.0, X2, 0.0, Y2)
    res["hll_row_sorted_autotuned"]["exact_mode_bitexact_vs_unsorted_hll"] = bool(np.array_equal(Y2.get_vect(), yh))
    T.free()
    return res


def _c5_matrix(spec):
    """One pool matrix of the serving mix (runs in a worker process)."""
    import numpy as np
    from psblas3_b200 import gen
    kind, size, seed = spec
    if kind == "poisson":
        return gen.poisson7(size)
    irp, ja, va = gen.powerlaw_spd(size, kmax=min(4096, size - 1), seed=seed)
    irp, ja, va, _ = gen.sort_rows_by_length(irp, ja, va)
    return irp, ja, va


def _c5_stream(rate, window, n_each, seed, keep_every=499):
    """Poisson arrivals (rate per second over window seconds); each request
    names a pool matrix, 50/50 Poisson grid or power-law, uniform within the
    kind, and carries a seeded right-hand side.  Every keep_every-th keeps
    its solution for the host check."""
    from psblas3_b200 import serve
    rng = np.random.default_rng(seed)
    t, reqs = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > window:
            return reqs
        k = int(rng.integers(0, n_each)) + (n_each if rng.random() < 0.5 else 0)
        rid = len(reqs)
        reqs.append(serve.Request(rid, k, int(rng.integers(1 << 31)), 1e-10, t, keep=rid % keep_every == 0))


def c5_serving(psb, gen, rate=2000.0, window=60.0, pool_each=16, seed=0, replays_per_step=2, window_b=30.0,
               fp64_seconds=15.0, world=1, rank=0):
    """C5: Poisson arrivals of solve requests drawn 50/50 from 3-D 7-point
    Poisson grids (side uniform in [10, 128]) and power-law unstructured SPD
    matrices (rows log-uniform in [1e3, 2e6], alpha 2.1, diagonally dominant)
    of a device-resident pool of 2*pool_each matrices, one seeded right-hand
    side each, FP64 tolerance 1e-10, admitted by a 150 GB HBM budget into the
    continuous-batching server.
      A: the stated stream, `rate` per second for `window` seconds; the
         throughput is the requests completed within the window (the backlog
         of an offered load above capacity is not drained: it is reported).
      B: 0.8 x the capacity measured in A, for window_b seconds, drained:
         latency there is service time, not backlog.
      FP64: the plain FP64 device CG serving the same streams one request at
         a time in arrival order, for fp64_seconds each: its capacity (stream
         A) and its latency at the rate of B.
    Under torchrun the pool's matrices are split over the ranks by
    shard.assign (work ~ rows); every rank draws the same global stream and
    serves the requests for its own matrices on its own GPU (nothing crosses
    ranks on the data path); counts are summed and latencies pooled at rank
    0."""
    import concurrent.futures as cf
    import multiprocessing as mp
    from psblas3_b200 import serve, shard
    rng = np.random.default_rng(seed)
    specs = [("poisson", int(rng.integers(10, 129)), 0) for _ in range(pool_each)]
    specs += [("powerlaw", int(np.exp(rng.uniform(np.log(1e3), np.log(2e6)))), int(rng.integers(1 << 30)))
              for _ in range(pool_each)]
    mine = shard.assign([sz ** 3 if kind == "poisson" else sz for kind, sz, _ in specs], world)[rank]
    local = {g: l for l, g in enumerate(mine)}
    t_gen = time.perf_counter()
    with cf.ProcessPoolExecutor(max_workers=min(len(mine), os.cpu_count() or 1),
                                mp_context=mp.get_context("spawn")) as ex:
        host = list(ex.map(_c5_matrix, [specs[i] for i in mine]))
    t_gen = time.perf_counter() - t_gen
    pool = serve.Pool()
    for irp, ja, va in host:
        pool.add_csr(irp, ja, va)

    def my_share(reqs):
        return [serve.Request(r.rid, local[r.mat], r.seed, r.eps, r.t_arrive, keep=r.keep)
                for r in reqs if r.mat in local]

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    # warm-up: one small request through each path
    w = serve.Server(pool, hbm_budget=150e9, replays_per_step=replays_per_step)
    serve.run_stream(w, [serve.Request(0, 0, 1, 1e-10, 0.0)])
    w.close()
    serve.serve_fp64(pool, [serve.Request(0, 0, 1, 1e-10, 0.0)], 60.0)

    def check(done):
        worst = 0.0
        for r in [q for q in done if q.keep and q.x is not None][:6]:
            irp, ja, va = host[r.mat]
            b = serve.request_rhs(r, pool.mats[r.mat]["n"]).cpu().numpy()
            worst = max(worst, host_residual(irp, ja, va, r.x, b))
        return shard.max_over_ranks(worst, world)

    def pooled_latency(done):
        lat = shard.gather_to_root([r.t_done - r.t_arrive for r in done], world, rank)
        if rank != 0:
            return {}
        lat = np.array([v for g in lat for v in g])
        if lat.size == 0:
            return {}
        return {"count": int(lat.size), "p50_ms": float(np.percentile(lat, 50) * 1e3),
                "p99_ms": float(np.percentile(lat, 99) * 1e3), "mean_ms": float(lat.mean() * 1e3)}

    def served(rate_, window_, seed_, stop):
        allreqs = _c5_stream(rate_, window_, pool_each, seed_)
        reqs = my_share(allreqs)
        srv = serve.Server(pool, hbm_budget=150e9, replays_per_step=replays_per_step)
        barrier()
        l0 = psb.kernel_launches()
        wall, left = serve.run_stream(srv, reqs, stop_at=window_ if stop else None)
        done = srv.done
        srv.close()
        wall = shard.max_over_ranks(wall, world)
        span = window_ if stop else wall
        completed = int(shard.sum_over_ranks(len(done), world))
        return {"arrival_rate_per_s": rate_, "window_s": window_, "requests": len(allreqs),
                "completed": completed,
                "unfinished_at_window_end": int(shard.sum_over_ranks(len(left) if stop else 0, world)),
                "converged": int(shard.sum_over_ranks(sum(1 for r in done if r.state == 1), world)),
                "wall_s": wall, "solves_per_s": completed / span, "latency": pooled_latency(done),
                "host_checked_max_relres": check(done),
                "kernel_launches": int(shard.sum_over_ranks(psb.kernel_launches() - l0, world))}

    out = {"pool_matrices": len(specs), "pool_rows": [m["n"] for m in pool.mats], "ranks": world,
           "pool_generation_s": t_gen, "request_mix": "50/50 Poisson / power-law, uniform over the pool's matrices"}
    a = served(rate, window, seed + 1, stop=True)
    out["A_stated_stream"] = a
    cap = a["solves_per_s"]
    b = served(0.8 * cap, window_b, seed + 2, stop=False)
    out["B_0p8_capacity"] = b
    # the plain FP64 path on the same streams, one request at a time per GPU
    barrier()
    fa_wall, fa = serve.serve_fp64(pool, my_share(_c5_stream(rate, window, pool_each, seed + 1)), fp64_seconds)
    fb_wall, fb = serve.serve_fp64(pool, my_share(_c5_stream(0.8 * cap, window_b, pool_each, seed + 2)),
                                   fp64_seconds)
    fa_rate = shard.sum_over_ranks(len(fa) / fa_wall if fa_wall > 0 else 0.0, world)
    fb_rate = shard.sum_over_ranks(len(fb) / fb_wall if fb_wall > 0 else 0.0, world)
    out["fp64_one_at_a_time"] = {
        "method": "the same arrival streams served one request at a time in arrival order (psb_krylov CG, DIAG)",
        "A_completed": int(shard.sum_over_ranks(len(fa), world)), "A_solves_per_s": fa_rate,
        "A_seconds": shard.max_over_ranks(fa_wall, world),
        "A_converged": int(shard.sum_over_ranks(sum(1 for r in fa if r.state == 1), world)),
        "B_completed": int(shard.sum_over_ranks(len(fb), world)), "B_solves_per_s": fb_rate,
        "B_seconds": shard.max_over_ranks(fb_wall, world),
        "B_latency": pooled_latency(fb), "host_checked_max_relres": check(fa + fb)}
    out["speedup_vs_fp64_A"] = cap / fa_rate
    out["speedup_vs_fp64_B"] = b["solves_per_s"] / fb_rate
    for m in pool.mats:
        m["A"].free()
    return out if rank == 0 else None


def run_ours(args):
    world, rank, local = dist_setup()
    import torch
    local = local_device(local)
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
        time.sleep(0.05)  # let the sampler take its first readings
        clk.start()
        e0.record(stream)
        for _ in range(args.steps):
            A.spmv(1.0, X, 0.0, Y)
        e1.record(stream)
        torch.cuda.synchronize()
        clk.stop()
    dist_barrier(world)
    torch.cuda.synchronize()
    launches = psb.kernel_launches() - l0
    ms = e0.elapsed_time(e1) / args.steps
    ms_max = dist_max(ms, world)
    value = world * bytes_alg / (ms_max * 1e-3) / 1e9

    # ---- end to end through the C-ABI with host buffers (pinned): the
    # reference's call sequence (write x, spmv, read y), and the one-call
    # host-buffer SpMV whose copies overlap the product block by block
    xh = torch.from_numpy(x_host).pin_memory()
    yh = torch.empty(n, dtype=torch.float64).pin_memory()
    xp, yp = C.c_void_p(xh.data_ptr()), C.c_void_p(yh.data_ptr())

    def three_calls():
        check(lib.writeMultiVecDeviceDouble(X.h, xp), "write")
        check(lib.spmvHllDeviceDouble(A.h, 1.0, X.h, 0.0, Y.h), "spmv")
        check(lib.readMultiVecDeviceDouble(Y.h, yp), "read")

    def one_call():
        check(lib.psbx_hll_spmv_host(A.h, 1.0, xp, 0.0, yp, 0), "psbx_hll_spmv_host")

    def e2e_time(step):
        for _ in range(2):
            step()
        dist_barrier(world)
        torch.cuda.synchronize()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for _ in range(args.steps):
            step()
        s1.record(stream)
        torch.cuda.synchronize()
        return dist_max(s0.elapsed_time(s1) / args.steps, world)

    e2e3_ms = e2e_time(three_calls)
    y3 = yh.numpy().copy()
    e2e_ms = e2e_time(one_call)
    e2e_same_bits = bool(np.array_equal(yh.numpy(), y3))
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
                    "ms_per_step": e2e_ms, "call": "psbx_hll_spmv_host (copies overlapped with the product)",
                    "same_bits_as_three_calls": e2e_same_bits,
                    "three_calls": {"value": world * bytes_alg / (e2e3_ms * 1e-3) / 1e9, "ms_per_step": e2e3_ms,
                                    "calls": "writeMultiVecDeviceDouble + spmvHllDeviceDouble + "
                                             "readMultiVecDeviceDouble"}},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": profile_traffic(), "peak_source": peak_kind},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
        })
        if not args.no_cpu_baseline:
            gbs, reps, threads = cpu_spmv_gbs(irp, ja, va, x_host)
            line["cpu_baseline"] = {"value": gbs, "unit": "GB/s", "cores": threads, "kind": "port",
                                    "sample": f"{reps} full-matrix SpMVs of the same operator (CSR, oracle csmv)"}
        if world == 1 and not args.no_secondary:
            line["secondary"] = secondary(args, psb, gen, irp, ja, va, x_host, Y.get_vect(), stream)
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
    ap.add_argument("--no-secondary", action="store_true", help="headline workload only")
    ap.add_argument("--skip-c3", action="store_true", help="skip the 256^3 CG solves among the secondaries")
    ap.add_argument("--skip-c4", action="store_true", help="skip the batched 512-system solve")
    ap.add_argument("--skip-c5", action="store_true", help="skip the serving stream")
    ap.add_argument("--only", choices=["c2b", "c3", "c4", "c5"], default=None,
                    help="run one secondary workload alone on one GPU and print its result (profiling runs)")
    args = ap.parse_args()
    if args.only:
        run_only(args.only)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


def run_only(name):
    """One secondary workload by itself (C2b power-law SpMV, C3 CG solves,
    C4 batched, C5 serving); prints {"only": name, "result": {...}} at rank
    0.  Under torchrun C4 and C5 are sharded over the ranks (shard.assign:
    independent systems, one GPU each); C2b and C3 run on rank 0's GPU."""
    world, rank, local = dist_setup()
    import torch
    from psblas3_b200 import gen, psb
    local = local_device(local)
    torch.cuda.set_device(local)
    psb.init(local)
    res = None
    if name in ("c4", "c5"):
        res = {"c4": c4_batched, "c5": c5_serving}[name](psb, gen, world=world, rank=rank)
    elif rank == 0:
        if name == "c2b":
            from psblas3_b200._lib import lib
            stream = torch.cuda.ExternalStream(lib.psb_cudaGetStream(), device=f"cuda:{local}")
            res = c2b_powerlaw(psb, gen, stream)
        else:
            res = c3_cg(psb, gen)
    if rank == 0:
        print(json.dumps({"only": name, "n_gpus": world, "result": res}), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
