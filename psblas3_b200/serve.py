"""Continuous-batching solve server over the batched mixed-precision CG
engine (psbx_batch_*).

Requests are (matrix, right-hand side, tolerance).  Matrices live on the
device in a resident pool (HLL-32 with FP64 values, FP32 copy and inverse
diagonal) and are shared by the requests that name them.  Requests wait in
a FIFO queue and are admitted into free engine slots while their vectors fit
the HBM budget; admitted requests advance together, 8 CG iterations per
engine step; finished requests leave at once and their slots and memory go
to the next requests in the queue -- requests that arrive while others run
join the running batch.  A request's result does not depend on which other
requests shared the engine (the engine's per-system reductions have a fixed
order), so a solve is bit-identical alone and in the mix.
"""
from __future__ import annotations

import collections
import time

import numpy as np

from . import psb

# device bytes per row and right-hand side the engine needs per request:
# b, x (FP64), r (FP64), r/z/p/q/d (FP32) and the FP32 inverse diagonal
BYTES_PER_ROW = 8 + 8 + 8 + 5 * 4 + 4


class Pool:
    """Device-resident matrices: HLL-32 (FP64 + FP32 copy) and DIAG."""

    def __init__(self):
        self.mats = []

    def add_csr(self, irp, ja, va, perm=None):
        import torch
        n = len(irp) - 1
        d = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (irp, ja, va)]
        A = psb.HllMat.from_csr_device(n, n, len(ja), d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), 32)
        A.make_single()
        P = psb.DiagPrec("DIAG").build(A)
        self.mats.append(dict(A=A, P=P, n=n, nnz=len(ja), perm=perm,
                              dinv=P.dv.data_ptr,
                              bytes=A.params()["allocsize"] * 16 + n * 20))
        return len(self.mats) - 1

    @property
    def device_bytes(self):
        return sum(m["bytes"] for m in self.mats)


def request_rhs(req, n):
    """The request's right-hand side, uniform in [-1, 1], generated on the
    device from the request's seed (reproducible, no host copy)."""
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(int(req.seed))
    return torch.empty(n, dtype=torch.float64, device="cuda").uniform_(-1.0, 1.0, generator=g)


class Request:
    __slots__ = ("rid", "mat", "seed", "eps", "t_arrive", "t_admit", "t_done", "x", "iters", "outer", "err",
                 "state", "slot", "db", "dx", "keep")

    def __init__(self, rid, mat, seed, eps, t_arrive, keep=True):
        self.rid, self.mat, self.seed, self.eps, self.t_arrive = rid, mat, seed, eps, t_arrive
        self.t_admit = self.t_done = None
        self.x = None
        self.slot = None
        self.keep = keep            # keep the solution as a host array (else it is delivered and dropped)


class PinnedBuffers:
    """Reusable page-locked host buffers for the solutions coming back, in
    power-of-two sizes (a pageable copy would wait for everything queued on
    the device, and pinning per request costs more than the copy)."""

    def __init__(self):
        self.free = collections.defaultdict(list)

    def get(self, n):
        import torch
        cap = 1 << max(10, int(n - 1).bit_length())
        lst = self.free[cap]
        return lst.pop() if lst else torch.empty(cap, dtype=torch.float64, pin_memory=True)

    def put(self, buf):
        self.free[buf.numel()].append(buf)


class Server:
    def __init__(self, pool, hbm_budget=150e9, max_slots=512, max_rows_total=200_000_000, inner_tol=1e-2,
                 itmax=200_000, replays_per_step=2, engine=None, clock=time.perf_counter):
        """engine: a psb.BatchSolver-like object (add/launch/wait/poll/remove/free);
        by default a new 1-rhs batch engine with max_slots slots.  clock: the
        time source of the completion times (the arrival stream's)."""
        self.pool = pool
        self.clock = clock
        self.budget = float(hbm_budget) - pool.device_bytes
        self.eng = engine if engine is not None else psb.BatchSolver(max_slots, max_rows_total, 1)
        self.max_slots = max_slots
        self.max_rows = max_rows_total
        self.queue = collections.deque()
        self.running = {}
        self.done = []
        self.in_use = 0.0
        self.rows_in_use = 0
        self.inner_tol, self.itmax = inner_tol, itmax
        self.replays = replays_per_step
        self.inflight = False       # replays launched and not yet waited for
        self.held = 0               # slots of finished requests not yet removed
        self.pinned = PinnedBuffers()
        self.copy_stream = None     # side stream of the solutions' device-to-host copies
        self.pending = collections.deque()  # (request, host buffer, copy event), in copy order

    def submit(self, req):
        self.queue.append(req)

    def _admit(self, now):
        import torch
        while self.queue and len(self.running) + self.held < self.max_slots:
            req = self.queue[0]
            m = self.pool.mats[req.mat]
            need = m["n"] * BYTES_PER_ROW
            if self.in_use + need > self.budget or self.rows_in_use + m["n"] > self.max_rows:
                break
            self.queue.popleft()
            req.db = request_rhs(req, m["n"])
            req.dx = torch.zeros_like(req.db)
            req.slot = self.eng.add(m["A"], req.db, req.dx, m["dinv"], eps=req.eps, inner_tol=self.inner_tol,
                                    itmax=self.itmax)
            req.t_admit = now
            self.running[req.slot] = req
            self.in_use += need
            self.rows_in_use += m["n"]

    def _collect(self):
        """Requests whose solve ended, as of the last wait (removed from the
        running set)."""
        finished = []
        # one call lists the ended slots (a poll per running slot would keep
        # the device idle for a host loop over all of them between replays)
        slots = self.eng.finished() if hasattr(self.eng, "finished") else list(self.running)
        for slot in slots:
            if slot not in self.running:
                continue
            st, outer, its, err = self.eng.poll(slot)
            if st == 0:
                continue
            req = self.running.pop(slot)
            req.state, req.outer, req.iters, req.err = st, outer, its[0], err[0]
            finished.append(req)
        return finished

    def _retire(self, finished):
        """Free the finished requests' slots and start copying their solutions
        to pinned host buffers on a side stream (the slots' phase is done, and
        the wait that reported them has seen their kernels end, so replays in
        flight do not touch them); the requests complete when their copies do
        (_deliver)."""
        import torch
        for req in finished:
            self.eng.remove(req.slot)
            if not req.dx.is_cuda:  # host vectors (a stand-in engine): nothing to copy
                self.pending.append((req, None, None))
                continue
            if self.copy_stream is None:
                self.copy_stream = torch.cuda.Stream()
            n = self.pool.mats[req.mat]["n"]
            buf = self.pinned.get(n)
            with torch.cuda.stream(self.copy_stream):
                buf[:n].copy_(req.dx, non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(self.copy_stream)
            self.pending.append((req, buf, ev))

    def _deliver(self, now, block=False):
        """Requests whose solution has reached host memory complete now: the
        solution is kept as a host array if the request asked for it, the
        pinned buffer and the device vectors are released."""
        while self.pending:
            req, buf, ev = self.pending[0]
            if ev is not None:
                if block:
                    ev.synchronize()
                elif not ev.query():
                    break
            self.pending.popleft()
            n = self.pool.mats[req.mat]["n"]
            req.t_done = now if not block else self.clock()
            if req.keep:
                req.x = buf[:n].numpy().copy() if buf is not None else req.dx.numpy().copy()
            if buf is not None:
                self.pinned.put(buf)
            self.in_use -= n * BYTES_PER_ROW
            self.rows_in_use -= n
            req.db = req.dx = None
            self.done.append(req)

    def step(self, now):
        """One round: take the results of the replays in flight, launch the
        next replays for the running requests, and -- while the device runs
        them -- admit what fits (the new requests join at the next launch),
        copy the finished solutions back and free their slots."""
        finished = []
        self._deliver(now)
        if self.inflight:
            self.eng.wait()
            self.inflight = False
            finished = self._collect()
        self.held = len(finished)  # their slots are freed only after the launch
        if self.running:
            self.eng.launch(self.replays)
            self.inflight = True
        self._admit(now)
        if not self.inflight and self.running:  # nothing was running: start at once
            self.eng.launch(self.replays)
            self.inflight = True
        if finished:
            self._retire(finished)
        self.held = 0
        self._deliver(self.clock())

    @property
    def busy(self):
        return bool(self.queue or self.running or self.inflight or self.pending)

    def drain(self, clock=time.perf_counter):
        while self.busy:
            self.step(clock())

    def abort(self):
        """Stop: wait for the replays in flight, deliver what finished, drop
        the running requests and the queue (returned, unfinished)."""
        if self.inflight:
            self.eng.wait()
            self.inflight = False
        finished = self._collect()
        if finished:
            self._retire(finished)
        self._deliver(self.clock(), block=True)
        left = list(self.running.values()) + list(self.queue)
        for req in self.running.values():
            self.eng.remove(req.slot)
            n = self.pool.mats[req.mat]["n"]
            self.in_use -= n * BYTES_PER_ROW
            self.rows_in_use -= n
            req.db = req.dx = None
        self.running.clear()
        self.queue.clear()
        return left

    def close(self):
        self.eng.free()


def run_stream(server, arrivals, clock=time.perf_counter, stop_at=None):
    """arrivals: list of Request sorted by t_arrive (seconds from start).
    Replays them in real time.  stop_at (seconds from start): stop there --
    the requests not complete by then are returned unfinished (an offered
    load above capacity is measured over the window, not drained); None:
    serve everything.  Returns (wall seconds, unfinished requests)."""
    t0 = clock()
    i = 0
    for r in arrivals:
        r.t_arrive = t0 + r.t_arrive
    end = None if stop_at is None else t0 + stop_at
    while i < len(arrivals) or server.busy:
        now = clock()
        if end is not None and now >= end:
            break
        while i < len(arrivals) and arrivals[i].t_arrive <= now:
            server.submit(arrivals[i])
            i += 1
        if not server.busy and i < len(arrivals):
            time.sleep(max(0.0, min(0.001, arrivals[i].t_arrive - now)))
            continue
        server.step(now)
    left = server.abort() if end is not None else []
    left += arrivals[i:]
    if end is not None:
        # completions after the window's end do not count for it
        late = [r for r in server.done if r.t_done > end]
        server.done = [r for r in server.done if r.t_done <= end]
        left += late
    return clock() - t0, left


def serve_fp64(pool, arrivals, max_seconds, clock=time.perf_counter):
    """The plain FP64 path as a server: the same arrival stream, one request
    at a time in arrival order (psb_krylov('CG') with DIAG, FP64, on the
    request's device right-hand side, solution copied back to host memory),
    for at most max_seconds.  Returns (wall seconds, completed requests)."""
    import ctypes as C
    import torch
    from ._lib import lib
    t0 = clock()
    for r in arrivals:
        r.t_arrive = t0 + r.t_arrive
    done = []
    for req in arrivals:
        now = clock()
        if now - t0 >= max_seconds:
            break
        if req.t_arrive > now:
            time.sleep(req.t_arrive - now)
        m = pool.mats[req.mat]
        db = request_rhs(req, m["n"])
        dx = torch.zeros_like(db)
        B, X = C.c_void_p(), C.c_void_p()
        lib.psbx_wrapMultiVecDevice(C.byref(B), C.c_void_p(db.data_ptr()), m["n"], 2)
        lib.psbx_wrapMultiVecDevice(C.byref(X), C.c_void_p(dx.data_ptr()), m["n"], 2)
        opt = psb.L.SolverOptions()
        lib.psbx_DefaultSolverOptions(C.byref(opt))
        opt.eps, opt.itmax, opt.istop = req.eps, 100000, 2
        req.t_admit = clock()
        psb.check(lib.psbx_dkrylov(b"CG", m["A"].h, 0, m["P"].dv.h, B, X, C.byref(opt)), "psbx_dkrylov")
        x = dx.cpu().numpy()
        req.t_done = clock()
        req.iters, req.err, req.state = opt.iter, opt.err, 1 if opt.err <= req.eps else 2
        if req.keep:
            req.x = x
        lib.freeMultiVecDevice(B)
        lib.freeMultiVecDevice(X)
        done.append(req)
    return clock() - t0, done


def latency_stats(done):
    lat = np.array([r.t_done - r.t_arrive for r in done])
    if lat.size == 0:
        return {}
    return {"count": int(lat.size), "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3), "mean_ms": float(lat.mean() * 1e3)}
