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
                 "state", "slot", "db", "dx")

    def __init__(self, rid, mat, seed, eps, t_arrive):
        self.rid, self.mat, self.seed, self.eps, self.t_arrive = rid, mat, seed, eps, t_arrive
        self.t_admit = self.t_done = None
        self.x = None
        self.slot = None


class Server:
    def __init__(self, pool, hbm_budget=150e9, max_slots=512, max_rows_total=200_000_000, inner_tol=1e-2,
                 itmax=200_000, replays_per_step=2, engine=None):
        """engine: a psb.BatchSolver-like object (add/launch/wait/poll/remove/free);
        by default a new 1-rhs batch engine with max_slots slots."""
        self.pool = pool
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
        for slot in list(self.running):
            st, outer, its, err = self.eng.poll(slot)
            if st == 0:
                continue
            req = self.running.pop(slot)
            req.state, req.outer, req.iters, req.err = st, outer, its[0], err[0]
            finished.append(req)
        return finished

    def _retire(self, finished):
        """Copy the finished solutions back to host arrays and free their slots
        and memory (the slots' phase is done, so replays in flight do not
        touch them)."""
        for req in finished:
            req.x = req.dx.cpu().numpy()
        now = time.perf_counter()
        for req in finished:
            req.t_done = now
            self.eng.remove(req.slot)
            m = self.pool.mats[req.mat]
            self.in_use -= m["n"] * BYTES_PER_ROW
            self.rows_in_use -= m["n"]
            req.db = req.dx = None
            self.done.append(req)

    def step(self, now):
        """One round: take the results of the replays in flight, launch the
        next replays for the running requests, and -- while the device runs
        them -- admit what fits (the new requests join at the next launch),
        copy the finished solutions back and free their slots."""
        finished = []
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

    @property
    def busy(self):
        return bool(self.queue or self.running or self.inflight)

    def drain(self, clock=time.perf_counter):
        while self.busy:
            self.step(clock())

    def close(self):
        self.eng.free()


def run_stream(server, arrivals, clock=time.perf_counter):
    """arrivals: list of Request sorted by t_arrive (seconds from start).
    Replays them in real time; returns wall time to drain."""
    t0 = clock()
    i = 0
    for r in arrivals:
        r.t_arrive = t0 + r.t_arrive
    while i < len(arrivals) or server.busy:
        now = clock()
        while i < len(arrivals) and arrivals[i].t_arrive <= now:
            server.submit(arrivals[i])
            i += 1
        if not server.busy and i < len(arrivals):
            time.sleep(max(0.0, min(0.001, arrivals[i].t_arrive - now)))
            continue
        server.step(now)
    return clock() - t0


def latency_stats(done):
    lat = np.array([r.t_done - r.t_arrive for r in done])
    if lat.size == 0:
        return {}
    return {"count": int(lat.size), "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3), "mean_ms": float(lat.mean() * 1e3)}
