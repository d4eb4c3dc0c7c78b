"""Host logic of the continuous-batching server, on CPU with a stand-in
engine: FIFO admission under the HBM budget and the slot limit, requests
that arrive while others run join the running batch, finished requests
leave at once and their memory goes to the queue, latency statistics."""
import numpy as np
import torch

from psblas3_b200 import serve


class FakeEngine:
    """Stands in for psb.BatchSolver: a request finishes after `work`
    engine steps (its matrix's n // 100), one step per replay."""

    def __init__(self):
        self.slots, self.log = {}, []

    def add(self, A, db, dx, dinv, eps, inner_tol, itmax):
        s = min(set(range(len(self.slots) + 1)) - set(self.slots))
        if getattr(self, "max_slots", None) is not None and len(self.slots) >= self.max_slots:
            raise RuntimeError("no free slot")
        self.slots[s] = [0, A["n"] // 100, dx]
        self.log.append(("add", s, A["n"]))
        return s

    def step(self, replays=1):
        for v in self.slots.values():
            v[0] += replays
            if v[0] >= v[1]:
                v[2].fill_(1.0)
        return sum(1 for v in self.slots.values() if v[0] < v[1])

    def launch(self, replays=1):
        self.pending = replays

    def wait(self):
        return self.step(self.pending)

    def poll(self, s):
        done, need, _ = self.slots[s]
        return (1 if done >= need else 0), 1, [done], [0.0]

    def remove(self, s):
        del self.slots[s]

    def free(self):
        pass


class FakePool:
    def __init__(self, sizes):
        self.mats = [dict(A=dict(n=n), n=n, dinv=0) for n in sizes]
        self.device_bytes = 0


def _server(sizes, budget_rows, max_slots=8, monkeypatch=None):
    monkeypatch.setattr(serve, "request_rhs", lambda req, n: torch.zeros(n, dtype=torch.float64))
    eng = FakeEngine()
    eng.max_slots = max_slots
    return serve.Server(FakePool(sizes), hbm_budget=budget_rows * serve.BYTES_PER_ROW, max_slots=max_slots,
                        engine=eng)


def test_fifo_admission_under_budget(monkeypatch):
    sizes = [1000, 400, 400, 300]
    srv = _server(sizes, budget_rows=1500, monkeypatch=monkeypatch)
    reqs = [serve.Request(i, m, i, 1e-10, 0.0) for i, m in enumerate([0, 1, 2, 3, 1])]
    for r in reqs:
        srv.submit(r)
    srv.step(0.0)
    # 1000 + 400 rows fit, the next 400 does not: FIFO stops at the head
    assert sorted(r.rid for r in srv.running.values()) == [0, 1]
    assert [r.rid for r in srv.queue] == [2, 3, 4]
    t = 1.0
    while srv.queue or srv.running:
        srv.step(t)
        t += 1.0
        assert srv.in_use <= 1500 * serve.BYTES_PER_ROW
    assert sorted(r.rid for r in srv.done) == [0, 1, 2, 3, 4]
    adds = [e for e in srv.eng.log if e[0] == "add"]
    assert [a[2] for a in adds] == [sizes[m] for m in (0, 1, 2, 3, 1)]   # admitted in arrival order
    assert all(np.all(r.x == 1.0) for r in srv.done)
    assert srv.in_use == 0 and srv.rows_in_use == 0


def test_late_arrivals_join_running_batch(monkeypatch):
    """A short request that arrives while a long one runs is admitted at
    once and finishes first (no head-of-line blocking by the running one)."""
    srv = _server([5000, 200], budget_rows=10_000, monkeypatch=monkeypatch)
    long_req = serve.Request(0, 0, 0, 1e-10, 0.0)
    srv.submit(long_req)
    srv.step(0.0)
    srv.step(1.0)
    short = serve.Request(1, 1, 1, 1e-10, 1.5)
    srv.submit(short)
    t = 2.0
    while srv.queue or srv.running:
        srv.step(t)
        t += 1.0
    assert short.t_admit == 2.0 and long_req.t_done > short.t_done
    assert short.t_admit < long_req.t_done


def test_slot_limit(monkeypatch):
    srv = _server([100] * 10, budget_rows=10**9, max_slots=3, monkeypatch=monkeypatch)
    for i in range(10):
        srv.submit(serve.Request(i, i, i, 1e-10, 0.0))
    srv._admit(0.0)
    assert len(srv.running) == 3 and len(srv.queue) == 7
    srv.drain(clock=lambda: 0.0)
    assert len(srv.done) == 10


def test_latency_stats():
    reqs = []
    for i in range(100):
        r = serve.Request(i, 0, i, 1e-10, 0.0)
        r.t_done = (i + 1) * 1e-3
        reqs.append(r)
    s = serve.latency_stats(reqs)
    assert s["count"] == 100
    assert abs(s["p50_ms"] - 50.5) < 1e-9 and abs(s["p99_ms"] - 99.01) < 1e-9
    assert serve.latency_stats([]) == {}


def test_finished_slots_count_until_retired(monkeypatch):
    """With every slot taken, requests that finish in a round free their
    slots only after the next launch: admission waits for them instead of
    asking the engine for a slot it does not have."""
    srv = _server([100] * 6, budget_rows=10**9, max_slots=2, monkeypatch=monkeypatch)
    for i in range(6):
        srv.submit(serve.Request(i, i, i, 1e-10, 0.0))
    t = 0.0
    while srv.busy:
        srv.step(t)
        assert len(srv.eng.slots) <= 2
        t += 1.0
    assert sorted(r.rid for r in srv.done) == list(range(6))


def test_stream_window_reports_unfinished(monkeypatch):
    """run_stream with stop_at: arrivals past the window are not served, the
    requests not complete at the window's end come back unfinished, and only
    completions inside the window count."""
    srv = _server([100, 5000], budget_rows=10**9, max_slots=4, monkeypatch=monkeypatch)
    t = [0.0]

    def clock():
        t[0] += 0.01
        return t[0]

    srv.clock = clock
    reqs = [serve.Request(i, i % 2, i, 1e-10, 0.05 * i) for i in range(40)]
    wall, left = serve.run_stream(srv, reqs, clock=clock, stop_at=1.0)
    done = srv.done
    assert done and left
    assert {r.rid for r in done}.isdisjoint({r.rid for r in left})
    assert len(done) + len(left) == 40
    end = reqs[0].t_arrive - 0.0 + 1.0  # arrival times were shifted to the stream's start
    assert all(r.t_done <= end for r in done)
    assert not srv.running and not srv.queue
