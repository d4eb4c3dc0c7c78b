"""World-size-2 gloo tests on CPU of the multi-rank plumbing: independent
systems are assigned to ranks with no data-path collective; the timing is
the max over ranks; summaries are gathered at rank 0."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from psblas3_b200 import shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, work, q):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    mine = shard.assign(work, world)[rank]
    local = sum(work[i] for i in mine)  # stands in for this rank's solve time
    tmax = shard.max_over_ranks(local, world)
    total = shard.sum_over_ranks(len(mine), world)
    got = shard.gather_to_root(sorted(mine), world, rank)
    if rank == 0:
        q.put((tmax, total, got))
    dist.barrier()
    dist.destroy_process_group()


def test_assign_is_balanced_and_complete():
    work = [5, 1, 1, 1, 4, 2, 2, 3, 8, 1]
    parts = shard.assign(work, 3)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(work)))
    loads = [sum(work[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(work)
    assert shard.assign(work, 3) == parts  # deterministic: every rank agrees


def test_two_rank_gloo_sharding():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    work = [float(w) for w in (9, 7, 5, 3, 2, 2, 1)]
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, work, q)) for r in range(2)]
    for p in procs:
        p.start()
    tmax, total, got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    parts = shard.assign(work, 2)
    assert tmax == max(sum(work[i] for i in p) for p in parts)
    assert total == len(work)
    assert sorted(i for g in got for i in g) == list(range(len(work)))


# ---- row-block distribution with halo exchange (psb_dspmm.f90:196-216) ----
def _global_matrix():
    from psblas3_b200 import gen
    import numpy as np
    return gen.pde3d(7, a=(1, 1, 1), b=(0.5, 0.5, 0.5))


def test_local_parts_cover_the_matrix():
    """Every entry of every row lands in exactly one of A_d / A_nd, halos
    are sorted and foreign, and the split product equals the global one
    within the FP64 tolerance (the split changes only the summation order)."""
    import numpy as np

    import oracle as O
    from psblas3_b200 import dist
    irp, ja, va = _global_matrix()
    n = len(irp) - 1
    x = np.random.default_rng(1).uniform(-1, 1, n)
    for world in (1, 2, 3, 5):
        blocks = dist.partition_rows(n, world)
        assert blocks[0][0] == 0 and blocks[-1][1] == n
        assert max(h - l for l, h in blocks) - min(h - l for l, h in blocks) <= 1
        parts = [dist.local_part(irp, ja, va, *b) for b in blocks]
        plans = [dist.exchange_plan(r, blocks, [p.halo for p in parts]) for r in range(world)]
        y = np.zeros(n)
        for r, (p, pl) in enumerate(zip(parts, plans)):
            assert p.ad[0][-1] - 1 + p.and_[0][-1] - 1 == irp[p.hi] - irp[p.lo]
            assert np.all(np.diff(p.halo) > 0) and not np.any((p.halo >= p.lo) & (p.halo < p.hi))
            assert sum(pl.recv_counts) == p.nh
            # what rank q sends to r is exactly r's halo entries owned by q
            for q in range(world):
                off = sum(plans[q].send_counts[:r])
                sent = plans[q].send_idx[off:off + plans[q].send_counts[r]] - 1 + blocks[q][0]
                want = p.halo[dist.owner_of(p.halo, blocks) == q]
                assert np.array_equal(sent, want)
            xe = np.concatenate([x[p.lo:p.hi], x[p.halo]])
            t = O.csr_csmv(*p.ad, 1.0, xe, 0.0, np.zeros(p.nl), nc=p.ncol)
            y[p.lo:p.hi] = O.csr_csmv(*p.and_, 1.0, xe, 1.0, t, nc=p.ncol)
        glob = O.csr_csmv(irp, ja, va, 1.0, x, 0.0, np.zeros(n))
        scale = O.csr_csmv(irp, ja, np.abs(va), 1.0, np.abs(x), 0.0, np.zeros(n))
        assert np.all(np.abs(y - glob) <= 1e-13 * scale)


def _halo_worker(rank, world, port, q):
    import datetime

    import numpy as np
    import torch
    import torch.distributed as dist

    from psblas3_b200 import dist as D
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    irp, ja, va = _global_matrix()
    n = len(irp) - 1
    x = np.random.default_rng(5).uniform(-1, 1, n)   # every rank can check against the global vector
    part, plan, blocks = D.build_part_on_rank(irp, ja, va, rank, world)
    xe = np.zeros(part.ncol)
    xe[:part.nl] = x[part.lo:part.hi]
    send = torch.from_numpy(xe[plan.send_idx - 1].copy())   # the gather, on the host here
    recv = torch.zeros(sum(plan.recv_counts), dtype=torch.float64)
    D.halo_exchange(send, recv, plan)
    xe[part.nl:] = recv.numpy()
    ok = bool(np.array_equal(xe[part.nl:], x[part.halo]))
    got = [None] * world
    dist.all_gather_object(got, (part.lo, part.hi, ok, len(part.halo)))
    if rank == 0:
        q.put(got)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_halo_exchange():
    """Two gloo ranks build their parts from their own rows, agree on the
    plan through all_gather_object, and the all-to-all delivers every halo
    entry (bit-exact copies of the owners' values)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_halo_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[2] for g in got] == [True, True]
    assert got[0][0] == 0 and got[0][1] == got[1][0]
    assert all(g[3] > 0 for g in got)


# ---- distributed CG (psb_dcg.F90:218-295 over the row-block product) ----
class _HostCGOps:
    """dist_cg's local operations on the host for the gloo ranks: the halo
    through the all-to-all, the local blocks through the oracle's csmv."""

    def __init__(self, part, plan, dinv):
        self.part, self.plan, self.dinv = part, plan, dinv
        self.nl, self.ncol = part.nl, part.ncol

    def new(self, ext=False):
        import numpy as np
        return np.zeros(self.ncol if ext else self.nl)

    def spmv(self, alpha, x, beta, y):
        import numpy as np
        import torch

        import oracle as O
        from psblas3_b200 import dist as D
        import torch.distributed as dist
        if dist.is_initialized():  # every rank takes part in the all-to-all
            send = torch.from_numpy(x[self.plan.send_idx - 1].copy())
            recv = torch.zeros(sum(self.plan.recv_counts), dtype=torch.float64)
            D.halo_exchange(send, recv, self.plan)
            x[self.nl:] = recv.numpy()
        t = O.csr_csmv(*self.part.ad, alpha, x, beta, np.asarray(y[:self.nl]), nc=self.ncol)
        y[:self.nl] = O.csr_csmv(*self.part.and_, alpha, x, 1.0, t, nc=self.ncol)

    def dot(self, u, v):
        import oracle as O
        return O.dot(u[:self.nl], v[:self.nl])

    def axpby(self, a, u, b, v):
        import oracle as O
        v[:self.nl] = O.axpby(a, u[:self.nl], b, v[:self.nl])

    def copy(self, u, v):
        v[:self.nl] = u[:self.nl]

    def prec(self, r, z):
        z[:self.nl] = self.dinv * r[:self.nl]


def _cg_system():
    import numpy as np

    import oracle as O
    from psblas3_b200 import gen
    irp, ja, va = gen.pde3d(12, a=(1, 1, 1), b=(0.0, 0.0, 0.0))   # SPD 7-point operator
    n = len(irp) - 1
    ustar = np.random.default_rng(3).uniform(0, 1, n)
    b = O.csr_csmv(irp, ja, va, 1.0, ustar, 0.0, np.zeros(n))
    rows = np.repeat(np.arange(n), np.diff(irp))
    diag = np.zeros(n)
    on = ja - 1 == rows
    diag[rows[on]] = va[on]
    return irp, ja, va, b, O.diag_prec_build(diag)


def _cg_worker(rank, world, port, q, single=False):
    import datetime

    import numpy as np
    import torch.distributed as dist

    from psblas3_b200 import dist as D
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    irp, ja, va, b, dinv = _cg_system()
    part, plan, blocks = D.build_part_on_rank(irp, ja, va, rank, world)
    ops = _HostCGOps(part, plan, dinv[part.lo:part.hi])
    x = ops.new(ext=True)
    calls = {"n": 0}

    def counted(vals):
        calls["n"] += 1
        return D.allreduce_sum(vals)

    solver = D.dist_cg1 if single else D.dist_cg
    it, err = solver(ops, b[part.lo:part.hi].copy(), x, eps=1e-9, itmax=500, allreduce=counted)
    got = [None] * world
    dist.all_gather_object(got, (part.lo, part.hi, it, err, calls["n"], x[:part.nl].copy()))
    if rank == 0:
        q.put(got)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("single", [False, True])
@pytest.mark.parametrize("world", [2, 3])
def test_gloo_distributed_cg(world, single):
    """Row-block CG over gloo ranks (halo all-to-all in every product; the
    per-iteration scalars in two all_reduces with the reference's
    recurrences, or in one with the single-reduction form): every rank
    reports the same iterations and error, within +-2 iterations of the
    oracle's serial CG, the tolerance reached, and the assembled x equal to
    the oracle's to 1e-8."""
    import numpy as np

    import oracle as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_cg_worker, args=(r, world, port, q, single)) for r in range(world)]
    for p in procs:
        p.start()
    got = q.get(timeout=180)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    irp, ja, va, b, dinv = _cg_system()
    xo, ito, erro = O.krylov("CG", irp, ja, va, b, dinv=dinv, eps=1e-9, itmax=500)
    its = {g[2] for g in got}
    assert len(its) == 1 and len({g[3] for g in got}) == 1
    it, err = got[0][2], got[0][3]
    assert abs(it - ito) <= 2, (it, ito)
    assert err <= 1e-9
    # all_reduces: the reference's recurrences take one at the start and two
    # per iteration; the single-reduction form one for ||b||, one per pass
    assert got[0][4] == (2 + it if single else 1 + 2 * it)
    x = np.concatenate([g[5] for g in sorted(got, key=lambda g: g[0])])
    assert np.max(np.abs(x - xo)) <= 1e-8 * np.max(np.abs(xo))


@pytest.mark.parametrize("single", [False, True])
def test_dist_cg_one_rank_stop_tests(single):
    """One rank, no process group: istop 3 (||r|| against ||r0||) within +-2
    iterations of the oracle's serial CG from a nonzero x0, and itmax ends
    the solve at exactly itmax iterations with the error of the last one."""
    import numpy as np

    import oracle as O
    from psblas3_b200 import dist as D
    irp, ja, va, b, dinv = _cg_system()
    n = len(irp) - 1
    part = D.local_part(irp, ja, va, 0, n)
    plan = D.exchange_plan(0, [(0, n)], [part.halo])
    ops = _HostCGOps(part, plan, dinv)
    solver = D.dist_cg1 if single else D.dist_cg
    x0 = np.random.default_rng(9).uniform(-1, 1, n)
    x = ops.new(ext=True)
    x[:n] = x0
    it, err = solver(ops, b.copy(), x, eps=1e-8, itmax=500, istop=3, allreduce=lambda v: [float(t) for t in v])
    xo, ito, erro = O.krylov("CG", irp, ja, va, b, x0=x0, dinv=dinv, eps=1e-8, itmax=500, istop=3)
    assert abs(it - ito) <= 2 and err <= 1e-8
    x = ops.new(ext=True)
    it, err = solver(ops, b.copy(), x, eps=1e-14, itmax=5, allreduce=lambda v: [float(t) for t in v])
    _, ito, erro = O.krylov("CG", irp, ja, va, b, dinv=dinv, eps=1e-14, itmax=5)
    assert it == 5 == ito
    assert abs(err - erro) <= 1e-6 * erro
