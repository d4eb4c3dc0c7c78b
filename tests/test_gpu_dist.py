"""Distributed CG (psb_dcg.F90:218-295 over the row-block product of
psb_dspmm.f90:196-216) on the device: the DistSpMV halo product and the
library's vector kernels under dist_cg, one rank alone and two gloo ranks
sharing one GPU (the halo staged through host memory; no kernel waits on
another rank), against the oracle's serial CG."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle as O
from psblas3_b200 import gen

pytestmark = pytest.mark.gpu


def _system():
    irp, ja, va = gen.pde3d(16, a=(1, 1, 1), b=(0.0, 0.0, 0.0))
    n = len(irp) - 1
    ustar = np.random.default_rng(7).uniform(0, 1, n)
    b = O.csr_csmv(irp, ja, va, 1.0, ustar, 0.0, np.zeros(n))
    rows = np.repeat(np.arange(n), np.diff(irp))
    diag = np.zeros(n)
    on = ja - 1 == rows
    diag[rows[on]] = va[on]
    return irp, ja, va, b, O.diag_prec_build(diag)


def _solve_rank(rank, world, exchange=None, single=False):
    from psblas3_b200 import dist as D
    from psblas3_b200 import psb
    irp, ja, va, b, dinv = _system()
    part, plan, blocks = D.build_part_on_rank(irp, ja, va, rank, world)
    op = D.DistSpMV(part, plan)
    ops = D.DeviceCGOps(op, psb.DVect.bld(dinv[part.lo:part.hi]), exchange=exchange)
    B = psb.DVect.bld(b[part.lo:part.hi])
    X = ops.new(ext=True)
    it, err = (D.dist_cg1 if single else D.dist_cg)(ops, B, X, eps=1e-9, itmax=1000)
    return part, it, err, X.get_vect()[:part.nl]


@pytest.mark.parametrize("single", [False, True])
def test_device_dist_cg_one_rank(psb, single):
    irp, ja, va, b, dinv = _system()
    part, it, err, x = _solve_rank(0, 1, single=single)
    xo, ito, erro = O.krylov("CG", irp, ja, va, b, dinv=dinv, eps=1e-9, itmax=1000)
    assert abs(it - ito) <= 2 and err <= 1e-9
    assert np.max(np.abs(x - xo)) <= 1e-8 * np.max(np.abs(xo))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _host_staged(send, recv, plan):
    """The halo all-to-all through host memory (gloo moves CPU tensors)."""
    import torch
    import torch.distributed as dist
    s = send.cpu()
    r = torch.empty(recv.numel(), dtype=torch.float64)
    dist.all_to_all_single(r, s, output_split_sizes=list(plan.recv_counts), input_split_sizes=list(plan.send_counts))
    recv.copy_(r)
    return None


def _worker(rank, world, port, q, single):
    import datetime

    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(0)
    from psblas3_b200 import psb
    psb.init(0)
    part, it, err, x = _solve_rank(rank, world, exchange=_host_staged, single=single)
    got = [None] * world
    dist.all_gather_object(got, (part.lo, part.hi, part.nh, it, err, x))
    if rank == 0:
        q.put(got)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("single", [False, True])
def test_device_dist_cg_two_ranks(psb, single):
    irp, ja, va, b, dinv = _system()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q, single)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert all(g[2] > 0 for g in got)            # both ranks have halo entries
    assert len({g[3] for g in got}) == 1 and len({g[4] for g in got}) == 1
    it, err = got[0][3], got[0][4]
    xo, ito, erro = O.krylov("CG", irp, ja, va, b, dinv=dinv, eps=1e-9, itmax=1000)
    assert abs(it - ito) <= 2 and err <= 1e-9
    x = np.concatenate([g[5] for g in sorted(got, key=lambda g: g[0])])
    assert np.max(np.abs(x - xo)) <= 1e-8 * np.max(np.abs(xo))
