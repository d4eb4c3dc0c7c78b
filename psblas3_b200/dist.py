"""Row-block distribution of one matrix over ranks, with a halo exchange.

This is the distributed SpMV of base/psblas/psb_dspmm.f90:196-216: each
rank owns a contiguous block of rows and the matching entries of x; its
local matrix is split into the block whose columns it owns (a%ad) and the
block whose columns belong to other ranks (a%and).  The product is

    send: gather the owned entries other ranks need        (psi_swapdata send)
    y  = alpha * A_d x_owned + beta * y                    (overlaps the exchange)
    recv: scatter the received entries into the halo part  (psi_swapdata recv)
    y  = alpha * A_nd x + 1 * y

with the local vector laid out as in the reference's descriptor: the nl
owned entries first, then the nh halo entries (global indices sorted), so
that A_nd's columns are local indices nl .. nl+nh-1.

The host side (partition, halo lists, exchange plan) is plain Python and is
what every rank computes identically; the device side (gather, SpMV,
scatter) runs the library's kernels through the C-ABI.  The exchange itself
is a torch.distributed all_to_all_single of the gathered buffers: NCCL on
GPUs, gloo on CPU.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

__all__ = ["partition_rows", "LocalPart", "local_part", "ExchangePlan", "exchange_plan",
           "build_part_on_rank", "halo_exchange", "DistSpMV", "allreduce_sum", "dist_cg", "dist_cg1",
           "DeviceCGOps"]


def partition_rows(n, world):
    """Contiguous row blocks [lo, hi) whose sizes differ by at most one
    (the block distribution of psb_cdall with a uniform local size)."""
    n, world = int(n), int(world)
    base, extra = divmod(n, world)
    out, lo = [], 0
    for r in range(world):
        hi = lo + base + (1 if r < extra else 0)
        out.append((lo, hi))
        lo = hi
    return out


def owner_of(g, blocks):
    """Rank owning each global index in g (0-based)."""
    starts = np.array([b[0] for b in blocks], dtype=np.int64)
    return np.searchsorted(starts, np.asarray(g, dtype=np.int64), side="right") - 1


@dataclass
class LocalPart:
    """One rank's rows.  ad / and_ are 1-based CSR triples in local column
    numbering: ad has columns 1..nl, and_ has columns nl+1..nl+nh."""
    lo: int
    hi: int
    halo: np.ndarray                      # global (0-based) ids of the halo entries, sorted
    ad: tuple = field(repr=False)
    and_: tuple = field(repr=False)

    @property
    def nl(self):
        return self.hi - self.lo

    @property
    def nh(self):
        return len(self.halo)

    @property
    def ncol(self):
        return self.nl + self.nh


def local_part(irp, ja, val, lo, hi):
    """Split rows lo..hi-1 of a 1-based global CSR into the owned-column
    block and the halo block (entry order inside each row is kept)."""
    irp = np.asarray(irp, dtype=np.int64)
    ja = np.asarray(ja, dtype=np.int64)
    val = np.asarray(val, dtype=np.float64)
    s, e = irp[lo] - 1, irp[hi] - 1
    rows = np.repeat(np.arange(hi - lo), np.diff(irp[lo:hi + 1]))
    cols = ja[s:e] - 1
    vals = val[s:e]
    own = (cols >= lo) & (cols < hi)
    halo = np.unique(cols[~own])
    nl = hi - lo

    def csr(mask, local_cols):
        r = rows[mask]
        cnt = np.bincount(r, minlength=nl)
        p = np.zeros(nl + 1, np.int32)
        p[1:] = np.cumsum(cnt)
        return p + 1, (local_cols + 1).astype(np.int32), np.ascontiguousarray(vals[mask])

    ad = csr(own, cols[own] - lo)
    and_ = csr(~own, nl + np.searchsorted(halo, cols[~own]))
    return LocalPart(int(lo), int(hi), halo.astype(np.int64), ad, and_)


@dataclass
class ExchangePlan:
    """send_idx: 1-based local (owned) indices to gather, grouped by
    destination rank in rank order; send_counts / recv_counts per rank.
    Received entries arrive grouped by source rank in rank order, which is
    the order of the sorted halo, so they scatter to local nl+1..nl+nh."""
    send_idx: np.ndarray
    send_counts: list
    recv_counts: list


def exchange_plan(rank, blocks, halos):
    """Plan of `rank` from every rank's halo list (global ids, sorted)."""
    world = len(blocks)
    lo, hi = blocks[rank]
    recv_counts = [0] * world
    own = owner_of(halos[rank], blocks) if len(halos[rank]) else np.zeros(0, np.int64)
    for q in range(world):
        recv_counts[q] = int(np.count_nonzero(own == q))
    assert recv_counts[rank] == 0, "a halo entry is owned by this rank"
    send, send_counts = [], []
    for q in range(world):
        h = np.asarray(halos[q], dtype=np.int64)
        mine = h[(h >= lo) & (h < hi)] if q != rank else h[:0]
        send.append(mine - lo + 1)
        send_counts.append(int(len(mine)))
    idx = np.concatenate(send).astype(np.int32) if send else np.zeros(0, np.int32)
    return ExchangePlan(idx, send_counts, recv_counts)


def build_part_on_rank(irp, ja, val, rank, world, all_gather=None):
    """This rank's LocalPart and ExchangePlan.  The rank needs only its own
    rows; the halo lists of the others come through `all_gather`
    (obj -> list over ranks; torch.distributed.all_gather_object by default)."""
    n = len(irp) - 1
    blocks = partition_rows(n, world)
    part = local_part(irp, ja, val, *blocks[rank])
    if world == 1:
        halos = [part.halo]
    elif all_gather is None:
        import torch.distributed as dist
        halos = [None] * world
        dist.all_gather_object(halos, part.halo)
    else:
        halos = all_gather(part.halo)
    return part, exchange_plan(rank, blocks, halos), blocks


def halo_exchange(sendbuf, recvbuf, plan, async_op=False):
    """All-to-all of the gathered send buffer into the receive buffer (torch
    tensors on the process group's device: CUDA under NCCL, CPU under
    gloo).  Returns the work handle when async_op."""
    import torch.distributed as dist
    return dist.all_to_all_single(recvbuf, sendbuf, output_split_sizes=list(plan.recv_counts),
                                  input_split_sizes=list(plan.send_counts), async_op=async_op)


class DistSpMV:
    """y = alpha*A*x + beta*y for this rank's rows on its GPU.

    x is a DVect of length ncol (owned entries, then halo); y a DVect of
    length nl.  `exchange(sendbuf, recvbuf, plan)` moves the gathered
    buffers (torch CUDA tensors) and may return a handle with .wait(); the
    default is halo_exchange over the default process group, asynchronous,
    so the A_d product overlaps it."""

    def __init__(self, part: LocalPart, plan: ExchangePlan, hksz=32):
        import torch
        from . import psb
        self.psb, self.part, self.plan = psb, part, plan
        nl, ncol = part.nl, part.ncol
        self._keep = []

        def dev_hll(trip, cols):
            irp, ja, va = trip
            nz = int(irp[-1] - 1)
            d = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in
                 (irp.astype(np.int32), ja.astype(np.int32) if nz else np.zeros(1, np.int32),
                  va if nz else np.zeros(1))]
            self._keep.append(d)
            return psb.HllMat.from_csr_device(nl, cols, nz, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), hksz)

        self.Ad = dev_hll(part.ad, nl)
        self.And = dev_hll(part.and_, ncol) if part.nh else None
        ns, nr = int(sum(plan.send_counts)), int(sum(plan.recv_counts))
        self.send_idx = torch.from_numpy(np.ascontiguousarray(plan.send_idx)).cuda() if ns else None
        self.recv_idx = torch.arange(nl + 1, ncol + 1, dtype=torch.int32, device="cuda") if nr else None
        self.sendbuf = torch.empty(max(ns, 1), dtype=torch.float64, device="cuda")
        self.recvbuf = torch.empty(max(nr, 1), dtype=torch.float64, device="cuda")
        self.ns, self.nr = ns, nr
        self.comm = torch.cuda.Stream() if (ns or nr) else None

    def gather(self, x):
        if self.ns:
            self.psb.check(self.psb.lib.igathMultiVecDeviceDouble(
                x.h, 0, self.ns, 1, C.c_void_p(self.send_idx.data_ptr()), 1, C.c_void_p(self.sendbuf.data_ptr()), 1),
                "igathMultiVecDeviceDouble")

    def scatter(self, x):
        if self.nr:
            self.psb.check(self.psb.lib.iscatMultiVecDeviceDouble(
                x.h, 0, self.nr, 1, C.c_void_p(self.recv_idx.data_ptr()), 1, C.c_void_p(self.recvbuf.data_ptr()), 1,
                0.0), "iscatMultiVecDeviceDouble")

    def __call__(self, alpha, x, beta, y, exchange=None):
        import torch
        psb = self.psb
        lib_stream = torch.cuda.ExternalStream(psb.lib.psb_cudaGetStream())
        self.gather(x)
        work = None
        if self.comm is not None:
            # the exchange runs on its own stream once the gather is done
            self.comm.wait_stream(lib_stream)
            with torch.cuda.stream(self.comm):
                if exchange is None:
                    work = halo_exchange(self.sendbuf[:self.ns], self.recvbuf[:self.nr], self.plan, async_op=True)
                else:
                    work = exchange(self.sendbuf[:self.ns], self.recvbuf[:self.nr], self.plan)
        self.Ad.spmv(alpha, x, beta, y)          # owned columns, overlapping the exchange
        if self.comm is not None:
            with torch.cuda.stream(lib_stream):
                if work is not None and hasattr(work, "wait"):
                    work.wait()
            lib_stream.wait_stream(self.comm)
        if self.And is not None:
            self.scatter(x)
            self.And.spmv(alpha, x, 1.0, y)


# ------------------------------------------------------------ distributed CG
def allreduce_sum(vals):
    """The sums over ranks of a few scalars in ONE all_reduce (psb_sum of
    base/psblas/psb_ddot.f90:150, for several dots at once): a CPU tensor
    under gloo, a CUDA tensor under NCCL.  Identity on one rank."""
    import torch
    import torch.distributed as dist
    vals = [float(v) for v in vals]
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return vals
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor(vals, dtype=torch.float64, device=dev)
    dist.all_reduce(t)
    return t.tolist()


def dist_cg(ops, b, x, eps=1e-6, itmax=1000, istop=2, allreduce=allreduce_sum):
    """psb_dcg (krylov/psb_dcg.F90:218-295, DIAG preconditioner) on a
    row-block distribution; returns (iter, err) like psb_krylov.

    `ops` holds this rank's rows: spmv(alpha, x, beta, y) is the distributed
    product (halo exchange, then the local blocks), dot(u, v) the local part
    of a dot product, axpby / copy / prec the local vector updates, new(ext)
    a zero vector (ext: with room for the halo, for the vectors the product
    reads: x and p).  b holds the owned entries, x the owned entries of x0 on
    entry (room for the halo) and of the solution on exit.

    Per iteration the reference takes three global reductions: rho = (r, z)
    and sigma = (p, q) through psb_gedot and ||r|| through psb_genrm2 in
    psb_check_conv.  Here z = D^-1 r is formed right after the update of r,
    so ||r||^2 and the next rho travel in one all_reduce: two per iteration.
    The stop test is the reference's (krylov/psb_d_krylov_conv_mod.f90:
    127-202): istop 2, ||r|| <= eps ||b||; istop 3, ||r|| <= eps ||r0||;
    err = ||r|| / ||b|| (or / ||r0||).  The sums over ranks change the
    rounding of the dots, so iterations agree with the serial method to
    within a step or two."""
    import math
    if istop not in (2, 3):
        raise ValueError("dist_cg: istop 2 or 3")
    r, z, q = ops.new(), ops.new(), ops.new()
    p = ops.new(ext=True)
    ops.copy(b, r)
    ops.spmv(-1.0, x, 1.0, r)                       # r = b - A x0
    ops.prec(r, z)                                  # z = D^-1 r
    bb, rr, rho = allreduce([ops.dot(b, b), ops.dot(r, r), ops.dot(r, z)])
    den = math.sqrt(bb) if istop == 2 else math.sqrt(rr)
    it, err = 0, 0.0
    rho_old = 0.0
    while it < itmax:
        it += 1
        if it == 1:
            ops.copy(z, p)
        else:
            if rho_old == 0.0:
                break                               # breakdown on rho
            ops.axpby(1.0, z, rho / rho_old, p)     # p = z + beta p
        ops.spmv(1.0, p, 0.0, q)                    # q = A p
        (sigma,) = allreduce([ops.dot(p, q)])
        if sigma == 0.0:
            break                                   # breakdown on sigma
        alpha = rho / sigma
        ops.axpby(alpha, p, 1.0, x)
        ops.axpby(-alpha, q, 1.0, r)
        ops.prec(r, z)
        rr, rz = allreduce([ops.dot(r, r), ops.dot(r, z)])
        rn = math.sqrt(rr)
        err = rn / den if den != 0.0 else rn
        if (rn <= eps * den) if den != 0.0 else (rn <= eps):
            break
        rho_old, rho = rho, rz
    return it, err


def dist_cg1(ops, b, x, eps=1e-6, itmax=1000, istop=2, allreduce=allreduce_sum):
    """CG with ONE all_reduce per iteration (Chronopoulos & Gear 1989, the
    s-step form with s = 1): the product w = A z is formed right after
    z = M^-1 r, so (r, z), (z, w) and (r, r) of the same residual travel
    together, and sigma = (p, A p) comes from the recurrence
    sigma = (z, w) - beta * rho / alpha_old instead of a second dot; q = A p
    is carried as q = w + beta q.  Same iterates as psb_dcg in exact
    arithmetic, one more vector update per iteration, one reduction fewer;
    the rounding differs, so iterations agree with the serial method to
    within a step or two.  Stop test and (iter, err) as dist_cg."""
    import math
    if istop not in (2, 3):
        raise ValueError("dist_cg1: istop 2 or 3")
    r, z, w, q = ops.new(), ops.new(), ops.new(), ops.new()
    p = ops.new(ext=True)
    zx = ops.new(ext=True)                          # z with room for the halo: the product reads it
    ops.copy(b, r)
    ops.spmv(-1.0, x, 1.0, r)                       # r = b - A x0
    (bb,) = allreduce([ops.dot(b, b)]) if istop == 2 else (None,)
    it, err, den = 0, 0.0, None
    rho_old = alpha_old = 0.0
    while True:
        ops.prec(r, zx)                             # z = M^-1 r
        ops.copy(zx, z)
        ops.spmv(1.0, zx, 0.0, w)                   # w = A z
        rho, delta, rr = allreduce([ops.dot(r, z), ops.dot(z, w), ops.dot(r, r)])
        rn = math.sqrt(rr)
        if den is None:                             # r0: no test before the first update
            den = math.sqrt(bb) if istop == 2 else rn
        else:
            err = rn / den if den != 0.0 else rn
            if ((rn <= eps * den) if den != 0.0 else (rn <= eps)) or it >= itmax:
                break
        it += 1
        if it == 1:
            beta, sigma = 0.0, delta
        else:
            if rho_old == 0.0:
                break
            beta = rho / rho_old
            sigma = delta - beta * rho / alpha_old
        if sigma == 0.0:
            break
        alpha = rho / sigma
        if it == 1:
            ops.copy(z, p)
            ops.copy(w, q)
        else:
            ops.axpby(1.0, z, beta, p)              # p = z + beta p
            ops.axpby(1.0, w, beta, q)              # q = w + beta q  (= A p)
        ops.axpby(alpha, p, 1.0, x)
        ops.axpby(-alpha, q, 1.0, r)
        rho_old, alpha_old = rho, alpha
    return it, err


class DeviceCGOps:
    """The local operations of dist_cg on this rank's GPU: the DistSpMV
    product and the library's vector kernels over the nl owned entries (the
    extended vectors x and p carry the halo after them).  `exchange` is
    passed to the DistSpMV (None: all_to_all over the default group)."""

    def __init__(self, op: DistSpMV, dinv, exchange=None):
        from . import psb
        self.psb, self.op, self.dinv, self.exchange = psb, op, dinv, exchange
        self.nl, self.ncol = op.part.nl, op.part.ncol

    def new(self, ext=False):
        return self.psb.DVect(self.ncol if ext else self.nl)

    def spmv(self, alpha, x, beta, y):
        self.op(alpha, x, beta, y, exchange=self.exchange)

    def dot(self, u, v):
        return self.psb.psb_gedot(u, v, n=self.nl)

    def axpby(self, a, u, b, v):
        self.psb.psb_geaxpby(a, u, b, v, n=self.nl)

    def copy(self, u, v):
        self.psb.psb_geaxpby(1.0, u, 0.0, v, n=self.nl)

    def prec(self, r, z):
        self.psb.psb_gemlt(1.0, self.dinv, r, 0.0, z, n=self.nl)
