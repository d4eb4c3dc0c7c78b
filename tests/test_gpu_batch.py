"""GPU tests of the batched mixed-precision CG engine (psbx_batch_*).

Bar: every right-hand side reaches ||b - A x||_2 <= 1e-10 ||b||_2, checked
here in FP64 on the host with the oracle's CSR product; the solution agrees
with the FP64 device CG (psbx_dkrylov) to the accuracy the tolerance allows;
a system's result is bit-identical alone and in a mix of other systems, and
when it joins the engine while others are already iterating."""
import numpy as np
import pytest

import oracle as O
from psblas3_b200 import gen

pytestmark = pytest.mark.gpu
EPS = 1e-10


def _system(psb, irp, ja, va):
    import torch
    n = len(irp) - 1
    d = [torch.from_numpy(a).cuda() for a in (irp, ja, va)]
    A = psb.HllMat.from_csr_device(n, n, len(ja), d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), 32)
    P = psb.DiagPrec("DIAG").build(A)
    return A, P


def _true_relres(irp, ja, va, x, b):
    r = O.csr_csmv(irp, ja, va, -1.0, x, 1.0, b)
    return np.linalg.norm(r) / np.linalg.norm(b)


def test_mixed_single_system_poisson(psb):
    import torch
    irp, ja, va = gen.poisson7(24)
    n = len(irp) - 1
    ustar = np.random.default_rng(0).uniform(0, 1, n)
    b = O.csr_csmv(irp, ja, va, 1.0, ustar, 0.0, np.zeros(n))
    A, P = _system(psb, irp, ja, va)
    db = torch.from_numpy(b).cuda()
    dx = torch.zeros(n, dtype=torch.float64, device="cuda")
    eng = psb.BatchSolver(1, n, 1)
    s = eng.add(A, db, dx, P.dv.data_ptr, eps=EPS)
    eng.run()
    st, outer, its, err = eng.poll(s)
    x = dx.cpu().numpy()
    assert st == 1 and err[0] <= EPS and outer >= 2
    assert _true_relres(irp, ja, va, x, b) <= 1.01 * EPS
    # FP64 device CG on the same system
    B, X = psb.DVect.bld(b), psb.DVect(n)
    X.zero()
    it64, err64 = psb.psb_krylov("CG", A, P, B, X, eps=EPS, itmax=5000)
    x64 = X.get_vect()
    assert np.max(np.abs(x - x64)) <= 1e-7 * np.max(np.abs(x64))
    assert its[0] <= 2 * it64


def _aniso_set(seed, count, k):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        m = int(rng.integers(32, 72))
        epsx = float(np.exp(rng.uniform(np.log(1e-2), 0.0)))
        irp, ja, va = gen.aniso2d(m, epsx)
        rhs = rng.uniform(-1, 1, (len(irp) - 1, k))
        out.append((irp, ja, va, rhs))
    return out


def _solve_set(psb, systems, k, order=None, late=None):
    """Solve `systems` in one engine; `late` systems join after 3 steps."""
    import torch
    total = sum(len(s[0]) - 1 for s in systems)
    eng = psb.BatchSolver(len(systems), total, k)
    xs, slots, keep = {}, {}, []
    idx = list(range(len(systems))) if order is None else order

    def add(i):
        irp, ja, va, rhs = systems[i]
        A, P = _system(psb, irp, ja, va)
        db = torch.from_numpy(np.ascontiguousarray(rhs.reshape(-1))).cuda()
        dx = torch.zeros_like(db)
        slots[i] = eng.add(A, db, dx, P.dv.data_ptr, eps=EPS)
        xs[i] = dx
        keep.append((A, P, db))

    for i in idx:
        if late is None or i not in late:
            add(i)
    if late:
        eng.step(3)
        for i in late:
            add(i)
    eng.run()
    res = {}
    for i in idx:
        st, outer, its, err = eng.poll(slots[i])
        res[i] = (st, its, err, xs[i].cpu().numpy().reshape(-1, k))
    eng.free()
    return res


@pytest.mark.parametrize("k", [1, 8])
def test_batched_converge_and_alone_equals_mix(psb, k):
    systems = _aniso_set(7, 6, k)
    mix = _solve_set(psb, systems, k)
    for i, (irp, ja, va, rhs) in enumerate(systems):
        st, its, err, x = mix[i]
        assert st == 1, (i, st, err)
        for j in range(k):
            assert _true_relres(irp, ja, va, x[:, j], rhs[:, j]) <= 1.01 * EPS
    alone = _solve_set(psb, [systems[2]], k)[0]
    assert np.array_equal(alone[3].view(np.uint64), mix[2][3].view(np.uint64))
    assert alone[1] == mix[2][1]
    # joining while others iterate does not change anything either
    late = _solve_set(psb, systems, k, late=[2, 4])
    for i in range(len(systems)):
        assert np.array_equal(late[i][3].view(np.uint64), mix[i][3].view(np.uint64)), i


def test_eight_rhs_equal_single_rhs(psb):
    """Column j of an 8-rhs solve is bit-identical to the 1-rhs solve of
    that right-hand side (same per-rhs operation order; rows longer than 64
    entries, summed by the block for one right-hand side and by a warp for
    eight, are the exception and absent here)."""
    systems = _aniso_set(11, 2, 8)
    r8 = _solve_set(psb, systems, 8)
    irp, ja, va, rhs = systems[1]
    r1 = _solve_set(psb, [(irp, ja, va, rhs[:, 5:6])], 1)[0]
    assert np.array_equal(r1[3][:, 0].view(np.uint64), r8[1][3][:, 5].view(np.uint64))


def test_powerlaw_long_rows_in_mix(psb):
    """Row-sorted power-law systems put their rows longer than 64 entries
    in long-row tiles (summed by the whole block); they converge and stay
    bit-identical alone and in a mix with stencil systems."""
    rng = np.random.default_rng(3)
    systems = []
    for rows, seed in ((6000, 1), (2500, 2)):
        irp, ja, va = gen.powerlaw_spd(rows, kmax=min(4096, rows - 1), seed=seed)
        irp, ja, va, _ = gen.sort_rows_by_length(irp, ja, va)
        assert np.diff(irp)[0] > 128
        systems.append((irp, ja, va, rng.uniform(-1, 1, (rows, 1))))
    systems += _aniso_set(5, 3, 1)
    mix = _solve_set(psb, systems, 1)
    for i, (irp, ja, va, rhs) in enumerate(systems):
        assert mix[i][0] == 1
        assert _true_relres(irp, ja, va, mix[i][3][:, 0], rhs[:, 0]) <= 1.01 * EPS
    alone = _solve_set(psb, [systems[0]], 1)[0]
    assert np.array_equal(alone[3].view(np.uint64), mix[0][3].view(np.uint64))


def test_remove_and_reuse_slot(psb):
    import torch
    irp, ja, va = gen.aniso2d(40, 0.1)
    n = len(irp) - 1
    A, P = _system(psb, irp, ja, va)
    eng = psb.BatchSolver(2, 4 * n, 1)
    dinv = P.dv.data_ptr
    xs = []
    for seed in (1, 2, 3):
        b = np.random.default_rng(seed).uniform(-1, 1, n)
        db = torch.from_numpy(b).cuda()
        dx = torch.zeros_like(db)
        s = eng.add(A, db, dx, dinv, eps=EPS)
        eng.run()
        st, outer, its, err = eng.poll(s)
        assert st == 1
        assert _true_relres(irp, ja, va, dx.cpu().numpy(), b) <= 1.01 * EPS
        eng.remove(s)
        xs.append((db, dx))
    eng.free()


@pytest.mark.parametrize("k", [1, 8])
def test_fp64_inner_engine(psb, k):
    """The engine with FP64 inner iterations (the batched FP64 solve): every
    right-hand side reaches the FP64 tolerance, and its iterations stay
    close to the FP64 device CG's on the same system (its refinements keep
    the search direction)."""
    import torch
    systems = _aniso_set(11, 5, k)
    total = sum(len(s[0]) - 1 for s in systems)
    eng = psb.BatchSolver(len(systems), total, k, inner_fp64=True)
    keep, slots = [], []
    for irp, ja, va, rhs in systems:
        A, P = _system(psb, irp, ja, va)
        db = torch.from_numpy(np.ascontiguousarray(rhs.reshape(-1))).cuda()
        dx = torch.zeros_like(db)
        slots.append(eng.add(A, db, dx, P.dv.data_ptr, eps=EPS))
        keep.append((A, P, db, dx))
    eng.run()
    for (irp, ja, va, rhs), s, (A, P, db, dx) in zip(systems, slots, keep):
        st, outer, its, err = eng.poll(s)
        assert st == 1, (st, its, err)
        x = dx.cpu().numpy().reshape(-1, k)
        for j in range(k):
            assert _true_relres(irp, ja, va, x[:, j], rhs[:, j]) <= 1.01 * EPS
        B, X = psb.DVect.bld(rhs[:, 0]), psb.DVect(len(irp) - 1)
        it64, _ = psb.psb_krylov("CG", A, P, B, X, eps=EPS, itmax=100000)
        assert its[0] <= 1.1 * it64 + 10, (its[0], it64)
    eng.free()


def test_finished_lists_ended_slots(psb):
    """psbx_batch_finished returns, after each step, exactly the slots that
    poll reports ended (state != 0) and that are not removed yet, in slot
    order; removing one takes it off the list."""
    import torch
    sizes = (6, 10, 16, 24)
    eng = psb.BatchSolver(8, sum(s ** 3 for s in sizes), 1)
    slots, keep = [], []
    for m in sizes:
        irp, ja, va = gen.poisson7(m)
        n = len(irp) - 1
        A, P = _system(psb, irp, ja, va)
        db = torch.from_numpy(np.random.default_rng(m).uniform(-1, 1, n)).cuda()
        dx = torch.zeros_like(db)
        keep.append((A, P, db, dx))
        slots.append(eng.add(A, db, dx, P.dv.data_ptr, eps=EPS))
    seen_partial = False
    for _ in range(200):
        running = eng.step(1)
        ended = [s for s in slots if eng.poll(s)[0] != 0]
        assert eng.finished() == sorted(ended)
        seen_partial |= 0 < len(ended) < len(slots)
        if running == 0:
            break
    assert eng.finished() == sorted(slots) and seen_partial
    eng.remove(slots[1])
    assert eng.finished() == sorted(s for s in slots if s != slots[1])
    eng.free()
