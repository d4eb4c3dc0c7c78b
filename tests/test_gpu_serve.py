"""The continuous-batching server on the device: requests of different
sizes (3-D Poisson grids and row-sorted power-law SPD matrices) arrive while
others run, join the running batch, and each result is bit-identical to the
same request served alone; every result meets the FP64 tolerance against
the oracle's residual."""
import numpy as np
import pytest

import oracle as O
from psblas3_b200 import gen

pytestmark = pytest.mark.gpu


def _pool(serve):
    pool, host = serve.Pool(), []
    for side in (9, 14):
        irp, ja, va = gen.poisson7(side)
        pool.add_csr(irp, ja, va)
        host.append((irp, ja, va))
    for rows, seed in ((3000, 1), (700, 2)):
        irp, ja, va = gen.powerlaw_spd(rows, kmax=rows - 1, seed=seed)
        irp, ja, va, _ = gen.sort_rows_by_length(irp, ja, va)
        pool.add_csr(irp, ja, va)
        host.append((irp, ja, va))
    return pool, host


def test_served_alone_equals_mix(psb):
    from psblas3_b200 import serve
    pool, host = _pool(serve)
    plan = [(0, 11), (2, 12), (1, 13), (3, 14), (2, 15), (0, 16), (1, 17), (3, 18)]
    srv = serve.Server(pool, hbm_budget=4e9, max_slots=16, max_rows_total=1 << 20)
    reqs = [serve.Request(i, m, seed, 1e-10, 0.0) for i, (m, seed) in enumerate(plan)]
    # three arrive first; the rest arrive while those are running
    for r in reqs[:3]:
        srv.submit(r)
    srv.step(0.0)
    srv.step(0.0)
    for r in reqs[3:]:
        srv.submit(r)
    srv.drain(clock=lambda: 1.0)
    srv.close()
    assert sorted(r.rid for r in srv.done) == list(range(len(plan)))
    joined_late = [r for r in reqs[3:] if r.t_admit == 1.0]
    assert joined_late, "no request joined a running batch"
    for r in reqs:
        assert r.state == 1, (r.rid, r.state, r.err)
        alone_srv = serve.Server(pool, hbm_budget=4e9, max_slots=2, max_rows_total=1 << 20)
        a = serve.Request(100 + r.rid, r.mat, r.seed, 1e-10, 0.0)
        alone_srv.submit(a)
        alone_srv.drain(clock=lambda: 0.0)
        alone_srv.close()
        assert np.array_equal(a.x.view(np.uint64), r.x.view(np.uint64)), r.rid
        assert a.iters == r.iters and a.outer == r.outer
        irp, ja, va = host[r.mat]
        b = serve.request_rhs(r, len(irp) - 1).cpu().numpy()
        res = O.csr_csmv(irp, ja, va, -1.0, r.x, 1.0, b)
        assert np.linalg.norm(res) <= 1e-10 * np.linalg.norm(b) * 1.0001, r.rid
    for m in pool.mats:
        m["A"].free()
