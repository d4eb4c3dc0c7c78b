"""A pure C program as the caller (tests/c/psbx_cg_c_caller.c): it includes
only include/psbx.h and links only libpsbx.so, and makes the calls a C or
Fortran caller of the reference's GPU glue makes -- gpuInit, an HLL-32
matrix written from host arrays, device vectors, spmvHllDeviceDouble and the
device-resident CG (psbx_dkrylov) with the diagonal preconditioner.  On the
CPU it must compile as C99 with every warning an error and link; on a GPU
its product must be exact and its CG must match the oracle's serial CG on
the same matrix (iterations within +-2, the tolerance reached)."""
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c", "psbx_cg_c_caller.c")


def _build(tmp_path):
    import psblas3_b200
    if not os.path.exists(psblas3_b200.LIB_PATH):
        psblas3_b200.build()
    libdir = os.path.dirname(psblas3_b200.LIB_PATH)
    exe = str(tmp_path / "psbx_c_caller")
    cmd = ["gcc", "-std=c99", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), SRC,
           "-L", libdir, "-lpsbx", "-lm", f"-Wl,-rpath,{libdir}", "-o", exe]
    out = subprocess.run(cmd, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    return exe


def test_c_caller_compiles_and_links(tmp_path):
    assert os.access(_build(tmp_path), os.X_OK)


@pytest.mark.gpu
def test_c_caller_runs_cg(tmp_path):
    import oracle as O
    m = 60
    exe = _build(tmp_path)
    out = subprocess.run([exe, str(m)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    f = dict(re.findall(r"(\w+) (\S+)", out.stdout.strip()))
    assert int(f["rows"]) == m * m
    assert float(f["spmv_maxdiff"]) == 0.0
    # the same system through the oracle's serial CG
    irp, ja, va = [1], [], []
    for i in range(m):
        for j in range(m):
            r = i * m + j
            ent = []
            if i > 0:
                ent.append((r - m, -1.0))
            if j > 0:
                ent.append((r - 1, -1.0))
            ent.append((r, 4.0))
            if j < m - 1:
                ent.append((r + 1, -1.0))
            if i < m - 1:
                ent.append((r + m, -1.0))
            ja += [c + 1 for c, _ in ent]
            va += [v for _, v in ent]
            irp.append(len(ja) + 1)
    irp, ja, va = np.array(irp, np.int32), np.array(ja, np.int32), np.array(va)
    n = m * m
    b = O.csr_csmv(irp, ja, va, 1.0, np.ones(n), 0.0, np.zeros(n))
    _, ito, erro = O.krylov("CG", irp, ja, va, b, dinv=np.full(n, 0.25), eps=1e-9, itmax=5000)
    assert abs(int(f["iters"]) - ito) <= 2, (f, ito)
    assert float(f["err"]) <= 1e-9 and float(f["resid"]) <= 1e-8
    assert float(f["maxerr"]) <= 1e-6
