"""psblas3_b200 -- B200-native (sm_100a) drop-in for PSBLAS's single-GPU
sparse Krylov path: HLL/ELL/CSR SpMV, the BLAS-1 vector kernels and the
CG/BiCGSTAB iteration with diagonal preconditioning, behind the C-ABI of
include/psbx.h (libpsbx.so).

``import psblas3_b200`` loads nothing; ``psblas3_b200.psb`` loads the
CUDA library and fails loudly when it is missing.
"""
import os

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libpsbx.so")


def build(quiet: bool = True) -> str:
    """Compile libpsbx.so for sm_100a in-tree (nvcc; no GPU needed)."""
    import subprocess
    cmd = ["make", "-C", os.path.join(PKG_DIR, "csrc"), "-j8"]
    if quiet:
        cmd.insert(1, "-s")
    subprocess.run(cmd, check=True)
    return LIB_PATH
