"""CPU checks of the drop-in boundary: libpsbx.so builds for sm_100a, loads
without a GPU, and exports every entry point include/psbx.h declares (no
compute call is made here)."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "psbx.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set()
    for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b([A-Za-z_]\w*)\s*\(", src, re.M):
        line = src[m.start(): src.find("\n", m.start())]
        if line.lstrip().startswith(("#", "typedef", "return")):
            continue
        names.add(m.group(1))
    return sorted(names)


@pytest.fixture(scope="module")
def libpath():
    import psblas3_b200
    if not os.path.exists(psblas3_b200.LIB_PATH):
        psblas3_b200.build()
    return psblas3_b200.LIB_PATH


def test_header_parses():
    names = declared_functions()
    for must in ("spmvHllDeviceDouble", "dotMultiVecDeviceDouble", "FallocHllDevice", "psbx_dkrylov",
                 "d_spmvCSRGDevice", "spmvEllDeviceDouble", "psiCopyCooToHlgDouble"):
        assert must in names
    assert len(names) > 80


def test_library_exports_every_declared_symbol(libpath):
    out = subprocess.run(["nm", "-D", "--defined-only", libpath], capture_output=True, text=True, check=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing


def test_library_loads_and_binds_without_gpu(libpath):
    from psblas3_b200 import _lib
    assert set(_lib.EXPORTED) <= set(declared_functions())
    # a call that touches no device: error string starts empty
    assert isinstance(_lib.lib.psbx_last_error(), bytes)


def test_library_is_sm100a(libpath):
    out = subprocess.run(["cuobjdump", "--list-elf", libpath], capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    assert "sm_100a" in out.stdout
