"""Generate bindc_symbols.json: every C symbol that the reference's Fortran GPU
modules bind through ``bind(c, name=...)``, per module file.

The link test (tests/test_abi.py) checks the exported symbols of libpsbx.so
against this list, so that linking the unmodified Fortran modules against the
library leaves nothing unresolved.  Run it where the psblas3 sources are:

    python tests/golden/make_bindc.py [PSBLAS_SOURCE_DIR]

(argument, else $PSBLAS_SRC, else /root/reference).  The modules are read as
text: Fortran comments ('!' to the end of a line) are dropped, continuation
lines joined, and the preprocessor blocks the files hold are resolved for a
CUDA 12 build (``#if CUDA_SHORT_VERSION <= 10`` false; ``#if
defined(SERIAL_MPI)`` false), as the reference's own build would see them.
"""
from __future__ import annotations

import json
import os
import re
import sys

MODULES = [
    "cuda/psb_cuda_env_mod.F90", "cuda/core_mod.f90", "cuda/psb_base_vectordev_mod.F90",
    "cuda/psb_d_vectordev_mod.F90", "cuda/psb_s_vectordev_mod.F90", "cuda/psb_i_vectordev_mod.F90",
    "cuda/psb_c_vectordev_mod.F90", "cuda/psb_z_vectordev_mod.F90",
    "cuda/hlldev_mod.F90", "cuda/elldev_mod.F90", "cuda/base_cusparse_mod.F90",
    "cuda/d_cusparse_mod.F90", "cuda/s_cusparse_mod.F90", "cuda/c_cusparse_mod.F90", "cuda/z_cusparse_mod.F90",
    "cuda/diagdev_mod.F90", "cuda/hdiagdev_mod.F90", "cuda/dnsdev_mod.F90",
]
CUDA_SHORT_VERSION = 12
_BIND = re.compile(r"bind\s*\(\s*c\s*,\s*name\s*=\s*['\"]([A-Za-z0-9_]+)['\"]\s*\)", re.I)


def _cond(expr: str) -> bool:
    expr = expr.strip()
    m = re.fullmatch(r"CUDA_SHORT_VERSION\s*(<=|<|>=|>|==)\s*(\d+)", expr)
    if m:
        op, v = m.group(1), int(m.group(2))
        return {"<=": CUDA_SHORT_VERSION <= v, "<": CUDA_SHORT_VERSION < v, ">=": CUDA_SHORT_VERSION >= v,
                ">": CUDA_SHORT_VERSION > v, "==": CUDA_SHORT_VERSION == v}[op]
    if re.fullmatch(r"defined\s*\(\s*SERIAL_MPI\s*\)", expr):
        return False
    raise ValueError(f"unhandled preprocessor condition: {expr}")


def active_lines(text: str):
    """Lines that a CUDA 12 build compiles, comments removed."""
    stack = []  # (taking, any_taken)
    out = []
    for line in text.splitlines():
        s = line.strip()
        if s.startswith("#"):
            d = s[1:].strip()
            if d.startswith("if"):
                c = _cond(d[2:]) if not d.startswith("ifdef") else False
                parent = all(t for t, _ in stack)
                stack.append((parent and c, c))
            elif d.startswith("else"):
                t, any_taken = stack.pop()
                parent = all(t2 for t2, _ in stack)
                stack.append((parent and not any_taken, True))
            elif d.startswith("endif"):
                stack.pop()
            continue
        if not all(t for t, _ in stack):
            continue
        out.append(line.split("!", 1)[0])
    return out


def bound_names(path: str):
    lines = active_lines(open(path, encoding="latin-1").read())
    joined = []
    buf = ""
    for ln in lines:
        t = ln.rstrip()
        lead = t.lstrip()
        if lead.startswith("&"):
            lead = lead[1:]
        if t.endswith("&"):
            buf += lead[:-1] + " " if buf else t[:-1] + " "
            continue
        joined.append(buf + lead if buf else t)
        buf = ""
    names = []
    for ln in joined:
        names += _BIND.findall(ln)
    return sorted(set(names))


def main(src: str) -> None:
    here = os.path.dirname(os.path.abspath(__file__))
    mods = {}
    for m in MODULES:
        mods[m] = bound_names(os.path.join(src, m))
    with open(os.path.join(here, "bindc_symbols.json"), "w") as f:
        json.dump({"cuda_short_version": CUDA_SHORT_VERSION, "modules": mods}, f, indent=1)
    print({m: len(v) for m, v in mods.items()})


if __name__ == "__main__":
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PSBLAS_SRC", "/root/reference")
    if not os.path.isfile(os.path.join(src, "cuda", "hlldev_mod.F90")):
        sys.exit(f"make_bindc: psblas3 sources not found at {src} (pass the directory or set PSBLAS_SRC)")
    main(src)
