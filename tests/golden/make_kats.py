"""Generate the golden known-answer fixtures from the reference's own tests.

Reads, as text, the reference test sources and writes JSON fixtures next to
this script.  Run it where the psblas3 source tree is available:

    python tests/golden/make_kats.py [PSBLAS_SOURCE_DIR]

The directory comes from the argument, else $PSBLAS_SRC, else
/root/reference; the script stops with a message when it is not there.

Fixtures written:
  usmv_kats.json   every ``d_usmv_*`` case of test/torture/psb_d_mvsv_tester.f90
                   (2x2 matrices; alpha, beta, trans, x, y before, y after).
  vecop_kats.json  the constant-vector cases of test/kernel/vecoperation.f90
                   (axpby / axpbyz / mlt / dot / amax with closed-form
                   answers); each case records the source line it checks and
                   the script verifies that the line's call text is there.
"""
from __future__ import annotations

import json
import os
import re
import sys


def _nums(s):
    return [float(t) for t in re.findall(r"-?\d+(?:\.\d*)?(?:[eEdD][-+]?\d+)?", s)]


def parse_usmv(path):
    src = open(path).read()
    cases = []
    for m in re.finditer(r"subroutine (d_usmv_\w+)\(res,afmt,ctxt\)(.*?)end subroutine \1", src, re.S):
        name, body = m.group(1), m.group(2)

        def grab(pat):
            mm = re.search(pat, body)
            if not mm:
                raise ValueError(f"{name}: {pat}")
            return mm.group(1)

        trans = grab(r"character::transa='(\w)'")
        alpha = float(grab(r"real\*8 :: alpha=(-?[\d.]+)"))
        beta = float(grab(r"real\*8 :: beta=(-?[\d.]+)"))
        m_ = int(grab(r"integer\(psb_ipk_\) :: m=(\d+)"))
        k_ = int(grab(r"integer\(psb_ipk_\) :: k=(\d+)"))
        ia = [int(v) for v in _nums(grab(r"IA\(\d+\)=\(/(.*?)/\)"))]
        ja = [int(v) for v in _nums(grab(r"JA\(\d+\)=\(/(.*?)/\)"))]
        va = _nums(grab(r"VA\(\d+\)=\(/(.*?)/\)"))
        x = _nums(grab(r"real\*8 :: x\(\d+\)=\(/(.*?)/\)"))
        cy = _nums(grab(r"real\*8 :: cy\(\d+\)=\(/(.*?)/\)"))
        bcy = _nums(grab(r"real\*8 :: bcy\(\d+\)=\(/(.*?)/\)"))
        line = src[: m.start()].count("\n") + 1
        cases.append(dict(name=name, line=line, trans=trans, alpha=alpha, beta=beta, m=m_, k=k_,
                          ia=ia, ja=ja, val=va, x=x, y_before=bcy, y_after=cy))
    return cases


# Each entry: (line in vecoperation.f90, call text expected on that line, case)
VECOP = [
    (241, "call psb_geaxpby(one,x,one,y,desc_a,info)",
     dict(op="axpby", alpha=1.0, x=1.0, beta=1.0, y=-2.0, expect=-1.0)),
    (250, "call psb_geaxpby(negativeone,x,one,y,desc_a,info)",
     dict(op="axpby", alpha=-1.0, x=1.0, beta=1.0, y=2.0, expect=1.0)),
    (259, "call psb_geaxpby(onehalf,x,one,y,desc_a,info)",
     dict(op="axpby", alpha=0.5, x=2.0, beta=1.0, y=-2.0, expect=-1.0)),
    (269, "call psb_geaxpby(one,x,one,y,z,desc_a,info)",
     dict(op="axpbyz", alpha=1.0, x=-2.0, beta=1.0, y=1.0, expect=-1.0)),
    (279, "call psb_geaxpby(one,x,negativeone,y,z,desc_a,info)",
     dict(op="axpbyz", alpha=1.0, x=2.0, beta=-1.0, y=1.0, expect=1.0)),
    (289, "call psb_geaxpby(negativeone,x,one,y,z,desc_a,info)",
     dict(op="axpbyz", alpha=-1.0, x=2.0, beta=1.0, y=1.0, expect=-1.0)),
    (299, "call psb_gemlt(one,x,y,dzero,z,desc_a,info)",
     dict(op="mlt", alpha=1.0, x=2.0, y=-0.5, beta=0.0, expect=-1.0)),
    (353, "ans = psb_gedot(x,y,desc_a,info)",
     dict(op="dot", x=2.0, y=0.5, expect_per_entry=1.0)),
    (360, "ans = psb_geamax(x,desc_a,info)",
     dict(op="amax", x=-0.5, expect=0.5)),
]


def check_vecop(path):
    lines = open(path).read().split("\n")
    out = []
    for ln, text, case in VECOP:
        # allow a few lines of drift between psblas3 revisions
        window = [l.strip() for l in lines[max(0, ln - 4): ln + 3]]  # lines ln-3 .. ln+3
        if text not in window:
            raise ValueError(f"vecoperation.f90: '{text}' not found near line {ln}")
        hit = ln - 3 + window.index(text)
        out.append(dict(case, line=hit, source=text))
    return out


def main(ref):
    here = os.path.dirname(os.path.abspath(__file__))
    usmv = parse_usmv(os.path.join(ref, "test/torture/psb_d_mvsv_tester.f90"))
    vec = check_vecop(os.path.join(ref, "test/kernel/vecoperation.f90"))
    with open(os.path.join(here, "usmv_kats.json"), "w") as f:
        json.dump(dict(source="test/torture/psb_d_mvsv_tester.f90", cases=usmv), f, indent=1)
    with open(os.path.join(here, "vecop_kats.json"), "w") as f:
        json.dump(dict(source="test/kernel/vecoperation.f90", cases=vec), f, indent=1)
    print(f"usmv cases: {len(usmv)}  vecop cases: {len(vec)}")


if __name__ == "__main__":
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PSBLAS_SRC", "/root/reference")
    if not os.path.isfile(os.path.join(src, "test/torture/psb_d_mvsv_tester.f90")):
        sys.exit(f"make_kats: psblas3 sources not found at {src} (pass the directory or set PSBLAS_SRC)")
    main(src)
