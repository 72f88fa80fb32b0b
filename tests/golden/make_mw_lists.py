"""Extract the microwave boundary lists of InitialModule::makeBoundary
(include/initialModule.hpp:420-1055) of the reference into a segment table,
tests/golden/mw_lists_cathode.json.

Each segment is one field (x: Ex, r: Er, p: Ephi), one side (W, E, S, N), one
boundary code, and either a loop over i or j with the other coordinate fixed,
or a single (i, j) entry; every bound is kept as an expression over the
cathode's cell blocks gc.i_flc_bl / gc.j_flc_bl, written ic[b][k] / jc[b][k],
so that the table serves any grid resolution.  Segments keep the reference's
order (the order of the boundary surgery) and cite their source line.

Usage: python <this script> <reference checkout>  (or set CATHODE_REFERENCE).
"""
import json
import os
import sys
import re

FIRST, LAST = 420, 1056
HERE = os.path.dirname(os.path.abspath(__file__))


def reference_root() -> str:
    """The reference checkout: the first command-line argument, else $CATHODE_REFERENCE."""
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CATHODE_REFERENCE")
    if not root or not os.path.isdir(root):
        sys.exit(f"usage: python {os.path.basename(__file__)} <reference checkout> (or set CATHODE_REFERENCE)")
    return root

EXPR = r"([^;]+?)"
LOOP = re.compile(r"for\s*\(\s*int\s+([ij])\s*=\s*" + EXPR + r"\s*;\s*\1\s*<=\s*" + EXPR + r"\s*;\s*\1\s*\+\+\s*\)\s*\{"
                  r"\s*int\s+([ij])\s*=\s*" + EXPR + r"\s*;"
                  r"\s*mb\.iBnd(\w\w)\.push_back\(i\)\s*;\s*mb\.jBnd\6\.push_back\(j\)\s*;"
                  r"\s*mb\.sBnd\6\.push_back\((\d)\)\s*;\s*\}", re.S)
POINT = re.compile(r"\{\s*int\s+i\s*=\s*" + EXPR + r"\s*;\s*int\s+j\s*=\s*" + EXPR + r"\s*;"
                   r"\s*mb\.iBnd(\w\w)\.push_back\(i\)\s*;\s*mb\.jBnd\3\.push_back\(j\)\s*;"
                   r"\s*mb\.sBnd\3\.push_back\((\d)\)\s*;\s*\}", re.S)


def expr(e: str) -> str:
    e = e.replace("gc.i_flc_bl", "ic").replace("gc.j_flc_bl", "jc").replace(" ", "")
    if not re.fullmatch(r"[ij]c\[\d\]\[[01]\](?:[+-]\d+)?", e):
        raise ValueError(f"unexpected bound expression: {e}")
    return e


def main():
    SRC = os.path.join(reference_root(), "include", "initialModule.hpp")
    lines = open(SRC, encoding="utf-8").read().splitlines()
    text = "\n".join(lines[FIRST - 1:LAST])
    # drop comments but keep the line structure (for the citations)
    text = re.sub(r"//[^\n]*", "", text)
    # one segment pushes j before i (z5 of the Ex right side): same lists, either order
    text = re.sub(r"mb\.jBnd(\w\w)\.push_back\(j\)\s*;(\s*)mb\.iBnd\1\.push_back\(i\)\s*;",
                  r"mb.iBnd\1.push_back(i);\2mb.jBnd\1.push_back(j);", text)
    segs = []
    for m in LOOP.finditer(text):
        var, lo, hi, fixvar, fix, key, code = m.groups()
        assert fixvar != var
        segs.append(dict(pos=m.start(), line=FIRST + text.count("\n", 0, m.start()), side=key[0], field=key[1],
                         code=int(code), kind="loop", var=var, lo=expr(lo), hi=expr(hi), fix=expr(fix)))
    for m in POINT.finditer(text):
        ie, je, key, code = m.groups()
        segs.append(dict(pos=m.start(), line=FIRST + text.count("\n", 0, m.start()), side=key[0], field=key[1],
                         code=int(code), kind="point", i=expr(ie), j=expr(je)))
    segs.sort(key=lambda s: s["pos"])
    for s in segs:
        del s["pos"]
    n_push = len(re.findall(r"mb\.sBnd\w\w\.push_back", text))
    assert len(segs) == n_push, (len(segs), n_push)
    out = os.path.join(HERE, "mw_lists_cathode.json")
    with open(out, "w") as f:
        json.dump(dict(source="include/initialModule.hpp:420-1055 (InitialModule::makeBoundary)", segments=segs),
                  f, indent=1)
    print(out, len(segs), "segments")


if __name__ == "__main__":
    main()
