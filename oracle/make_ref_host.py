#!/usr/bin/env python3
"""Build recipe (test infrastructure): the reference's FM and LOD kernel bodies for the host.

Reads include/FMkernel.cuh and include/LODkernel.cuh of the reference in place, rewrites each
kernel launch `name<<<grid, block>>>(args);` into `gref_host_launch(grid, block, [&] { name(args); });`
(oracle/host_shim/gref_host_launch.h runs it as an OpenMP loop), splices both into
oracle/ref_host_harness.cpp at its marker, and pipes the result to g++ -fopenmp.  Only the
launch syntax changes; the rewritten text exists only in the compiler's input pipe and is not
written anywhere.  Output: one shared library (e.g. oracle/_ref/libgellref_host_c2.so).

  python oracle/make_ref_host.py --ref-root <reference> --out <lib.so> [-DGREF_N=400 ...]
"""
from __future__ import annotations

import argparse
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
MARKER = "// @REFERENCE_HEADERS_WITH_HOST_LAUNCHES@"
HEADERS = ("FMkernel.cuh", "LODkernel.cuh")


def _match(text: str, i: int, open_c: str, close_c: str) -> int:
    """Index just past the bracket that closes text[i] (== open_c)."""
    depth = 0
    for j in range(i, len(text)):
        if text[j] == open_c:
            depth += 1
        elif text[j] == close_c:
            depth -= 1
            if depth == 0:
                return j + 1
    raise ValueError("unbalanced brackets")


def _split_top(s: str) -> list[str]:
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch in "([{":
            depth += 1
        elif ch in ")]}":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur)
            cur = ""
        else:
            cur += ch
    out.append(cur)
    return [x.strip() for x in out]


LAUNCH = re.compile(r"([A-Za-z_]\w*)\s*<<\s*<")
CLOSE = re.compile(r">>\s*>")


def rewrite_launches(text: str) -> tuple[str, int]:
    """Rewrite every `name<<<cfg>>>(args);` (any spacing, e.g. `name << <g, b >> > (a);`)."""
    out, pos, count = [], 0, 0
    while True:
        m = LAUNCH.search(text, pos)
        if not m:
            out.append(text[pos:])
            return "".join(out), count
        c = CLOSE.search(text, m.end())
        cfg = _split_top(text[m.end():c.start()])
        if len(cfg) != 2:
            raise ValueError(f"launch with {len(cfg)} configuration arguments: {text[m.start():c.end()]}")
        j = c.end()
        while text[j].isspace():
            j += 1
        if text[j] != "(":
            raise ValueError("launch without an argument list")
        k = _match(text, j, "(", ")")
        args = text[j + 1:k - 1]
        while text[k].isspace():
            k += 1
        if text[k] != ";":
            raise ValueError("launch not ended by ';'")
        out.append(text[pos:m.start()])
        out.append(f"gref_host_launch({cfg[0]}, {cfg[1]}, [&] {{ {m.group(1)}({args}); }});")
        pos = k + 1
        count += 1


def translation_unit(ref_root: str) -> tuple[str, int]:
    harness = open(os.path.join(HERE, "ref_host_harness.cpp")).read()
    if MARKER not in harness:
        raise SystemExit("marker missing in ref_host_harness.cpp")
    parts, total = [], 0
    for h in HEADERS:
        path = os.path.join(ref_root, "include", h)
        text = open(path, encoding="utf-8", errors="replace").read()
        text = re.sub(r"^\s*#pragma\s+once\s*$", "", text, flags=re.M)
        text, n = rewrite_launches(text)
        total += n
        parts.append(f'#line 1 "{path} (launches rewritten for the host)"\n{text}\n')
    head, tail = harness.split(MARKER, 1)
    line = head.count("\n") + 1
    tu = (f'#line 1 "{os.path.join(HERE, "ref_host_harness.cpp")}"\n' + head + "".join(parts)
          + f'#line {line + 1} "{os.path.join(HERE, "ref_host_harness.cpp")}"\n' + tail)
    return tu, total


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", required=True)
    ap.add_argument("--out", required=True)
    ap.add_argument("--cxx", default="g++")
    ap.add_argument("defines", nargs="*", help="-D flags of the parameter set")
    a = ap.parse_args()
    tu, n = translation_unit(a.ref_root)
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    cmd = [a.cxx, "-std=c++17", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", "-w",
           "-I", os.path.join(HERE, "host_shim"), "-I", os.path.join(a.ref_root, "include"), *a.defines,
           "-x", "c++", "-", "-o", a.out]
    r = subprocess.run(cmd, input=tu, text=True)
    if r.returncode != 0:
        sys.exit(r.returncode)
    print(f"{a.out}: {n} launches rewritten")


if __name__ == "__main__":
    main()
