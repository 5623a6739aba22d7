"""Writes a copy of the reference's src/SparseMat.cpp in which the definition
of FillAdjListGPU (src/SparseMat.cpp:454-534) is replaced by an #include of
indexgen_b200/host/FillAdjListGPU.cpp -- the library binding a maintainer
would paste there.  Test infrastructure for oracle/Makefile, target `host`:
the copy goes to a build directory under oracle/_ref/ (never committed) and
nothing else in the file changes.

    python oracle/splice_fill_gpu.py <reference src/SparseMat.cpp> <output .cpp>
"""
from __future__ import annotations

import sys

SIGNATURE = "void FillAdjListGPU("


def body_end(text: str, start: int) -> int:
    """Index just past the closing brace of the function whose signature
    starts at `start` (string/char literals and comments are skipped)."""
    i = text.index("{", start)
    depth = 0
    n = len(text)
    while i < n:
        c = text[i]
        if c == '"' or c == "'":
            q = c
            i += 1
            while text[i] != q:
                i += 2 if text[i] == "\\" else 1
        elif text.startswith("//", i):
            i = text.index("\n", i)
        elif text.startswith("/*", i):
            i = text.index("*/", i) + 1
        elif c == "{":
            depth += 1
        elif c == "}":
            depth -= 1
            if depth == 0:
                return i + 1
        i += 1
    raise ValueError("unbalanced braces after FillAdjListGPU")


def main() -> int:
    src, dst = sys.argv[1], sys.argv[2]
    text = open(src).read()
    if text.count(SIGNATURE) != 1:
        sys.exit(f"expected exactly one definition starting with {SIGNATURE!r} in {src}")
    start = text.index(SIGNATURE)
    end = body_end(text, start)
    line = text.count("\n", 0, start) + 1
    out = (text[:start] + f"// FillAdjListGPU (reference lines {line}-{text.count(chr(10), 0, end) + 1}) replaced by the "
           "libindexgen_cuda binding\n#include \"FillAdjListGPU.cpp\"\n" + text[end:])
    with open(dst, "w") as f:
        f.write(out)
    return 0


if __name__ == "__main__":
    sys.exit(main())
