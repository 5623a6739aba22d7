"""Drop-in for src/gpu_graph_generator.py (the script FillAdjListGPU runs).

    python -m indexgen_b200.gpu_graph_generator <input_vectors.txt> <output_edges.bin> <threshold> [max_gpu_memory_gb]

Same arguments, same output: little-endian int32 (u, v) pairs with u < v,
grouped by u ascending (src/gpu_graph_generator.py:49-77), which
AdjList::FromBinaryFile loads (src/SparseMat.cpp:338-390).  Exit status 1 on
any failure, as the reference script's try/except does
(src/gpu_graph_generator.py:40-44).  The columns of each u are ascending, so the
loader builds the sorted neighbour order (the canonical order the library's
greedy calls order_threads = 1).
"""
from __future__ import annotations

import sys
import time

import numpy as np


def load_candidates(filename):
    """Lines stripped, empty lines skipped (src/gpu_graph_generator.py:11-15)."""
    with open(filename, "r") as f:
        return [line.strip() for line in f if line.strip()]


def main(argv=None) -> int:
    argv = list(sys.argv if argv is None else argv)
    if len(argv) < 4:
        print("Usage: python -m indexgen_b200.gpu_graph_generator <input_vectors.txt> <output_edges.bin> "
              "<threshold> [max_gpu_memory_gb]")
        return 1
    input_file, output_file = argv[1], argv[2]
    try:
        threshold = int(argv[3])
        max_gpu_gb = float(argv[4]) if len(argv) > 4 else 9.0
    except ValueError as e:
        print(f"[Error] bad argument: {e}")
        return 1
    try:
        from . import build_conflict_graph, pack_sequences

        strings = load_candidates(input_file)
        print(f"[GPU] Loaded {len(strings)} strings. threshold={threshold}, memory limit={max_gpu_gb} GB")
        t0 = time.time()
        if strings:
            words, L, _ = pack_sequences(strings)
            with build_conflict_graph(words, L, threshold) as g:
                pairs = g.pairs()
        else:
            pairs = np.zeros((0, 2), np.int32)
        t1 = time.time()
        with open(output_file, "wb") as f:
            f.write(np.ascontiguousarray(pairs, dtype="<i4").tobytes())
        print(f"[GPU] Done. Wrote {len(pairs)} unique edges (graph {t1 - t0:.4f}s).")
    except Exception as e:  # the reference script reports and exits 1
        print(f"[Error] CUDA computation failed: {e}")
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
