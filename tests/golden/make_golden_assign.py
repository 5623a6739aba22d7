"""Golden vectors for the nearest-centre assignment (tests/golden/assign.npz).

Runs the reference's own solve_assignments_cuda (src/gpu_cluster.py) on
seeded inputs under Numba's CUDA simulator (NUMBA_ENABLE_CUDASIM=1; no GPU
needed) and stores the packed words, centres and the reference assignments.

    python tests/golden/make_golden_assign.py <reference checkout>

Cases cover L = 4..16, centre counts 1..40, duplicated centres (ties must go
to the lowest index, as np.argmin does) and words equal to a centre.
"""
import os
import sys

import numpy as np

os.environ["NUMBA_ENABLE_CUDASIM"] = "1"
HERE = os.path.dirname(os.path.abspath(__file__))


def pack(strings):
    d = np.array([[int(ch) for ch in s] for s in strings], dtype=np.uint64)
    return (d << (2 * np.arange(d.shape[1], dtype=np.uint64))[None, :]).sum(axis=1).astype(np.uint32)


def main(ref_root):
    sys.path.insert(0, os.path.join(ref_root, "src"))
    import warnings

    warnings.simplefilter("ignore")
    import gpu_cluster as G

    cases = [(4, 200, 5), (7, 150, 1), (8, 300, 12), (10, 400, 16), (11, 250, 40), (12, 400, 20), (13, 200, 6),
             (14, 300, 9), (15, 300, 7), (16, 400, 24)]
    out = {}
    for ci, (L, n, k) in enumerate(cases):
        rng = np.random.default_rng(700 + ci)
        vec = ["".join(map(str, rng.integers(0, 4, L))) for _ in range(n)]
        cen = [vec[int(i)] for i in rng.choice(n, k, replace=False)]  # centres are candidates (words at distance 0)
        if k >= 4:
            cen[k - 1] = cen[1]  # a duplicated centre: its words must go to index 1
            cen[k - 2] = cen[0]
        a = np.asarray(G.solve_assignments_cuda(vec, cen, batch_size=128), dtype=np.int32)
        key = f"L{L}_n{n}_k{k}"
        out[key + "_words"] = pack(vec)
        out[key + "_centers"] = pack(cen)
        out[key + "_assign"] = a
        print(key, np.bincount(a, minlength=k)[:8], flush=True)
    np.savez_compressed(os.path.join(HERE, "assign.npz"), **out)


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: make_golden_assign.py <reference checkout>")
    main(sys.argv[1])
