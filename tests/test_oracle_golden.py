"""Pins the CPU oracle to the reference's own outputs (tests/golden/, produced
by tests/golden/make_golden.py from the reference C++ sources)."""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_golden


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_predicate_vectors(oracle):
    g = load_golden("predicate.npz")
    a, b, L, d, at_least = g["a"], g["b"], g["L"], g["min_ed"], g["at_least"]
    for i in range(len(a)):
        ed = oracle.lev(int(a[i]), int(b[i]), int(L[i]))
        assert (ed >= d[i]) == bool(at_least[i]), (i, int(L[i]), int(d[i]), ed)


def test_myers_matches_dp(oracle):
    rng = np.random.default_rng(11)
    for L in range(1, 17):
        for _ in range(300):
            a = int(rng.integers(0, 4 ** L))
            b = int(rng.integers(0, 4 ** L))
            assert oracle.lev(a, b, L) == oracle.lev(a, b, L, "dp")


def small_keys():
    g = load_golden("small_cases.npz")
    return sorted({k.rsplit("_", 1)[0] for k in g.files if k.endswith("_words")})


@pytest.mark.parametrize("key", small_keys())
def test_small_cases(oracle, key):
    g = load_golden("small_cases.npz")
    L, d = (int(x[1:]) for x in key.split("_"))
    w = g[key + "_words"]
    rp, cols = oracle.conflict_upper(w, L, d, threads=2)
    pairs = oracle.pairs_from_csr(rp, cols)
    assert np.array_equal(pairs, g[key + "_edges"])
    ap, adj = oracle.adjacency(rp, cols, len(w), 3)
    assert np.array_equal(ap, g[key + "_adj3_ptr"])
    assert np.array_equal(adj, g[key + "_adj3"])
    assert np.array_equal(oracle.codebook(rp, cols, len(w), 1), g[key + "_sel1"])
    assert np.array_equal(oracle.codebook(rp, cols, len(w), 3), g[key + "_sel3"])


def test_uniform11(oracle):
    g = load_golden("uniform11.npz")
    w = g["words"]
    rp, cols = oracle.conflict_upper(w, 11, 3)
    assert np.array_equal(oracle.pairs_from_csr(rp, cols), g["edges"])
    for T in (16, 8, 1):
        assert np.array_equal(oracle.codebook(rp, cols, len(w), T), g[f"sel{T}"]), T


def test_shipped_codebooks_are_conflict_free(oracle):
    g = load_golden("shipped.npz")
    for k in g.files:
        if not k.endswith("_meta"):
            continue
        L, d = (int(x) for x in g[k])
        w = g[k.replace("_meta", "_words")]
        rp, _ = oracle.conflict_upper(w, L, d)
        assert rp[-1] == 0, k


@pytest.mark.slow
def test_n11_header_pin(oracle):
    """Codebooks/N11/N11-ED3-GC0.3-0.7-RUN0.txt: N=50,688, Number of Ones 129,128."""
    from indexgen_b200 import workloads as W

    info = json.load(open(os.path.join(GOLDEN, "linear.json")))["n11_header"]
    w = W.linear_code_words(11, info["bias"], info["row_perm"], info["col_perm"])
    w = w[W.filter_words(w, 11, info["max_run"], info["min_gc"], info["max_gc"])]
    assert len(w) == info["N"] == 50688
    assert sha(w.astype("<u4")) == info["words_sha256"]
    rp, cols = oracle.conflict_upper(w, 11, 3)
    assert 2 * rp[-1] == 129128
    assert sha(oracle.pairs_from_csr(rp, cols).astype("<i4")) == info["edges_sha256"]


def test_assignment_matches_reference(oracle):
    """The oracle's nearest-centre assignment equals the reference's own
    solve_assignments_cuda (src/gpu_cluster.py, run under Numba's CUDA
    simulator by tests/golden/make_golden_assign.py), ties included."""
    g = load_golden("assign.npz")
    keys = sorted({k.rsplit("_", 1)[0] for k in g.files})
    assert len(keys) == 10
    for key in keys:
        L = int(key.split("_")[0][1:])
        got = oracle.assign_centers(g[key + "_words"], g[key + "_centers"], L)
        assert np.array_equal(got, g[key + "_assign"]), key


def test_row_neighbours_match_all_pairs(oracle):
    from indexgen_b200 import workloads as W

    w = W.uniform_words(2500, 10, 5)
    rp, cols = oracle.conflict_upper(w, 10, 4)
    full = [[] for _ in range(len(w))]
    for i in range(len(w)):
        for c in cols[rp[i]:rp[i + 1]]:
            full[i].append(int(c))
            full[int(c)].append(i)
    rows = np.array([0, 7, 100, 1234, 2499], np.int32)
    got = oracle.row_neighbours(w, 10, 4, rows)
    for k, r in enumerate(rows):
        assert sorted(full[int(r)]) == got[k].tolist(), int(r)


def test_cluster_oracle_single_cluster_is_plain_greedy(oracle):
    from indexgen_b200 import workloads as W

    w = W.uniform_until(1500, 10, 4)
    book, sizes = oracle.cluster_solve(w, 10, 3, 0, converge_iters=1)
    rp, cols = oracle.conflict_upper(w, 10, 3)
    assert np.array_equal(book, oracle.codebook(rp, cols, len(w), 1)) and list(sizes) == [len(book)]
    idx = oracle.pick_centres(100, 10, 7, 1)
    assert len(set(idx.tolist())) == 10 and idx.min() >= 0 and idx.max() < 100


def test_library_centre_picker_matches_oracle(oracle):
    from indexgen_b200 import cluster_centres

    for n, k, seed, it in ((100, 10, 7, 1), (5000, 64, 2**63 + 5, 3), (17, 17, 0, 2)):
        assert np.array_equal(cluster_centres(n, k, seed, it), oracle.pick_centres(n, k, seed, it))
