"""Parity of the CUDA path (through the C ABI) with the oracle and with the
reference's own outputs.  Integer work: every comparison is bit-exact."""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_golden

pytestmark = pytest.mark.gpu


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def gpu_pairs(igctx, w, L, d):
    from indexgen_b200 import build_conflict_graph

    with build_conflict_graph(w, L, d, igctx) as g:
        return g.pairs(), g


def oracle_pairs(oracle, w, L, d):
    rp, cols = oracle.conflict_upper(w, L, d)
    return oracle.pairs_from_csr(rp, cols)


def test_uniform11_edges_and_codebooks(igctx):
    from indexgen_b200 import build_conflict_graph

    g = load_golden("uniform11.npz")
    with build_conflict_graph(g["words"], 11, 3, igctx) as G:
        assert G.edges == 20871
        assert G.matrix_ones_num == 41742
        assert np.array_equal(G.pairs(), g["edges"])
        for T in (16, 8, 1):
            assert np.array_equal(G.codebook(T), g[f"sel{T}"]), T


def test_small_cases(igctx):
    from indexgen_b200 import build_conflict_graph

    g = load_golden("small_cases.npz")
    keys = sorted({k.rsplit("_", 1)[0] for k in g.files if k.endswith("_words")})
    for key in keys:
        L, d = (int(x[1:]) for x in key.split("_"))
        with build_conflict_graph(g[key + "_words"], L, d, igctx) as G:
            assert np.array_equal(G.pairs(), g[key + "_edges"]), key
            assert np.array_equal(G.codebook(1), g[key + "_sel1"]), key
            assert np.array_equal(G.codebook(3), g[key + "_sel3"]), key


def test_predicate_vectors(igctx):
    """Each golden (a, b, minED) query becomes the pair (i, k+i) of one graph
    per (L, minED) group; the edge must exist iff the reference said ED < minED."""
    from indexgen_b200 import build_conflict_graph

    g = load_golden("predicate.npz")
    a, b, Ls, ds, at_least = g["a"], g["b"], g["L"], g["min_ed"], g["at_least"]
    for L in np.unique(Ls):
        for d in np.unique(ds):
            sel = np.nonzero((Ls == L) & (ds == d))[0]
            if len(sel) == 0:
                continue
            k = len(sel)
            w = np.concatenate([a[sel], b[sel]]).astype(np.uint32)
            with build_conflict_graph(w, int(L), int(d), igctx) as G:
                pairs = G.pairs()
            have = set(map(tuple, pairs.tolist()))
            for j, q in enumerate(sel):
                lo, hi = min(j, k + j), max(j, k + j)
                is_edge = (lo, hi) in have
                assert is_edge == (not at_least[q]), (int(L), int(d), int(q))


@pytest.mark.parametrize("L", list(range(1, 17)))
def test_random_sets_all_lengths(igctx, oracle, L):
    rng = np.random.default_rng(100 + L)
    from indexgen_b200 import workloads as W

    for n, d in ((1000, 1 + L // 3), (777, max(1, L // 2)), (513, 3)):
        w = W.uniform_words(n, L, int(rng.integers(1 << 30)))
        if L >= 4:  # plant near neighbours
            w[: n // 4] = w[n // 4 : n // 2] ^ (np.uint32(1) << np.uint32(2 * int(rng.integers(0, L))))
        got, _ = gpu_pairs(igctx, w, L, d)
        assert np.array_equal(got, oracle_pairs(oracle, w, L, d)), (L, n, d)


@pytest.mark.parametrize("n", [0, 1, 2, 3, 255, 256, 257, 511, 512, 513, 2049, 4095])
def test_sizes_around_tiles(igctx, oracle, n):
    from indexgen_b200 import workloads as W

    w = W.uniform_words(n, 10, 7 + n)
    if n >= 8:
        w[1::7] = w[0::7][: len(w[1::7])]  # duplicates (distance 0)
    got, G = gpu_pairs(igctx, w, 10, 4)
    assert np.array_equal(got, oracle_pairs(oracle, w, 10, 4))


def test_threshold_extremes(igctx):
    from indexgen_b200 import build_conflict_graph, workloads as W

    w = W.uniform_words(300, 12, 9)
    for d, expect in ((0, 0), (-3, 0), (13, 300 * 299 // 2), (40, 300 * 299 // 2)):
        with build_conflict_graph(w, 12, d, igctx) as G:
            assert G.edges == expect, d
            if expect:
                rp, cols = G.upper_csr()
                assert np.array_equal(np.diff(rp), 299 - np.arange(300))


def test_all_duplicates(igctx):
    from indexgen_b200 import build_conflict_graph

    w = np.full(700, 0x155555, np.uint32)
    with build_conflict_graph(w, 11, 1, igctx) as G:
        assert G.edges == 700 * 699 // 2
        assert G.codebook(1).tolist() == [699]


def test_bad_input_is_rejected(igctx):
    from indexgen_b200 import IndexGenError, build_conflict_graph

    with pytest.raises(IndexGenError) as e:
        build_conflict_graph(np.zeros(4, np.uint32), 17, 3, igctx)
    assert e.value.code == "IG_ERR_INPUT"
    with pytest.raises(IndexGenError):
        build_conflict_graph(np.zeros(4, np.uint32), 0, 3, igctx)


def test_device_input_equals_host_input(igctx):
    import torch

    from indexgen_b200 import build_conflict_graph, workloads as W

    w = W.uniform_filtered(30000, 12, 77)
    t = torch.from_numpy(w.view(np.int32)).cuda()
    torch.cuda.synchronize()
    with build_conflict_graph(w, 12, 4, igctx) as A, build_conflict_graph(t, 12, 4, igctx) as B:
        ra, ca = A.upper_csr()
        rb, cb = B.upper_csr()
        assert np.array_equal(ra, rb) and np.array_equal(ca, cb)


def test_shipped_codebooks_verify(igctx):
    from indexgen_b200 import count_conflicts, verify_dist, workloads as W

    g = load_golden("shipped.npz")
    for k in g.files:
        if k.endswith("_meta"):
            L, d = (int(x) for x in g[k])
            w = g[k.replace("_meta", "_words")]
            assert count_conflicts(w, L, d, igctx) == 0, k
            assert verify_dist(W.to_strings(w, L), d, igctx)
            assert count_conflicts(w, L, d + 3, igctx) > 0


def test_reference_named_mirrors(igctx, oracle):
    from indexgen_b200 import (fill_adj_list_gpu, solve_edit_distance_cuda, solve_independent_set,
                               workloads as W)

    g = load_golden("small_cases.npz")
    w = g["L12_d4_words"]
    strings = W.to_strings(w, 12)
    adj = solve_edit_distance_cuda(strings, 4, ctx=igctx)
    rp, cols = oracle.conflict_upper(w, 12, 4)
    ap, a = oracle.adjacency(rp, cols, len(w), 1)
    for i in range(len(w)):
        assert adj[i] == a[ap[i]:ap[i + 1]].tolist()
    cb = solve_independent_set(strings, 4, thread_num=3, ctx=igctx)
    assert cb == [strings[i] for i in g["L12_d4_sel3"]]
    G, ones = fill_adj_list_gpu(strings, 4, ctx=igctx)
    assert ones == 2 * len(g["L12_d4_edges"])
    G.close()


def test_linear12_full_size_against_reference(igctx):
    """Single large job: 207,432 words, ED<4.  Edge list and T=1 codebook
    hashed against the reference's own FillAdjList + FromBinaryFile + greedy."""
    from indexgen_b200 import build_conflict_graph, workloads as W

    info = json.load(open(os.path.join(GOLDEN, "linear.json")))["linear12"]
    w = W.linear12_candidates()
    with build_conflict_graph(w, 12, 4, igctx) as G:
        assert G.edges == info["edges"]
        pairs = G.pairs()
        assert sha(pairs.astype("<i4")) == info["edges_sha256"]
        sel = G.codebook(1)
        assert len(sel) == info["codebook_t1"]
        assert sel[:64].tolist() == info["codebook_t1_head"]
        assert sha(sel.astype("<i4")) == info["codebook_t1_sha256"]


def test_repeated_builds_are_identical(igctx):
    from indexgen_b200 import build_conflict_graph, workloads as W

    w = W.uniform_filtered(60000, 11, 5)
    ref = None
    for _ in range(3):
        with build_conflict_graph(w, 11, 3, igctx) as G:
            r = G.upper_csr()
        if ref is None:
            ref = r
        else:
            assert np.array_equal(ref[0], r[0]) and np.array_equal(ref[1], r[1])


def test_adjacency_matches_oracle_order(igctx, oracle):
    """Device-built symmetric lists equal the reference loader's order (T=1)."""
    from indexgen_b200 import build_conflict_graph

    g = load_golden("small_cases.npz")
    cases = [(g[k + "_words"], int(k.split("_")[0][1:]), int(k.split("_")[1][1:])) for k in
             sorted({k.rsplit("_", 1)[0] for k in g.files if k.endswith("_words")})]
    u = load_golden("uniform11.npz")
    cases.append((u["words"], 11, 3))
    for w, L, d in cases:
        rp, cols = oracle.conflict_upper(w, L, d)
        ap_o, adj_o = oracle.adjacency(rp, cols, len(w), 1)
        with build_conflict_graph(w, L, d, igctx) as G:
            ap, adj = G.adjacency()
        assert np.array_equal(ap, ap_o) and np.array_equal(adj, adj_o), (L, d)


def test_adjacency_long_rows(igctx):
    """Rows with more than 1024 lower neighbours take the bitmap path; the last
    row's neighbours span two 512 Ki-value bitmap windows."""
    from indexgen_b200 import build_conflict_graph, workloads as W

    n = 530_000
    w = W.uniform_words(n, 16, 1234)
    clique = np.r_[np.arange(1100), n - 1]
    w[clique] = w[0]
    with build_conflict_graph(w, 16, 1, igctx) as G:
        ap, adj = G.adjacency()
        rp, cols = G.upper_csr()
    _, counts = np.unique(w, return_counts=True)
    assert G.edges == int((counts * (counts - 1) // 2).sum())  # editDist 1: exact duplicates
    last = adj[ap[n - 1]:ap[n]]
    assert last.tolist() == np.nonzero(w[: n - 1] == w[n - 1])[0].tolist()
    assert len(last) >= 1100
    # every row: lower part ascending and < x, upper part equals the CSR row
    deg_up = np.diff(rp)
    deg = np.diff(ap)
    for x in (0, 1, 500, 1099):
        row = adj[ap[x]:ap[x + 1]]
        lo, up = row[: deg[x] - deg_up[x]], row[deg[x] - deg_up[x]:]
        assert np.all(np.diff(lo) > 0) and np.all(lo < x)
        assert np.array_equal(up, cols[rp[x]:rp[x + 1]])
