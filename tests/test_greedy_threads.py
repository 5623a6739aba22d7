"""The two-threaded host greedy (one thread walks the balls and keeps the
degrees, a helper thread keeps the degree buckets) against the single-threaded
one and the oracle's restatement of the reference's AdjList greedy: the same
codebook sequence on every graph, including rows longer than the walker's
chunk, more bucket moves than the ring holds, cliques, stars, isolated
vertices, both neighbour-list orders, and several greedies running at once
with fewer helper threads than greedies.  Host-only (no device work).
Integer work: bit-exact."""
import threading

import numpy as np
import pytest

from conftest import load_golden


@pytest.fixture(scope="module")
def G():
    from indexgen_b200 import build as B

    B.build()
    import indexgen_b200 as G

    yield G
    G.set_greedy_threads(-1, -1)


def upper_csr(n, pairs):
    """Upper CSR of the undirected edge set `pairs` (any orientation, repeats dropped)."""
    p = np.asarray(pairs, dtype=np.int64).reshape(-1, 2)
    p = p[p[:, 0] != p[:, 1]]
    p = np.sort(p, axis=1)
    p = np.unique(p, axis=0)
    row_ptr = np.zeros(n + 1, np.int64)
    np.add.at(row_ptr, p[:, 0] + 1, 1)
    return np.cumsum(row_ptr), p[:, 1].astype(np.int32)


def graphs():
    rng = np.random.default_rng(11)
    out = {}
    n = 5000
    out["sparse"] = (n, upper_csr(n, rng.integers(0, n, (60000, 2))))
    n = 40000  # ~4e5 bucket moves: the ring (65536 entries) wraps several times
    out["wrap"] = (n, upper_csr(n, rng.integers(0, n, (400000, 2))))
    n = 12001  # a hub of degree 12000: rows longer than one walker chunk (4096)
    star = np.stack([np.zeros(n - 1, np.int64), np.arange(1, n)], axis=1)
    out["star"] = (n, upper_csr(n, np.concatenate([star, rng.integers(1, n, (30000, 2))])))
    n = 300  # every degree equal
    iu = np.triu_indices(n, 1)
    out["clique"] = (n, upper_csr(n, np.stack(iu, axis=1)))
    n = 3000  # isolated vertices, pairs and a dense core
    core = rng.integers(0, 400, (20000, 2))
    pairs = np.stack([np.arange(1000, 2000, 2), np.arange(1001, 2001, 2)], axis=1)
    out["mixed"] = (n, upper_csr(n, np.concatenate([core, pairs])))
    return out


def both(G, fn):
    G.set_greedy_threads(0, -1)
    seq = fn()
    G.set_greedy_threads(1, 0)
    before = G.greedy_stats()[0]
    par = fn()
    assert G.greedy_stats()[0] > before, "the two-threaded greedy did not run"
    G.set_greedy_threads(-1, -1)
    return seq, par


@pytest.mark.parametrize("name", ["sparse", "wrap", "star", "clique", "mixed"])
def test_two_threads_equal_one_and_oracle(G, oracle, name):
    n, (rp, cols) = graphs()[name]
    want = oracle.codebook(rp, cols, n, 1)
    seq, par = both(G, lambda: G.codebook_from_upper_csr(rp, cols, n, 1))
    assert np.array_equal(seq, want)
    assert np.array_equal(par, want)
    # the FillAdjList(T) neighbour order changes the codebook; both forms follow it
    want3 = oracle.codebook(rp, cols, n, 3)
    ap, adj = oracle.adjacency(rp, cols, n, 3)
    seq, par = both(G, lambda: G.codebook_from_adjacency(ap, adj, n))
    assert np.array_equal(seq, want3)
    assert np.array_equal(par, want3)


def test_two_threads_reference_fixtures(G):
    g = load_golden("uniform11.npz")
    n = len(g["words"])
    e = g["edges"]
    rp = np.zeros(n + 1, np.int64)
    np.add.at(rp, e[:, 0].astype(np.int64) + 1, 1)
    rp = np.cumsum(rp)
    for T in (1, 8, 16):
        seq, par = both(G, lambda: G.codebook_from_upper_csr(rp, e[:, 1], n, T))
        assert np.array_equal(seq, g[f"sel{T}"])
        assert np.array_equal(par, g[f"sel{T}"])
    s = load_golden("small_cases.npz")
    for key in sorted({k[: -len("_adj3_ptr")] for k in s.files if k.endswith("_adj3_ptr")}):
        m = len(s[key + "_adj3_ptr"]) - 1
        seq, par = both(G, lambda: G.codebook_from_adjacency(s[key + "_adj3_ptr"], s[key + "_adj3"], m))
        assert np.array_equal(seq, par), key
        assert np.array_equal(par, s[key + "_sel3"]), key


def test_concurrent_greedies(G, oracle):
    """Several greedies at once with one helper thread allowed: a greedy runs
    two-threaded only when it is the only one running, so at most one of
    them does (none if they all overlap); every result is the oracle's."""
    import os

    n, (rp, cols) = graphs()["wrap"]
    want = oracle.codebook(rp, cols, n, 1)
    G.set_greedy_threads(1, 0)
    p0, s0 = G.greedy_stats()
    k = max(2, min(6, (os.cpu_count() or 2) - 2))
    results = [None] * k

    def run(k):
        results[k] = G.codebook_from_upper_csr(rp, cols, n, 1)

    ts = [threading.Thread(target=run, args=(q,)) for q in range(k)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    p1, s1 = G.greedy_stats()
    G.set_greedy_threads(-1, -1)
    assert (p1 - p0) + (s1 - s0) == k
    assert p1 - p0 <= k
    for r in results:
        assert np.array_equal(r, want)


def test_small_graphs_stay_single_threaded(G):
    G.set_greedy_threads(-1, -1)
    p0, s0 = G.greedy_stats()
    rp = np.array([0, 1, 2, 2], np.int64)
    cols = np.array([1, 2], np.int32)
    assert G.codebook_from_upper_csr(rp, cols, 3, 1).tolist() == [2, 0]
    p1, s1 = G.greedy_stats()
    assert (p1, s1) == (p0, s0 + 1)


@pytest.mark.gpu
def test_two_threads_on_the_linear12_job(igctx):
    """words -> codebook for the [12,9,3] GF(4) code + coset job (207,432
    words, editDist 4) through ig_solve, with the greedy on two threads (the
    default at this size) and on one: both equal the reference's codebook."""
    import hashlib
    import json
    import os

    from conftest import GOLDEN
    from indexgen_b200 import greedy_stats, set_greedy_threads, solve
    from indexgen_b200 import workloads as W

    gold = json.load(open(os.path.join(GOLDEN, "linear.json")))["linear12"]
    words = W.linear12_candidates()
    try:
        set_greedy_threads(1, -1)
        p0 = greedy_stats()[0]
        two, edges = solve(words, 12, 4, 1, igctx)
        assert greedy_stats()[0] == p0 + 1
        set_greedy_threads(0, -1)
        one, _ = solve(words, 12, 4, 1, igctx)
    finally:
        set_greedy_threads(-1, -1)
    assert edges == gold["edges"]
    assert np.array_equal(two, one)
    assert hashlib.sha256(two.astype("<i4").tobytes()).hexdigest() == gold["codebook_t1_sha256"]
    # the batch path's greedies run in the library's pool: one thread each
    from indexgen_b200 import solve_batch

    p0, s0 = greedy_stats()
    books, _ = solve_batch([(words, 12, 4)], 1, 0, igctx)
    p1, s1 = greedy_stats()
    assert (p1, s1) == (p0, s0 + 1)
    assert np.array_equal(books[0], two)


@pytest.mark.gpu
def test_two_threads_on_batch_jobs_with_offsets(igctx):
    """A batch graph's per-job codebooks computed on the caller's thread
    alone (host_threads=1): each job's greedy is a lone greedy over rows whose
    neighbour ids carry the job's word offset, in plain and in bit-packed
    host lists.  With the two-thread form forced for every size, each equals
    the job's own single-threaded solve."""
    from indexgen_b200 import LISTS_AUTO, LISTS_PACKED, build_batch, greedy_stats, set_greedy_threads, solve
    from indexgen_b200 import workloads as W

    jobs = [(W.uniform_words(6000, 10, 41), 10, 4), (W.uniform_words(20000, 10, 42), 10, 5),
            (W.uniform_words(9000, 12, 43), 12, 4)]
    try:
        set_greedy_threads(0, -1)
        want = [solve(w, L, d, 1, igctx)[0] for w, L, d in jobs]
        for lists in (LISTS_AUTO, LISTS_PACKED):
            igctx.set_host_lists(lists)
            set_greedy_threads(1, 0)
            p0 = greedy_stats()[0]
            with build_batch(jobs, igctx) as G:
                books = G.job_codebooks(order_threads=1, host_threads=1)
            assert greedy_stats()[0] == p0 + len(jobs)
            for got, ref in zip(books, want):
                assert np.array_equal(got, ref)
    finally:
        igctx.set_host_lists(LISTS_AUTO)
        set_greedy_threads(-1, -1)


@pytest.mark.gpu
def test_large_pooled_greedy_takes_a_free_helper(igctx):
    """In the library's greedy pool only graphs with at least 64 times the
    lone threshold of entries run two-threaded (the densest jobs of a
    stream); with the threshold lowered, a batch's dense job does, a small
    one does not, and both codebooks equal their single-threaded solves."""
    from indexgen_b200 import greedy_stats, set_greedy_threads, solve, solve_batch
    from indexgen_b200 import workloads as W

    dense = (W.uniform_words(20000, 10, 42), 10, 5)   # about 9e6 edges
    small = (W.uniform_words(3000, 12, 44), 12, 3)    # a few hundred edges
    try:
        set_greedy_threads(0, -1)
        want = [solve(w, L, d, 1, igctx)[0] for w, L, d in (dense, small)]
        set_greedy_threads(1, 1 << 14)  # pooled threshold 2^20 entries
        p0, s0 = greedy_stats()
        books, _ = solve_batch([dense, small], 1, 0, igctx)
        p1, s1 = greedy_stats()
    finally:
        set_greedy_threads(-1, -1)
    assert (p1 - p0, s1 - s0) == (1, 1)
    for got, ref in zip(books, want):
        assert np.array_equal(got, ref)
