"""Batched clusters: one device pipeline for many jobs must give every job the
same edges and codebook as solving it alone (SolveIndependentSet per cluster,
src/SparseMat.cpp:784-851 inside the cluster loop :927-1095)."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def test_batch_of_golden_cases(igctx):
    from indexgen_b200 import build_batch

    g = load_golden("small_cases.npz")
    keys = sorted({k.rsplit("_", 1)[0] for k in g.files if k.endswith("_words")})
    jobs = [(g[k + "_words"], int(k.split("_")[0][1:]), int(k.split("_")[1][1:])) for k in keys]
    with build_batch(jobs, igctx) as G:
        assert G.jobs == len(jobs)
        rp, cols = G.upper_csr()
        for T in (1, 3):
            books = G.job_codebooks(order_threads=T, host_threads=4)
            for j, k in enumerate(keys):
                assert np.array_equal(books[j], g[k + f"_sel{T}"]), (k, T)
        for j, k in enumerate(keys):
            first, n, e = G.job_stats(j)
            assert e == len(g[k + "_edges"]), k
            rows = np.repeat(np.arange(n), np.diff(rp[first:first + n + 1]))
            c = cols[rp[first]:rp[first + n]] - first
            assert np.array_equal(np.stack([rows, c], 1), g[k + "_edges"]), k


def test_batch_mixed_jobs_equal_single_solves(igctx):
    from indexgen_b200 import build_conflict_graph, solve_batch, workloads as W

    rng = np.random.default_rng(5)
    jobs = []
    for n in (0, 1, 2, 3, 257, 511, 1000, 4097, 12000):
        L = int(rng.integers(10, 17))
        d = int(rng.integers(3, 6))
        w = W.uniform_words(n, L, int(rng.integers(1 << 30)))
        if n > 20:
            w[: n // 5] = w[n // 5: 2 * (n // 5)] ^ np.uint32(1 << (2 * int(rng.integers(0, L))))
        jobs.append((w, L, d))
    books, edges = solve_batch(jobs, host_threads=3, ctx=igctx)
    for (w, L, d), b, e in zip(jobs, books, edges):
        with build_conflict_graph(w, L, d, igctx) as G:
            assert G.edges == e
            assert np.array_equal(G.codebook(1), b)


def test_batch_clustered_sample(igctx):
    from indexgen_b200 import build_conflict_graph, build_batch, workloads as W

    w = W.uniform_until(30000, 14, 3)
    parts = W.assign_clusters(w, 14, W.zipf_sizes(30000, 12, lo=500, hi=6000), 4)
    jobs = [(w[p], 14, 4) for p in parts]
    with build_batch(jobs, igctx) as G:
        books = G.job_codebooks()
        for j, (cw, L, d) in enumerate(jobs):
            with build_conflict_graph(cw, L, d, igctx) as S:
                assert S.edges == G.job_stats(j)[2]
                assert np.array_equal(S.codebook(1), books[j])
