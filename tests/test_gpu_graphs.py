"""Builds as captured CUDA graphs (one graph launch per build: pair pass and
compaction): the same graphs as direct launches, with the executable graph
updated in place across batches of one shape.
Integer work: bit-exact comparisons."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _jobs(seed, sizes, L=12, d=4):
    from indexgen_b200 import workloads as W

    return [(W.uniform_words(n, L, seed + k), L, d) for k, n in enumerate(sizes)]


def test_graphs_equal_direct_launches(oracle):
    from indexgen_b200 import Context, build_batch, build_conflict_graph

    g_ctx, d_ctx = Context(0), Context(0)
    try:
        d_ctx.set_graphs(False)
        for seed, sizes in ((1, [3000, 500, 1200]), (2, [2500, 2500, 40]), (3, [7000])):
            jobs = _jobs(seed, sizes)
            with build_batch(jobs, g_ctx) as A, build_batch(jobs, d_ctx) as B:
                ra, ca = A.upper_csr()
                rb, cb = B.upper_csr()
                assert np.array_equal(ra, rb) and np.array_equal(ca, cb)
                for j in range(len(jobs)):
                    assert A.job_stats(j) == B.job_stats(j)
        w = jobs[0][0]
        rp, cols = oracle.conflict_upper(w, 12, 4)
        with build_conflict_graph(w, 12, 4, g_ctx) as G:
            r, c = G.upper_csr()
        assert np.array_equal(r, rp) and np.array_equal(c, cols)
        launches, inst, upd = g_ctx.graph_stats()
        assert launches >= 4 and upd > 0 and inst < launches
        assert d_ctx.graph_stats() == (0, 0, 0)
    finally:
        g_ctx.close()
        d_ctx.close()


def test_graph_updates_in_place_for_same_shape():
    """Batches of the same lane forms but other sizes reuse the executable
    graph: one instantiation, then in-place updates."""
    from indexgen_b200 import Context, build_batch

    ctx = Context(0)
    try:
        ctx.set_autotune(False)
        for seed in range(5):
            with build_batch(_jobs(10 + seed, [1000 + 300 * seed, 700], L=10), ctx) as G:
                assert G.edges > 0
        launches, inst, upd = ctx.graph_stats()
        assert launches == 5 and inst == 1 and upd == 4
    finally:
        ctx.close()


def test_identical_builds_relaunch_the_cached_graph():
    from indexgen_b200 import Context, build_batch

    ctx = Context(0)
    try:
        ctx.set_autotune(False)
        jobs = _jobs(40, [1500, 900], L=10)
        edges = set()
        for _ in range(4):
            with build_batch(jobs, ctx) as G:
                edges.add(G.edges)
        launches, inst, upd = ctx.graph_stats()
        assert len(edges) == 1 and launches == 4 and inst == 1
        assert launches - inst - upd >= 0
    finally:
        ctx.close()


def test_graphs_with_mixed_lane_forms_and_growth(oracle):
    """A batch with both pair kernels and a record-buffer growth (rerun of the
    pair pass) through graphs equals the oracle."""
    from indexgen_b200 import Context, build_batch, workloads as W

    jobs = [(W.uniform_words(20000, 10, 77), 10, 5), (W.uniform_words(900, 12, 5), 12, 3)]
    ctx = Context(0)
    try:
        with build_batch(jobs, ctx) as G:
            rp, cols = G.upper_csr()
            for j, (w, L, d) in enumerate(jobs):
                first, n, e = G.job_stats(j)
                orp, ocols = oracle.conflict_upper(w, L, d)
                assert e == orp[-1]
                assert np.array_equal(rp[first:first + n + 1] - rp[first], orp)
                assert np.array_equal(cols[rp[first]:rp[first + n]] - first, ocols)
    finally:
        ctx.close()
