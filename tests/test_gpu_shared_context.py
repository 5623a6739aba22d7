"""One context shared by host threads, as the reference's cluster worker pool
(src/SparseMat.cpp:985-1010) shares its GPU path: builds, batch solves and
counts from several threads at once give the results of running them one
after another (calls on a context serialise; the cached CUDA graphs, the
autotuner and the workspaces are per context).  Integer work: bit-exact."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_threads_sharing_one_context():
    from indexgen_b200 import Context, build_conflict_graph, count_conflicts, solve_batch, workloads as W

    cases = [(W.uniform_words(n, L, 900 + i), L, d)
             for i, (n, L, d) in enumerate([(3000, 12, 4), (5000, 10, 5), (800, 16, 9), (6000, 14, 3),
                                            (2500, 11, 6), (4000, 13, 4)])]
    batch = [(W.uniform_words(n, 12, 50 + n), 12, 4) for n in (1500, 700, 2200, 40)]
    ref_ctx = Context(0)
    try:
        want_pairs = []
        for w, L, d in cases:
            with build_conflict_graph(w, L, d, ref_ctx) as G:
                want_pairs.append(G.pairs())
        want_counts = [count_conflicts(w, L, d, ref_ctx) for w, L, d in cases]
        want_books, want_edges = solve_batch(batch, ctx=ref_ctx)
    finally:
        ref_ctx.close()

    ctx = Context(0)
    errors = []
    got = {}

    def worker(t):
        try:
            for rep in range(3):
                k = (t + rep) % len(cases)
                w, L, d = cases[k]
                with build_conflict_graph(w, L, d, ctx) as G:
                    if not np.array_equal(G.pairs(), want_pairs[k]):
                        errors.append(("pairs", t, k))
                if count_conflicts(w, L, d, ctx) != want_counts[k]:
                    errors.append(("count", t, k))
            books, edges = solve_batch(batch, ctx=ctx)
            got[t] = (books, edges)
        except Exception as e:  # surfaced below
            errors.append(("raised", t, repr(e)))

    try:
        threads = [threading.Thread(target=worker, args=(t,)) for t in range(4)]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        assert not errors, errors
        for books, edges in got.values():
            assert np.array_equal(edges, want_edges)
            assert all(np.array_equal(a, b) for a, b in zip(books, want_books))
    finally:
        ctx.close()
