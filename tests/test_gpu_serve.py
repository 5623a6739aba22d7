"""Serving loop: each job's result is the same alone and in the mix."""
import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_server_results_equal_solo_solves(igctx):
    from indexgen_b200 import Server, solve, workloads as W

    stream = W.serving_stream(24, seed=77, rate=400.0, nmin=300, nmax=20000)
    solo = [solve(w, L, d, 1, igctx) for _, w, L, d in stream]
    with Server(igctx, host_threads=4, max_batch_jobs=8) as sv:
        tickets = []
        t0 = time.perf_counter()
        for arr, w, L, d in stream:  # arrivals while earlier jobs run
            while time.perf_counter() - t0 < arr:
                time.sleep(0.0005)
            tickets.append(sv.submit(w, L, d))
        for tk, (order, edges), (_, w, L, d) in zip(tickets, solo, stream):
            got, e, lat = sv.wait(tk)
            assert e == edges
            assert np.array_equal(got, order), (len(w), L, d)
            assert lat >= 0
        st = sv.stats()
        assert st["completed"] == len(stream)
        assert st["batches"] <= len(stream)


def test_server_concurrent_submitters_and_cancel(igctx):
    from indexgen_b200 import IndexGenError, Server, solve, workloads as W

    jobs = [(W.uniform_until(n, 12, 500 + n), 12, 4) for n in (3000, 15000, 800, 40000, 5, 0, 1)]
    solo = [solve(w, L, d, 1, igctx)[0] for w, L, d in jobs]
    with Server(igctx, host_threads=2) as sv:
        tickets = [None] * len(jobs)

        def submit(i):
            tickets[i] = sv.submit(*jobs[i])

        th = [threading.Thread(target=submit, args=(i,)) for i in range(len(jobs))]
        for t in th:
            t.start()
        for t in th:
            t.join()
        extra = sv.submit(*jobs[3])
        cancelled = sv.cancel(extra)
        for i, tk in enumerate(tickets):
            got, _, _ = sv.wait(tk)
            assert np.array_equal(got, solo[i]), i
        if cancelled:
            with pytest.raises(IndexGenError) as e:
                sv.wait(extra)
            assert e.value.code == "IG_ERR_CANCELLED"
        else:
            got, _, _ = sv.wait(extra)
            assert np.array_equal(got, solo[3])


def test_server_with_threaded_neighbour_order(igctx):
    """A server whose greedies follow FillAdjList's order for 3 threads (the
    host-assembled order, downloaded synchronously) gives ig_solve's results
    for that order."""
    from indexgen_b200 import Server, solve, workloads as W

    jobs = [(W.uniform_words(n, L, 40 + n), L, d) for n, L, d in ((3000, 12, 4), (1500, 10, 3), (4000, 13, 5))]
    solo = [solve(w, L, d, 3, igctx) for w, L, d in jobs]
    with Server(igctx, host_threads=2, order_threads=3) as sv:
        tickets = [sv.submit(w, L, d) for w, L, d in jobs]
        for tk, (order, edges) in zip(tickets, solo):
            got, e, _ = sv.wait(tk)
            assert e == edges and np.array_equal(got, order)
