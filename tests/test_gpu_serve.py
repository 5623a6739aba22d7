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


def test_server_rejects_a_job_larger_than_its_hbm_budget(igctx):
    """With a 64 MB HBM budget, a dense job (20,000 n=10 words, editDist 5:
    about 9e6 edges, some 200 MB at its peak) is refused with IG_ERR_OOM as
    soon as its sampled edge count is known; the jobs around it are served
    and equal their solo solves."""
    from indexgen_b200 import IndexGenError, Server, solve, workloads as W

    small = [(W.uniform_words(2500 + 300 * i, 12, 40 + i), 12, 4) for i in range(5)]
    dense = (W.uniform_words(20000, 10, 77), 10, 5)
    want = [solve(w, L, d, 1, igctx)[0] for w, L, d in small]
    with Server(igctx, host_threads=2, hbm_budget_bytes=64 << 20) as sv:
        tk = [sv.submit(w, L, d) for w, L, d in small[:2]]
        td = sv.submit(*dense)
        tk += [sv.submit(w, L, d) for w, L, d in small[2:]]
        with pytest.raises(IndexGenError) as ei:
            sv.wait(td)
        assert ei.value.status == 3  # IG_ERR_OOM
        for t, w in zip(tk, want):
            got, _, _ = sv.wait(t)
            assert np.array_equal(got, w)
        assert sv.stats()["completed"] == len(small)


def test_server_estimate_failure_fails_cleanly_and_serves_on(igctx):
    """The next device allocation is made to fail while jobs wait: the jobs
    whose admission needed it fail with IG_ERR_OOM, jobs submitted afterwards
    are served exactly."""
    import time

    from indexgen_b200 import FAULT_DEVICE_ALLOC, FAULT_NONE, IndexGenError, Server, solve, workloads as W

    jobs = [(W.uniform_words(3000 + 200 * i, 11, 60 + i), 11, 3) for i in range(4)]
    want = [solve(w, L, d, 1, igctx)[0] for w, L, d in jobs]
    with Server(igctx, host_threads=2) as sv:
        first = sv.submit(*jobs[0])
        sv.wait(first)  # the server is warm and idle
        igctx.inject_fault(FAULT_DEVICE_ALLOC, 1)
        t1 = sv.submit(*jobs[1])
        try:
            sv.wait(t1)
            failed = False
        except IndexGenError as e:
            assert e.status == 3, str(e)
            failed = True
        igctx.inject_fault(FAULT_NONE)
        assert failed, "the injected allocation failure was not reached"
        time.sleep(0.01)
        later = [sv.submit(*j) for j in jobs[2:]]
        for t, w in zip(later, want[2:]):
            got, _, _ = sv.wait(t)
            assert np.array_equal(got, w)
