"""Concurrent solve() calls on one context (the reference's cluster worker
pool calling its GPU path from several threads, src/SparseMat.cpp:978-1010)
are built together and give every caller the codebook it gets alone.
Integer work: bit-exact."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_concurrent_solves_equal_solo_solves():
    from indexgen_b200 import Context, solve, workloads as W

    jobs = [(W.uniform_words(n, L, 700 + i), L, d)
            for i, (n, L, d) in enumerate([(4000, 12, 4), (2500, 10, 3), (6000, 14, 5), (900, 16, 9),
                                           (3000, 11, 4), (0, 12, 4), (1, 12, 4), (5000, 13, 6),
                                           (3500, 12, 4), (2000, 15, 5), (4500, 10, 4), (1200, 12, 2)])]
    solo_ctx = Context(0)
    try:
        solo_ctx.set_coalescing(False)
        want = [solve(w, L, d, 1, solo_ctx) for w, L, d in jobs]
        assert solo_ctx.coalesce_stats() == (0, 0)
    finally:
        solo_ctx.close()
    ctx = Context(0)
    got = [None] * len(jobs)
    errors = []
    start = threading.Barrier(len(jobs))

    def worker(i):
        try:
            w, L, d = jobs[i]
            start.wait()
            for _ in range(3):
                got[i] = solve(w, L, d, 1, ctx)
        except Exception as e:
            errors.append((i, repr(e)))

    try:
        threads = [threading.Thread(target=worker, args=(i,)) for i in range(len(jobs))]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        assert not errors, errors
        for (book, edges), (wbook, wedges) in zip(got, want):
            assert edges == wedges
            assert np.array_equal(book, wbook)
        batches, requests = ctx.coalesce_stats()
        assert requests == 3 * len(jobs) and 1 <= batches <= requests
    finally:
        ctx.close()


def test_bad_call_among_concurrent_solves():
    """An invalid call fails on its own; the calls around it are built and
    solved as usual."""
    from indexgen_b200 import Context, IndexGenError, solve, workloads as W

    ctx = Context(0)
    good = [(W.uniform_words(2000 + 100 * i, 12, 60 + i), 12, 4) for i in range(4)]
    want = []
    try:
        ctx.set_coalescing(False)
        want = [solve(w, L, d, 1, ctx) for w, L, d in good]
        ctx.set_coalescing(True)
        results, errors = {}, {}
        start = threading.Barrier(len(good) + 1)

        def ok(i):
            start.wait()
            results[i] = solve(*good[i], 1, ctx)

        def bad():
            start.wait()
            try:
                solve(np.zeros(10, np.uint32), 17, 4, 1, ctx)  # length 17 is out of range
            except IndexGenError as e:
                errors["bad"] = e

        threads = [threading.Thread(target=ok, args=(i,)) for i in range(len(good))] + [threading.Thread(target=bad)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        assert "bad" in errors and errors["bad"].code == "IG_ERR_INPUT"
        for i, (book, edges) in enumerate(want):
            assert results[i][1] == edges and np.array_equal(results[i][0], book)
    finally:
        ctx.close()


def test_merged_build_that_fails_is_split_per_request():
    """Two calls that arrive while a long build holds the device are built
    together next.  The first device allocation of that merged build is made
    to fail (as a summed workspace that does not fit would); each request is
    then built on its own and both callers get their exact codebooks."""
    import time

    from indexgen_b200 import FAULT_DEVICE_ALLOC, FAULT_NONE, Context, solve, workloads as W

    big = (W.uniform_words(400000, 12, 5), 12, 4)
    small = [(W.uniform_words(3000, 12, 6), 12, 4), (W.uniform_words(2500, 11, 7), 11, 3)]
    ref = Context(0)
    try:
        ref.set_coalescing(False)
        want = [solve(w, L, d, 1, ref) for w, L, d in small]
        # allocations of the big call alone on a fresh context
        probe = Context(0)
        try:
            solve(*big, 1, probe)
            big_allocs = probe.device_allocs
        finally:
            probe.close()
    finally:
        ref.close()
    ctx = Context(0)
    got = [None, None]
    errors = []

    def run_big():
        try:
            solve(*big, 1, ctx)
        except Exception as e:
            errors.append(("big", repr(e)))

    def run_small(i):
        try:
            w, L, d = small[i]
            got[i] = solve(w, L, d, 1, ctx)
        except Exception as e:
            errors.append((i, repr(e)))

    try:
        ctx.inject_fault(FAULT_DEVICE_ALLOC, big_allocs + 1)
        tb = threading.Thread(target=run_big)
        tb.start()
        time.sleep(0.03)  # the big build holds the device for much longer than this
        ts = [threading.Thread(target=run_small, args=(i,)) for i in range(2)]
        for t in ts:
            t.start()
        for t in [tb] + ts:
            t.join()
        ctx.inject_fault(FAULT_NONE)
        assert not errors, errors
        for (book, edges), (wbook, wedges) in zip(got, want):
            assert edges == wedges
            assert np.array_equal(book, wbook)
        batches, requests = ctx.coalesce_stats()
        assert requests == 3 and batches == 2  # the big call, then the two small ones merged
    finally:
        ctx.close()
