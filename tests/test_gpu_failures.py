"""Failure paths, made to happen on purpose without faulting the GPU.

The reference stops the whole process on a failed GPU step (exit(1) after
system(), src/SparseMat.cpp:500-513) and silently drops edges past 5,000,000
per tile (src/cuda_edit_distance.py:401-402).  The library instead returns a
status and keeps the context usable:

  * a bounded device wait that runs out: the test hook withholds one staged
    tile copy (IG_FAULT_TILE_COPY) under a 10 ms wait limit, so the waiting
    CTA gives up, waits for its other copy in flight and leaves; the build
    returns IG_ERR_TIMEOUT and the next build on the same context is exact;
  * a device allocation that fails: IG_FAULT_DEVICE_ALLOC makes the k-th
    allocation of a fresh context fail, for every k the solve reaches; each
    time the call returns IG_ERR_OOM and the same context then solves the job
    exactly.
"""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

OOM, TIMEOUT = 3, 5


def _words(n, L, seed):
    from indexgen_b200 import workloads as W

    return W.uniform_words(n, L, seed)


@pytest.mark.parametrize("L,d", [(12, 4), (16, 5)])
def test_bounded_wait_runs_out_and_context_recovers(oracle, L, d):
    """(12, 4) runs the nibble-lane kernel, (16, 5) the byte-lane one.  A work
    split of one item per CTA makes the first item's segment two staged tiles
    wide, so a copy is in flight when the withheld one times out."""
    from indexgen_b200 import (FAULT_TILE_COPY, Context, IndexGenError, build_conflict_graph, lane_form)

    w = _words(40000, L, 31 + L)
    rp, cols = oracle.conflict_upper(w, L, d)
    want = oracle.pairs_from_csr(rp, cols)
    ctx = Context(0)
    try:
        ctx.set_work_split(lane_form(L, d), 1)
        ctx.set_wait_limit(20_000_000)  # about 10 ms of SM clock
        with build_conflict_graph(w, L, d, ctx) as G:
            assert G.job_tiling(0)[0] >= 1024
            assert np.array_equal(G.pairs(), want)
        ctx.inject_fault(FAULT_TILE_COPY)
        with pytest.raises(IndexGenError) as ei:
            build_conflict_graph(w, L, d, ctx)
        assert ei.value.status == TIMEOUT
        assert "did not arrive" in str(ei.value) and "did not land" not in str(ei.value)
        # the hook is one-shot: the same context builds the exact graph again
        for _ in range(2):
            with build_conflict_graph(w, L, d, ctx) as G:
                assert np.array_equal(G.pairs(), want)
        ctx.set_wait_limit(0)
        with build_conflict_graph(w, L, d, ctx) as G:
            assert np.array_equal(G.pairs(), want)
    finally:
        ctx.close()


def test_timeout_in_a_count_pass(oracle):
    from indexgen_b200 import FAULT_TILE_COPY, Context, IndexGenError, count_conflicts

    w = _words(30000, 11, 5)
    rp, _ = oracle.conflict_upper(w, 11, 4)
    ctx = Context(0)
    try:
        ctx.set_wait_limit(20_000_000)
        ctx.inject_fault(FAULT_TILE_COPY)
        with pytest.raises(IndexGenError) as ei:
            count_conflicts(w, 11, 4, ctx)
        assert ei.value.status == TIMEOUT
        assert count_conflicts(w, 11, 4, ctx) == int(rp[-1])
    finally:
        ctx.close()


def _alloc_sweep(run, check, max_k=64):
    """Fail the k-th device allocation of a fresh context for k = 1, 2, ...
    until a run no longer reaches the k-th one.  Each failing run must return
    IG_ERR_OOM, and the same context must then give the exact result."""
    from indexgen_b200 import FAULT_DEVICE_ALLOC, FAULT_NONE, Context, IndexGenError

    failed_at = []
    for k in range(1, max_k + 1):
        ctx = Context(0)
        try:
            ctx.inject_fault(FAULT_DEVICE_ALLOC, k)
            try:
                run(ctx)
                reached = False
            except IndexGenError as e:
                assert e.status == OOM, (k, str(e))
                reached = True
            ctx.inject_fault(FAULT_NONE)
            check(run(ctx))
            check(run(ctx))
        finally:
            ctx.close()
        if not reached:
            return failed_at
        failed_at.append(k)
    raise AssertionError("the sweep never ran past the last allocation")


def test_every_allocation_of_a_solve_can_fail(oracle):
    """Graph build (workspaces, record buffer growth, CSR), canonical
    adjacency and greedy: a 20,000-word n=10 editDist 5 job overflows the first
    record buffer, so the growth path is in the sweep too."""
    from indexgen_b200 import solve

    g = load_golden("small_cases.npz")
    small = g["L12_d4_words"]
    dense = _words(20000, 10, 77)
    rp, cols = oracle.conflict_upper(dense, 10, 5)
    want_dense = oracle.codebook(rp, cols, len(dense), 1)

    def run(ctx):
        a, _ = solve(small, 12, 4, 1, ctx)
        b, _ = solve(dense, 10, 5, 1, ctx)
        return a, b

    def check(out):
        assert np.array_equal(out[0], g["L12_d4_sel1"])
        assert np.array_equal(out[1], want_dense)

    failed = _alloc_sweep(run, check)
    assert len(failed) >= 6, failed


def test_every_allocation_of_a_batch_can_fail(oracle):
    from indexgen_b200 import solve_batch

    jobs = [(_words(3000 + 500 * j, L, 90 + j), L, d) for j, (L, d) in enumerate([(11, 3), (12, 4), (14, 5), (16, 9)])]
    want = []
    for w, L, d in jobs:
        rp, cols = oracle.conflict_upper(w, L, d)
        want.append(oracle.codebook(rp, cols, len(w), 1))

    def run(ctx):
        return solve_batch(jobs, 1, 2, ctx)

    def check(out):
        books = out[0] if isinstance(out, tuple) else out
        for got, exp in zip(books, want):
            assert np.array_equal(got, exp)

    failed = _alloc_sweep(run, check)
    assert len(failed) >= 6, failed


def test_tiny_host_budget_serialises_downloads_without_deadlock(oracle):
    """A 1 MB host budget is smaller than every graph below: each download then
    waits until no other graph is held on the host, so batch groups, threads
    calling solve (coalesced or not) and the server take turns -- and still
    finish with the exact codebooks."""
    import threading

    from indexgen_b200 import Context, Server, solve, solve_batch

    jobs = [(_words(6000 + 700 * j, L, 300 + j), L, d) for j, (L, d) in enumerate([(11, 3), (10, 4), (12, 4), (10, 5)])]
    want = []
    for w, L, d in jobs:
        rp, cols = oracle.conflict_upper(w, L, d)
        want.append(oracle.codebook(rp, cols, len(w), 1))
    ctx = Context(0)
    try:
        ctx.set_host_budget(1 << 20)
        assert ctx.host_budget()[0] == 1 << 20
        books, _ = solve_batch(jobs, 1, 0, ctx)
        for got, exp in zip(books, want):
            assert np.array_equal(got, exp)
        for coalesce in (True, False):
            ctx.set_coalescing(coalesce)
            got = [None] * len(jobs)

            def run(i):
                got[i] = solve(*jobs[i], 1, ctx)[0]

            ts = [threading.Thread(target=run, args=(i,)) for i in range(len(jobs)) for _ in range(2)]
            for t in ts:
                t.start()
            for t in ts:
                t.join()
            for g, exp in zip(got, want):
                assert np.array_equal(g, exp)
        with Server(ctx, host_threads=3) as sv:
            tickets = [sv.submit(*j) for j in jobs]
            for t, exp in zip(tickets, want):
                assert np.array_equal(sv.wait(t)[0], exp)
        assert ctx.host_budget()[1] == 0  # every download's share came back
    finally:
        ctx.close()
