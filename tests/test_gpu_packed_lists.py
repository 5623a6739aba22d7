"""Neighbour lists sent to the host greedy bit-packed per row (each row: gap
width, first neighbour, gaps minus one in that width; built on the device by
ig_packrows.cu, decoded by the greedy).  Forced on for every greedy path --
one job, coalesced calls, batches, the server -- the codebooks must equal the
reference's fixtures and the plain lists' results, including rows whose gaps
are all zero (width 0: a clique of duplicates), single-neighbour rows and
isolated vertices.  Integer work: bit-exact."""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def packed_ctx():
    from indexgen_b200 import LISTS_PACKED, Context

    ctx = Context(0)
    ctx.set_host_lists(LISTS_PACKED)
    yield ctx
    ctx.close()


def test_packed_lists_reference_fixtures(packed_ctx):
    from indexgen_b200 import solve

    g = load_golden("uniform11.npz")
    book, _ = solve(g["words"], 11, 3, 1, packed_ctx)
    assert np.array_equal(book, g["sel1"])
    s = load_golden("small_cases.npz")
    for key in sorted({k.rsplit("_", 1)[0] for k in s.files if k.endswith("_words")}):
        L, d = (int(x[1:]) for x in key.split("_"))
        book, _ = solve(s[key + "_words"], L, d, 1, packed_ctx)
        assert np.array_equal(book, s[key + "_sel1"]), key


def test_packed_lists_linear12_full_size(packed_ctx):
    from indexgen_b200 import solve
    from indexgen_b200 import workloads as W

    gold = json.load(open(os.path.join(GOLDEN, "linear.json")))["linear12"]
    book, edges = solve(W.linear12_candidates(), 12, 4, 1, packed_ctx)
    assert edges == gold["edges"]
    assert hashlib.sha256(book.astype("<i4").tobytes()).hexdigest() == gold["codebook_t1_sha256"]


def test_packed_lists_equal_plain_on_dense_and_degenerate_jobs(packed_ctx, oracle):
    from indexgen_b200 import LISTS_PLAIN, Context, Server, solve, solve_batch
    from indexgen_b200 import workloads as W

    dense = W.uniform_words(20000, 10, 77)                     # ~9e6 edges, wide rows
    clique = np.full(300, W.uniform_words(1, 12, 3)[0], np.uint32)  # every gap 0: width 0
    pairs = np.repeat(W.uniform_words(400, 14, 4), 2)          # one neighbour each
    lonely = W.uniform_words(500, 16, 5)                       # isolated at editDist 2
    jobs = [(dense, 10, 5), (clique, 12, 4), (pairs, 14, 3), (lonely, 16, 2), (dense[:1], 10, 5),
            (dense[:0], 10, 5)]
    plain_ctx = Context(0)
    try:
        plain_ctx.set_host_lists(LISTS_PLAIN)
        want = [solve(w, L, d, 1, plain_ctx)[0] for w, L, d in jobs]
    finally:
        plain_ctx.close()
    rp, cols = oracle.conflict_upper(dense, 10, 5)
    assert np.array_equal(want[0], oracle.codebook(rp, cols, len(dense), 1))
    for (w, L, d), ref in zip(jobs, want):
        assert np.array_equal(solve(w, L, d, 1, packed_ctx)[0], ref)
    books, _ = solve_batch(jobs, 1, 0, packed_ctx)
    for got, ref in zip(books, want):
        assert np.array_equal(got, ref)
    with Server(packed_ctx, host_threads=3) as sv:
        tickets = [sv.submit(w, L, d) for w, L, d in jobs]
        for t, ref in zip(tickets, want):
            assert np.array_equal(sv.wait(t)[0], ref)
