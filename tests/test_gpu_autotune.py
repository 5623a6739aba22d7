"""Work-split autotuner: the split changes how the pair triangle is cut into
item tiles, never the graph.  Integer work: bit-exact comparisons."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_graph_independent_of_work_split(oracle):
    """Every candidate split (and extreme pinned ones) gives the oracle's
    graph on a job large enough for the splits to cut it differently."""
    from indexgen_b200 import Context, LANES_NIBBLE, build_conflict_graph, lane_form, workloads as W

    w = W.uniform_words(60000, 12, 2024)
    assert lane_form(12, 4) == LANES_NIBBLE
    rp, cols = oracle.conflict_upper(w[:6000], 12, 4)
    ctx = Context(0)
    try:
        ctx.set_autotune(False)
        ref = None
        for split in (1, 6, 24, 96, 4096):
            ctx.set_work_split(LANES_NIBBLE, split)
            assert ctx.work_split(LANES_NIBBLE) == (split, True)
            with build_conflict_graph(w, 12, 4, ctx) as G:
                got = G.upper_csr()
            if ref is None:
                ref = got
            assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1]), split
            with build_conflict_graph(w[:6000], 12, 4, ctx) as G:
                r2, c2 = G.upper_csr()
            assert np.array_equal(r2, rp) and np.array_equal(c2, cols), split
    finally:
        ctx.close()


@pytest.mark.parametrize("L,d,form", [(12, 4, 1), (14, 6, 2), (16, 10, 0)])
def test_autotune_picks_a_candidate_per_lane_form(L, d, form):
    from indexgen_b200 import Context, build_conflict_graph, lane_form, workloads as W

    assert lane_form(L, d) == form
    w = W.uniform_words(120000, L, 7 + L)
    ctx = Context(0)
    try:
        assert ctx.work_split(form) == (24, False)
        chosen = ctx.autotune(w, L, d)
        assert chosen in (6, 12, 24, 48, 96)
        assert ctx.work_split(form) == (chosen, True)
        # the other lane forms are untouched
        for f in {0, 1, 2} - {form}:
            assert ctx.work_split(f) == (24, False)
        with build_conflict_graph(w[:3000], L, d, ctx) as G:
            e_tuned = G.edges
        ctx2 = Context(0)
        try:
            ctx2.set_autotune(False)
            with build_conflict_graph(w[:3000], L, d, ctx2) as G:
                assert G.edges == e_tuned
        finally:
            ctx2.close()
    finally:
        ctx.close()


def test_automatic_tuning_on_first_large_build(oracle):
    """A fresh context tunes a lane form by itself on the first batch build
    whose splits differ (not on a single-job build), and the graph equals the
    untuned build's."""
    from indexgen_b200 import Context, LANES_BYTE, build_batch, build_conflict_graph, workloads as W

    parts = [W.uniform_words(n, 13, 300 + n) for n in (70000, 20000, 5000)]
    jobs = [(p, 13, 6) for p in parts]
    ctx = Context(0)
    plain = Context(0)
    try:
        plain.set_autotune(False)
        # a single-job build never pays the timing passes
        with build_conflict_graph(parts[0], 13, 6, ctx) as G:
            assert G.edges > 0
        assert ctx.work_split(LANES_BYTE) == (24, False)
        with build_batch(jobs, ctx) as A, build_batch(jobs, plain) as B:
            ra, ca = A.upper_csr()
            rb, cb = B.upper_csr()
        assert ctx.work_split(LANES_BYTE)[1] is True
        assert plain.work_split(LANES_BYTE) == (24, False)
        assert np.array_equal(ra, rb) and np.array_equal(ca, cb)
        orp, ocols = oracle.conflict_upper(parts[2], 13, 6)
        first = len(parts[0]) + len(parts[1])
        sub_r = ra[first:] - ra[first]
        assert np.array_equal(sub_r, orp)
        assert np.array_equal(ca[ra[first]:] - first, ocols)
    finally:
        ctx.close()
        plain.close()


def test_autotune_rejects_bad_input():
    from indexgen_b200 import Context, IndexGenError

    ctx = Context(0)
    try:
        with pytest.raises(IndexGenError):
            ctx.autotune(np.zeros(1, np.uint32), 12, 4)
        with pytest.raises(IndexGenError):
            ctx.set_work_split(3, 24)
        with pytest.raises(IndexGenError):
            ctx.set_work_split(1, 0)
    finally:
        ctx.close()
