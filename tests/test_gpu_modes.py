"""Lane forms, record-buffer growth and full-size spot checks of the CUDA
path (through the C ABI) against the oracle.  The kernel picks its lane form
by editDist (eight nibble lanes for editDist <= 4, four byte lanes for 5..8,
full Myers above), so every (L, editDist) pair below exercises one form on
sets with planted near neighbours.  Integer work: bit-exact comparisons."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def planted(n, L, seed):
    """Uniform words plus neighbours at 1..3 edits (substitutions, deletions
    with a fill at the end, insertions dropping the last char)."""
    from indexgen_b200 import workloads as W

    rng = np.random.default_rng(seed)
    w = W.uniform_words(n, L, seed)
    d = W.unpack_digits(w, L).astype(np.int64)
    half = n // 2
    for i in range(half, n):
        x = list(d[int(rng.integers(0, half))])
        for _ in range(int(rng.integers(1, 4))):
            p = int(rng.integers(0, L))
            op = int(rng.integers(0, 3))
            if op == 0:
                x[p] = int(rng.integers(0, 4))
            elif op == 1:
                x = x[:p] + x[p + 1:] + [int(rng.integers(0, 4))]
            else:
                x = x[:p] + [int(rng.integers(0, 4))] + x[p:-1]
        d[i] = x[:L]
    return W.pack_digits(d)


def pairs_of(G):
    return G.pairs()


@pytest.mark.parametrize("L", [1, 2, 4, 7, 8, 10, 12, 13, 15, 16])
def test_lane_forms_all_thresholds(igctx, oracle, L):
    from indexgen_b200 import build_conflict_graph

    w = planted(600, L, 1000 + L)
    for d in range(1, min(L + 2, 12)):
        rp, cols = oracle.conflict_upper(w, L, d)
        with build_conflict_graph(w, L, d, igctx) as G:
            assert np.array_equal(pairs_of(G), oracle.pairs_from_csr(rp, cols)), (L, d)


def test_dense_job_grows_records_and_reruns(oracle):
    """A fresh context starts with room for 4,194,304 records; a 20,000-word
    n=10 editDist 5 job has about 9e6 edges, so the first pass overflows, the
    buffer grows and the pass reruns.  The result must equal the oracle and a
    build on the grown context."""
    from indexgen_b200 import Context, build_conflict_graph, workloads as W

    w = W.uniform_words(20000, 10, 77)
    rp, cols = oracle.conflict_upper(w, 10, 5)
    assert rp[-1] > 4_500_000
    ctx = Context(0)
    try:
        with build_conflict_graph(w, 10, 5, ctx) as G:
            r1, c1 = G.upper_csr()
        with build_conflict_graph(w, 10, 5, ctx) as G:
            r2, c2 = G.upper_csr()
    finally:
        ctx.close()
    assert np.array_equal(r1, rp) and np.array_equal(c1, cols)
    assert np.array_equal(r2, rp) and np.array_equal(c2, cols)


def test_batch_of_all_lane_forms_equals_solo(igctx, oracle):
    from indexgen_b200 import build_batch, build_conflict_graph

    jobs = []
    for k, (L, d) in enumerate([(10, 5), (12, 2), (16, 9), (11, 4), (14, 7), (9, 10), (13, 3), (16, 5)]):
        jobs.append((planted(400 + 97 * k, L, 50 + k), L, d))
    with build_batch(jobs, igctx) as B:
        rp, cols = B.upper_csr()
        for j, (w, L, d) in enumerate(jobs):
            first, n, e = B.job_stats(j)
            orp, ocols = oracle.conflict_upper(w, L, d)
            assert e == orp[-1], j
            rows = np.repeat(np.arange(n), np.diff(rp[first:first + n + 1]))
            got = np.stack([rows, cols[rp[first]:rp[first + n]] - first], 1)
            assert np.array_equal(got, oracle.pairs_from_csr(orp, ocols)), j
            with build_conflict_graph(w, L, d, igctx) as G:
                assert np.array_equal(G.pairs(), got), j


def test_vt16_full_size_sampled_rows(igctx, oracle):
    """The 1,000,000-word VT-style n=16 editDist 5 job (5e11 pair tests): the
    symmetric neighbour sets of 48 seeded rows equal the oracle's, the graph
    is the same on a second build, and its degree sum is twice its edges."""
    from indexgen_b200 import build_conflict_graph, workloads as W

    w = W.vt16_words(1_000_000, seed=16)
    with build_conflict_graph(w, 16, 5, igctx) as G:
        rp, cols = G.upper_csr()
        edges = G.edges
    with build_conflict_graph(w, 16, 5, igctx) as G:
        rp2, cols2 = G.upper_csr()
    assert np.array_equal(rp, rp2) and np.array_equal(cols, cols2)
    assert rp[-1] == edges and edges > 0
    rows = np.sort(np.random.default_rng(3).choice(len(w), 48, replace=False)).astype(np.int32)
    want = oracle.row_neighbours(w, 16, 5, rows)
    # lower neighbours: rows u whose upper list holds r
    hit = np.isin(cols, rows)
    owner = np.repeat(np.arange(len(w), dtype=np.int32), np.diff(rp))[hit]
    target = cols[hit]
    for k, r in enumerate(rows):
        lower = owner[target == r]
        upper = cols[rp[r]:rp[r + 1]]
        got = np.concatenate([np.sort(lower), upper])
        assert np.array_equal(got, want[k]), int(r)
