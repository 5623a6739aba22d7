"""Full-size workloads pinned to the reference's own outputs (tests/golden/
large.json, written once by tests/golden/make_golden_large.py from the
reference's C++ FillAdjList / AdjList / SolveIndependentSet):

  * the 64 Zipf clusters of 1,000,000 n=14 words (editDist 4), solved in one
    batch: every cluster's matrix ones and codebook (as word ids within the
    cluster) equal the reference's SolveIndependentSet with one FillAdjList
    thread (src/SparseMat.cpp:784-851);
  * 1,000,000 VT-style n=16 words (editDist 5): the edge list equals the
    reference FillAdjList's (src/SparseMat.cpp:567-615), by count and sha256,
    and the T=1 codebook equals the FindMinDel loop over the reference GPU
    path's loader (AdjList::FromBinaryFile, src/SparseMat.cpp:338-390).
"""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def large():
    return json.load(open(os.path.join(GOLDEN, "large.json")))


def test_clustered14_batch_equals_reference_per_cluster(large, igctx):
    from indexgen_b200 import solve_batch
    from indexgen_b200 import workloads as W

    gold = large["clustered14"]
    clusters = W.clustered14()
    assert len(clusters) == gold["k"] == 64
    books, edges = solve_batch([(w, 14, 4) for w in clusters], 1, 0, igctx)
    for c, (w, book, e, ref) in enumerate(zip(clusters, books, edges, gold["clusters"])):
        assert len(w) == ref["N"] and sha(np.asarray(w, "<u4")) == ref["words_sha256"], c
        assert 2 * int(e) == ref["ones"], c
        assert len(book) == ref["codebook"], c
        assert sha(book.astype("<i4")) == ref["codebook_sha256"], c


def test_vt16_full_size_equals_reference(large, igctx):
    from indexgen_b200 import build_conflict_graph
    from indexgen_b200 import workloads as W

    gold = large["vt16"]
    w = W.vt16_words(1_000_000, 16)
    assert len(w) == gold["N"] and sha(w.astype("<u4")) == gold["words_sha256"]
    with build_conflict_graph(w, 16, 5, igctx) as G:
        assert G.edges == gold["edges"] and G.matrix_ones_num == gold["ones"]
        pairs = G.pairs()
        assert sha(pairs.astype("<i4")) == gold["edges_sha256"]
        del pairs
        book = G.codebook(1)
    assert len(book) == gold["codebook_t1"]
    assert book[:64].tolist() == gold["codebook_t1_head"]
    assert sha(book.astype("<i4")) == gold["codebook_t1_sha256"]
