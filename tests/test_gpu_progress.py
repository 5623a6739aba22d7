"""Checkpoint bridge: progress_adj_list.txt written from the device graph is
byte-identical to the reference's AdjList::ToFile after its GPU loader
(FromBinaryFile), and reading it back resumes to the reference's codebook
(reference driver built from the reference sources, oracle/_ref)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_golden

pytestmark = pytest.mark.gpu

REF = os.path.join(ROOT, "oracle", "_ref", "ref_driver")


def ref(*args):
    if not os.path.exists(REF):
        pytest.skip("reference driver not built (make -C oracle ref)")
    subprocess.run([REF, *map(str, args)], check=True, capture_output=True)


def graphs():
    from indexgen_b200 import workloads as W

    g = load_golden("small_cases.npz")
    yield "planted_L10_d4", g["L10_d4_words"], 10, 4
    yield "uniform11_d3", load_golden("uniform11.npz")["words"], 11, 3
    yield "uniform_n11_d4_40k", W.uniform_until(40000, 11, 21), 11, 4


@pytest.mark.parametrize("case", [0, 1, 2])
def test_write_matches_reference_tofile_and_resumes(igctx, tmp_path, case):
    from indexgen_b200 import build_conflict_graph, read_adj_list

    name, w, L, d = list(graphs())[case]
    n = len(w)
    with build_conflict_graph(w, L, d, igctx) as G:
        pairs = G.pairs()
        book = G.codebook(1)
        ours = tmp_path / "ours.txt"
        size = G.write_adj_list(ours)
    pairs_file = tmp_path / "pairs.bin"
    pairs.astype("<i4").tofile(pairs_file)
    theirs = tmp_path / "ref.txt"
    ref("tofile", n, pairs_file, theirs)
    assert size == os.path.getsize(ours)
    assert open(ours, "rb").read() == open(theirs, "rb").read(), name
    # resume: FromFile semantics (n = largest id + 1), greedy, then the rest
    with read_adj_list(ours, igctx) as R:
        assert R.edges == len(pairs)
        resumed = R.codebook(1)
    rest = [i for i in range(n) if i >= R.n]
    out = tmp_path / "resume.bin"
    ref("resume", n, ours, out)
    expect = np.fromfile(out, "<i4")[1:]
    assert np.array_equal(np.concatenate([resumed, np.array(rest, np.int32)]), expect), name
    if R.n == n:
        assert np.array_equal(resumed, book)


def test_bad_files_are_rejected(igctx, tmp_path):
    from indexgen_b200 import IndexGenError, read_adj_list

    p = tmp_path / "asym.txt"
    p.write_text("0\t1\n1\t2\n2\t1\n")
    with pytest.raises(IndexGenError):
        read_adj_list(p, igctx)
    p.write_text("0\t1\nx y\n")
    with pytest.raises(IndexGenError):
        read_adj_list(p, igctx)
    with pytest.raises(IndexGenError):
        read_adj_list(tmp_path / "missing.txt", igctx)
    p.write_text("")
    with read_adj_list(p, igctx) as R:
        assert R.n == 0 and R.edges == 0
