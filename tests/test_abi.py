"""The C-ABI library: it loads, exports every declared entry point, and its
host-only functions (no device work) agree with the oracle / reference."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, load_golden


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "indexgen_cuda.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ig_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def L():
    from indexgen_b200 import build as B
    from indexgen_b200 import _lib

    B.build()
    return _lib.lib()


def test_exports_every_declared_symbol(L):
    from indexgen_b200 import _lib

    syms = declared_symbols()
    assert len(syms) >= 20
    assert sorted(_lib.EXPORTS) == syms
    for s in syms:
        assert hasattr(L, s), s
    assert b"sm_100a" in L.ig_version()


def test_status_strings(L):
    for code in range(8):
        assert L.ig_status_string(code)


def test_pack_matches_oracle(L, oracle):
    rng = np.random.default_rng(1)
    strings = ["".join(map(str, rng.integers(0, 4, 13))) for _ in range(500)]
    raw = "".join(strings).encode()
    out = np.zeros(500, np.uint32)
    bad = ctypes.c_int64(7)
    assert L.ig_pack(raw, 500, 13, 13, out.ctypes.data, ctypes.byref(bad)) == 0
    assert bad.value == -1
    assert np.array_equal(out, oracle.pack(strings))


def test_pack_rejects_bad_symbol(L):
    raw = b"0123" + b"01A3" + b"0000"
    out = np.zeros(3, np.uint32)
    bad = ctypes.c_int64(0)
    assert L.ig_pack(raw, 3, 4, 4, out.ctypes.data, ctypes.byref(bad)) == 1
    assert bad.value == 1
    assert L.ig_pack(raw, 3, 17, 17, out.ctypes.data, None) == 1  # length > 16
    assert L.ig_pack(raw, 3, 0, 4, out.ctypes.data, None) == 1


def test_filter_matches_oracle(L, oracle):
    from indexgen_b200 import apply_filters
    from indexgen_b200 import workloads as W

    for Ln in (3, 10, 12, 16):
        w = W.uniform_words(3000, Ln, Ln)
        for args in ((3, 0.3, 0.7), (0, 0.4, 0.6), (2, 0.0, 0.0)):
            assert np.array_equal(apply_filters(w, Ln, *args), oracle.filter_mask(w, Ln, *args))


@pytest.mark.parametrize("T", [1, 3, 8, 16])
def test_host_greedy_uniform11(L, T):
    """The library's greedy (host) reproduces SolveIndependentSet at T threads."""
    from indexgen_b200 import codebook_from_upper_csr

    g = load_golden("uniform11.npz")
    n = len(g["words"])
    e = g["edges"]
    row_ptr = np.zeros(n + 1, np.int64)
    np.add.at(row_ptr, e[:, 0] + 1, 1)
    row_ptr = np.cumsum(row_ptr)
    sel = codebook_from_upper_csr(row_ptr, e[:, 1], n, T)
    if f"sel{T}" in g.files:
        assert np.array_equal(sel, g[f"sel{T}"])
    else:
        assert len(sel) > 0


def test_host_greedy_small_cases(L):
    from indexgen_b200 import codebook_from_upper_csr

    g = load_golden("small_cases.npz")
    keys = sorted({k.rsplit("_", 1)[0] for k in g.files if k.endswith("_words")})
    for key in keys:
        n = len(g[key + "_words"])
        e = g[key + "_edges"]
        row_ptr = np.zeros(n + 1, np.int64)
        np.add.at(row_ptr, e[:, 0] + 1, 1)
        row_ptr = np.cumsum(row_ptr)
        cols = e[:, 1] if len(e) else np.zeros(0, np.int32)
        assert np.array_equal(codebook_from_upper_csr(row_ptr, cols, n, 1), g[key + "_sel1"]), key
        assert np.array_equal(codebook_from_upper_csr(row_ptr, cols, n, 3), g[key + "_sel3"]), key


def test_host_greedy_over_reference_neighbour_lists(L):
    """Greedy over neighbour lists as the reference's AdjList holds them: the
    reference's own m[] at T=3 (small_cases.npz) gives its T=3 codebooks."""
    from indexgen_b200 import IndexGenError, codebook_from_adjacency

    g = load_golden("small_cases.npz")
    keys = sorted({k.rsplit("_", 1)[0] for k in g.files if k.endswith("_words")})
    for key in keys:
        n = len(g[key + "_words"])
        assert np.array_equal(codebook_from_adjacency(g[key + "_adj3_ptr"], g[key + "_adj3"], n),
                              g[key + "_sel3"]), key
    with pytest.raises(IndexGenError):
        codebook_from_adjacency(np.array([0, 1, 1], np.int64), np.array([4], np.int32), 2)


def test_host_greedy_rejects_bad_csr(L):
    from indexgen_b200 import IndexGenError, codebook_from_upper_csr

    with pytest.raises(IndexGenError):
        codebook_from_upper_csr(np.array([0, 1, 1], np.int64), np.array([5], np.int32), 2)
    with pytest.raises(IndexGenError):
        codebook_from_upper_csr(np.array([0, 1, 1], np.int64), np.array([1], np.int32), 2, order_threads=0)


def test_host_greedy_edge_cases(L):
    from indexgen_b200 import codebook_from_upper_csr

    assert len(codebook_from_upper_csr(np.zeros(1, np.int64), np.zeros(0, np.int32), 0)) == 0
    # isolated vertices are taken from bucket 0 back-to-front
    assert codebook_from_upper_csr(np.zeros(4, np.int64), np.zeros(0, np.int32), 3).tolist() == [2, 1, 0]


def test_ctx_create_without_gpu_fails_cleanly(L):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    st = L.ig_ctx_create(ctypes.byref(h), 0)
    assert st != 0 and not h.value
    assert L.ig_ctx_create(None, 0) == 1


def test_lane_forms_and_null_context_calls(L):
    """Lane form per (len, min_ed) (host only) and the tuning / graph calls'
    argument checks, which need no device."""
    from indexgen_b200 import LANES_BYTE, LANES_FULL, LANES_NIBBLE, lane_form

    for d in range(1, 5):
        assert lane_form(12, d) == LANES_NIBBLE
    for d in range(5, 9):
        assert lane_form(16, d) == LANES_BYTE
    assert lane_form(16, 9) == LANES_FULL and lane_form(10, 0) == LANES_FULL
    assert lane_form(0, 4) == -1 and lane_form(17, 4) == -1
    v = ctypes.c_int32()
    t = ctypes.c_int()
    n = ctypes.c_int64()
    assert L.ig_ctx_autotune(None, None, 0, 12, 4, 0, ctypes.byref(v)) == 1
    assert L.ig_ctx_set_work_split(None, 1, 24) == 1
    assert L.ig_ctx_work_split(None, 1, ctypes.byref(v), ctypes.byref(t)) == 1
    assert L.ig_ctx_set_autotune(None, 1) == 1
    assert L.ig_ctx_set_graphs(None, 1) == 1
    assert L.ig_ctx_graph_stats(None, ctypes.byref(n), None, None) == 1
