"""Candidate generators and filters against the reference's candidate lists."""
import hashlib
import json
import os

import numpy as np

from conftest import GOLDEN, load_golden
from indexgen_b200 import workloads as W


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_uniform11_matches_reference_input():
    g = load_golden("uniform11.npz")
    assert np.array_equal(W.uniform11_candidates(), g["words"])


def test_linear12_matches_reference_generator():
    info = json.load(open(os.path.join(GOLDEN, "linear.json")))["linear12"]
    w = W.linear12_candidates()
    assert len(w) == info["N"] == 207432
    assert sha(w.astype("<u4")) == info["words_sha256"]


def test_n11_header_candidates():
    info = json.load(open(os.path.join(GOLDEN, "linear.json")))["n11_header"]
    w = W.linear_code_words(11, info["bias"], info["row_perm"], info["col_perm"])
    w = w[W.filter_words(w, 11, info["max_run"], info["min_gc"], info["max_gc"])]
    assert len(w) == info["N"]
    assert sha(w.astype("<u4")) == info["words_sha256"]


def test_hamming_code_distance():
    """The [n, n-3, 3] code has minimum Hamming distance 3."""
    w = W.linear_code_words(8, [0] * 8)
    d = W.unpack_digits(w, 8).astype(np.int64)
    nz = (d != 0).sum(axis=1)
    assert nz[1:].min() == 3  # linear: min weight of a non-zero codeword


def test_filters_agree_with_oracle(oracle):
    rng = np.random.default_rng(3)
    for L in (1, 2, 5, 10, 11, 12, 16):
        w = W.uniform_words(4000, L, int(rng.integers(1 << 30)))
        for args in ((3, 0.3, 0.7), (0, 0.3, 0.7), (2, 0.0, 0.0), (0, 0.0, 0.5), (4, 0.45, 0.55)):
            assert np.array_equal(W.filter_words(w, L, *args), oracle.filter_mask(w, L, *args)), (L, args)


def test_strings_roundtrip():
    s = ["0123012301", "3333333333", "0000000000"]
    assert W.to_strings(W.from_strings(s), 10) == s


def test_vt16_membership():
    w = W.vt16_words(2000, seed=5)
    d = W.unpack_digits(w, 16).astype(np.int64)
    assert np.all((d * np.arange(1, 17)).sum(axis=1) % 17 == 0)
    assert np.all(d.sum(axis=1) % 4 == 0)
    assert W.filter_words(w, 16).all()


def test_zipf_sizes():
    s = W.zipf_sizes(1_000_000, 64)
    assert s.sum() == 1_000_000 and s.min() >= 2000 and s.max() <= 60000
    assert np.all(np.diff(s) <= 0)


def test_assign_clusters_partition():
    w = W.uniform_until(5000, 14, 9)
    parts = W.assign_clusters(w, 14, W.zipf_sizes(5000, 8, lo=100, hi=2000), 10)
    allidx = np.concatenate(parts)
    assert len(allidx) == 5000 and len(np.unique(allidx)) == 5000
    again = W.assign_clusters(w, 14, W.zipf_sizes(5000, 8, lo=100, hi=2000), 10)
    assert all(np.array_equal(a, b) for a, b in zip(parts, again))
