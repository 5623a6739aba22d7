"""Nearest-centre assignment (random_cluster's GPU step, src/gpu_cluster.py)
through the C ABI: equal to the reference's own outputs and to the oracle.
Integer work: exact equality, ties to the lowest centre index."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def test_golden_cases(igctx):
    from indexgen_b200 import assign_centers

    g = load_golden("assign.npz")
    keys = sorted({k.rsplit("_", 1)[0] for k in g.files})
    for key in keys:
        L = int(key.split("_")[0][1:])
        got = assign_centers(g[key + "_words"], g[key + "_centers"], L, igctx)
        assert np.array_equal(got, g[key + "_assign"]), key


@pytest.mark.parametrize("L", list(range(1, 17)))
def test_random_against_oracle(igctx, oracle, L):
    from indexgen_b200 import assign_centers, workloads as W

    rng = np.random.default_rng(40 + L)
    for n, k in ((1, 1), (2, 3), (777, 1), (1001, 17), (3000, 64)):
        w = W.uniform_words(n, L, int(rng.integers(1 << 30)))
        c = w[rng.choice(n, min(k, n), replace=False)] if k <= n else W.uniform_words(k, L, 3)
        if len(c) >= 3:
            c[-1] = c[0]  # a tie the lower index must win
        assert np.array_equal(assign_centers(w, c, L, igctx), oracle.assign_centers(w, c, L)), (L, n, k)


def test_many_centres_span_several_shared_memory_passes(igctx, oracle):
    from indexgen_b200 import assign_centers, workloads as W

    w = W.uniform_words(5000, 12, 1)
    c = W.uniform_words(5000, 12, 2)  # 5000 > 2048 centres per pass
    c[4999] = c[17]
    assert np.array_equal(assign_centers(w, c, 12, igctx), oracle.assign_centers(w, c, 12))


def test_device_pointers_equal_host(igctx):
    import torch

    from indexgen_b200 import assign_centers, workloads as W

    w = W.uniform_until(200_001, 14, 9)
    c = w[::5000].copy()
    host = assign_centers(w, c, 14, igctx)
    dev = assign_centers(torch.from_numpy(w.view(np.int32)).cuda(), c, 14, igctx)
    assert np.array_equal(dev.cpu().numpy(), host)
    assert np.bincount(host, minlength=len(c)).sum() == len(w)


def test_reference_named_mirrors(igctx, oracle):
    from indexgen_b200 import random_cluster_fit, solve_assignments_cuda, workloads as W

    w = W.uniform_words(400, 11, 8)
    strings = W.to_strings(w, 11)
    centers = strings[10:30]
    a = solve_assignments_cuda(strings, centers, ctx=igctx)
    assert a.dtype == np.int32
    assert np.array_equal(a, oracle.assign_centers(w, w[10:30], 11))
    assert len(solve_assignments_cuda([], centers, ctx=igctx)) == 0
    with pytest.raises(ValueError):
        solve_assignments_cuda(strings, ["0123"], ctx=igctx)
    clusters = random_cluster_fit(strings, 8, seed=3, ctx=igctx)
    assert sorted(s for c in clusters for s in c) == sorted(strings)
    assert all(c for c in clusters) and len(clusters) <= 8
    for c in clusters:  # order inside a cluster is candidate order
        pos = [strings.index(s) for s in c]
        assert pos == sorted(pos)


def test_bad_input_is_rejected(igctx):
    import ctypes

    from indexgen_b200._lib import lib

    w = np.zeros(4, np.uint32)
    out = np.zeros(4, np.int32)
    L = lib()
    p = lambda a: ctypes.c_void_p(a.ctypes.data)  # noqa: E731
    assert L.ig_assign_centers(igctx.handle, p(w), 4, p(w), 0, 10, 0, p(out)) == 1  # no centres
    assert L.ig_assign_centers(igctx.handle, p(w), 4, p(w), 2, 17, 0, p(out)) == 1  # length
    assert L.ig_assign_centers(igctx.handle, p(w), -1, p(w), 2, 10, 0, p(out)) == 1
    assert L.ig_assign_centers(igctx.handle, None, 0, None, 0, 10, 0, None) == 0  # nothing to do
