"""The allocation-free conflict count (ig_count_conflicts_noalloc).

Some hosts own every byte of device memory themselves -- a JVM, Go or Rust
runtime handing out slices of one preallocated arena, or a service held to a
hard memory budget -- and cannot let a library call the CUDA allocator.  This
entry point serves them: its scratch is a fixed array inside the library, and
the caller passes device buffers for the input words and the output count.
The test compares it with the allocating entry point, ig_count_conflicts, on
the same inputs, calling it twice in a row per input so that a count left in
the shared scratch by an earlier call would show up.  This file is collected
last so that a failure here cannot stop the other GPU tests.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_count_matches_allocating_count():
    import torch

    from indexgen_b200 import Context, count_conflicts, workloads as W
    from indexgen_b200._lib import lib

    ctx = Context(0)
    out = torch.zeros(1, dtype=torch.int64, device="cuda:0")
    cases = [
        (W.uniform_filtered(60000, 12, 21), 12, 4),  # two-lane kernel, near the size limit
        (W.uniform_words(40001, 16, 22), 16, 5),     # one-lane kernel, odd size
        (W.uniform_words(5000, 11, 23), 11, 3),
        (W.uniform_words(3, 10, 24), 10, 11),        # every pair conflicts
        (W.uniform_words(1, 10, 25), 10, 4),         # no pairs
    ]
    for w, L, d in cases:
        want = count_conflicts(w, L, d, ctx)
        words = torch.from_numpy(w.view(np.int32)).to("cuda:0")
        for _ in range(2):
            torch.cuda.synchronize()
            st = lib().ig_count_conflicts_noalloc(ctypes.c_void_p(words.data_ptr()), len(w), L, d,
                                                  ctypes.c_void_p(out.data_ptr()), None)
            assert st == 0
            torch.cuda.synchronize()
            assert int(out.item()) == want, (len(w), L, d)
    ctx.close()


def test_noalloc_rejects_oversize_and_bad_arguments():
    import torch

    from indexgen_b200._lib import lib

    out = torch.zeros(1, dtype=torch.int64, device="cuda:0")
    words = torch.zeros(65537, dtype=torch.int32, device="cuda:0")
    p = ctypes.c_void_p(words.data_ptr())
    o = ctypes.c_void_p(out.data_ptr())
    assert lib().ig_count_conflicts_noalloc(p, 65537, 12, 4, o, None) == 2  # IG_ERR_CAPACITY
    assert lib().ig_count_conflicts_noalloc(p, 100, 17, 4, o, None) == 1    # IG_ERR_INPUT
    assert lib().ig_count_conflicts_noalloc(p, 100, 12, 4, None, None) == 1
