"""ctypes front end of the CPU oracle (oracle/ig_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
as the checker, and by the ``cpu_baseline`` leg of bench.py.  The product
package never imports it.

The C library restates the reference path (edge predicate of
include/EditDistance.hpp:368-372, neighbour order of src/SparseMat.cpp:599-609,
greedy of src/SparseMat.cpp:81-266/679-731) and is pinned against golden
vectors produced by the reference's own C++ code (tests/golden/).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libigoracle.so")
_lib = None

_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


def build() -> str:
    """Compile the oracle library with gcc (Makefile beside this file)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
            os.path.join(_HERE, "ig_oracle.c")
        ):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.igo_pack.restype = ctypes.c_int64
        L.igo_pack.argtypes = [ctypes.c_char_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int64, _u32p]
        L.igo_lev_dp.restype = ctypes.c_int
        L.igo_lev_dp.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int]
        L.igo_lev_myers.restype = ctypes.c_int
        L.igo_lev_myers.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int]
        L.igo_filter.restype = None
        L.igo_filter.argtypes = [_u32p, ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                 ctypes.c_double, _u8p]
        L.igo_conflict_upper.restype = ctypes.c_int
        L.igo_conflict_upper.argtypes = [_u32p, ctypes.c_int32, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         _i64p, ctypes.c_void_p]
        L.igo_conflict_upper_alloc.restype = ctypes.c_int
        L.igo_conflict_upper_alloc.argtypes = [_u32p, ctypes.c_int32, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                               _i64p, ctypes.POINTER(ctypes.c_void_p)]
        L.igo_row_neighbours.restype = ctypes.c_int
        L.igo_row_neighbours.argtypes = [_u32p, ctypes.c_int32, ctypes.c_int, ctypes.c_int, _i32p, ctypes.c_int32,
                                         ctypes.c_int, _i64p, ctypes.POINTER(ctypes.c_void_p)]
        L.igo_assign_centers.restype = ctypes.c_int
        L.igo_assign_centers.argtypes = [_u32p, ctypes.c_int64, _u32p, ctypes.c_int32, ctypes.c_int, ctypes.c_int,
                                         _i32p]
        L.igo_free.restype = None
        L.igo_free.argtypes = [ctypes.c_void_p]
        L.igo_adjacency.restype = None
        L.igo_adjacency.argtypes = [_i64p, _i32p, ctypes.c_int32, ctypes.c_int, _i64p, _i32p]
        L.igo_greedy.restype = ctypes.c_int32
        L.igo_greedy.argtypes = [_i64p, _i32p, ctypes.c_int32, _i32p]
        _lib = L
    return _lib


def pack(strings) -> np.ndarray:
    """'0'..'3' strings of one length -> uint32 words (char p at bits 2p..2p+1)."""
    n = len(strings)
    if n == 0:
        return np.zeros(0, np.uint32)
    L = len(strings[0])
    raw = "".join(strings).encode("latin1")
    out = np.zeros(n, np.uint32)
    bad = lib().igo_pack(raw, n, L, L, out)
    if bad >= 0:
        raise ValueError(f"row {bad} is not a '0'..'3' string of length {L}")
    return out


def unpack(words, L: int):
    w = np.asarray(words, dtype=np.uint32)
    digits = (w[:, None] >> (2 * np.arange(L, dtype=np.uint32))[None, :]) & 3
    return ["".join(map(str, row)) for row in digits.tolist()]


def lev(a: int, b: int, L: int, method: str = "myers") -> int:
    f = lib().igo_lev_myers if method == "myers" else lib().igo_lev_dp
    return int(f(int(a), int(b), L))


def filter_mask(words, L: int, max_run: int, min_gc: float, max_gc: float) -> np.ndarray:
    w = np.ascontiguousarray(words, dtype=np.uint32)
    keep = np.zeros(len(w), np.uint8)
    lib().igo_filter(w, len(w), L, max_run, min_gc, max_gc, keep)
    return keep.astype(bool)


def conflict_upper(words, L: int, min_ed: int, threads: int | None = None):
    """Upper CSR (row_ptr int64[n+1], cols int32[nnz]) of pairs i<j with ED < min_ed."""
    w = np.ascontiguousarray(words, dtype=np.uint32)
    n = len(w)
    threads = threads or max(1, len(os.sched_getaffinity(0)))
    row_ptr = np.zeros(n + 1, np.int64)
    buf = ctypes.c_void_p()
    rc = lib().igo_conflict_upper_alloc(w, n, L, min_ed, threads, row_ptr, ctypes.byref(buf))
    if rc != 0:
        raise MemoryError("oracle conflict_upper failed")
    nnz = int(row_ptr[-1])
    try:
        cols = np.ctypeslib.as_array(ctypes.cast(buf, ctypes.POINTER(ctypes.c_int32)), shape=(max(nnz, 1),))
        cols = cols[:nnz].copy()
    finally:
        lib().igo_free(buf)
    return row_ptr, cols


def row_neighbours(words, L: int, min_ed: int, rows, threads: int | None = None):
    """Symmetric neighbour sets of the sampled rows: list of ascending int32 arrays."""
    w = np.ascontiguousarray(words, dtype=np.uint32)
    rows = np.ascontiguousarray(rows, dtype=np.int32)
    threads = threads or max(1, len(os.sched_getaffinity(0)))
    ptr = np.zeros(len(rows) + 1, np.int64)
    buf = ctypes.c_void_p()
    if lib().igo_row_neighbours(w, len(w), L, min_ed, rows, len(rows), threads, ptr, ctypes.byref(buf)) != 0:
        raise MemoryError("oracle row_neighbours failed")
    try:
        flat = np.ctypeslib.as_array(ctypes.cast(buf, ctypes.POINTER(ctypes.c_int32)), shape=(max(int(ptr[-1]), 1),))
        return [flat[ptr[k]:ptr[k + 1]].copy() for k in range(len(rows))]
    finally:
        lib().igo_free(buf)


def assign_centers(words, centers, L: int, threads: int | None = None) -> np.ndarray:
    """Nearest centre (Levenshtein, lowest index on ties) of every word."""
    w = np.ascontiguousarray(words, dtype=np.uint32)
    c = np.ascontiguousarray(centers, dtype=np.uint32)
    threads = threads or max(1, len(os.sched_getaffinity(0)))
    out = np.zeros(max(len(w), 1), np.int32)
    if lib().igo_assign_centers(w if len(w) else np.zeros(1, np.uint32), len(w),
                                c if len(c) else np.zeros(1, np.uint32), len(c), L, threads, out) != 0:
        raise ValueError("oracle assign_centers failed")
    return out[: len(w)]


def adjacency(row_ptr, cols, n: int, order_threads: int = 1):
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int64)
    cols = np.ascontiguousarray(cols, dtype=np.int32)
    nnz = int(row_ptr[-1])
    adj_ptr = np.zeros(n + 1, np.int64)
    adj = np.zeros(max(2 * nnz, 1), np.int32)
    lib().igo_adjacency(row_ptr, cols if len(cols) else np.zeros(1, np.int32), n, order_threads, adj_ptr, adj)
    return adj_ptr, adj[: 2 * nnz]


def greedy(adj_ptr, adj, n: int) -> np.ndarray:
    adj_ptr = np.ascontiguousarray(adj_ptr, dtype=np.int64)
    adj = np.ascontiguousarray(adj, dtype=np.int32)
    order = np.zeros(max(n, 1), np.int32)
    cnt = lib().igo_greedy(adj_ptr, adj if len(adj) else np.zeros(1, np.int32), n, order)
    return order[:cnt]


def codebook(row_ptr, cols, n: int, order_threads: int = 1) -> np.ndarray:
    ap, a = adjacency(row_ptr, cols, n, order_threads)
    return greedy(ap, a, n)


def pairs_from_csr(row_ptr, cols) -> np.ndarray:
    """(u, v) int32 pairs, u < v, rows ascending: the reference's binary edge-file layout."""
    row_ptr = np.asarray(row_ptr, dtype=np.int64)
    rows = np.repeat(np.arange(len(row_ptr) - 1, dtype=np.int32), np.diff(row_ptr))
    return np.stack([rows, np.asarray(cols, dtype=np.int32)], axis=1)


_M64 = (1 << 64) - 1


def _splitmix64(state):
    state = (state + 0x9E3779B97F4A7C15) & _M64
    z = state
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
    return state, z ^ (z >> 31)


def pick_centres(n: int, k: int, seed: int, iteration: int) -> np.ndarray:
    """First k entries of a splitmix64-driven partial Fisher-Yates shuffle of
    range(n), state seed ^ iteration * 0xD1B54A32D192ED03 (the library's
    stand-in for RandomCluster's std::random_device shuffle)."""
    idx = np.arange(n, dtype=np.int64)
    x = (seed ^ ((iteration * 0xD1B54A32D192ED03) & _M64)) & _M64
    for i in range(k):
        x, r = _splitmix64(x)
        j = i + r % (n - i)
        idx[i], idx[j] = idx[j], idx[i]
    return idx[:k]


def cluster_solve(words, L: int, min_ed: int, k: int, converge_iters: int = 3, seed: int = 0, max_iters: int = 50):
    """The iterative clustered solve of src/SparseMat.cpp:920-1095 with
    random_cluster (RandomCluster.cpp:42-136), restated on the oracle's
    assignment, edge set and greedy: (codebook ids into words, sizes)."""
    w = np.ascontiguousarray(words, dtype=np.uint32)
    cur = np.arange(len(w), dtype=np.int64)
    sizes = []
    it = 0
    while len(cur) and it < max_iters:
        it += 1
        N = len(cur)
        eff_k = k
        if eff_k > 0 and N // eff_k > 200000:
            eff_k = max(2, (N + 199999) // 200000)
        if eff_k > 0:
            kk = min(eff_k, N)
            cen = w[cur[pick_centres(N, kk, seed, it)]]
            asg = assign_centers(w[cur], cen, L)
        else:
            kk = 1
            asg = np.zeros(N, np.int32)
        nxt = []
        for c in range(kk):
            members = cur[asg == c]
            if len(members) == 0:
                continue
            rp, cols = conflict_upper(w[members], L, min_ed)
            nxt.extend(members[codebook(rp, cols, len(members), 1)].tolist())
        sizes.append(len(nxt))
        cur = np.asarray(nxt, dtype=np.int64)
        if converge_iters >= 0 and len(sizes) >= converge_iters and \
                all(sizes[-1] == sizes[-1 - c] for c in range(1, converge_iters)):
            break
    return cur.astype(np.int32), np.asarray(sizes, np.int64)
