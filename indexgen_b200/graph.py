"""Python host API over libindexgen_cuda, mirroring the reference's GPU path.

Reference interface this mirrors (same names, argument meaning, errors):

* ``pack_sequences(strings)``                 src/cuda_edit_distance.py:246-255
* ``solve_edit_distance_cuda(strings, threshold, tile_size, max_gpu_memory_gb)``
                                              src/cuda_edit_distance.py:278-446
  returns the adjacency lists (both directions; here in ascending order).
* ``fill_adj_list_gpu(candidates, min_ed, ...)`` FillAdjListGPU, src/SparseMat.cpp:454-534:
  the conflict graph and matrixOnesNum (= 2 * edges).
* ``solve_independent_set(candidates, min_ed, thread_num)``
                                              SolveIndependentSet, src/SparseMat.cpp:784-851
* ``verify_dist(codebook, min_ed)``          VerifyDist GPU branch, src/Utils.cpp:203-288
* ``apply_filters(words, L, ...)``           CandidateGenerator::applyFilters, src/CandidateGenerator.cpp:24-50
* ``solve_assignments_cuda(vectors, centers, batch_size)``
                                              src/gpu_cluster.py:239-300 (nearest centre, np.argmin ties)
* ``random_cluster_fit(data, k, seed)``      RandomCluster::fit, src/clustering/impl/random_cluster/RandomCluster.cpp:42-136
* ``cluster_solve(words, L, min_ed, k, ...)`` the iterative clustered solve, src/SparseMat.cpp:920-1095

All device work goes through the C ABI; nothing here computes a distance.
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

from . import _lib
from ._lib import IndexGenError, check, lib, ptr


class Context:
    """One device, one CUDA stream, a reusable HBM workspace (ig_ctx)."""

    def __init__(self, device: int = 0):
        h = ctypes.c_void_p()
        check(lib().ig_ctx_create(ctypes.byref(h), int(device)), "ig_ctx_create")
        self.handle = h
        self.device = int(device)

    @property
    def stream(self) -> int:
        s = ctypes.c_void_p()
        check(lib().ig_ctx_stream(self.handle, ctypes.byref(s)), "ig_ctx_stream", self.handle)
        return int(s.value or 0)

    @property
    def launches(self) -> int:
        return int(lib().ig_ctx_launches(self.handle))

    def set_profiling(self, enable: bool):
        check(lib().ig_ctx_set_profiling(self.handle, int(bool(enable))), "ig_ctx_set_profiling", self.handle)

    def phase_time(self, phase: int):
        """(milliseconds, launches) accumulated for IG_PHASE_{PAIRS=0, COMPACT=1, PREP=2}."""
        ms = ctypes.c_double()
        n = ctypes.c_int64()
        check(lib().ig_ctx_phase_time(self.handle, int(phase), ctypes.byref(ms), ctypes.byref(n)),
              "ig_ctx_phase_time", self.handle)
        return float(ms.value), int(n.value)

    def reserve(self, edges: int):
        check(lib().ig_ctx_reserve(self.handle, int(edges)), "ig_ctx_reserve", self.handle)

    def autotune(self, words, L: int, min_ed: int) -> int:
        """Time the work-split candidates on this job (host words, or a
        device tensor on this context's GPU) and keep the fastest for its lane
        form; returns the chosen items per CTA (ig_ctx_autotune)."""
        got = ctypes.c_int32()
        if hasattr(words, "data_ptr") and getattr(words, "is_cuda", False):
            wptr, n, on_dev = ctypes.c_void_p(words.data_ptr()), int(words.numel()), 1
        else:
            w = _words_array(words)
            wptr, n, on_dev = ptr(w), len(w), 0
        check(lib().ig_ctx_autotune(self.handle, wptr, n, int(L), int(min_ed), on_dev, ctypes.byref(got)),
              "ig_ctx_autotune", self.handle)
        return int(got.value)

    def set_work_split(self, lane_form: int, items_per_cta: int):
        """Pin a lane form's split (IG_LANES_FULL=0, NIBBLE=1, BYTE=2)."""
        check(lib().ig_ctx_set_work_split(self.handle, int(lane_form), int(items_per_cta)),
              "ig_ctx_set_work_split", self.handle)

    def work_split(self, lane_form: int):
        """(items per CTA, tuned-or-pinned) of a lane form."""
        v = ctypes.c_int32()
        t = ctypes.c_int()
        check(lib().ig_ctx_work_split(self.handle, int(lane_form), ctypes.byref(v), ctypes.byref(t)),
              "ig_ctx_work_split", self.handle)
        return int(v.value), bool(t.value)

    def set_graphs(self, enable: bool):
        """Run builds as captured CUDA graphs (default) or as direct launches."""
        check(lib().ig_ctx_set_graphs(self.handle, int(bool(enable))), "ig_ctx_set_graphs", self.handle)

    def graph_stats(self):
        """(graph launches, instantiations, in-place updates) so far."""
        v = [ctypes.c_int64() for _ in range(3)]
        check(lib().ig_ctx_graph_stats(self.handle, *[ctypes.byref(x) for x in v]), "ig_ctx_graph_stats",
              self.handle)
        return tuple(int(x.value) for x in v)

    def set_coalescing(self, enable: bool):
        """Build concurrent solve() calls on this context together (default)."""
        check(lib().ig_ctx_set_coalescing(self.handle, int(bool(enable))), "ig_ctx_set_coalescing", self.handle)

    def coalesce_stats(self):
        """(batches, solve calls) that went through the combiner."""
        b, r = ctypes.c_int64(), ctypes.c_int64()
        check(lib().ig_ctx_coalesce_stats(self.handle, ctypes.byref(b), ctypes.byref(r)), "ig_ctx_coalesce_stats",
              self.handle)
        return int(b.value), int(r.value)

    @property
    def device_allocs(self) -> int:
        """Device allocations this context has asked for so far."""
        k = ctypes.c_int64()
        check(lib().ig_ctx_alloc_stats(self.handle, ctypes.byref(k)), "ig_ctx_alloc_stats")
        return int(k.value)

    def set_host_lists(self, form: int):
        """Form of the lists sent to the host greedy: LISTS_AUTO, LISTS_PLAIN or LISTS_PACKED."""
        check(lib().ig_ctx_set_host_lists(self.handle, int(form)), "ig_ctx_set_host_lists", self.handle)

    def set_host_budget(self, nbytes: int):
        """Host memory downloaded graphs may hold at once (0 = half of RAM)."""
        check(lib().ig_ctx_set_host_budget(self.handle, int(nbytes)), "ig_ctx_set_host_budget", self.handle)

    def host_budget(self):
        """(limit, bytes held now) of the host budget."""
        lim = ctypes.c_int64()
        used = ctypes.c_int64()
        check(lib().ig_ctx_host_budget(self.handle, ctypes.byref(lim), ctypes.byref(used)), "ig_ctx_host_budget")
        return int(lim.value), int(used.value)

    def set_wait_limit(self, cycles: int):
        """Bound on the pair kernels' device waits (SM cycles; 0 = default)."""
        check(lib().ig_ctx_set_wait_limit(self.handle, int(cycles)), "ig_ctx_set_wait_limit", self.handle)

    def inject_fault(self, kind: int, arg: int = 0):
        """Arm a one-shot failure for a test (FAULT_DEVICE_ALLOC: the arg-th
        device allocation fails; FAULT_TILE_COPY: the next pair pass withholds
        one staged tile copy so its bounded wait runs out; FAULT_NONE clears)."""
        check(lib().ig_ctx_inject_fault(self.handle, int(kind), int(arg)), "ig_ctx_inject_fault", self.handle)

    def set_autotune(self, enable: bool):
        check(lib().ig_ctx_set_autotune(self.handle, int(bool(enable))), "ig_ctx_set_autotune", self.handle)

    def close(self):
        if self.handle:
            lib().ig_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default = None
_default_lock = threading.Lock()


def default_context() -> Context:
    global _default
    with _default_lock:
        if _default is None:
            _default = Context(0)
        return _default


def _words_array(words) -> np.ndarray:
    w = np.ascontiguousarray(words, dtype=np.uint32)
    if w.ndim != 1:
        raise ValueError("words must be a 1-D array of packed uint32")
    return w


class ConflictGraph:
    """A conflict graph resident in HBM as an upper CSR (ig_graph)."""

    def __init__(self, handle, ctx: Context, L: int, min_ed: int):
        self.handle = handle
        self.ctx = ctx
        self.L = L
        self.min_ed = min_ed
        n = ctypes.c_int32()
        e = ctypes.c_int64()
        check(lib().ig_graph_stats(handle, ctypes.byref(n), ctypes.byref(e)), "ig_graph_stats")
        self.n = int(n.value)
        self.edges = int(e.value)

    @property
    def matrix_ones_num(self) -> int:
        """The reference's 'Number of Ones in Matrix' (both directions)."""
        return 2 * self.edges

    def upper_csr(self):
        row_ptr = np.zeros(self.n + 1, np.int64)
        cols = np.zeros(self.edges, np.int32)
        check(lib().ig_graph_upper_csr(self.handle, ptr(row_ptr), ptr(cols)), "ig_graph_upper_csr",
              self.ctx.handle)
        return row_ptr, cols

    def pairs(self) -> np.ndarray:
        """(u, v) int32 pairs, u < v: the reference's binary edge-file layout."""
        out = np.zeros((self.edges, 2), np.int32)
        check(lib().ig_graph_pairs(self.handle, ptr(out)), "ig_graph_pairs", self.ctx.handle)
        return out

    def device_csr(self):
        rp = ctypes.c_void_p()
        cl = ctypes.c_void_p()
        check(lib().ig_graph_device_csr(self.handle, ctypes.byref(rp), ctypes.byref(cl)), "ig_graph_device_csr")
        return int(rp.value or 0), int(cl.value or 0)

    def adjacency(self):
        """Symmetric neighbour lists in the canonical (sorted) order, as CSR."""
        adj_ptr = np.zeros(self.n + 1, np.int64)
        adj = np.zeros(2 * self.edges, np.int32)
        check(lib().ig_graph_adjacency(self.handle, ptr(adj_ptr), ptr(adj)), "ig_graph_adjacency",
              self.ctx.handle)
        return adj_ptr, adj

    def codebook(self, order_threads: int = 1) -> np.ndarray:
        order = np.zeros(max(self.n, 1), np.int32)
        cnt = ctypes.c_int32()
        check(lib().ig_graph_codebook(self.handle, int(order_threads), ptr(order), ctypes.byref(cnt)),
              "ig_graph_codebook", self.ctx.handle)
        return order[: cnt.value]

    @property
    def jobs(self) -> int:
        k = ctypes.c_int32()
        check(lib().ig_graph_job_count(self.handle, ctypes.byref(k)), "ig_graph_job_count")
        return int(k.value)

    def job_stats(self, job: int):
        """(first word, n, edges) of one job of a batch graph."""
        f = ctypes.c_int64()
        n = ctypes.c_int32()
        e = ctypes.c_int64()
        check(lib().ig_graph_job_stats(self.handle, int(job), ctypes.byref(f), ctypes.byref(n), ctypes.byref(e)),
              "ig_graph_job_stats")
        return int(f.value), int(n.value), int(e.value)

    def job_tiling(self, job: int = 0):
        """(segment width, segments) of the pair pass that built one job."""
        w = ctypes.c_int32()
        k = ctypes.c_int32()
        check(lib().ig_graph_job_tiling(self.handle, int(job), ctypes.byref(w), ctypes.byref(k)),
              "ig_graph_job_tiling")
        return int(w.value), int(k.value)

    def job_codebooks(self, order_threads: int = 1, host_threads: int = 0):
        """Per-job codebooks (job-local ids in selection order), as a list."""
        k = self.jobs
        order = np.zeros(max(self.n, 1), np.int32)
        counts = np.zeros(max(k, 1), np.int32)
        check(lib().ig_graph_job_codebooks(self.handle, int(order_threads), int(host_threads), ptr(order),
                                           ptr(counts)), "ig_graph_job_codebooks", self.ctx.handle)
        out = []
        for j in range(k):
            f, _, _ = self.job_stats(j)
            out.append(order[f:f + counts[j]].copy())
        return out

    def write_adj_list(self, path) -> int:
        """Write the reference's progress_adj_list.txt for this graph
        (AdjList::ToFile format); returns the file size in bytes."""
        b = ctypes.c_int64()
        check(lib().ig_graph_write_adj_list(self.handle, os.fsencode(path), ctypes.byref(b)),
              "ig_graph_write_adj_list", self.ctx.handle)
        return int(b.value)

    def adj_list(self):
        """Neighbour lists in both directions, ascending (list of lists)."""
        adj_ptr, adj = self.adjacency()
        flat = adj.tolist()
        return [flat[adj_ptr[u]:adj_ptr[u + 1]] for u in range(self.n)]

    def close(self):
        if self.handle:
            lib().ig_graph_free(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


LANES_FULL, LANES_NIBBLE, LANES_BYTE = 0, 1, 2


FAULT_NONE, FAULT_DEVICE_ALLOC, FAULT_TILE_COPY = 0, 1, 2
LISTS_AUTO, LISTS_PLAIN, LISTS_PACKED = 0, 1, 2


def lane_form(L: int, min_ed: int) -> int:
    """Lane form of the pair kernel for (L, min_ed) (ig_lane_form)."""
    return int(lib().ig_lane_form(int(L), int(min_ed)))


def build_conflict_graph(words, L: int, min_ed: int, ctx: Context | None = None) -> ConflictGraph:
    """Conflict graph of packed words (numpy uint32, or a CUDA tensor/array
    exposing ``data_ptr()`` whose data is already on the context's device)."""
    ctx = ctx or default_context()
    h = ctypes.c_void_p()
    if hasattr(words, "data_ptr") and getattr(words, "is_cuda", False):
        n = int(words.numel())
        check(lib().ig_graph_build(ctx.handle, ctypes.c_void_p(words.data_ptr()), n, int(L), int(min_ed), 1,
                                   ctypes.byref(h)), "ig_graph_build", ctx.handle)
    else:
        w = _words_array(words)
        check(lib().ig_graph_build(ctx.handle, ptr(w), len(w), int(L), int(min_ed), 0, ctypes.byref(h)),
              "ig_graph_build", ctx.handle)
    return ConflictGraph(h, ctx, int(L), int(min_ed))


def _batch_arrays(jobs):
    """jobs: iterable of (words, L, min_ed) -> concatenated words, offsets, lens, min_eds."""
    ws, lens, eds = [], [], []
    for w, L, d in jobs:
        ws.append(_words_array(w))
        lens.append(int(L))
        eds.append(int(d))
    offsets = np.zeros(len(ws) + 1, np.int64)
    if ws:
        offsets[1:] = np.cumsum([len(w) for w in ws])
    words = np.concatenate(ws) if ws else np.zeros(0, np.uint32)
    return np.ascontiguousarray(words), offsets, np.asarray(lens, np.int32), np.asarray(eds, np.int32)


def build_batch(jobs, ctx: Context | None = None) -> ConflictGraph:
    """One block-diagonal conflict graph for a list of (words, L, min_ed) jobs,
    built by one device pipeline (one persistent pair-test launch)."""
    ctx = ctx or default_context()
    words, offsets, lens, eds = _batch_arrays(jobs)
    h = ctypes.c_void_p()
    check(lib().ig_batch_build(ctx.handle, ptr(words), ptr(offsets), len(lens), ptr(lens), ptr(eds), 0,
                               ctypes.byref(h)), "ig_batch_build", ctx.handle)
    return ConflictGraph(h, ctx, 0, 0)


def solve_batch(jobs, order_threads: int = 1, host_threads: int = 0, ctx: Context | None = None):
    """Codebooks (job-local ids in selection order) and edge counts of a batch."""
    ctx = ctx or default_context()
    words, offsets, lens, eds = _batch_arrays(jobs)
    k = len(lens)
    order = np.zeros(max(len(words), 1), np.int32)
    counts = np.zeros(max(k, 1), np.int32)
    edges = np.zeros(max(k, 1), np.int64)
    check(lib().ig_solve_batch(ctx.handle, ptr(words), ptr(offsets), k, ptr(lens), ptr(eds), int(order_threads),
                               int(host_threads), ptr(order), ptr(counts), ptr(edges)), "ig_solve_batch",
          ctx.handle)
    return [order[offsets[j]:offsets[j] + counts[j]].copy() for j in range(k)], edges[:k].copy()


def read_adj_list(path, ctx: Context | None = None) -> ConflictGraph:
    """A graph from a progress_adj_list.txt (AdjList::FromFile semantics: n =
    largest id + 1, neighbours in file order)."""
    ctx = ctx or default_context()
    h = ctypes.c_void_p()
    check(lib().ig_graph_read_adj_list(ctx.handle, os.fsencode(path), ctypes.byref(h)), "ig_graph_read_adj_list",
          ctx.handle)
    return ConflictGraph(h, ctx, 0, 0)


def count_conflicts(words, L: int, min_ed: int, ctx: Context | None = None) -> int:
    ctx = ctx or default_context()
    w = _words_array(words)
    e = ctypes.c_int64()
    check(lib().ig_count_conflicts(ctx.handle, ptr(w), len(w), int(L), int(min_ed), ctypes.byref(e)),
          "ig_count_conflicts", ctx.handle)
    return int(e.value)


def assign_centers(words, centers, L: int, ctx: Context | None = None):
    """Index of the nearest centre of every word (Levenshtein, ties to the
    lowest index): int32 array, or a CUDA int32 tensor when the words are a
    CUDA tensor (the centres are then moved to the same device)."""
    ctx = ctx or default_context()
    if hasattr(words, "data_ptr") and getattr(words, "is_cuda", False):
        import torch

        c = centers if getattr(centers, "is_cuda", False) else torch.as_tensor(
            np.ascontiguousarray(centers, dtype=np.uint32).view(np.int32), device=words.device)
        out = torch.empty(words.numel(), dtype=torch.int32, device=words.device)
        check(lib().ig_assign_centers(ctx.handle, ctypes.c_void_p(words.data_ptr()), words.numel(),
                                      ctypes.c_void_p(c.data_ptr()), c.numel(), int(L), 1,
                                      ctypes.c_void_p(out.data_ptr())), "ig_assign_centers", ctx.handle)
        return out
    w = _words_array(words)
    c = _words_array(centers)
    out = np.zeros(max(len(w), 1), np.int32)
    check(lib().ig_assign_centers(ctx.handle, ptr(w), len(w), ptr(c), len(c), int(L), 0, ptr(out)),
          "ig_assign_centers", ctx.handle)
    return out[: len(w)]


def codebook_from_adjacency(adj_ptr, adj, n: int) -> np.ndarray:
    """Greedy codebook over host neighbour lists taken in the given order
    (the reference's AdjList::m, e.g. ConflictGraph.adjacency())."""
    ap = np.ascontiguousarray(adj_ptr, dtype=np.int64)
    a = np.ascontiguousarray(adj, dtype=np.int32)
    order = np.zeros(max(int(n), 1), np.int32)
    cnt = ctypes.c_int32()
    check(lib().ig_codebook_from_adjacency(ptr(ap), ptr(a), int(n), ptr(order), ctypes.byref(cnt)),
          "ig_codebook_from_adjacency")
    return order[: cnt.value].copy()


def set_greedy_threads(max_helpers: int = -1, min_entries: int = -1) -> None:
    """Process-wide threading of the host greedy: a greedy over a graph with at
    least `min_entries` neighbour-list entries runs on two threads while fewer
    than `max_helpers` helper threads are in use (defaults: 2^20 entries,
    (hardware threads - 1) // 2 helpers; 0 helpers = always one thread).  The
    codebook is the same either way."""
    check(lib().ig_set_greedy_threads(int(max_helpers), int(min_entries)), "ig_set_greedy_threads")


def greedy_stats() -> tuple:
    """(two-threaded, single-threaded) greedies run so far in this process."""
    a, b = ctypes.c_int64(), ctypes.c_int64()
    check(lib().ig_greedy_stats(ctypes.byref(a), ctypes.byref(b)), "ig_greedy_stats")
    return a.value, b.value


def codebook_from_upper_csr(row_ptr, cols, n: int, order_threads: int = 1) -> np.ndarray:
    rp = np.ascontiguousarray(row_ptr, dtype=np.int64)
    cl = np.ascontiguousarray(cols, dtype=np.int32)
    order = np.zeros(max(n, 1), np.int32)
    cnt = ctypes.c_int32()
    check(lib().ig_codebook_from_upper_csr(ptr(rp), ptr(cl), int(n), int(order_threads), ptr(order),
                                           ctypes.byref(cnt)), "ig_codebook_from_upper_csr")
    return order[: cnt.value]


def solve(words, L: int, min_ed: int, order_threads: int = 1, ctx: Context | None = None):
    """Graph + greedy in one call: (selected ids in order, edges)."""
    ctx = ctx or default_context()
    w = _words_array(words)
    order = np.zeros(max(len(w), 1), np.int32)
    cnt = ctypes.c_int32()
    e = ctypes.c_int64()
    check(lib().ig_solve(ctx.handle, ptr(w), len(w), int(L), int(min_ed), int(order_threads), ptr(order),
                         ctypes.byref(cnt), ctypes.byref(e)), "ig_solve", ctx.handle)
    return order[: cnt.value], int(e.value)


class Server:
    """Continuous-batching codebook server (ig_server_*): submit jobs from any
    thread, wait for their codebooks.  Each result equals solve() of the job
    alone."""

    STATES = ("queued", "on_device", "greedy", "done", "cancelled", "failed")

    def __init__(self, ctx: Context | None = None, host_threads: int = 0, max_batch_jobs: int = 0,
                 max_batch_pairs: int = 0, hbm_budget_bytes: int = 0, order_threads: int = 1,
                 pool_reserve_bytes: int = 0):
        self.ctx = ctx or default_context()
        o = _lib.ServerOpts(host_threads, max_batch_jobs, order_threads, 0, max_batch_pairs, hbm_budget_bytes,
                            pool_reserve_bytes)
        h = ctypes.c_void_p()
        check(lib().ig_server_create(self.ctx.handle, ctypes.byref(o), ctypes.byref(h)), "ig_server_create",
              self.ctx.handle)
        self.handle = h
        self._n = {}

    def submit(self, words, L: int, min_ed: int) -> int:
        w = _words_array(words)
        t = ctypes.c_int64()
        check(lib().ig_server_submit(self.handle, ptr(w), len(w), int(L), int(min_ed), ctypes.byref(t)),
              "ig_server_submit")
        self._n[t.value] = len(w)
        return int(t.value)

    def poll(self, ticket: int) -> str:
        st = ctypes.c_int()
        check(lib().ig_server_poll(self.handle, int(ticket), ctypes.byref(st)), "ig_server_poll")
        return self.STATES[st.value]

    def wait(self, ticket: int):
        """(codebook ids in selection order, edges, latency_ms)."""
        n = self._n.pop(ticket, 0)
        order = np.zeros(max(n, 1), np.int32)
        cnt = ctypes.c_int32()
        e = ctypes.c_int64()
        lat = ctypes.c_double()
        check(lib().ig_server_wait(self.handle, int(ticket), ptr(order), ctypes.byref(cnt), ctypes.byref(e),
                                   ctypes.byref(lat)), "ig_server_wait")
        return order[: cnt.value].copy(), int(e.value), float(lat.value)

    def cancel(self, ticket: int) -> bool:
        """True if the job was still queued and is now cancelled."""
        st = lib().ig_server_cancel(self.handle, int(ticket))
        if st == 7:  # IG_ERR_STATE: already running
            return False
        check(st, "ig_server_cancel")
        return True

    def stats(self):
        b = ctypes.c_int64()
        c = ctypes.c_int64()
        m = ctypes.c_int64()
        check(lib().ig_server_stats(self.handle, ctypes.byref(b), ctypes.byref(c), ctypes.byref(m)),
              "ig_server_stats")
        return {"batches": int(b.value), "completed": int(c.value), "max_batch_jobs": int(m.value)}

    def close(self):
        if self.handle:
            lib().ig_server_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Reference-named entry points
# ---------------------------------------------------------------------------

def pack_sequences(strings):
    """Strings over '0'..'3' -> (packed words, L, N).  Mirrors
    src/cuda_edit_distance.py:246-255 (which returns flat uint8 symbols); the
    words here hold 2 bits per symbol.  Raises ValueError on a bad symbol or
    ragged lengths, as the reference does for L > 32."""
    N = len(strings)
    if N == 0:
        return np.zeros(0, np.uint32), 0, 0
    L = len(strings[0])
    if L > _lib_max_len():
        raise ValueError(f"[GPU] This kernel only supports lengths <= {_lib_max_len()}.")
    if any(len(s) != L for s in strings):
        raise ValueError("all candidates must have the same length")
    raw = "".join(strings).encode("latin1")
    out = np.zeros(N, np.uint32)
    bad = ctypes.c_int64(-1)
    st = lib().ig_pack(raw, N, L, L, ptr(out), ctypes.byref(bad))
    if st != 0:
        raise ValueError(f"candidate {bad.value} is not a string over '0'..'3'")
    return out, L, N


def _lib_max_len() -> int:
    return 16


def apply_filters(words, L: int, max_run: int, min_gc: float, max_gc: float) -> np.ndarray:
    w = _words_array(words)
    keep = np.zeros(len(w), np.uint8)
    check(lib().ig_filter(ptr(w), len(w), int(L), int(max_run), float(min_gc), float(max_gc), ptr(keep)),
          "ig_filter")
    return keep.astype(bool)


def solve_edit_distance_cuda(strings, threshold, tile_size=16384, max_gpu_memory_gb=9.0, ctx=None):
    """Adjacency lists of the ED < threshold graph (list of lists, both
    directions).  tile_size / max_gpu_memory_gb are accepted for interface
    parity; the library schedules its own tiles and sizes its workspace."""
    if len(strings) == 0:
        return []
    words, L, _ = pack_sequences(strings)
    with build_conflict_graph(words, L, int(threshold), ctx) as g:
        return g.adj_list()


def solve_assignments_cuda(vectors, centers, batch_size=32768, ctx=None):
    """Mirror of src/gpu_cluster.py:239-300: the nearest centre (np.argmin
    order: lowest index on ties) of every vector, int32.  batch_size is
    accepted for interface parity; the kernel needs no distance matrix."""
    K, N = len(centers), len(vectors)
    if N == 0 or K == 0:
        return np.array([], dtype=np.int32)
    vw, Lv, _ = pack_sequences(list(vectors))
    cw, Lc, _ = pack_sequences(list(centers))
    if Lv != Lc:
        raise ValueError("Length mismatch between vectors and centers.")
    return assign_centers(vw, cw, Lv, ctx)


def random_cluster_fit(data, k: int, seed: int, ctx=None):
    """RandomCluster::fit (src/clustering/impl/random_cluster/RandomCluster.cpp:
    42-136): k distinct random candidates become the centres, every candidate
    joins its nearest centre, clusters keep candidate order, empty clusters are
    dropped.  The reference seeds its shuffle from std::random_device; here the
    shuffle is numpy's, seeded, so runs repeat."""
    data = list(data)
    if not data:
        return []
    if k <= 0:
        return [data]
    kk = min(k, len(data))
    idx = np.random.default_rng(seed).permutation(len(data))[:kk]
    a = solve_assignments_cuda(data, [data[i] for i in idx], ctx=ctx)
    clusters = [[] for _ in range(kk)]
    for s, c in zip(data, a.tolist()):
        clusters[c if 0 <= c < kk else 0].append(s)
    return [c for c in clusters if c]


def cluster_centres(n: int, k: int, seed: int, iteration: int) -> np.ndarray:
    """Indices (into the current candidates) of the centres ig_cluster_solve
    takes in iteration `iteration` (1-based): the first k entries of a
    splitmix64-driven partial Fisher-Yates shuffle of range(n), state
    seed ^ iteration * 0xD1B54A32D192ED03."""
    m64 = (1 << 64) - 1
    idx = np.arange(n, dtype=np.int64)
    x = (int(seed) ^ ((int(iteration) * 0xD1B54A32D192ED03) & m64)) & m64
    for i in range(int(k)):
        x = (x + 0x9E3779B97F4A7C15) & m64
        z = x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m64
        z ^= z >> 31
        j = i + z % (n - i)
        idx[i], idx[j] = idx[j], idx[i]
    return idx[:k]


def cluster_solve(words, L: int, min_ed: int, k: int, converge_iters: int = 3, seed: int = 0,
                  max_iters: int = 50, host_threads: int = 0, ctx: Context | None = None):
    """Iterative clustered solve with random_cluster (src/SparseMat.cpp:920-1095)
    with the words resident on the device: (codebook ids into words, sizes
    after each iteration)."""
    ctx = ctx or default_context()
    w = _words_array(words)
    book = np.zeros(max(len(w), 1), np.int32)
    sizes = np.zeros(max(int(max_iters), 1), np.int64)
    cnt = ctypes.c_int32()
    it = ctypes.c_int32()
    check(lib().ig_cluster_solve(ctx.handle, ptr(w), len(w), int(L), int(min_ed), int(k), int(converge_iters),
                                 int(seed) & ((1 << 64) - 1), int(max_iters), int(host_threads), ptr(book),
                                 ctypes.byref(cnt), ctypes.byref(it), ptr(sizes)), "ig_cluster_solve", ctx.handle)
    return book[: cnt.value], sizes[: it.value]


def fill_adj_list_gpu(candidates, min_ed: int, ctx=None):
    """FillAdjListGPU: returns (ConflictGraph, matrixOnesNum)."""
    words, L, _ = pack_sequences(list(candidates))
    g = build_conflict_graph(words, max(L, 1), int(min_ed), ctx)
    return g, g.matrix_ones_num


def solve_independent_set(candidates, min_ed: int, thread_num: int = 1, ctx=None):
    """SolveIndependentSet: the codebook strings in selection order.
    thread_num selects the neighbour order of the reference's FillAdjList
    with that many threads (1 = the sorted order of the GPU-path loader)."""
    cands = list(candidates)
    if len(cands) == 0:
        return []
    if len(cands) == 1:
        return cands
    words, L, _ = pack_sequences(cands)
    order, _ = solve(words, L, min_ed, thread_num, ctx)
    return [cands[i] for i in order.tolist()]


def verify_dist(vecs, min_ed: int, ctx=None) -> bool:
    """True iff no pair of `vecs` is closer than min_ed."""
    if len(vecs) < 2:
        return True
    words, L, _ = pack_sequences(list(vecs))
    return count_conflicts(words, L, min_ed, ctx) == 0


__all__ = [
    "Context", "ConflictGraph", "IndexGenError", "Server", "FAULT_NONE", "FAULT_DEVICE_ALLOC", "FAULT_TILE_COPY", "LISTS_AUTO", "LISTS_PLAIN",
    "LISTS_PACKED", "build_conflict_graph", "build_batch", "solve_batch",
    "count_conflicts",
    "codebook_from_upper_csr", "codebook_from_adjacency", "solve", "pack_sequences", "apply_filters", "solve_edit_distance_cuda",
    "fill_adj_list_gpu", "solve_independent_set", "verify_dist", "default_context", "assign_centers",
    "solve_assignments_cuda", "random_cluster_fit", "cluster_solve", "cluster_centres", "read_adj_list",
]
