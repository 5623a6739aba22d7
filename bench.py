#!/usr/bin/env python
"""Benchmark of the conflict-graph hot path: ED pair tests per second.

One step = build the conflict graph of one job (all pairs i<j, edge iff
Levenshtein < editDist) into an upper CSR in HBM.  Default workload: the single
large job -- all 262,144 codewords of the GF(4) [12,9,3] code plus the seeded
coset vector, filtered (maxRun 3, GC [0.3,0.7]) to 207,432 words, editDist 4:
21.5e9 pair tests and 18.6e6 edges per step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

* value     -- pair tests/s with the words already in HBM (device timeline,
               CUDA events on the library's stream; L2 flushed between steps).
* e2e       -- the same metric through the public API with host buffers: each
               step uploads the words from pinned memory and downloads the CSR
               into pinned memory (wall clock around the synchronous calls).
* roofline  -- the pair-test kernel against the ALU-pipe peak (SMs x 64
               LOP3/PRMT lanes x max SM clock); algorithmic work = the ALU-pipe
               ops the lane recurrence issues per pair test (alu_ops_per_pair),
               measured traffic from the committed ncu summary.  The 16*L
               integer-op convention against the INT32 peak is reported beside
               it (int_ops_16L_convention).
* batch / serve -- clustered batch (64 jobs) and a Poisson serving stream,
               each against the plain one-job-per-call path, same codebooks.
* cpu_baseline -- the reference's own CPU FillAdjList (oracle/_ref, built from
               the reference sources) on all host cores, on a seeded sample.
* --impl reference -- times only that reference CPU path (rank 0).
Multi-GPU: every rank solves its own replica (the path has no exchange step);
value = all ranks' pair tests / max-over-ranks time ("weak" scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from indexgen_b200 import workloads as W  # noqa: E402

METRIC = "ED pair tests/s"
UNIT = "Gpair/s"
REF_DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver")


def workload(name: str):
    if name == "linear12":
        return dict(name="linear12_gf4_coset", desc="[12,9,3] GF(4) code + coset (seed 20251203), maxRun 3, "
                    "GC [0.3,0.7]", words=W.linear12_candidates(), L=12, min_ed=4)
    if name == "uniform11":
        return dict(name="uniform11", desc="20,000 uniform n=11 (seed 12345), maxRun 3, GC [0.3,0.7]",
                    words=W.uniform11_candidates(), L=11, min_ed=3)
    if name == "vt16":
        return dict(name="vt16_1M", desc="1,000,000 VT-style n=16 words (seed 16), maxRun 3, GC [0.3,0.7]",
                    words=W.vt16_words(1_000_000, seed=16), L=16, min_ed=5)
    raise SystemExit(f"unknown workload {name}")


def pairs_of(n: int) -> int:
    return n * (n - 1) // 2


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ---------------------------------------------------------------- clocks ----
class ClockSampler:
    FIELDS = ("index,pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, bus_id: str | None):
        self.bus_id = (bus_id or "").lower()
        self.proc = None
        self.lines = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
        except OSError:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.t:
            self.t.join(timeout=2)
        rows = [l.split(", ") for l in self.lines if l.count(",") >= 9]
        mine = [r for r in rows if self.bus_id and self.bus_id in r[1].lower()] or rows
        sm = [float(r[2]) for r in mine if r[2].replace(".", "").isdigit()]
        mx = [float(r[3]) for r in mine if r[3].replace(".", "").isdigit()]
        reasons = set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in mine:
            for name, v in zip(names, r[6:10]):
                if v.strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(mine)}


# ----------------------------------------------------------- cpu baseline ---
def write_strings(path, words, L):
    with open(path, "w") as f:
        f.write("\n".join(W.to_strings(words, L)) + "\n")


def ref_time(words, L, d, threads) -> dict:
    with tempfile.TemporaryDirectory() as tmp:
        p = os.path.join(tmp, "cands.txt")
        write_strings(p, words, L)
        out = subprocess.run([REF_DRIVER, "time", p, str(d), str(threads)], check=True, capture_output=True,
                             text=True, cwd=tmp).stdout
    return json.loads([l for l in out.splitlines() if l.startswith("{")][-1])


def port_time(words, L, d, threads) -> dict:
    from oracle import oracle as O

    t0 = time.perf_counter()
    rp, _ = O.conflict_upper(words, L, d, threads)
    s = time.perf_counter() - t0
    return {"N": len(words), "pairs": pairs_of(len(words)), "ones": int(2 * rp[-1]), "seconds": s,
            "threads": threads}


def cpu_sample(wl, target_s: float, seed: int = 1234):
    """Seeded random subset of the workload whose CPU build takes ~target_s."""
    words, L, d = wl["words"], wl["L"], wl["min_ed"]
    cores = host_cores()
    kind = "reference" if os.path.exists(REF_DRIVER) else "port"
    timer = ref_time if kind == "reference" else port_time
    rng = np.random.default_rng(seed)
    m0 = min(len(words), 6000)
    idx = np.sort(rng.choice(len(words), m0, replace=False))
    r0 = timer(words[idx], L, d, cores)
    rate = r0["pairs"] / max(r0["seconds"], 1e-3)
    m = int(min(len(words), max(m0, (2 * rate * target_s) ** 0.5)))
    idx = np.sort(rng.choice(len(words), m, replace=False))
    return kind, timer, words[idx], cores


def cpu_baseline(wl, target_s: float = 15.0) -> dict:
    kind, timer, sample, cores = cpu_sample(wl, target_s)
    r = timer(sample, wl["L"], wl["min_ed"], cores)
    v = r["pairs"] / r["seconds"] / 1e9
    who = "reference FillAdjList (oracle/_ref, built from the reference sources)" if kind == "reference" else \
        "C oracle port of FillAdjList"
    return {"value": v, "unit": UNIT, "cores": cores, "kind": kind,
            "sample": f"{who}: seeded random subset of {len(sample)} of the {len(wl['words'])} words "
                      f"({r['pairs']} pair tests, {r['seconds']:.2f} s, {r['ones'] // 2} edges)"}


# ------------------------------------------------------------- reference ----
def run_reference(args, wl, rank):
    if rank != 0:
        return
    kind, timer, sample, cores = cpu_sample(wl, target_s=4.0)
    for _ in range(args.warmup):
        timer(sample, wl["L"], wl["min_ed"], cores)
    secs = []
    for _ in range(args.steps):
        r = timer(sample, wl["L"], wl["min_ed"], cores)
        secs.append(r["seconds"])
    v = r["pairs"] * len(secs) / sum(secs) / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * sum(secs) / len(secs), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": wl["name"], "desc": wl["desc"], "n": len(wl["words"]), "L": wl["L"],
                   "min_ed": wl["min_ed"], "pairs_per_step": r["pairs"], "sample_n": len(sample)},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": f"seeded random subset of {len(sample)} of {len(wl['words'])} words per step "
                                   f"({r['pairs']} pair tests), FillAdjList with {cores} threads"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_reference_gpu(args, wl, rank):
    """The reference's own GPU path, unmodified: solve_edit_distance_cuda of
    src/cuda_edit_distance.py (Numba kernel compute_chunk_kernel, 16,384-square
    tiles, per-edge Python lists), installed into baseline/_ref/src by
    oracle/Makefile (target `numba`).  Timed as one call on the whole workload
    after a warm-up call on its first 2,048 words (which JIT-compiles the
    kernels); the edge count is reported beside the rate, since the reference
    drops edges past 5,000,000 per tile (src/cuda_edit_distance.py:401-402)."""
    if rank != 0:
        return
    src = os.path.join(ROOT, "baseline", "_ref", "src")
    base = {"impl": "reference_gpu", "metric": METRIC, "unit": UNIT, "config": {"workload": wl["name"]}}
    if not os.path.exists(os.path.join(src, "cuda_edit_distance.py")):
        print(json.dumps({**base, "unavailable": "baseline/_ref/src holds no reference GPU path "
                                                  "(make -C oracle numba REF=<reference checkout>)"}), flush=True)
        return
    sys.path.insert(0, src)
    try:
        import cuda_edit_distance as R  # the reference's module
    except Exception as e:  # numba or its CUDA binding missing
        print(json.dumps({**base, "unavailable": f"import failed: {e!r}"[:300]}), flush=True)
        return
    L, d = wl["L"], wl["min_ed"]
    strings = W.to_strings(wl["words"], L)
    try:
        t0 = time.perf_counter()
        R.solve_edit_distance_cuda(strings[:2048], d)
        t_warm = time.perf_counter() - t0
        t0 = time.perf_counter()
        adj = R.solve_edit_distance_cuda(strings, d)
        secs = time.perf_counter() - t0
    except Exception as e:
        print(json.dumps({**base, "unavailable": f"the reference GPU path failed: {e!r}"[:300]}), flush=True)
        return
    n = len(strings)
    edges = sum(len(a) for a in adj) // 2
    pairs = n * (n - 1) // 2
    line = {**base, "value": pairs / secs / 1e9, "n_gpus": 1, "steps": 1, "warmup": 1, "ms_per_step": 1e3 * secs,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": wl["name"], "desc": wl["desc"], "n": n, "L": L, "min_ed": d, "pairs_per_step": pairs},
            "edges": edges, "warmup_call_s": t_warm,
            "note": "solve_edit_distance_cuda(strings, editDist) with its defaults (tile 16384, 9 GB), wall clock: "
                    "host preparation, kernels, per-tile 40 MB edge-buffer copies and the per-edge Python lists"}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ ours ----
def profile_traffic(wl_name):
    """dram bytes per pair-kernel launch from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", f"pair_kernel_{wl_name}.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1])
            except ValueError:
                return None
    return None


def profile_path_traffic(wl_name):
    """dram bytes per build of the whole device path (pair kernel, row
    prefix, scan, scatter) from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", f"compaction_{wl_name}.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("path_traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1])
            except ValueError:
                return None
    return None


def path_traffic_line(wl_name, edges: int, n: int):
    """The device path's measured DRAM bytes per build against 16 B per edge
    + 20 B per row (each edge written once as a record and read once)."""
    t = profile_path_traffic(wl_name)
    plan = 16 * edges + 20 * n
    return {"bytes_per_build": t, "bytes_per_edge": (t / edges) if t and edges else None,
            "plan_bytes_16E_20N": plan, "ratio_to_plan": (t / plan) if t else None,
            "source": f"profiles/compaction_{wl_name}.md (ncu dram__bytes_read + write, pair kernel to scatter)"}


def touched_cells(n: int, seg_width: int, segments: int, band_rows: int = 256) -> int:
    """(row, segment) count cells the pair kernel writes and the compaction
    reads: a row's cells run from its band's first segment on (band_rows-row
    bands, segments of seg_width columns, upper triangle only)."""
    bands = np.arange((n + band_rows - 1) // band_rows, dtype=np.int64)
    rows = np.minimum(band_rows, n - bands * band_rows)
    first = (bands * band_rows) // seg_width
    return int(np.sum(rows * np.maximum(segments - first, 0)))


def alu_ops_per_pair(L: int, d: int) -> float:
    """ALU-pipe operations (LOP3, PRMT, the add and the shift) the pair-test
    recurrence issues per pair test, counted from the kernel source (the lane
    counter runs as an IMAD on the FMA pipe and is not counted).  Banded
    8-lane form (two rows x four columns, editDist <= 4): 11 per character
    step for 8 pairs, 5 fewer in the last step (its vertical deltas are not
    needed), 3 per nibble-counter flush (every 7 steps and at the end) and 4
    for the threshold.  4-lane form (editDist 5..8): 11 per step for 4 pairs,
    5 fewer in the last step, 2 for the threshold.  Full Myers: 8 per step
    for 2 pairs (L <= 15) or for 1."""
    if 1 <= d <= 4:
        return (11.0 * L - 5 + 3 * -(-L // 7) + 4) / 8
    if 5 <= d <= 8:
        return (11.0 * L - 5 + 2) / 4
    return 8.0 / 2 * L if L <= 15 else 8.0 * L


def max_over_ranks(x: float, dist, device: str) -> float:
    """The largest value of x over all ranks (x itself without a process group)."""
    if not dist:
        return x
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(world: int, units_per_rank: int, steps: int, seconds: float) -> float:
    """Whole-job rate in G units/s: every rank processes its own replica."""
    return world * units_per_rank * steps / seconds / 1e9


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return json.load(open(p)), "measured"
    return {"hbm_gbs": 6650.0, "sm_max_mhz": 1965.0}, "fallback"


def run_batch_section(ctx, reps: int = 6) -> dict:
    """Batched clusters (1,000,000 filtered uniform n=14 words, 64 clusters with
    Zipf(1.1) sizes in [2k, 60k], editDist 4): the whole batch as one device
    pipeline + per-cluster greedies on all host cores, against the plain path
    that solves the clusters one after another (one graph build + one greedy
    per cluster).  Both through the public API with host buffers."""
    from indexgen_b200 import solve, solve_batch

    parts = W.clustered14()
    jobs = [(w, 14, 4) for w in parts]
    pairs = sum(len(w) * (len(w) - 1) // 2 for w in parts)
    cores = host_cores()
    books, edges = solve_batch(jobs, host_threads=cores, ctx=ctx)  # warm-up (workspace growth)
    # captured CUDA graphs (the default) and direct launches, alternated so
    # that neither side gets the warmer host
    t_batch, t_direct = [], []
    for _ in range(reps + 1):
        for graphs, out in ((True, t_batch), (False, t_direct)):
            ctx.set_graphs(graphs)
            t0 = time.perf_counter()
            b, e = solve_batch(jobs, host_threads=cores, ctx=ctx)
            out.append(time.perf_counter() - t0)
            if graphs:
                books, edges = b, e
    ctx.set_graphs(True)
    # one more pass with per-phase events (they add syncs, so it is not timed)
    ctx.set_profiling(True)
    solve_batch(jobs, host_threads=cores, ctx=ctx)
    pair_ms, pair_launches = ctx.phase_time(0)  # all pair-kernel launches of that pass
    ctx.set_profiling(False)
    solve(jobs[0][0], 14, 4, 1, ctx)  # warm-up
    t0 = time.perf_counter()
    plain_books = []
    for w, L, d in jobs:
        plain_books.append(solve(w, L, d, 1, ctx)[0])
    t_plain = time.perf_counter() - t0

    # the reference host's pattern: a pool of worker threads, each calling
    # solve() per cluster on one shared context (concurrent calls coalesced
    # into batches by the library, then without that)
    def threaded(coalesce: bool) -> float:
        import threading

        ctx.set_coalescing(coalesce)
        nxt = iter(range(len(jobs)))
        lock = threading.Lock()
        out = [None] * len(jobs)

        def worker():
            while True:
                with lock:
                    j = next(nxt, None)
                if j is None:
                    return
                w, L, d = jobs[j]
                out[j] = solve(w, L, d, 1, ctx)[0]

        th = [threading.Thread(target=worker) for _ in range(cores)]
        t0 = time.perf_counter()
        for t in th:
            t.start()
        for t in th:
            t.join()
        dt = time.perf_counter() - t0
        ctx.set_coalescing(True)
        assert all(np.array_equal(a, b) for a, b in zip(out, plain_books))
        return dt

    t_thr = min(threaded(True) for _ in range(3))
    t_thr_off = min(threaded(False) for _ in range(3))
    same = all(np.array_equal(a, b) for a, b in zip(books, plain_books))
    tb = min(t_batch)
    return {"workload": "clusters64_n14_d4 (1,000,000 uniform n=14 words, 64 Zipf(1.1) clusters in [2k,60k])",
            "jobs": len(jobs), "pair_tests": pairs, "edges": int(np.sum(edges)),
            "codebook_words": int(sum(len(b) for b in books)),
            "batched_jobs_per_s": len(jobs) / tb, "batched_s": tb,
            "batched_direct_launches_jobs_per_s": len(jobs) / min(t_direct),
            "work_split_items_per_cta": ctx.work_split(1)[0], "work_split_tuned": ctx.work_split(1)[1],
            "plain_jobs_per_s": len(jobs) / t_plain, "plain_s": t_plain,
            "speedup_vs_plain": t_plain / tb,
            "threaded_solve_jobs_per_s": len(jobs) / t_thr,
            "threaded_solve_uncoalesced_jobs_per_s": len(jobs) / t_thr_off,
            "batched_pair_kernel_gpairs_per_s": (pairs / (pair_ms / 1e3) / 1e9) if pair_ms else None,
            "host_threads": cores, "identical_to_plain": bool(same),
            # the plain loop is one thread; the split below separates what
            # host threads give from what device batching gives
            "gain_split": {"host_threading": t_plain / t_thr_off,
                           "device_batching_vs_uncoalesced_threads": t_thr_off / tb,
                           "device_batching_vs_coalesced_threads": t_thr / tb,
                           "note": "plain loop (1 thread) -> 16 threads calling solve one job per launch -> "
                                   "solve_batch; the factors multiply to speedup_vs_plain"},
            "note": "wall clock through solve_batch vs a loop of solve (graph + greedy per cluster)"}


def run_assign_section(ctx, reps: int = 5) -> dict:
    """random_cluster's assignment step (src/gpu_cluster.py): 1,000,000
    filtered uniform n=14 words against 64 seeded random centres, nearest
    centre each.  Device rate (words resident, CUDA events on the library
    stream), end to end with host buffers, and the C oracle on all host cores
    on a 20,000-word sample of the same job (results compared)."""
    import ctypes

    import torch

    from indexgen_b200 import assign_centers
    from indexgen_b200._lib import check, lib
    from oracle import oracle as O

    L, K = 14, 64
    w = W.uniform_until(1_000_000, L, 14, max_run=3, min_gc=0.3, max_gc=0.7)
    c = w[np.random.default_rng(64).choice(len(w), K, replace=False)]
    dw = torch.from_numpy(w.view(np.int32)).cuda()
    dc = torch.from_numpy(c.view(np.int32)).cuda()
    out = torch.empty(len(w), dtype=torch.int32, device="cuda")
    ext = torch.cuda.ExternalStream(ctx.stream)

    def dev_call():
        check(lib().ig_assign_centers(ctx.handle, ctypes.c_void_p(dw.data_ptr()), len(w),
                                      ctypes.c_void_p(dc.data_ptr()), K, L, 1, ctypes.c_void_p(out.data_ptr())),
              "ig_assign_centers", ctx.handle)

    for _ in range(3):
        dev_call()
    ms = []
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        dev_call()
        e1.record(ext)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    dist = len(w) * K
    t0 = time.perf_counter()
    for _ in range(reps):
        host = assign_centers(w, c, L, ctx)
    e2e_s = (time.perf_counter() - t0) / reps
    sample = w[:20000]
    t0 = time.perf_counter()
    ref = O.assign_centers(sample, c, L)
    cpu_s = time.perf_counter() - t0
    same = bool(np.array_equal(ref, host[:20000]) and np.array_equal(out.cpu().numpy(), host))
    alu_ops = 4 * L  # two-lane Myers: 7 LOP3 + 1 PRMT per step for two distances
    peaks, _ = measured_peaks()
    dev_s = min(ms) / 1e3
    alu_peak = torch.cuda.get_device_properties(0).multi_processor_count * 64 * float(
        peaks.get("sm_max_mhz", 1965.0)) * 1e6
    return {"workload": "1,000,000 filtered uniform n=14 words, 64 random centres (seed 64)",
            "distances": dist, "device_gdist_per_s": dist / dev_s / 1e9, "device_ms": dev_s * 1e3,
            "e2e_gdist_per_s": dist / e2e_s / 1e9, "e2e_ms": e2e_s * 1e3,
            "roofline": {"bound": "int32-alu-pipe", "alu_ops_per_distance": alu_ops,
                         "frac": dist * alu_ops / dev_s / alu_peak},
            "cpu_oracle_gdist_per_s": len(sample) * K / cpu_s / 1e9, "cpu_cores": host_cores(),
            "identical_to_oracle": same}


def run_cluster_section(ctx) -> dict:
    """The iterative clustered solve (src/SparseMat.cpp:920-1095, random_cluster):
    200,000 filtered uniform n=12 words, editDist 4, k = 16, two iterations,
    resident on the device (ig_cluster_solve) against the plain flow of the
    same iterations (assignment with host buffers, then one ig_solve call per
    cluster), same centres; both must give the same codebook."""
    from indexgen_b200 import assign_centers, cluster_centres, cluster_solve, solve

    L, d, k, iters = 12, 4, 16, 2
    w = W.uniform_until(200_000, L, 1212, max_run=3, min_gc=0.3, max_gc=0.7)
    cluster_solve(w, L, d, k, converge_iters=-1, seed=5, max_iters=1, ctx=ctx)  # warm-up
    t0 = time.perf_counter()
    book, sizes = cluster_solve(w, L, d, k, converge_iters=-1, seed=5, max_iters=iters, ctx=ctx)
    t_res = time.perf_counter() - t0
    t0 = time.perf_counter()
    cur = np.arange(len(w))
    for it in range(1, iters + 1):
        cen = w[cur[cluster_centres(len(cur), min(k, len(cur)), 5, it)]]
        asg = assign_centers(w[cur], cen, L, ctx)
        nxt = []
        for cidx in range(min(k, len(cur))):
            members = cur[asg == cidx]
            if len(members):
                nxt.extend(members[solve(w[members], L, d, 1, ctx)[0]].tolist())
        cur = np.asarray(nxt)
    t_plain = time.perf_counter() - t0
    return {"workload": "200,000 filtered uniform n=12 words, editDist 4, k=16 random centres, 2 iterations",
            "resident_s": t_res, "plain_s": t_plain, "speedup": t_plain / t_res,
            "sizes": [int(x) for x in sizes], "identical_to_plain": bool(np.array_equal(book, cur))}


def run_serve_section(ctx, jobs: int, nmax: int, rate: float = 50.0) -> dict:
    """Serving stream: seeded Poisson arrivals (mean `rate` jobs/s), n uniform
    in 10..16, editDist uniform in 3..5, candidates log-uniform in [5k, nmax].
    The continuous-batching server (all host cores for greedies) against the
    plain one-job-per-launch path (one worker solving jobs in arrival order).
    Latency = arrival to codebook ready."""
    import threading

    from indexgen_b200 import Server, solve

    stream = W.serving_stream(jobs, seed=5, rate=rate, nmin=5000, nmax=nmax)
    pairs = sum(len(w) * (len(w) - 1) // 2 for _, w, _, _ in stream)
    cores = host_cores()
    # warm-up (untimed): the whole stream once through a server, so that the
    # device pool and the pinned download blocks both paths share are grown
    with Server(ctx, host_threads=cores) as sv:
        for t in [sv.submit(w, L, d) for _, w, L, d in stream]:
            sv.wait(t)

    # served
    lat = [0.0] * len(stream)
    results = [None] * len(stream)
    with Server(ctx, host_threads=cores) as sv:
        tickets = [None] * len(stream)
        t0 = time.perf_counter()

        def submitter():
            for i, (arr, w, L, d) in enumerate(stream):
                dt = arr - (time.perf_counter() - t0)
                if dt > 0:
                    time.sleep(dt)
                tickets[i] = sv.submit(w, L, d)

        th = threading.Thread(target=submitter)
        th.start()
        th.join()
        for i in range(len(stream)):
            order, _, ms = sv.wait(tickets[i])
            lat[i] = ms
            results[i] = order
        t_served = time.perf_counter() - t0
        st = sv.stats()
    # saturated: every job submitted at t=0 (server capacity)
    with Server(ctx, host_threads=cores) as sv:
        t0 = time.perf_counter()
        tk = [sv.submit(w, L, d) for _, w, L, d in stream]
        for t in tk:
            sv.wait(t)
        t_sat = time.perf_counter() - t0
    t0 = time.perf_counter()
    for _, w, L, d in stream:
        solve(w, L, d, 1, ctx)
    t_sat_plain = time.perf_counter() - t0
    # plain: one job per launch, in arrival order
    lat_plain = []
    same = True
    t0 = time.perf_counter()
    for i, (arr, w, L, d) in enumerate(stream):
        dt = arr - (time.perf_counter() - t0)
        if dt > 0:
            time.sleep(dt)
        order, _ = solve(w, L, d, 1, ctx)
        lat_plain.append(1e3 * (time.perf_counter() - t0 - arr))
        same = same and np.array_equal(order, results[i])
    t_plain = time.perf_counter() - t0
    return {"workload": f"{jobs} jobs, Poisson {rate:g}/s, n 10..16, editDist 3..5, candidates log-uniform "
                        f"[5000, {nmax}] (seed 5)",
            "pair_tests": pairs, "served_jobs_per_s": len(stream) / t_served,
            "served_p50_ms": float(np.percentile(lat, 50)), "served_p99_ms": float(np.percentile(lat, 99)),
            "plain_jobs_per_s": len(stream) / t_plain, "plain_p50_ms": float(np.percentile(lat_plain, 50)),
            "plain_p99_ms": float(np.percentile(lat_plain, 99)),
            "saturated_served_jobs_per_s": len(stream) / t_sat, "saturated_plain_jobs_per_s": len(stream) / t_sat_plain,
            "saturated_speedup": t_sat_plain / t_sat,
            "batches": st["batches"], "max_batch_jobs": st["max_batch_jobs"], "host_threads": cores,
            "identical_to_plain": bool(same)}


# ----------------------------------------------- config 5: serving stream ---
SERVE5 = dict(jobs=2000, seed=5, rate=50.0, nmin=5000, nmax=500000)


def serve5_stream(procs: int, jobs: int = 0):
    """The config-5 stream as stated: 2,000 jobs, Poisson arrivals at 50/s, n
    uniform in 10..16, editDist uniform in 3..5, candidates log-uniform in
    [5,000, 500,000] after the maxRun 3 / GC [0.3,0.7] filters (seed 5).  The
    words of the jobs are drawn in a spawned process pool (the same seeded
    draws as workloads.serving_stream, job by job)."""
    import multiprocessing as mp

    specs = W.serving_stream_specs(SERVE5["jobs"], SERVE5["seed"], SERVE5["rate"], SERVE5["nmin"], SERVE5["nmax"])
    specs = specs[:jobs] if jobs else specs
    with mp.get_context("spawn").Pool(max(1, procs)) as pool:
        words = pool.map(W.serving_job_words, specs, chunksize=4)
    return [(t, w, L, d) for (t, _, L, d, _), w in zip(specs, words)]


def run_serve5(args):
    """One JSON line for config 5: the continuous-batching server against the
    plain path -- one job per launch (coalescing off), solved by as many host
    threads as the server's greedy pool has, each taking the next arrived job
    in arrival order (the reference's cluster worker pool pattern,
    src/SparseMat.cpp:978-1010).  Both arms see the same arrival times;
    latency = arrival to codebook on the host; jobs/s = jobs / (last
    completion - first arrival)."""
    t_gen = time.perf_counter()
    cores = host_cores()
    stream = serve5_stream(cores, args.serve5_jobs)
    t_gen = time.perf_counter() - t_gen
    import torch

    from indexgen_b200 import Context, Server, solve

    torch.cuda.set_device(0)
    props = torch.cuda.get_device_properties(0)
    bus = None
    if hasattr(props, "pci_bus_id") and hasattr(props, "pci_domain_id") and hasattr(props, "pci_device_id"):
        bus = f"{props.pci_domain_id:08x}:{props.pci_bus_id:02x}:{props.pci_device_id:02x}"
    pairs = sum(len(w) * (len(w) - 1) // 2 for _, w, _, _ in stream)
    words_bytes = sum(4 * len(w) for _, w, _, _ in stream)
    ctx = Context(0)
    # warm-up (untimed): a few small jobs through both paths
    warm = sorted(stream, key=lambda j: len(j[1]))[:16]
    with Server(ctx, host_threads=cores) as sv:
        for t in [sv.submit(w, L, d) for _, w, L, d in warm]:
            sv.wait(t)
    for _, w, L, d in warm:
        solve(w, L, d, 1, ctx)
    launches0 = ctx.launches
    clocks = ClockSampler(bus)
    clocks.start()
    # ---- served
    lat = [0.0] * len(stream)
    books = [None] * len(stream)
    edges = [0] * len(stream)
    with Server(ctx, host_threads=cores) as sv:
        tickets = [None] * len(stream)
        submitted = threading.Event()
        t0 = time.perf_counter()

        def submitter():
            for i, (arr, w, L, d) in enumerate(stream):
                dt = arr - (time.perf_counter() - t0)
                if dt > 0:
                    time.sleep(dt)
                tickets[i] = sv.submit(w, L, d)
            submitted.set()

        th = threading.Thread(target=submitter)
        th.start()
        th.join()
        for i in range(len(stream)):
            books[i], edges[i], lat[i] = sv.wait(tickets[i])
        t_served = time.perf_counter() - t0 - stream[0][0]
        st = sv.stats()
    served_launches = ctx.launches - launches0
    clk_served = clocks.stop()
    ctx.close()  # its workspaces go back to the device pool for the plain arm
    # ---- plain: one job per launch, worker threads in arrival order
    ctx_plain = Context(0)
    ctx_plain.set_coalescing(False)
    clocks = ClockSampler(bus)
    clocks.start()
    lat_plain = [0.0] * len(stream)
    same = [True] * len(stream)
    nxt = [0]
    lock = threading.Lock()
    errors = []
    t0 = time.perf_counter()

    def worker():
        while True:
            with lock:
                i = nxt[0]
                nxt[0] += 1
            if i >= len(stream):
                return
            arr, w, L, d = stream[i]
            dt = arr - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            try:
                book, _ = solve(w, L, d, 1, ctx_plain)
            except Exception as e:  # reported in the line, never silently dropped
                errors.append((i, repr(e)))
                same[i] = False
                continue
            lat_plain[i] = 1e3 * (time.perf_counter() - t0 - arr)
            same[i] = bool(np.array_equal(book, books[i]))

    ws = [threading.Thread(target=worker) for _ in range(max(1, cores - 1))]
    for t in ws:
        t.start()
    for t in ws:
        t.join()
    t_plain = time.perf_counter() - t0 - stream[0][0]
    clk_plain = clocks.stop()
    plain_launches = ctx_plain.launches
    ctx_plain.close()
    n_jobs = len(stream)
    total_edges = int(sum(edges))
    book_bytes = sum(4 * len(b) for b in books)
    served = n_jobs / t_served
    line = {
        "metric": "served codebook jobs/s", "value": served, "unit": "jobs/s", "n_gpus": 1, "steps": 1,
        "warmup": 1, "ms_per_step": 1e3 * t_served, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": "serve5_poisson50_n10-16_d3-5_N5k-500k" + (
                       "" if n_jobs == SERVE5["jobs"] else f"_first{n_jobs}_jobs"),
                   "desc": f"{n_jobs} jobs, Poisson 50/s (seed 5), n uniform 10..16, editDist uniform 3..5, "
                           "candidates log-uniform [5000, 500000] after maxRun 3 / GC [0.3,0.7]",
                   "pair_tests": pairs, "edges": total_edges, "parallelism": "replicas x1",
                   "l2": "inputs (860 MB of words) larger than L2",
                   "step": "one pass over the whole stream (warm-up: 16 small jobs through both paths)"},
        "e2e": {"value": served, "unit": "jobs/s", "h2d_bytes_per_step": words_bytes, "d2h_bytes_per_step": book_bytes,
                "note": "serving is end to end by definition: host words in through ig_server_submit, codebooks "
                        "out through ig_server_wait, wall clock from the first arrival to the last codebook"},
        "serve": {"served_jobs_per_s": served, "served_p50_ms": float(np.percentile(lat, 50)),
                  "served_p99_ms": float(np.percentile(lat, 99)), "served_max_ms": float(max(lat)),
                  "served_s": t_served, "plain_jobs_per_s": n_jobs / t_plain,
                  "plain_p50_ms": float(np.percentile(lat_plain, 50)),
                  "plain_p99_ms": float(np.percentile(lat_plain, 99)), "plain_max_ms": float(max(lat_plain)),
                  "plain_s": t_plain, "speedup_jobs_per_s": t_plain / t_served,
                  "batches": st["batches"], "max_batch_jobs": st["max_batch_jobs"],
                  "served_gpu_launches": served_launches, "plain_gpu_launches": plain_launches,
                  "plain": f"one job per launch (coalescing off), {max(1, cores - 1)} worker threads in arrival order",
                  "host_threads": cores, "identical_to_plain": bool(all(same)), "plain_errors": errors[:5],
                  "stream_generation_s": t_gen},
        "gpu_launches": served_launches,
        "clocks": clk_served, "clocks_plain": clk_plain,
    }
    print(json.dumps(line), flush=True)


def run_ours(args, wl, rank, world, dist):
    import ctypes

    import torch

    from indexgen_b200 import Context, build_conflict_graph, lane_form
    from indexgen_b200._lib import check, lib

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    words, L, d = wl["words"], wl["L"], wl["min_ed"]
    n = len(words)
    pairs = pairs_of(n)
    ctx = Context(dev)
    ext = torch.cuda.ExternalStream(ctx.stream)
    words_dev = torch.from_numpy(words.view(np.int32)).to(f"cuda:{dev}")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{dev}")
    torch.cuda.synchronize()

    # work split for this job, chosen by the library's autotuner (untimed)
    ctx.autotune(words_dev, L, d)
    edges = None
    for _ in range(args.warmup):
        with build_conflict_graph(words_dev, L, d, ctx) as G:
            edges = G.edges
    props = torch.cuda.get_device_properties(dev)
    bus = None
    for attr in ("pci_bus_id",):
        if hasattr(props, attr) and hasattr(props, "pci_domain_id") and hasattr(props, "pci_device_id"):
            bus = f"{props.pci_domain_id:08x}:{props.pci_bus_id:02x}:{props.pci_device_id:02x}"

    # ---- device-resident timing
    ctx.set_profiling(True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(bus)
    clocks.start()
    launches0 = ctx.launches
    step_ms = []
    for _ in range(args.steps):
        flush.zero_()  # L2 flush between timed steps (256 MiB > 126 MB L2), untimed
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        G = build_conflict_graph(words_dev, L, d, ctx)
        e1.record(ext)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        seg_width, segments = G.job_tiling(0)
        G.close()
    torch.cuda.synchronize()
    launches = ctx.launches - launches0
    clk = clocks.stop()
    total_ms = sum(step_ms)
    pair_ms, pair_launches = ctx.phase_time(0)
    comp_ms, comp_launches = ctx.phase_time(1)
    comp_parts = {name: ctx.phase_time(ph)[0] / max(ctx.phase_time(ph)[1], 1)
                  for name, ph in (("prefix_ms", 3), ("scan_ms", 4), ("scatter_ms", 5))}
    ctx.set_profiling(False)
    total_ms = max_over_ranks(total_ms, dist, f"cuda:{dev}")
    value = replica_rate(world, pairs, args.steps, total_ms / 1e3)

    # ---- end to end through the public API with pinned host buffers
    h_words = torch.from_numpy(words.view(np.int32)).pin_memory()
    h_row = torch.empty(n + 1, dtype=torch.int64, pin_memory=True)
    h_cols = torch.empty(max(edges, 1), dtype=torch.int32, pin_memory=True)
    e2e_steps = max(3, min(args.steps, 10))
    wall = []
    for _ in range(e2e_steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        h = ctypes.c_void_p()
        check(lib().ig_graph_build(ctx.handle, ctypes.c_void_p(h_words.data_ptr()), n, L, d, 0, ctypes.byref(h)),
              "ig_graph_build", ctx.handle)
        check(lib().ig_graph_upper_csr(h, ctypes.c_void_p(h_row.data_ptr()), ctypes.c_void_p(h_cols.data_ptr())),
              "ig_graph_upper_csr", ctx.handle)
        t1 = time.perf_counter()
        lib().ig_graph_free(h)
        wall.append(t1 - t0)
    e2e_s = sum(wall) / len(wall)
    e2e_s = max_over_ranks(e2e_s, dist, f"cuda:{dev}")
    e2e = {"value": replica_rate(world, pairs, 1, e2e_s), "unit": UNIT, "h2d_bytes_per_step": 4 * n,
           "d2h_bytes_per_step": 8 * (n + 1) + 4 * edges, "ms_per_step": 1e3 * e2e_s,
           "note": "ig_graph_build(host words) + ig_graph_upper_csr(host buffers), wall clock"}

    # ---- greedy codebook (host) on the same graph, reported apart: canonical
    # adjacency on the device, download, greedy (best of three after one
    # untimed run), with the greedy on two threads (the library's default for
    # a graph this size) and on one
    from indexgen_b200 import greedy_stats, set_greedy_threads

    greedy_ms = {}
    for mode, helpers in (("two_threads", -1), ("one_thread", 0)):
        set_greedy_threads(helpers, -1)
        runs = []
        for _ in range(4):
            with build_conflict_graph(words_dev, L, d, ctx) as G:
                p0 = greedy_stats()[0]
                t0 = time.perf_counter()
                sel = G.codebook(1)
                runs.append(1e3 * (time.perf_counter() - t0))
                if mode == "two_threads" and greedy_stats()[0] == p0:
                    greedy_ms["two_threads_note"] = "no helper thread free: ran on one thread"
        greedy_ms[mode] = min(runs[1:])
    set_greedy_threads(-1, -1)

    # ---- words -> codebook through the public API (host words in, codebook
    # out), and its parts measured apart on the same context
    from indexgen_b200 import codebook_from_adjacency, solve

    solve_ms = []
    for _ in range(3):
        t0 = time.perf_counter()
        book, _ = solve(words, L, d, 1, ctx)
        solve_ms.append(1e3 * (time.perf_counter() - t0))
    set_greedy_threads(0, -1)
    solve_1t_ms = []
    for _ in range(3):
        t0 = time.perf_counter()
        book1, _ = solve(words, L, d, 1, ctx)
        solve_1t_ms.append(1e3 * (time.perf_counter() - t0))
    set_greedy_threads(-1, -1)
    t0 = time.perf_counter()
    G = build_conflict_graph(words, L, d, ctx)
    t_build = time.perf_counter() - t0
    t0 = time.perf_counter()
    ap, adj = G.adjacency()
    t_adj = time.perf_counter() - t0
    G.close()
    t0 = time.perf_counter()
    book2 = codebook_from_adjacency(ap, adj, n)
    t_greedy = time.perf_counter() - t0
    set_greedy_threads(0, -1)
    t0 = time.perf_counter()
    book3 = codebook_from_adjacency(ap, adj, n)
    t_greedy_1t = time.perf_counter() - t0
    set_greedy_threads(-1, -1)
    solve_e2e = {"ms": min(solve_ms), "ms_greedy_one_thread": min(solve_1t_ms),
                 "build_from_host_words_ms": 1e3 * t_build,
                 "adjacency_build_and_download_ms": 1e3 * t_adj, "host_greedy_ms": 1e3 * t_greedy,
                 "host_greedy_one_thread_ms": 1e3 * t_greedy_1t,
                 "codebook": int(len(book)),
                 "same_codebook_every_way": bool(np.array_equal(book, book1) and np.array_equal(book, book2)
                                                 and np.array_equal(book, book3)),
                 "h2d_bytes": 4 * n, "d2h_adjacency_bytes": 8 * (n + 1) + 8 * edges,
                 "note": "solve() = ig_solve(host words) -> codebook, wall clock, best of 3, greedy on two threads "
                         "(default) and on one; the parts are separate calls: ig_graph_build, ig_graph_adjacency "
                         "(device canonical order + pinned download), ig_codebook_from_adjacency (two threads, "
                         "then one)"}

    peaks, src = measured_peaks()
    sm_mhz = float(peaks.get("sm_max_mhz", 1965.0))
    alu_peak = props.multi_processor_count * 64 * sm_mhz * 1e6 / 1e12  # ALU pipe: 64 lanes/clk/SM
    int32_peak = props.multi_processor_count * 128 * sm_mhz * 1e6 / 1e12
    pair_avg_s = (pair_ms / max(pair_launches, 1)) / 1e3
    alu_ops = pairs * alu_ops_per_pair(L, d)
    achieved = alu_ops / pair_avg_s / 1e12 if pair_launches else None
    conv_ops = pairs * 16 * L
    conv_achieved = conv_ops / pair_avg_s / 1e12 if pair_launches else None
    traffic = profile_traffic(wl["name"])
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    # compaction: 8 B edge record read + 4 B column written per edge, 4 B
    # count read + 4 B prefix written per (row, segment) cell a row uses (its
    # band's diagonal segment onwards), 24 B per row (degree, offset scan,
    # offset read)
    cells = touched_cells(n, seg_width, segments)
    comp_bytes = 12 * edges + 8 * cells + 24 * (n + 1)
    comp_avg_s = (comp_ms / max(comp_launches, 1)) / 1e3
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": statistics.mean(step_ms), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": wl["name"], "desc": wl["desc"], "n": n, "L": L, "min_ed": d,
                   "pairs_per_step": pairs, "edges": edges, "parallelism": f"replicas x{world}",
                   "l2": "flushed between steps (256 MiB device write, untimed)"},
        "e2e": e2e,
        "roofline": {"bound": "int32-alu-pipe", "achieved": achieved, "peak": alu_peak, "unit": "Tops/s",
                     "frac": (achieved / alu_peak) if achieved else None, "traffic": traffic,
                     "kernel": "pair_kernel", "kernel_ms_per_launch": pair_avg_s * 1e3,
                     "work": f"{pairs} pair tests x {alu_ops_per_pair(L, d):g} ALU-pipe ops (LOP3/PRMT/add/shift) per pair "
                             f"test per launch",
                     "peak_source": f"{props.multi_processor_count} SMs x 64 ALU-pipe lanes/clk x {sm_mhz:.0f} MHz "
                                    f"max SM clock ({src} MEASURED_PEAKS sm_max_mhz)",
                     "int_ops_16L_convention": {"ops_per_pair": 16 * L, "achieved_tops": conv_achieved,
                                           "int32_peak_tops": int32_peak,
                                           "ratio": (conv_achieved / int32_peak) if conv_achieved else None,
                                           "note": "16*L int ops per pair test credited; the banded multi-lane "
                                                   "kernel does several pair tests per op, so this exceeds 1"}},
        "compaction": {"bound": "hbm", "achieved": comp_bytes / comp_avg_s / 1e9 if comp_launches else None,
                       "peak": hbm_peak, "unit": "GB/s",
                       "frac": (comp_bytes / comp_avg_s / 1e9 / hbm_peak) if comp_launches else None,
                       "ms_per_launch": comp_avg_s * 1e3, "peak_source": f"{src} hbm_gbs",
                       "bytes_per_launch": comp_bytes, "count_cells": cells, "segment_width": seg_width,
                       "parts_ms_per_launch": comp_parts},
        "path_traffic": path_traffic_line(wl["name"], edges, n),
        "gpu_launches": launches,
        "work_split": {"lane_form": ["full", "nibble", "byte"][lane_form(L, d)],
                       "items_per_cta": ctx.work_split(lane_form(L, d))[0],
                       "tuned": ctx.work_split(lane_form(L, d))[1]},
        "cuda_graphs": dict(zip(("launches", "instantiations", "updates"), ctx.graph_stats())),
        "clocks": clk,
        "greedy": {"ms": greedy_ms["two_threads"], "ms_one_thread": greedy_ms["one_thread"],
                   "codebook": int(len(sel)), "order_threads": 1,
                   "where": "host C++ (library): walker + bucket-mover threads (one thread for the second figure)",
                   **({"note": greedy_ms["two_threads_note"]} if "two_threads_note" in greedy_ms else {})},
        "solve_e2e": solve_e2e,
    }
    if not args.no_batch:
        line["batch"] = run_batch_section(ctx)
        line["assign"] = run_assign_section(ctx)
        line["cluster"] = run_cluster_section(ctx)
    if args.serve_jobs > 0:
        line["serve"] = run_serve_section(ctx, args.serve_jobs, args.serve_nmax)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(wl)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "reference_gpu"])
    ap.add_argument("--workload", default="linear12", choices=["linear12", "uniform11", "vt16", "serve5"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-clusters section")
    ap.add_argument("--serve-jobs", type=int, default=200, help="jobs in the serving section (0 = skip)")
    ap.add_argument("--serve-nmax", type=int, default=50000, help="largest job (candidates) in the serving stream")
    ap.add_argument("--serve5-jobs", type=int, default=0,
                    help="serve5: only the first K jobs of the stream (a trial run; 0 = all 2,000)")
    ap.add_argument("--subset", type=int, default=0,
                    help="use a seeded random subset of this many words (profiling runs)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.workload == "serve5":
        if args.impl != "ours" or world > 1:
            if rank == 0:
                print(json.dumps({"impl": args.impl, "unavailable": "the config-5 serving stream is a one-GPU "
                                  "comparison of the library's server with its own one-job-per-launch path"}))
            return
        run_serve5(args)
        return
    wl = workload(args.workload)
    if args.subset and args.subset < len(wl["words"]):
        rng = np.random.default_rng(4321)
        wl["words"] = wl["words"][np.sort(rng.choice(len(wl["words"]), args.subset, replace=False))]
        wl["name"] += f"_subset{args.subset}"
    if args.impl == "reference":
        run_reference(args, wl, rank)
        return
    if args.impl == "reference_gpu":
        run_reference_gpu(args, wl, rank)
        return
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist
    try:
        run_ours(args, wl, rank, world, dist)
    finally:
        if dist:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
