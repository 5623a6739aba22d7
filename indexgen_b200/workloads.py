"""Seeded candidate sets for the conflict-graph workloads.

These produce the INPUT of the accelerated path (2-bit packed words, character
p at bits 2p..2p+1).  They restate the reference's candidate sources where a
workload names one:

* ``uniform_words``  -- i.i.d. uniform 4-ary strings (numpy PCG64), the stand-in
  for the reference's ``Random`` method (src/CandidateGenerator.cpp:410-446),
  which seeds from std::random_device and so cannot be replayed.
* ``linear_code_words`` -- all codewords of the shortened GF(4) Hamming code
  [n, n-3, 3] in the order src/Candidates/LinearCodes.cpp:225-289 emits them:
  data vectors counted in base 4 with the last digit fastest (src/Utils.cpp:525-542),
  encoded by the permuted generator matrix, plus the bias (coset) vector.
* ``vt16_words`` -- seeded uniform draws of the quaternary VT-style code
  sum(i*x_i) = 0 (mod 17), sum(x_i) = 0 (mod 4) used by the large sparse graph.
* ``filter_words`` -- MaxRun / GC-content filters with the reference's double
  comparisons (src/CandidateGenerator.cpp:24-50, src/Utils.cpp:420-462).
"""
from __future__ import annotations

import itertools

import numpy as np

# GF(4) = {0, 1, a, a^2} coded 0,1,2,3 with a^2 = a + 1: addition is XOR of the
# 2-bit codes, multiplication goes through discrete logs.
_LOG = {1: 0, 2: 1, 3: 2}
_EXP = [1, 2, 3]


def gf4_mul(a: int, b: int) -> int:
    if a == 0 or b == 0:
        return 0
    return _EXP[(_LOG[a] + _LOG[b]) % 3]


def hamming_parity_rows() -> list[tuple[int, int, int]]:
    """Parity rows of the systematic GF(4) Hamming code of length 21.

    One normalised representative (first non-zero coordinate 1) of every point
    of PG(2,4) that is not a unit vector, in lexicographic order.  Appending
    them to the identity gives the [21,18,3] generator that
    src/Candidates/GenMat.cpp:9-33 tabulates.
    """
    rows = []
    for v in itertools.product(range(4), repeat=3):
        nz = [x for x in v if x]
        if len(nz) >= 2 and nz[0] == 1:
            rows.append(v)
    assert len(rows) == 18
    return rows


def hamming_generator(n: int) -> np.ndarray:
    """Generator of the [21,18,3] code shortened to length n (4 <= n <= 21).

    Shortening drops the first 21-n data rows and coordinates, as
    src/Candidates/LinearCodes.cpp:118-136 / :160-166 do.
    """
    if not 4 <= n <= 21:
        raise ValueError("length must be in 4..21")
    full = np.zeros((18, 21), np.int64)
    full[:, :18] = np.eye(18, dtype=np.int64)
    full[:, 18:] = np.array(hamming_parity_rows(), np.int64)
    d = 21 - n
    return full[d:, d:]


def linear_code_words(n: int, bias, row_perm=None, col_perm=None) -> np.ndarray:
    """All 4^(n-3) codewords (+ bias) as packed words, in the reference's order."""
    G = hamming_generator(n)
    k = G.shape[0]
    if col_perm is not None:
        G = G[:, list(col_perm)]
    if row_perm is not None:
        G = G[list(row_perm), :]
    # data vectors in base-4 counting order, last digit fastest
    idx = np.arange(4 ** k, dtype=np.int64)
    data = (idx[:, None] >> (2 * np.arange(k - 1, -1, -1, dtype=np.int64))[None, :]) & 3
    code = np.zeros((len(idx), n), np.int64)
    mul = np.array([[gf4_mul(a, b) for b in range(4)] for a in range(4)], np.int64)
    for i in range(k):
        code ^= mul[data[:, i][:, None], G[i][None, :]]
    code ^= np.asarray(bias, np.int64)[None, :]
    return pack_digits(code)


def pack_digits(digits) -> np.ndarray:
    d = np.asarray(digits, dtype=np.uint32)
    L = d.shape[1]
    return (d << (2 * np.arange(L, dtype=np.uint32))[None, :]).sum(axis=1, dtype=np.uint64).astype(np.uint32)


def unpack_digits(words, L: int) -> np.ndarray:
    w = np.asarray(words, dtype=np.uint32)
    return ((w[:, None] >> (2 * np.arange(L, dtype=np.uint32))[None, :]) & 3).astype(np.uint8)


def to_strings(words, L: int) -> list[str]:
    d = unpack_digits(words, L) + ord("0")
    return [bytes(r).decode("ascii") for r in d]


def from_strings(strings) -> np.ndarray:
    if len(strings) == 0:
        return np.zeros(0, np.uint32)
    L = len(strings[0])
    raw = np.frombuffer("".join(strings).encode("latin1"), np.uint8).reshape(len(strings), L)
    if np.any((raw < 48) | (raw > 51)):
        raise ValueError("candidates must be strings over '0'..'3'")
    return pack_digits(raw - 48)


_CHUNK_TABLES = {}


def _chunk_tables(k: int):
    """Per 16-bit chunk value (8 chars at bits 2i) restricted to its first k
    chars: longest run, leading run, trailing run, first and last char and
    the count of chars in {1, 2} (C or G)."""
    t = _CHUNK_TABLES.get(k)
    if t is None:
        v = np.arange(1 << 16, dtype=np.uint32)
        c = ((v[:, None] >> (2 * np.arange(k, dtype=np.uint32))[None, :]) & 3).astype(np.int8)
        run = np.ones(len(v), np.int8)
        best = np.ones(len(v), np.int8)
        lead = np.ones(len(v), np.int8)
        still = np.ones(len(v), bool)
        for p in range(1, k):
            same = c[:, p] == c[:, p - 1]
            run = np.where(same, run + 1, 1).astype(np.int8)
            best = np.maximum(best, run)
            still &= same
            lead = np.where(still, lead + 1, lead).astype(np.int8)
        gc = ((c == 1) | (c == 2)).sum(axis=1).astype(np.int8)
        t = (best, lead, run, c[:, 0].copy(), c[:, k - 1].copy(), gc)
        _CHUNK_TABLES[k] = t
    return t


def filter_words(words, L: int, max_run: int = 3, min_gc: float = 0.3, max_gc: float = 0.7) -> np.ndarray:
    """Boolean keep-mask with the reference filter semantics (MaxRun <= maxRun
    when maxRun > 0; GC fraction compared in double when either bound is set),
    evaluated with per-8-character lookup tables."""
    w = np.asarray(words, dtype=np.uint32)
    keep = np.ones(len(w), bool)
    if len(w) == 0:
        return keep
    lo = w & np.uint32(0xffff)
    k_lo = min(L, 8)
    b0, _, t0, _, last0, g0 = _chunk_tables(k_lo)
    best = b0[lo].astype(np.int64)
    gc = g0[lo].astype(np.int64)
    if L > 8:
        hi = (w >> np.uint32(16)) & np.uint32(0xffff)
        b1, l1, _, first1, _, g1 = _chunk_tables(L - 8)
        join = np.where(last0[lo] == first1[hi], t0[lo].astype(np.int64) + l1[hi], 0)
        best = np.maximum(np.maximum(best, b1[hi]), join)
        gc += g1[hi]
    if max_run > 0:
        keep &= best <= max_run
    if min_gc > 0 or max_gc > 0:
        frac = gc.astype(np.float64) / float(L)
        keep &= (frac >= min_gc) & (frac <= max_gc)
    return keep


def uniform_words(count: int, L: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return pack_digits(rng.integers(0, 4, size=(count, L)))


def uniform_filtered(count: int, L: int, seed: int, **flt) -> np.ndarray:
    """`count` uniform draws, then the filters (order preserved)."""
    w = uniform_words(count, L, seed)
    return w[filter_words(w, L, **flt)]


def uniform_until(target: int, L: int, seed: int, **flt) -> np.ndarray:
    """Draw uniform strings in seeded batches until `target` survive the filters."""
    if target <= 0:
        return np.zeros(0, np.uint32)
    rng = np.random.default_rng(seed)
    out = []
    have = 0
    while have < target:
        w = pack_digits(rng.integers(0, 4, size=(max(4096, target), L)))
        w = w[filter_words(w, L, **flt)]
        out.append(w)
        have += len(w)
    return np.concatenate(out)[:target]


def vt16_words(target: int, seed: int, max_run: int = 3, min_gc: float = 0.3, max_gc: float = 0.7) -> np.ndarray:
    """`target` filtered words of sum(i*x_i)=0 mod 17, sum(x_i)=0 mod 4 (n=16)."""
    L = 16
    rng = np.random.default_rng(seed)
    # per byte b of a word (digits 4b..4b+3): sum of (i+1)*x_i and of x_i
    byte = np.arange(256, dtype=np.int64)
    dig = (byte[:, None] >> (2 * np.arange(4))) & 3
    wsum = [(dig * (4 * b + 1 + np.arange(4))).sum(axis=1) for b in range(4)]
    dsum = dig.sum(axis=1)
    out = []
    have = 0
    while have < target:
        w = rng.integers(0, 1 << 32, size=1 << 22, dtype=np.uint64).astype(np.uint32)  # 16 uniform digits each
        bs = [(w >> np.uint32(8 * b)) & np.uint32(0xff) for b in range(4)]
        ws = wsum[0][bs[0]] + wsum[1][bs[1]] + wsum[2][bs[2]] + wsum[3][bs[3]]
        ds = dsum[bs[0]] + dsum[bs[1]] + dsum[bs[2]] + dsum[bs[3]]
        w = w[(ws % 17 == 0) & (ds % 4 == 0)]
        w = w[filter_words(w, L, max_run, min_gc, max_gc)]
        out.append(w)
        have += len(w)
    return np.concatenate(out)[:target]


# The coset vector the reference's LinearCode generator draws for n=12 with
# biasMode=random and randomSeed=20251203 (mt19937 + uniform_int_distribution,
# src/CandidateGenerator.cpp:81-96); pinned by the golden fixture.
LINEAR12_SEED = 20251203
LINEAR12_BIAS = (1, 0, 0, 2, 1, 3, 3, 0, 1, 0, 3, 0)


def linear12_candidates() -> np.ndarray:
    """The single-large-job workload: [12,9,3] GF(4) code + seeded coset, filtered."""
    w = linear_code_words(12, LINEAR12_BIAS)
    return w[filter_words(w, 12, 3, 0.3, 0.7)]


def uniform11_candidates() -> np.ndarray:
    """The CPU-runnable workload: 20,000 uniform n=11 strings (seed 12345), filtered."""
    return uniform_filtered(20000, 11, 12345, max_run=3, min_gc=0.3, max_gc=0.7)


def zipf_sizes(total: int, k: int, s: float = 1.1, lo: int = 2000, hi: int = 60000) -> np.ndarray:
    """k cluster sizes proportional to i^-s (i = 1..k), clamped to [lo, hi] and
    renormalised so they sum to `total` (clamped sizes stay at their bound,
    the free ones absorb the rest; integer rounding by largest remainder)."""
    if not lo * k <= total <= hi * k:
        raise ValueError("total must lie in [lo*k, hi*k]")
    w = np.arange(1, k + 1, dtype=np.float64) ** -s
    size = w / w.sum() * total
    fixed = np.zeros(k, bool)
    for _ in range(4 * k):
        free = ~fixed
        rest = total - size[fixed].sum()
        size[free] = w[free] / w[free].sum() * rest
        over = free & ((size > hi) | (size < lo))
        if not over.any():
            break
        size[over] = np.clip(size[over], lo, hi)
        fixed |= over
    base = np.floor(size).astype(np.int64)
    short = int(total - base.sum())
    order = np.argsort(-(size - base), kind="stable")
    base[order[:short]] += 1
    return base


def assign_clusters(words, L: int, sizes, seed: int):
    """Capacity-constrained nearest-centre assignment (a k-means-style step
    with imposed sizes).  Centres are seeded random members; clusters, largest
    first, take their `size` nearest unassigned words by Hamming distance to
    the centre (ties by word index).  Returns one index array per cluster, in
    ascending word order."""
    w = np.asarray(words, np.uint32)
    n = len(w)
    sizes = np.asarray(sizes, np.int64)
    if sizes.sum() != n:
        raise ValueError("sizes must sum to the number of words")
    rng = np.random.default_rng(seed)
    centres = w[rng.choice(n, len(sizes), replace=False)]
    digits = unpack_digits(w, L)
    free = np.ones(n, bool)
    out = [None] * len(sizes)
    for c in np.argsort(-sizes, kind="stable"):
        cd = unpack_digits(centres[c:c + 1], L)[0]
        dist = (digits != cd[None, :]).sum(axis=1)
        need = int(sizes[c])
        take = []
        for d in range(L + 1):
            idx = np.nonzero(free & (dist == d))[0]
            if len(idx) >= need:
                take.append(idx[:need])
                need = 0
                break
            take.append(idx)
            need -= len(idx)
        sel = np.sort(np.concatenate(take))
        free[sel] = False
        out[c] = sel
    return out


def clustered14(total: int = 1_000_000, k: int = 64, seed: int = 14):
    """The batched-clusters workload: `total` filtered uniform n=14 words split
    into k clusters with Zipf(1.1) sizes in [2000, 60000].  Returns a list of
    packed word arrays, one per cluster."""
    w = uniform_until(total, 14, seed, max_run=3, min_gc=0.3, max_gc=0.7)
    parts = assign_clusters(w, 14, zipf_sizes(total, k), seed + 1)
    return [w[p] for p in parts]


def serving_stream_specs(jobs: int, seed: int, rate: float = 50.0, nmin: int = 5000, nmax: int = 500000,
                         lengths=(10, 16), dists=(3, 5)):
    """The jobs of serving_stream without their words: (arrival_s, count, n,
    editDist, word seed) each; serving_job_words(spec) draws the words."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(jobs):
        t += rng.exponential(1.0 / rate)
        L = int(rng.integers(lengths[0], lengths[1] + 1))
        d = int(rng.integers(dists[0], dists[1] + 1))
        count = int(round(float(np.exp(rng.uniform(np.log(nmin), np.log(nmax))))))
        out.append((t, count, L, d, int(rng.integers(1 << 31))))
    return out


def serving_job_words(spec) -> np.ndarray:
    """The filtered words of one serving_stream_specs entry."""
    _, count, L, _, wseed = spec
    return uniform_until(count, L, wseed, max_run=3, min_gc=0.3, max_gc=0.7)


def serving_stream(jobs: int, seed: int, rate: float = 50.0, nmin: int = 5000, nmax: int = 500000,
                   lengths=(10, 16), dists=(3, 5)):
    """Seeded stream of codebook jobs: Poisson arrivals (mean `rate` jobs/s),
    n uniform in [lengths], editDist uniform in [dists], candidate count
    log-uniform in [nmin, nmax] (counted after the maxRun 3 / GC [0.3,0.7]
    filters).  Returns a list of (arrival_s, words, n, editDist)."""
    return [(t, serving_job_words((t, c, L, d, ws)), L, d)
            for t, c, L, d, ws in serving_stream_specs(jobs, seed, rate, nmin, nmax, lengths, dists)]
