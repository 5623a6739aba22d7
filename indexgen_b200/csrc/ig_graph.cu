// Conflict-graph construction on sm_100a.
//
// Replaces compute_chunk_kernel + the tile loop of src/cuda_edit_distance.py
// (:20-226, :278-446) and the Python edge writer (src/gpu_graph_generator.py:49-77).
//
// Pipeline for a batch of independent jobs (one job = n words of one length L
// and a threshold d; edge iff ED < d).  A single job is a batch of one; the
// clustered solve (src/SparseMat.cpp:927-1095) submits all clusters at once.
//   prep_units      words -> PRMT selector streams, two columns per unit for L <= 15
//   pair_kernel     ONE persistent launch for the whole batch: CTAs take
//                   (job, row band, column segment) items from an atomic queue and
//                   dispatch on the job's L and lane form; 256 rows per band, one
//                   per thread, keep their match masks in registers; column tiles
//                   of the segment are staged into shared memory by cp.async.bulk
//                   (TMA bulk copy, no multicast) with a two-slot mbarrier
//                   pipeline; each thread tests its row against 4 (byte lanes,
//                   editDist 5..8) or 2/1 (full Myers) columns per 32-bit word
//                   (pair_kernel_nib: two rows against 4 columns, nibble lanes,
//                   editDist <= 4, 128 threads per band) and emits hits as
//                   (row, col, rank-in-(row,segment), cell) records into slots
//                   its warp takes in chunks, plus a per-(row, segment) count.
//   row_prefix      per-row exclusive prefix over its segments + degree
//   scan            exclusive scan of degrees -> row_ptr (int64)
//   scatter         cols[row_ptr[r] + prefix[cell] + rank] = col
// The result is one upper CSR over the concatenated rows with global column
// ids (block diagonal: jobs never share an edge), ascending per row and
// bit-exact by construction (no sort, no dependence on scheduling).
#include <algorithm>
#include <cstdio>
#include <cstring>

#include "ig_internal.h"
#include "ig_myers.cuh"

namespace ig {

namespace {

using myers::BandConst;
using myers::BandUnit;
using myers::kModeByte;
using myers::kModeFull;
using myers::kModeNib;
using myers::Unit;
using myers::imad;
using myers::myers_one;
using myers::myers_two;
using myers::nib;
using myers::row_pools;

constexpr unsigned kFull = 0xffffffffu;

// Pass status word: a bounded wait ran out (the CTA left after its copies in
// flight had landed), or, worse, a copy in flight never landed either.
enum : int { kStatusOk = 0, kStatusTimeout = 1, kStatusCopyLost = 2 };

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// 1-D TMA bulk copy global -> this CTA's shared memory (16-byte aligned,
// size a multiple of 16).  Plain copy: no cluster multicast.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// Index of the job whose `key` range contains v (jobs sorted by key).
__device__ __forceinline__ int find_job_by_item(const JobDesc *jobs, int njobs, long long v)
{
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].item_off <= v)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ int find_job_by_unit(const JobDesc *jobs, int njobs, long long v)
{
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].unit_start <= v)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ int find_job_by_row(const JobDesc *jobs, int njobs, long long v)
{
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].word_off <= v)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Column units of every job: two columns per unit (16 selector words) for
// L <= 15, one column per unit (8 words, two positions each) for L = 16.
__global__ void prep_units(const uint32_t *__restrict__ words, const JobDesc *__restrict__ jobs, int njobs,
                           long long total_units, uint4 *__restrict__ units)
{
    const long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (u >= total_units)
        return;
    const JobDesc J = jobs[find_job_by_unit(jobs, njobs, u)];
    const long long p = u - J.unit_start;
    const uint32_t *w = words + J.word_off;
    uint4 *out = units + J.unit_off;
    if (J.mode == kModeNib) {
        // 4 columns; word j: nibble l = char of column l at position j
        uint32_t cw[4];
#pragma unroll
        for (int c = 0; c < 4; ++c)
            cw[c] = (4 * p + c < J.n) ? w[4 * p + c] : 0u;
        uint32_t o[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            uint32_t x = 0u;
#pragma unroll
            for (int l = 0; l < 4; ++l)
                x |= ((cw[l] >> (2 * j)) & 3u) << (4 * l);
            o[j] = (j < J.L) ? x : 0u;
        }
#pragma unroll
        for (int v = 0; v < 4; ++v)
            out[4 * p + v] = make_uint4(o[4 * v], o[4 * v + 1], o[4 * v + 2], o[4 * v + 3]);
        return;
    }
    if (J.mode == kModeByte) {
        // 4 columns; word q: positions 2q (bits 0..15) and 2q+1 (16..31)
        uint32_t cw[4];
#pragma unroll
        for (int c = 0; c < 4; ++c)
            cw[c] = (4 * p + c < J.n) ? w[4 * p + c] : 0u;
        uint32_t o[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            uint32_t x = 0u;
#pragma unroll
            for (int l = 0; l < 4; ++l) {
                x |= ((cw[l] >> (4 * q)) & 3u) << (4 * l);
                x |= ((cw[l] >> (4 * q + 2)) & 3u) << (16 + 4 * l);
            }
            o[q] = x;
        }
        out[2 * p] = make_uint4(o[0], o[1], o[2], o[3]);
        out[2 * p + 1] = make_uint4(o[4], o[5], o[6], o[7]);
        return;
    }
    if (J.L <= 15) {
        const uint32_t wa = w[2 * p];
        const uint32_t wb = (2 * p + 1 < J.n) ? w[2 * p + 1] : wa;
        uint32_t o[16];
#pragma unroll
        for (int k = 0; k < 16; ++k)
            o[k] = (k < J.L) ? (nib((wa >> (2 * k)) & 3u) | (nib((wb >> (2 * k)) & 3u) << 8)) : 0u;
#pragma unroll
        for (int v = 0; v < 4; ++v)
            out[4 * p + v] = make_uint4(o[4 * v], o[4 * v + 1], o[4 * v + 2], o[4 * v + 3]);
    } else {
        const uint32_t x = w[p];
        uint32_t o[8];
#pragma unroll
        for (int j = 0; j < 8; ++j)
            o[j] = nib((x >> (4 * j)) & 3u) | (nib((x >> (4 * j + 2)) & 3u) << 16);
        out[2 * p] = make_uint4(o[0], o[1], o[2], o[3]);
        out[2 * p + 1] = make_uint4(o[4], o[5], o[6], o[7]);
    }
}

struct PairArgs {
    const uint4 *units;
    const uint32_t *words;
    const JobDesc *jobs;
    int njobs;
    long long items;
    uint32_t one;     // 1, 2, 2^16 as opaque operands for imad / umulhi
    uint32_t two;
    uint32_t hi;
    uint32_t gather;  // 0x00204081 and 16, opaque: hit flags -> column mask on the FMA pipe
    uint32_t h4;
    unsigned long long *work;
    unsigned long long *rec_count;  // record slots handed out (chunks of kSlotChunk)
    unsigned long long *hit_count;  // pair tests that are edges (exact)
    EdgeRecord *rec;
    unsigned long long rec_cap;
    uint32_t *counts;
    int *status;
    int emit;
    long long wait_cycles;  // bound on every mbarrier wait (SM clock cycles)
    int skip_first_copy;    // test hook: withhold the first tile copy of the kernel's first item
};

// Record slots.  Each warp takes slots from the global counter in chunks of
// kSlotChunk (one atomic per chunk instead of one per hit group: a single
// counter address is otherwise the limit on dense graphs) and keeps the rest
// of its chunk in shared memory.  Slots a warp never fills are written as
// sentinels (cell = kNoCell) when the kernel ends; the scatter skips them.
constexpr unsigned kSlotChunk = 64;
constexpr uint32_t kNoCell = 0xffffffffu;

// Two scalar arrays, each element read and written on its own (a 16-byte
// struct here, read whole, faulted with a misaligned shared access).
__shared__ unsigned long long g_slot_base[kBandRows / 32];  // next free slot of each warp's chunk
__shared__ unsigned g_slot_left[kBandRows / 32];            // free slots left in it

// Slots of the warp's next `total` records (warp-uniform call): record j goes
// to b0 + j for j < n0, else to b1 + (j - n0).
struct Slots {
    unsigned long long b0, b1;
    unsigned n0;
};

__device__ __forceinline__ Slots take_slots(const PairArgs &a, unsigned total, int lane)
{
    const int w = threadIdx.x >> 5;
    unsigned long long b0 = 0, b1 = 0;
    unsigned n0 = 0;
    if (lane == 0) {
        b0 = g_slot_base[w];
        const unsigned left = g_slot_left[w];
        if (left >= total) {
            n0 = total;
            g_slot_base[w] = b0 + total;
            g_slot_left[w] = left - total;
        } else {
            n0 = left;
            const unsigned need = total - left;
            const unsigned take = need > kSlotChunk ? need : kSlotChunk;
            b1 = atomicAdd(a.rec_count, (unsigned long long)take);
            g_slot_base[w] = b1 + need;
            g_slot_left[w] = take - need;
        }
    }
    Slots s;
    s.b0 = __shfl_sync(kFull, b0, 0);
    s.b1 = __shfl_sync(kFull, b1, 0);
    s.n0 = __shfl_sync(kFull, n0, 0);
    return s;
}

// Hit flags at bits 7, 15, 23, 31 of h (all other bits clear) -> bits 0..3.
// The multiply by 2^21 + 2^14 + 2^7 + 1 moves bit 8c+7 to bit 28+c and puts
// every other partial product on a distinct bit below 28 or above 31 (no
// carries), and the high half of a multiply by 16 is bits 28..31: two FMA-pipe
// operations instead of seven shifts and masks on the ALU pipe.
__device__ __forceinline__ uint32_t hit_columns(uint32_t h, const PairArgs &a)
{
    return __umulhi(myers::imad(h, a.gather, 0u), a.h4);
}

// Warp total of cnt and this lane's exclusive prefix.  When no lane has more
// than one hit (the usual case on sparse graphs) one ballot gives both;
// otherwise the bit planes of cnt (kPlanes of them) are balloted.
template <int kPlanes>
__device__ __forceinline__ void warp_count_prefix(uint32_t cnt, int lane, unsigned &total, unsigned &pre)
{
    const unsigned lt = (1u << lane) - 1u;
    const unsigned some = __ballot_sync(kFull, cnt != 0u);
    if (__all_sync(kFull, cnt <= 1u)) {
        total = (unsigned)__popc(some);
        pre = (unsigned)__popc(some & lt);
        return;
    }
    total = 0;
    pre = 0;
#pragma unroll
    for (int b = 0; b < kPlanes; ++b) {
        const unsigned bal = __ballot_sync(kFull, (cnt >> b) & 1u);
        total += (unsigned)__popc(bal) << b;
        pre += (unsigned)__popc(bal & lt) << b;
    }
}

constexpr int kSlotVec = kTileCols * 2;  // uint4 per staged tile (8 KiB, every unit layout)

// Thread 0: copy the tile of units starting at column c0 (at most kTile
// columns, up to c_hi) into ring slot `slot`.
template <int kTile, int kCols, int kVec>
__device__ __forceinline__ void ring_issue(uint4 (*tile)[kSlotVec], uint64_t *bar, int slot, const uint4 *units,
                                           int32_t c0, int32_t c_hi)
{
    const int nu = (min(kTile, c_hi - c0) + kCols - 1) / kCols;
    const uint32_t bytes = (uint32_t)nu * kVec * 16;
    mbar_arrive_expect_tx(&bar[slot], bytes);
    bulk_g2s(&tile[slot][0], units + (size_t)(c0 / kCols) * kVec, bytes, &bar[slot]);
}

// Ring state bits: bit s (s = 0, 1) is the phase parity slot s waits for
// next; kSkipped marks an item whose first tile copy the test hook withheld
// (cleared by that tile's wait).
constexpr uint32_t kSkipped = 4u;

// A CTA whose wait on a staged tile ran out leaves its item loop, but not
// before thread 0 has waited (bounded) for the copies it issued that may still
// be in flight into the CTA's shared memory -- slot b's, unless the test hook
// withheld it, and the other slot's, when the next tile was issued -- so that
// no bulk copy lands after the CTA is gone.  The wait happens once per kernel,
// after the item loop (ring_drain), where it costs the pair loop no
// registers; ring_note_abort leaves it what it needs: bit 0 = slot b, bit 1 =
// slot b's copy was issued, bit 2 = the other slot's copy was issued.
__shared__ uint32_t g_drain;

__device__ __forceinline__ void ring_note_abort(const PairArgs &a, int b, bool b_issued, bool other_issued)
{
    atomicCAS(a.status, kStatusOk, kStatusTimeout);
    g_drain = (uint32_t)b | (b_issued ? 2u : 0u) | (other_issued ? 4u : 0u);
}

// Thread 0, after the item loop of an aborted CTA.  `parity` has slot b's bit
// already advanced past the phase that timed out.  Waiting on a phase that
// has completed returns at once; a copy that never lands is reported as
// kStatusCopyLost.
__device__ __forceinline__ void ring_drain(const PairArgs &a, uint64_t *bar, uint32_t parity)
{
    const uint32_t d = g_drain;
    const int b = (int)(d & 1u);
    const uint32_t pend = parity ^ (1u << b);  // the phase each slot still waits for
    for (int slot = 0; slot < 2; ++slot) {
        if (!((d >> (slot == b ? 1 : 2)) & 1u))
            continue;
        const long long t0 = clock64();
        while (!mbar_try_wait(&bar[slot], (pend >> slot) & 1u)) {
            if (clock64() - t0 > a.wait_cycles) {
                atomicExch(a.status, kStatusCopyLost);
                break;
            }
        }
    }
}

// Everything one thread needs about its row while it walks a segment.
struct RowCtx {
    int32_t row;     // job-local row
    bool ok;         // row < n
    uint32_t p01, p23;
    int32_t seg0;    // job-local first column of the segment
    uint32_t cell;   // index of this (row, segment) count
    int32_t n;
    int lim;
};

// Bits [lo, hi) of the columns col0 + c, c < NC, that lie in the strict upper
// triangle of the job (col > row, col < n) for a valid row.
template <int NC>
__device__ __forceinline__ uint32_t upper_mask(const RowCtx &r, int32_t col0)
{
    if (!r.ok)
        return 0u;
    const int lo = max(r.row + 1 - col0, 0);
    const int hi = min(r.n - col0, NC);
    return hi > lo ? (((1u << hi) - 1u) & ~((1u << lo) - 1u)) : 0u;
}

// Emit this thread's hits m (bit c: column col0 + c, c < NC) for a warp in
// which at least one lane has a hit.  Ranks count the row's hits in its
// (row, segment) cell in column order, so the scatter needs no sort.
template <int NC>
__device__ __forceinline__ void emit_mask(const PairArgs &a, uint32_t m, const RowCtx &r, int32_t col0,
                                          uint32_t &rank, int lane)
{
    const uint32_t cnt = __popc(m);
    if (!a.emit) {
        rank += cnt;
        return;
    }
    // warp total and this lane's exclusive prefix
    constexpr int kPlanes = NC >= 8 ? 4 : (NC >= 4 ? 3 : (NC >= 2 ? 2 : 1));
    unsigned total, pre;
    warp_count_prefix<kPlanes>(cnt, lane, total, pre);
    if (total == 0u)
        return;
    const Slots sl = take_slots(a, total, lane);
    unsigned j = pre;
    while (m) {
        const int c = __ffs(m) - 1;
        m &= m - 1u;
        const unsigned long long idx = j < sl.n0 ? sl.b0 + j : sl.b1 + (j - sl.n0);
        if (idx < a.rec_cap) {
            *reinterpret_cast<uint2 *>(a.rec + idx) = make_uint2(r.cell, (uint32_t)(col0 + c - r.seg0) << 16 | rank);
        }
        ++rank;
        ++j;
    }
}

// One staged tile of nu units whose first (job-local) column is c0.  CHECK
// adds the strict-upper-triangle test (col > row), row < n and col < n; it is
// only needed on diagonal items, the last (partial) band and an odd last column.
template <int L, bool CHECK>
__device__ __forceinline__ void tile_pass(const PairArgs &a, const uint4 *tile, int nu, int32_t c0, const RowCtx &r,
                                          uint32_t &rank, int lane)
{
    using U = Unit<L>;
    for (int u = 0; u < nu; ++u) {
        const uint4 *src = tile + u * U::kVec;
        if constexpr (U::kTwo) {
            uint32_t sel[16];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                if (v < U::kUsed) {
                    const uint4 q = src[v];
                    sel[4 * v] = q.x;
                    sel[4 * v + 1] = q.y;
                    sel[4 * v + 2] = q.z;
                    sel[4 * v + 3] = q.w;
                } else {
                    sel[4 * v] = sel[4 * v + 1] = sel[4 * v + 2] = sel[4 * v + 3] = 0u;
                }
            }
            bool h0, h1;
            myers_two<L>(r.p01, r.p23, sel, a.one, a.two, r.lim, h0, h1);
            const int32_t col = c0 + 2 * u;
            uint32_t m = (h0 ? 1u : 0u) | (h1 ? 2u : 0u);
            if (CHECK)
                m &= upper_mask<2>(r, col);
            if (__any_sync(kFull, m != 0u))
                emit_mask<2>(a, m, r, col, rank, lane);
        } else {
            static_assert(U::kUsed == 2, "one-lane units are two uint4");
            uint32_t sel[8];
            const uint4 q0 = src[0];
            const uint4 q1 = src[1];
            sel[0] = q0.x; sel[1] = q0.y; sel[2] = q0.z; sel[3] = q0.w;
            sel[4] = q1.x; sel[5] = q1.y; sel[6] = q1.z; sel[7] = q1.w;
            const bool h0 = myers_one<L>(r.p01, r.p23, sel, a.one, a.two, a.hi, r.lim);
            const int32_t col = c0 + u;
            uint32_t m = h0 ? 1u : 0u;
            if (CHECK)
                m &= upper_mask<1>(r, col);
            if (__any_sync(kFull, m != 0u))
                emit_mask<1>(a, m, r, col, rank, lane);
        }
    }
}

// Byte lanes (editDist 5..8): one unit = 4 columns against the thread's row.
template <int L, int MODE, bool CHECK>
__device__ __forceinline__ void tile_pass_band(const PairArgs &a, const uint4 *tile, int nu, int32_t c0,
                                               const RowCtx &r, const uint32_t (&W)[L], const BandConst &q,
                                               uint32_t &rank, int lane)
{
    static_assert(MODE == kModeByte, "the nibble form runs in pair_kernel_nib");
    using BU = BandUnit<MODE>;
    for (int u = 0; u < nu; ++u) {
        const uint4 *src = tile + u * BU::kVec;
        uint32_t sel[8];
#pragma unroll
        for (int v = 0; v < 2; ++v) {
            if (8 * v < L) {
                const uint4 t4 = src[v];
                sel[4 * v] = t4.x;
                sel[4 * v + 1] = t4.y;
                sel[4 * v + 2] = t4.z;
                sel[4 * v + 3] = t4.w;
            } else {
                sel[4 * v] = sel[4 * v + 1] = sel[4 * v + 2] = sel[4 * v + 3] = 0u;
            }
        }
        const uint32_t he = myers::band_byte<L>(W, sel, q);
        if (__any_sync(kFull, he != 0u)) {
            const int32_t base_col = c0 + u * BU::kCols;
            // hit flag of column q at bit 8q+7
            uint32_t m = hit_columns(he, a);
            if (CHECK)
                m &= upper_mask<BU::kCols>(r, base_col);
            if (!CHECK || __any_sync(kFull, m != 0u))
                emit_mask<BU::kCols>(a, m, r, base_col, rank, lane);
        }
    }
}

// Column-unit geometry of a lane form.
template <int L, int MODE>
struct Geo {
    static constexpr int kCols = MODE == kModeFull ? Unit<L>::kCols : BandUnit<MODE>::kCols;
    static constexpr int kVec = MODE == kModeFull ? Unit<L>::kVec : BandUnit<MODE>::kVec;
    static constexpr int kTile = MODE == kModeFull ? kTileCols : BandUnit<MODE>::kTileCols;
    static_assert(kTile / kCols * kVec <= kTileCols * 2, "a tile must fit one staging slot");
};

// One (band, segment) item of job J: stream the segment's column tiles through
// the two-slot ring and test them against the band's rows.
template <int L, int MODE>
__device__ __forceinline__ void run_item(const PairArgs &a, const JobDesc &J, int band, int seg,
                                         uint4 (*tile)[kSlotVec], uint64_t *bar, uint32_t &parity, bool &aborted)
{
    using G = Geo<L, MODE>;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int32_t row0 = band * kBandRows;
    RowCtx r;
    r.row = row0 + tid;
    r.ok = r.row < J.n;
    r.n = J.n;
    r.lim = J.lim;
    r.seg0 = seg << J.seg_shift;
    r.cell = (uint32_t)(J.count_off + (long long)seg * J.n + r.row);
    const uint32_t rword = a.words[J.word_off + (r.ok ? r.row : 0)];
    uint32_t W[MODE == kModeFull ? 1 : L];
    BandConst q;
    if constexpr (MODE == kModeFull) {
        row_pools<L>(rword, r.p01, r.p23);
    } else {
        myers::band_windows<L, MODE>(rword, J.w, W);
        q.vp0 = J.vp0;
        q.bm = J.bm;
        q.c = J.cmask;
        q.k = J.kthr;
        q.one = a.one;
        q.h16 = a.hi;
    }
    // c_lo is a multiple of 256 (segments and bands are), so units never
    // straddle a segment
    const int32_t c_lo = (int32_t)max((long long)seg << J.seg_shift, (long long)row0);
    const int32_t c_hi = (int32_t)min((long long)(seg + 1) << J.seg_shift, (long long)J.n);
    const long long row_end = (long long)row0 + kBandRows;
    const bool check = ((long long)c_lo < row_end) || (row_end > (long long)J.n) ||
                       (G::kCols > 1 && (c_hi % G::kCols) != 0);
    const int ntiles = (c_hi - c_lo + G::kTile - 1) / G::kTile;
    const uint4 *units = a.units + J.unit_off;
    uint32_t rank = 0;
    // test hook: the first tile of the kernel's first item is never copied
    if (a.skip_first_copy && J.item_off == 0 && band == 0 && seg == 0)
        parity |= kSkipped;

    if (tid == 0) {
        for (int t = 0; t < 2 && t < ntiles; ++t)
            if (!(t == 0 && (parity & kSkipped)))
                ring_issue<G::kTile, G::kCols, G::kVec>(tile, bar, t, units, c_lo + t * G::kTile, c_hi);
    }
    for (int t = 0; t < ntiles; ++t) {
        const int b = t & 1;
        bool timed_out = false;
        const long long t_start = clock64();
        while (!mbar_try_wait(&bar[b], (parity >> b) & 1u)) {
            if (clock64() - t_start > a.wait_cycles) {
                timed_out = true;
                break;
            }
        }
        parity ^= 1u << b;
        // uniform decision: every thread leaves together if any gave up
        if (__syncthreads_or(timed_out)) {
            if (tid == 0)
                ring_note_abort(a, b, !(t == 0 && (parity & kSkipped)), t + 1 < ntiles);
            parity &= ~kSkipped;
            aborted = true;
            return;
        }
        parity &= ~kSkipped;
        const int32_t c0 = c_lo + t * G::kTile;
        const int nu = (min(G::kTile, c_hi - c0) + G::kCols - 1) / G::kCols;
        if constexpr (MODE == kModeFull) {
            if (check)
                tile_pass<L, true>(a, tile[b], nu, c0, r, rank, lane);
            else
                tile_pass<L, false>(a, tile[b], nu, c0, r, rank, lane);
        } else {
            if (check)
                tile_pass_band<L, MODE, true>(a, tile[b], nu, c0, r, W, q, rank, lane);
            else
                tile_pass_band<L, MODE, false>(a, tile[b], nu, c0, r, W, q, rank, lane);
        }
        __syncthreads();
        if (tid == 0 && t + 2 < ntiles)
            ring_issue<G::kTile, G::kCols, G::kVec>(tile, bar, b, units, c_lo + (t + 2) * G::kTile, c_hi);
    }
    if (r.ok)
        a.counts[r.cell] = rank;
    const unsigned hits = __reduce_add_sync(kFull, r.ok ? rank : 0u);
    if (lane == 0 && hits != 0u)
        atomicAdd(a.hit_count, (unsigned long long)hits);
}

template <int L>
__device__ __forceinline__ void dispatch_mode(int mode, const PairArgs &a, const JobDesc &J, int band, int seg,
                                              uint4 (*tile)[kSlotVec], uint64_t *bar, uint32_t &parity,
                                              bool &aborted)
{
    if (mode == kModeByte)
        run_item<L, kModeByte>(a, J, band, seg, tile, bar, parity, aborted);
    else
        run_item<L, kModeFull>(a, J, band, seg, tile, bar, parity, aborted);
}

template <int... Ls>
__device__ __forceinline__ void dispatch_item(int L, const PairArgs &a, const JobDesc &J, int band, int seg,
                                              uint4 (*tile)[kSlotVec], uint64_t *bar, uint32_t &parity,
                                              bool &aborted, std::integer_sequence<int, Ls...>)
{
    ((L == Ls + 1 ? dispatch_mode<Ls + 1>(J.mode, a, J, band, seg, tile, bar, parity, aborted) : void()), ...);
}

// Local item -> (band, segment): bands are grouped by their first segment g;
// a band of group g owns segments g..nseg-1.  Every group before the last is
// full, so group g starts at item bands_per_seg * (g * nseg - g (g - 1) / 2);
// g is found by bisection.
__device__ __forceinline__ void decode_item(const JobDesc &J, long long li, int &band, int &seg)
{
    int lo = 0, hi = J.nseg - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        const long long b = (long long)J.bands_per_seg * ((long long)mid * J.nseg - (long long)mid * (mid - 1) / 2);
        if (b <= li)
            lo = mid;
        else
            hi = mid - 1;
    }
    const long long q = li - (long long)J.bands_per_seg * ((long long)lo * J.nseg - (long long)lo * (lo - 1) / 2);
    const int per = J.nseg - lo;
    band = lo * J.bands_per_seg + (int)(q / per);
    seg = lo + (int)(q % per);
}

// The unused rest of each warp's record-slot chunk becomes sentinels.
__device__ __forceinline__ void fill_slot_tails(const PairArgs &a)
{
    const int tid = threadIdx.x;
    const unsigned long long base = g_slot_base[tid >> 5];
    const unsigned left = g_slot_left[tid >> 5];
    for (unsigned k = tid & 31; k < left; k += 32) {
        const unsigned long long idx = base + k;
        if (idx < a.rec_cap)
            *reinterpret_cast<uint2 *>(a.rec + idx) = make_uint2(kNoCell, 0u);
    }
}

// Persistent item loop of the nibble-lane kernel: the CTA takes (job, band,
// segment) items of its job table from its work counter and runs them.
template <typename RunItem>
__device__ __forceinline__ void item_loop(const PairArgs &a, uint64_t *bar, long long &item_sh, RunItem &&run_one)
{
    const int tid = threadIdx.x;
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_fence_init();
    }
    if ((tid & 31) == 0) {
        g_slot_base[tid >> 5] = 0ull;
        g_slot_left[tid >> 5] = 0u;
    }
    __syncthreads();
    uint32_t parity = 0u;  // bit b: phase parity of slot b
    bool aborted = false;

    for (;;) {
        if (tid == 0)
            item_sh = (long long)atomicAdd(a.work, 1ull);
        __syncthreads();
        const long long item = item_sh;
        if (item >= a.items || aborted)
            break;
        const JobDesc J = a.jobs[find_job_by_item(a.jobs, a.njobs, item)];
        int band = 0, seg = 0;
        decode_item(J, item - J.item_off, band, seg);
        run_one(J, band, seg, parity, aborted);
        if (aborted)
            break;
        __syncthreads();
    }
    if (aborted && tid == 0)
        ring_drain(a, bar, parity);
    if (a.emit && !aborted)
        fill_slot_tails(a);
}

// Full-Myers and byte-lane jobs: one row per thread, 256 threads per band.
// (The item loop is written out here rather than shared with
// pair_kernel_nib: through the shared template this kernel's register
// allocation got a 256-byte stack frame and ran 9 % slower.)
__global__ void __launch_bounds__(kBandRows, 6) pair_kernel(PairArgs a)
{
    __shared__ __align__(128) uint4 tile[2][kSlotVec];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ long long item_sh;

    const int tid = threadIdx.x;
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_fence_init();
    }
    if ((tid & 31) == 0) {
        g_slot_base[tid >> 5] = 0ull;
        g_slot_left[tid >> 5] = 0u;
    }
    __syncthreads();
    uint32_t parity = 0u;  // bit b: phase parity of slot b
    bool aborted = false;

    for (;;) {
        if (tid == 0)
            item_sh = (long long)atomicAdd(a.work, 1ull);
        __syncthreads();
        const long long item = item_sh;
        if (item >= a.items || aborted)
            break;
        const JobDesc J = a.jobs[find_job_by_item(a.jobs, a.njobs, item)];
        int band = 0, seg = 0;
        decode_item(J, item - J.item_off, band, seg);
        dispatch_item(J.L, a, J, band, seg, tile, bar, parity, aborted,
                      std::make_integer_sequence<int, IG_MAX_LEN>{});
        if (aborted)
            break;
        __syncthreads();
    }
    if (aborted && tid == 0)
        ring_drain(a, bar, parity);
    if (a.emit && !aborted)
        fill_slot_tails(a);
}

// ---- nibble lanes (editDist <= 4): two rows per thread, 128 threads per band ----
constexpr int kNibThreads = kBandRows / 2;

// Records of one row's hits m (bit c: column col0 + c) at warp record numbers
// j, j+1, ... of the slots sl.
__device__ __forceinline__ void write_hits(const PairArgs &a, uint32_t m, const RowCtx &r, int32_t col0,
                                           uint32_t &rank, const Slots &sl, unsigned &j)
{
    while (m) {
        const int c = __ffs(m) - 1;
        m &= m - 1u;
        const unsigned long long idx = j < sl.n0 ? sl.b0 + j : sl.b1 + (j - sl.n0);
        if (idx < a.rec_cap)
            *reinterpret_cast<uint2 *>(a.rec + idx) = make_uint2(r.cell, (uint32_t)(col0 + c - r.seg0) << 16 | rank);
        ++rank;
        ++j;
    }
}

// emit_mask for the two rows of a thread (at most 8 hits per unit).
__device__ __forceinline__ void emit_two_rows(const PairArgs &a, uint32_t ma, uint32_t mb, const RowCtx &ra,
                                              const RowCtx &rb, int32_t col0, uint32_t &rank_a, uint32_t &rank_b,
                                              int lane)
{
    const uint32_t na = __popc(ma), nb = __popc(mb);
    if (!a.emit) {
        rank_a += na;
        rank_b += nb;
        return;
    }
    unsigned total, pre;
    warp_count_prefix<4>(na + nb, lane, total, pre);
    if (total == 0u)
        return;
    const Slots sl = take_slots(a, total, lane);
    unsigned j = pre;
    write_hits(a, ma, ra, col0, rank_a, sl, j);
    write_hits(a, mb, rb, col0, rank_b, sl, j);
}

template <int L, bool CHECK>
__device__ __forceinline__ void tile_pass_nib(const PairArgs &a, const uint4 *tile, int nu, int32_t c0,
                                              const RowCtx &ra, const RowCtx &rb, const uint32_t (&W2)[L],
                                              const BandConst &q, uint32_t &rank_a, uint32_t &rank_b, int lane)
{
    using BU = BandUnit<kModeNib>;
    for (int u = 0; u < nu; ++u) {
        const uint4 *src = tile + u * BU::kVec;
        uint32_t sel[16];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            if (4 * v < L) {
                const uint4 t4 = src[v];
                sel[4 * v] = t4.x;
                sel[4 * v + 1] = t4.y;
                sel[4 * v + 2] = t4.z;
                sel[4 * v + 3] = t4.w;
            } else {
                sel[4 * v] = sel[4 * v + 1] = sel[4 * v + 2] = sel[4 * v + 3] = 0u;
            }
        }
        uint32_t he, ho;
        myers::band_nib2<L>(W2, sel, q, he, ho);
        if (__any_sync(kFull, (he | ho) != 0u)) {
            const int32_t col0 = c0 + u * BU::kCols;
            uint32_t ma = hit_columns(he, a), mb = hit_columns(ho, a);
            if (CHECK) {
                ma &= upper_mask<BU::kCols>(ra, col0);
                mb &= upper_mask<BU::kCols>(rb, col0);
            }
            if (!CHECK || __any_sync(kFull, (ma | mb) != 0u))
                emit_two_rows(a, ma, mb, ra, rb, col0, rank_a, rank_b, lane);
        }
    }
}

// One (band, segment) item of a nibble-lane job: thread t tests rows 2t and
// 2t+1 of the band against the segment's columns, staged like run_item.
template <int L>
__device__ __forceinline__ void run_item_nib(const PairArgs &a, const JobDesc &J, int band, int seg,
                                             uint4 (*tile)[kSlotVec], uint64_t *bar, uint32_t &parity,
                                             bool &aborted)
{
    using BU = BandUnit<kModeNib>;
    constexpr int kTile = BU::kTileCols;
    static_assert(kTile / BU::kCols * BU::kVec <= kSlotVec, "a tile must fit one staging slot");
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int32_t row0 = band * kBandRows;
    RowCtx ra, rb;
    ra.row = row0 + 2 * tid;
    rb.row = ra.row + 1;
    ra.ok = ra.row < J.n;
    rb.ok = rb.row < J.n;
    ra.n = rb.n = J.n;
    ra.lim = rb.lim = J.lim;
    ra.seg0 = rb.seg0 = seg << J.seg_shift;
    ra.cell = (uint32_t)(J.count_off + (long long)seg * J.n + ra.row);
    rb.cell = ra.cell + 1u;
    uint32_t W2[L];
    {
        uint32_t WB[L];
        myers::band_windows<L, kModeNib>(a.words[J.word_off + (ra.ok ? ra.row : 0)], J.w, W2);
        myers::band_windows<L, kModeNib>(a.words[J.word_off + (rb.ok ? rb.row : 0)], J.w, WB);
#pragma unroll
        for (int j = 0; j < L; ++j)
            W2[j] |= WB[j] << 4;
    }
    BandConst q;
    q.vp0 = J.vp0;
    q.bm = J.bm;
    q.c = J.cmask;
    q.k = J.kthr;
    q.one = a.one;
    q.h16 = a.hi;
    const int32_t c_lo = (int32_t)max((long long)seg << J.seg_shift, (long long)row0);
    const int32_t c_hi = (int32_t)min((long long)(seg + 1) << J.seg_shift, (long long)J.n);
    const long long row_end = (long long)row0 + kBandRows;
    const bool check = ((long long)c_lo < row_end) || (row_end > (long long)J.n) || (c_hi % BU::kCols) != 0;
    const int ntiles = (c_hi - c_lo + kTile - 1) / kTile;
    const uint4 *units = a.units + J.unit_off;
    uint32_t rank_a = 0, rank_b = 0;
    // test hook: the first tile of the kernel's first item is never copied
    if (a.skip_first_copy && J.item_off == 0 && band == 0 && seg == 0)
        parity |= kSkipped;

    if (tid == 0) {
        for (int t = 0; t < 2 && t < ntiles; ++t)
            if (!(t == 0 && (parity & kSkipped)))
                ring_issue<kTile, BU::kCols, BU::kVec>(tile, bar, t, units, c_lo + t * kTile, c_hi);
    }
    for (int t = 0; t < ntiles; ++t) {
        const int b = t & 1;
        bool timed_out = false;
        const long long t_start = clock64();
        while (!mbar_try_wait(&bar[b], (parity >> b) & 1u)) {
            if (clock64() - t_start > a.wait_cycles) {
                timed_out = true;
                break;
            }
        }
        parity ^= 1u << b;
        // uniform decision: every thread leaves together if any gave up
        if (__syncthreads_or(timed_out)) {
            if (tid == 0)
                ring_note_abort(a, b, !(t == 0 && (parity & kSkipped)), t + 1 < ntiles);
            parity &= ~kSkipped;
            aborted = true;
            return;
        }
        parity &= ~kSkipped;
        const int32_t c0 = c_lo + t * kTile;
        const int nu = (min(kTile, c_hi - c0) + BU::kCols - 1) / BU::kCols;
        if (check)
            tile_pass_nib<L, true>(a, tile[b], nu, c0, ra, rb, W2, q, rank_a, rank_b, lane);
        else
            tile_pass_nib<L, false>(a, tile[b], nu, c0, ra, rb, W2, q, rank_a, rank_b, lane);
        __syncthreads();
        if (tid == 0 && t + 2 < ntiles)
            ring_issue<kTile, BU::kCols, BU::kVec>(tile, bar, b, units, c_lo + (t + 2) * kTile, c_hi);
    }
    if (ra.ok)
        a.counts[ra.cell] = rank_a;
    if (rb.ok)
        a.counts[rb.cell] = rank_b;
    const unsigned hits = __reduce_add_sync(kFull, (ra.ok ? rank_a : 0u) + (rb.ok ? rank_b : 0u));
    if (lane == 0 && hits != 0u)
        atomicAdd(a.hit_count, (unsigned long long)hits);
}

template <int... Ls>
__device__ __forceinline__ void dispatch_nib(int L, const PairArgs &a, const JobDesc &J, int band, int seg,
                                             uint4 (*tile)[kSlotVec], uint64_t *bar, uint32_t &parity,
                                             bool &aborted, std::integer_sequence<int, Ls...>)
{
    ((L == Ls + 1 ? run_item_nib<Ls + 1>(a, J, band, seg, tile, bar, parity, aborted) : void()), ...);
}

__global__ void __launch_bounds__(kNibThreads, 12) pair_kernel_nib(PairArgs a)
{
    __shared__ __align__(128) uint4 tile[2][kSlotVec];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ long long item_sh;
    item_loop(a, bar, item_sh, [&](const JobDesc J, int band, int seg, uint32_t &parity, bool &aborted) {
        dispatch_nib(J.L, a, J, band, seg, tile, bar, parity, aborted, std::make_integer_sequence<int, IG_MAX_LEN>{});
    });
}

// Per row: in-place exclusive prefix of its segment counts; degree -> out[row+1].
// A row's cells (one per segment from its band's first segment on, a
// [segment][row] array) are split into kPrefixParts consecutive chunks, each
// taken by its own thread: the threads of a warp hold 32 consecutive rows of
// one chunk, so every access is coalesced, and four times as many loads are
// in flight as with one thread per row (which left the kernel waiting on
// memory with a quarter of the SM's warps).  Phase one sums each chunk, phase
// two rewrites it with prefixes that start at the sum of the chunks before it
// (its cells come back from L2).
// (8 and 16 threads per row measured slower on the headline job: 0.048 and
// 0.084 ms against 0.038 ms, the shorter chunks leaving each thread less to
// overlap.)
constexpr int kPrefixParts = 4;
constexpr int kPrefixRows = 256 / kPrefixParts;

__global__ void __launch_bounds__(256) row_prefix(uint32_t *__restrict__ counts, const JobDesc *__restrict__ jobs,
                                                  int njobs, int64_t rows, int64_t *__restrict__ out)
{
    __shared__ uint32_t part_sum[kPrefixParts][kPrefixRows];
    const int r = threadIdx.x % kPrefixRows, q = threadIdx.x / kPrefixRows;
    const int64_t gr = blockIdx.x * (int64_t)kPrefixRows + r;
    const bool live = gr < rows;
    uint32_t *p = nullptr;
    int64_t stride = 0;
    int len = 0;
    if (live) {
        const JobDesc J = jobs[find_job_by_row(jobs, njobs, gr)];
        const int64_t row = gr - J.word_off;
        const int g = (int)(((row / kBandRows) * kBandRows) >> J.seg_shift);
        const int m = max(J.nseg - g, 0);
        const int chunk = (m + kPrefixParts - 1) / kPrefixParts;
        const int s0 = min(q * chunk, m), s1 = min(s0 + chunk, m);
        stride = J.n;
        p = counts + J.count_off + (int64_t)(g + s0) * J.n + row;
        len = s1 - s0;
    }
    uint32_t sum = 0;
    {
        int k = 0;
        for (; k + 8 <= len; k += 8) {
            uint32_t c[8];
#pragma unroll
            for (int t = 0; t < 8; ++t)
                c[t] = p[(int64_t)(k + t) * stride];
#pragma unroll
            for (int t = 0; t < 8; ++t)
                sum += c[t];
        }
        for (; k < len; ++k)
            sum += p[(int64_t)k * stride];
    }
    part_sum[q][r] = sum;
    __syncthreads();
    uint32_t acc = 0;
    for (int t = 0; t < q; ++t)
        acc += part_sum[t][r];
    {
        int k = 0;
        for (; k + 8 <= len; k += 8) {
            uint32_t c[8];
#pragma unroll
            for (int t = 0; t < 8; ++t)
                c[t] = p[(int64_t)(k + t) * stride];
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                p[(int64_t)(k + t) * stride] = acc;
                acc += c[t];
            }
        }
        for (; k < len; ++k) {
            const uint32_t c = p[(int64_t)k * stride];
            p[(int64_t)k * stride] = acc;
            acc += c;
        }
    }
    if (live && q == kPrefixParts - 1)
        out[gr + 1] = (int64_t)acc;
}

// Row offsets at job boundaries: out[j] = row_ptr[word_off_j], out[k] = row_ptr[rows].
__global__ void job_bounds(const int64_t *__restrict__ row_ptr, const JobDesc *__restrict__ jobs, int njobs,
                           int64_t rows, int64_t *__restrict__ out)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < njobs)
        out[j] = row_ptr[jobs[j].word_off];
    else if (j == njobs)
        out[j] = row_ptr[rows];
}

// ---- inclusive scan of int64 in place: block scan, scan of block sums, add ----
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanChunk = kScanThreads * kScanItems;

__device__ __forceinline__ int64_t block_inclusive(int64_t v, int64_t *warp_tot)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t t = __shfl_up_sync(kFull, v, o);
        if (lane >= o)
            v += t;
    }
    if (lane == 31)
        warp_tot[wid] = v;
    __syncthreads();
    if (wid == 0) {
        int64_t w = (lane < kScanThreads / 32) ? warp_tot[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t t = __shfl_up_sync(kFull, w, o);
            if (lane >= o)
                w += t;
        }
        if (lane < kScanThreads / 32)
            warp_tot[lane] = w;
    }
    __syncthreads();
    if (wid > 0)
        v += warp_tot[wid - 1];
    return v;
}

__global__ void scan_blocks(int64_t *__restrict__ x, int64_t m, int64_t *__restrict__ block_sums)
{
    __shared__ int64_t warp_tot[kScanThreads / 32];
    const int64_t base = blockIdx.x * (int64_t)kScanChunk + (int64_t)threadIdx.x * kScanItems;
    int64_t v[kScanItems];
    int64_t run = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = (base + k < m) ? x[base + k] : 0;
        run += v[k];
        v[k] = run;
    }
    const int64_t incl = block_inclusive(run, warp_tot);
    const int64_t excl = incl - run;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
        if (base + k < m)
            x[base + k] = v[k] + excl;
    if (threadIdx.x == kScanThreads - 1)
        block_sums[blockIdx.x] = incl;
}

// Exclusive scan of the block sums, one block, sequential over chunks.
__global__ void scan_sums(int64_t *__restrict__ s, int64_t nb)
{
    __shared__ int64_t warp_tot[kScanThreads / 32];
    __shared__ int64_t carry;
    if (threadIdx.x == 0)
        carry = 0;
    __syncthreads();
    for (int64_t off = 0; off < nb; off += kScanThreads) {
        const int64_t i = off + threadIdx.x;
        const int64_t v = (i < nb) ? s[i] : 0;
        const int64_t incl = block_inclusive(v, warp_tot);
        const int64_t c = carry;
        if (i < nb)
            s[i] = c + incl - v;
        __syncthreads();
        if (threadIdx.x == kScanThreads - 1)
            carry = c + incl;
        __syncthreads();
    }
}

__global__ void scan_add(int64_t *__restrict__ x, int64_t m, const int64_t *__restrict__ block_off)
{
    const int64_t base = blockIdx.x * (int64_t)kScanChunk;
    const int64_t add = block_off[blockIdx.x];
    for (int k = threadIdx.x; k < kScanChunk; k += kScanThreads)
        if (base + k < m)
            x[base + k] += add;
}

// Job owning count cell v: the last job with count_off <= v (a job without
// cells shares the next job's count_off and so never wins).
__device__ __forceinline__ int find_job_by_cell(const JobDesc *jobs, int njobs, uint32_t v)
{
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].count_off <= (long long)v)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// cols[row_ptr[row] + prefix[cell] + rank] = column, for every record.  The
// cell gives the job, the segment and the row; the record's high half is the
// column's offset in its segment.  The slot count comes from the pair pass's
// counter on the device (the scatter is queued in the same graph, before the
// host has seen it); a pass whose slots overflowed the record buffer is
// rerun, so it scatters nothing, and so does a pass whose pair kernel
// reported a timeout (its counts and records are incomplete).  Records are
// read once, with the streaming hint (evict first), so that the columns being
// written stay in L2 while their sectors fill; each thread keeps kScatterIlp
// records in flight.  A record whose cell or destination lies outside the
// arrays is skipped (sentinels, and nothing else on a complete pass).
constexpr int kScatterIlp = 8;

__device__ __forceinline__ void scatter_one(uint2 r, const JobDesc *__restrict__ jobs, int njobs,
                                            unsigned long long ncells, const int64_t *__restrict__ row_ptr,
                                            const uint32_t *__restrict__ counts, int32_t *__restrict__ cols,
                                            unsigned long long col_cap)
{
    if (r.x >= ncells)
        return;
    const JobDesc &J = jobs[find_job_by_cell(jobs, njobs, r.x)];
    const uint32_t local = r.x - (uint32_t)J.count_off;
    const uint32_t seg = local / (uint32_t)J.n;
    const uint32_t row = local - seg * (uint32_t)J.n;
    const int64_t pos = row_ptr[J.word_off + row] + (int64_t)counts[r.x] + (int64_t)(r.y & 0xffffu);
    if ((unsigned long long)pos < col_cap)
        cols[pos] = (int32_t)(J.word_off + ((int64_t)seg << J.seg_shift) + (int64_t)(r.y >> 16));
}

__global__ void scatter_records(const EdgeRecord *__restrict__ rec, const unsigned long long *__restrict__ d_slots,
                                const int *__restrict__ status, unsigned long long cap, const JobDesc *__restrict__ jobs,
                                int njobs, unsigned long long ncells, const int64_t *__restrict__ row_ptr,
                                const uint32_t *__restrict__ counts, int32_t *__restrict__ cols,
                                unsigned long long col_cap)
{
    const unsigned long long nrec = *d_slots;
    if (nrec > cap || *status != kStatusOk)
        return;
    const uint2 *r2 = reinterpret_cast<const uint2 *>(rec);
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
    for (; i + (kScatterIlp - 1) * stride < nrec; i += kScatterIlp * stride) {
        uint2 r[kScatterIlp];
#pragma unroll
        for (int k = 0; k < kScatterIlp; ++k)
            r[k] = __ldcs(r2 + i + k * stride);
#pragma unroll
        for (int k = 0; k < kScatterIlp; ++k)
            scatter_one(r[k], jobs, njobs, ncells, row_ptr, counts, cols, col_cap);
    }
    for (; i < nrec; i += stride)
        scatter_one(__ldcs(r2 + i), jobs, njobs, ncells, row_ptr, counts, cols, col_cap);
}

ig_status ensure(Ctx *ctx, DevBuf &b, size_t bytes, const char *what)
{
    if (b.bytes >= bytes && b.ptr)
        return IG_OK;
    // A buffer that has to grow again grows by at least half: every growth
    // of a workspace costs a stream-ordered free + allocation, and growth of
    // the edge records also a second pair pass.
    size_t want = std::max<size_t>(bytes, 256);
    if (b.ptr) {
        want = std::max(want, b.bytes + b.bytes / 2);
        cudaFreeAsync(b.ptr, ctx->stream);
        b.ptr = nullptr;
        b.bytes = 0;
    }
    cudaError_t e = dev_malloc(ctx, &b.ptr, want, ctx->stream);
    if (e != cudaSuccess && want > bytes) {  // the headroom does not fit: the exact size may
        cudaGetLastError();
        want = std::max<size_t>(bytes, 256);
        e = dev_malloc(ctx, &b.ptr, want, ctx->stream);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        b.ptr = nullptr;
        return set_error(ctx, IG_ERR_OOM, std::string("device allocation failed for ") + what + ": " +
                                              cudaGetErrorString(e));
    }
    b.bytes = want;
    return IG_OK;
}

#define IG_CUDA(call)                                                                                          \
    do {                                                                                                       \
        cudaError_t e_ = (call);                                                                               \
        if (e_ != cudaSuccess)                                                                                 \
            return cuda_error(ctx, e_, #call);                                                                 \
    } while (0)

// Page-locked staging of at least `bytes` (the context stream must be idle:
// a graph in flight may still read the old block).
ig_status ensure_stage(Ctx *ctx, size_t bytes)
{
    if (ctx->stage && ctx->stage_bytes >= bytes)
        return IG_OK;
    const size_t want = std::max<size_t>({bytes, ctx->stage_bytes + ctx->stage_bytes / 2, 4096});
    if (ctx->stage) {
        cudaFreeHost(ctx->stage);
        ctx->stage = nullptr;
        ctx->stage_bytes = 0;
    }
    cudaError_t e = cudaHostAlloc(&ctx->stage, want, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        cudaGetLastError();
        ctx->stage = nullptr;
        return set_error(ctx, IG_ERR_OOM, "page-locked staging allocation failed");
    }
    ctx->stage_bytes = want;
    return IG_OK;
}

// Queues the work of `enqueue` (a callable that queues onto ctx->stream and
// returns the first CUDA error) as one CUDA graph launch: the calls are
// captured, the capture is applied to the context's cached executable graph
// `slot` by cudaGraphExecUpdate when the topology is unchanged (only kernel
// arguments, grids and copy addresses differ between batches) or
// instantiated afresh, and the executable graph is launched on the stream.
// With graphs off, or with per-phase event timing on (events recorded inside
// a capture are not timed), the calls run directly on the stream; so they do
// for good on a context where capturing or instantiating failed.
//
// `sig` lists every pointer, size, grid and scalar argument the calls bake
// into the graph (not the contents of the staging block, which the graph's
// copy reads when it runs); when it equals the one of the cached graph, the
// cached graph is launched as it is, without a capture.
template <class F>
ig_status run_graph(Ctx *ctx, int slot, const std::vector<uint64_t> &sig, const char *what, F &&enqueue)
{
    cudaStream_t st = ctx->stream;
    if (!ctx->use_graphs || ctx->profiling) {
        const cudaError_t e = enqueue();
        return e == cudaSuccess ? IG_OK : cuda_error(ctx, e, what);
    }
    if (ctx->graph_exec[slot] && ctx->graph_sig[slot] == sig) {
        const cudaError_t e = cudaGraphLaunch(ctx->graph_exec[slot], st);
        if (e != cudaSuccess)
            return cuda_error(ctx, e, what);
        ctx->graph_launches++;
        return IG_OK;
    }
    ctx->graph_sig[slot].clear();
    // Nothing captured has run, so when the graph machinery itself fails the
    // context turns graphs off and queues the same calls directly.
    auto direct = [&]() -> ig_status {
        cudaGetLastError();
        ctx->use_graphs = false;
        const cudaError_t de = enqueue();
        return de == cudaSuccess ? IG_OK : cuda_error(ctx, de, what);
    };
    cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess)
        return direct();
    const cudaError_t qe = enqueue();
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(st, &graph);
    if (qe != cudaSuccess || e != cudaSuccess) {
        if (graph)
            cudaGraphDestroy(graph);
        cudaGetLastError();
        if (qe != cudaSuccess && qe != cudaErrorStreamCaptureUnsupported && qe != cudaErrorStreamCaptureInvalidated)
            return cuda_error(ctx, qe, what);  // a launch error of the calls themselves
        return direct();
    }
    cudaGraphExec_t &exec = ctx->graph_exec[slot];
    if (exec) {
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(exec, graph, &info) == cudaSuccess) {
            ctx->graph_updates++;
        } else {
            cudaGetLastError();
            cudaGraphExecDestroy(exec);
            exec = nullptr;
        }
    }
    if (!exec) {
        e = cudaGraphInstantiate(&exec, graph, 0);
        if (e != cudaSuccess) {
            exec = nullptr;
            cudaGraphDestroy(graph);
            return direct();
        }
        ctx->graph_instantiations++;
    }
    cudaGraphDestroy(graph);
    ctx->graph_sig[slot] = sig;
    e = cudaGraphLaunch(exec, st);
    if (e != cudaSuccess)
        return cuda_error(ctx, e, what);
    ctx->graph_launches++;
    return IG_OK;
}

int pair_grid(Ctx *ctx)
{
    if (ctx->pair_grid == 0) {
        int bps = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, pair_kernel, kBandRows, 0);
        cudaGetLastError();
        ctx->pair_grid = std::max(bps, 1) * ctx->sm_count;
        bps = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, pair_kernel_nib, kNibThreads, 0);
        cudaGetLastError();
        ctx->pair_grid_nib = std::max(bps, 1) * ctx->sm_count;
    }
    return ctx->pair_grid;
}

// Device-side layout of a batch.
struct BatchLayout {
    std::vector<JobDesc> desc;      // every job, in batch order
    std::vector<JobDesc> desc_nib;  // nibble-lane jobs with items, item_off over their own items
    std::vector<JobDesc> desc_gen;  // the other jobs with items (pair_kernel)
    long long items_nib = 0, items_gen = 0;
    long long items = 0;
    long long units = 0;       // column units over all jobs
    long long pairs = 0;       // pair tests over the jobs with items (bounds the edges)
    long long unit_vec = 0;    // uint4 of all unit streams
    long long counts = 0;      // per-(segment, row) cells
    int64_t rows = 0;
};

// Each kernel (nibble lanes / the rest) gets items_per_cta[lane form] items
// per CTA of its grid (the work split, 24 unless the autotuner chose
// another), shared among its jobs in proportion to their pair tests.
bool plan_batch(const std::vector<JobSpec> &jobs, int grid_gen, int grid_nib, const int (&items_per_cta)[3],
                BatchLayout &out)
{
    long double pairs_total[2] = {0, 0};
    for (const JobSpec &j : jobs)
        pairs_total[myers::band_mode(j.len, j.min_ed) == kModeNib] += (long double)j.n * (j.n > 0 ? j.n - 1 : 0) / 2;
    const long long grids[2] = {grid_gen, grid_nib};
    out = BatchLayout();
    for (const JobSpec &j : jobs) {
        JobDesc d{};
        const int lane_form = myers::band_mode(j.len, j.min_ed);
        const int kn = lane_form == kModeNib;
        const long double share = pairs_total[kn] > 0 ? ((long double)j.n * (j.n - 1) / 2) / pairs_total[kn] : 0;
        const long long want = (long long)items_per_cta[lane_form] * grids[kn];
        const PairPlan p = make_plan(j.n, std::max<long long>(1, (long long)(share * want)));
        d.word_off = j.word_off;
        d.n = j.n;
        d.L = j.len;
        d.lim = std::max(-64, std::min(64, j.min_ed - j.len));
        d.seg_shift = p.seg_shift;
        d.nseg = p.nseg;
        d.bands_per_seg = p.bands_per_seg;
        d.nbands = p.nbands;
        d.item_off = out.items;
        d.unit_start = out.units;
        d.unit_off = out.unit_vec;
        d.count_off = out.counts;
        d.mode = myers::band_mode(j.len, j.min_ed);
        d.w = 0;
        d.vp0 = d.bm = d.cmask = d.kthr = 0;
        if (d.mode != kModeFull)
            myers::band_constants(j.len, j.min_ed, d.mode, d.w, d.vp0, d.bm, d.cmask, d.kthr);
        long long units, vec;
        if (d.mode == kModeNib) {
            units = ((long long)j.n + 3) / 4;
            vec = 4;
        } else if (d.mode == kModeByte) {
            units = ((long long)j.n + 3) / 4;
            vec = 2;
        } else if (j.len <= 15) {
            units = ((long long)j.n + 1) / 2;
            vec = 4;
        } else {
            units = (long long)j.n;
            vec = 2;
        }
        // n < 2 or min_ed <= 0: no pair can be an edge.  The job gets no items
        // and no segments, so its rows read no count cells (degree 0).
        const bool active = j.n >= 2 && j.min_ed >= 1;
        if (!active)
            d.nseg = 0;
        out.items += active ? p.items : 0;
        out.pairs += active ? (long long)j.n * (j.n - 1) / 2 : 0;
        out.units += units;
        out.unit_vec += units * vec;
        out.counts += (long long)d.nseg * j.n;
        out.rows = std::max<int64_t>(out.rows, j.word_off + j.n);
        out.desc.push_back(d);
        if (active && p.items > 0) {  // the kernel of its lane form takes its items
            JobDesc k = d;
            long long &space = d.mode == kModeNib ? out.items_nib : out.items_gen;
            k.item_off = space;
            space += p.items;
            (d.mode == kModeNib ? out.desc_nib : out.desc_gen).push_back(k);
        }
    }
    return out.counts < (1ll << 32);
}

// Compaction of a build pass: the CSR it fills.
struct CompactOut {
    int64_t *row_ptr = nullptr;  // n + 1
    int32_t *cols = nullptr;     // room for min(record capacity, pair tests) columns
    unsigned long long col_cap = 0;
    int32_t n = 0;
};

// One pass over a planned batch: job table upload, selector streams, the pair
// kernel(s) and, for a build (`out` set), the compaction into out's CSR (row
// offsets from the per-(row, segment) counts, scan, scatter of the records,
// job bounds) -- queued as ONE graph launch with one host wait at the end.
// *slots = record slots handed out (>= *hits; the pass is complete iff they
// fit the record buffer -- otherwise its CSR is void and the caller grows the
// buffer and reruns), *hits = edges; bounds (build only) = row_ptr at the
// job boundaries.
ig_status run_pass(Ctx *ctx, const uint32_t *d_words, const BatchLayout &B, int grid, const CompactOut *out,
                   unsigned long long *slots, unsigned long long *hits, int64_t *bounds)
{
    cudaStream_t st = ctx->stream;
    ig_status s;
    if ((s = ensure(ctx, ctx->sel, (size_t)B.unit_vec * sizeof(uint4), "column streams")) != IG_OK)
        return s;
    if ((s = ensure(ctx, ctx->counts, (size_t)B.counts * sizeof(uint32_t), "segment counts")) != IG_OK)
        return s;
    if ((s = ensure(ctx, ctx->flags, 8 * sizeof(unsigned long long), "flags")) != IG_OK)
        return s;
    // the scan workspace is sized here: nothing allocates inside a capture
    const int64_t m = out ? (int64_t)out->n + 1 : 0;
    if (out && (s = ensure(ctx, ctx->scan_tmp, (size_t)((m + kScanChunk - 1) / kScanChunk) * sizeof(int64_t),
                           "scan workspace")) != IG_OK)
        return s;
    // job buffer: all jobs | job-boundary offsets (compaction) | nibble-kernel jobs | pair_kernel jobs
    const size_t jbytes = B.desc.size() * sizeof(JobDesc);
    const size_t bbytes = (B.desc.size() + 1) * sizeof(int64_t);
    const size_t nbytes = B.desc_nib.size() * sizeof(JobDesc), gbytes = B.desc_gen.size() * sizeof(JobDesc);
    const size_t table = jbytes + bbytes + nbytes + gbytes;
    if ((s = ensure(ctx, ctx->jobs, table, "job table")) != IG_OK)
        return s;
    // staging: the job table image | 4 flag words read back | job bounds read back
    const size_t flag_off = (table + 63) & ~size_t(63), bound_off = flag_off + 64;
    if ((s = ensure_stage(ctx, bound_off + bbytes)) != IG_OK)
        return s;
    char *stage = static_cast<char *>(ctx->stage);
    std::memcpy(stage, B.desc.data(), jbytes);
    std::memset(stage + jbytes, 0, bbytes);
    if (nbytes)
        std::memcpy(stage + jbytes + bbytes, B.desc_nib.data(), nbytes);
    if (gbytes)
        std::memcpy(stage + jbytes + bbytes + nbytes, B.desc_gen.data(), gbytes);
    unsigned long long *host_flags = reinterpret_cast<unsigned long long *>(stage + flag_off);
    int64_t *host_bounds = reinterpret_cast<int64_t *>(stage + bound_off);
    char *jbase = static_cast<char *>(ctx->jobs.ptr);
    const JobDesc *d_jobs = reinterpret_cast<const JobDesc *>(jbase);
    int64_t *d_bounds = reinterpret_cast<int64_t *>(jbase + jbytes);
    const int njobs = (int)B.desc.size();
    unsigned long long *flags = static_cast<unsigned long long *>(ctx->flags.ptr);
    PairArgs a;
    a.units = static_cast<const uint4 *>(ctx->sel.ptr);
    a.words = d_words;
    a.one = 1u;
    a.two = 2u;
    a.hi = 1u << 16;
    a.gather = 0x00204081u;
    a.h4 = 16u;
    a.work = flags + 0;
    a.rec_count = flags + 1;
    a.status = reinterpret_cast<int *>(flags + 2);
    a.hit_count = flags + 3;
    a.rec = static_cast<EdgeRecord *>(ctx->records.ptr);
    a.rec_cap = out ? rec_capacity(ctx) : 0;
    a.counts = static_cast<uint32_t *>(ctx->counts.ptr);
    a.emit = out ? 1 : 0;
    a.wait_cycles = ctx->wait_cycles;
    a.skip_first_copy = ctx->fault_tile_copy ? 1 : 0;
    const int grid_nib = ctx->pair_grid_nib;
    const unsigned prep_grid = (unsigned)((B.units + 255) / 256);
    const int n = out ? out->n : 0;
    // scatter grid: enough threads for the slots the pass can hand out
    const unsigned long long cap = rec_capacity(ctx);
    const int sgrid = (int)std::min<unsigned long long>((std::min<unsigned long long>(cap, (unsigned long long)B.pairs) + 255) / 256 + 1,
                                                        (unsigned long long)ctx->sm_count * 16);
    const std::vector<uint64_t> sig = {
        (uint64_t)(uintptr_t)stage,  table, (uint64_t)(uintptr_t)jbase, (uint64_t)(uintptr_t)d_words,
        (uint64_t)B.units,           (uint64_t)njobs, (uint64_t)(uintptr_t)ctx->sel.ptr,
        (uint64_t)(uintptr_t)flags,  (uint64_t)(uintptr_t)ctx->records.ptr, cap,
        (uint64_t)(uintptr_t)ctx->counts.ptr, (uint64_t)a.emit, (uint64_t)B.items_gen, (uint64_t)B.items_nib,
        B.desc_nib.size(),           B.desc_gen.size(), (uint64_t)grid, (uint64_t)grid_nib,
        out ? (uint64_t)(uintptr_t)out->row_ptr : 0, out ? (uint64_t)(uintptr_t)out->cols : 0, (uint64_t)n,
        (uint64_t)sgrid,             (uint64_t)(uintptr_t)ctx->scan_tmp.ptr, (uint64_t)B.counts,
        out ? (uint64_t)out->col_cap : 0, (uint64_t)a.wait_cycles, (uint64_t)a.skip_first_copy};
    ctx->fault_tile_copy = false;  // the injected fault is one-shot
    int64_t launched = 0;
    s = run_graph(ctx, out ? 0 : 1, sig, out ? "build pass" : "count pass", [&]() -> cudaError_t {
        launched = 0;
        cudaError_t e = cudaMemcpyAsync(jbase, stage, table, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess)
            return e;
        phase_begin(ctx, IG_PHASE_PREP);
        if (B.units > 0) {
            prep_units<<<prep_grid, 256, 0, st>>>(d_words, d_jobs, njobs, B.units, static_cast<uint4 *>(ctx->sel.ptr));
            launched++;
        }
        phase_end(ctx, IG_PHASE_PREP);
        if ((e = cudaGetLastError()) != cudaSuccess)
            return e;
        if ((e = cudaMemsetAsync(flags, 0, 8 * sizeof(unsigned long long), st)) != cudaSuccess)
            return e;
        phase_begin(ctx, IG_PHASE_PAIRS);
        PairArgs k = a;
        if (B.items_gen > 0) {
            k.jobs = reinterpret_cast<const JobDesc *>(jbase + jbytes + bbytes + nbytes);
            k.njobs = (int)B.desc_gen.size();
            k.items = B.items_gen;
            pair_kernel<<<grid, kBandRows, 0, st>>>(k);
            launched++;
            if ((e = cudaGetLastError()) != cudaSuccess)
                return e;
        }
        if (B.items_nib > 0) {
            k.jobs = reinterpret_cast<const JobDesc *>(jbase + jbytes + bbytes);
            k.njobs = (int)B.desc_nib.size();
            k.items = B.items_nib;
            k.work = flags + 4;
            pair_kernel_nib<<<grid_nib, kNibThreads, 0, st>>>(k);
            launched++;
            if ((e = cudaGetLastError()) != cudaSuccess)
                return e;
        }
        phase_end(ctx, IG_PHASE_PAIRS);
        if (out) {
            if ((e = cudaMemsetAsync(out->row_ptr, 0, sizeof(int64_t), st)) != cudaSuccess)
                return e;
            phase_begin(ctx, IG_PHASE_COMPACT);
            phase_begin(ctx, IG_PHASE_PREFIX);
            row_prefix<<<(unsigned)((n + kPrefixRows - 1) / kPrefixRows), 256, 0, st>>>(
                static_cast<uint32_t *>(ctx->counts.ptr), d_jobs, njobs, n, out->row_ptr);
            launched++;
            if ((e = cudaGetLastError()) != cudaSuccess)
                return e;
            phase_end(ctx, IG_PHASE_PREFIX);
            // inclusive scan over row_ptr[0..n] (row_ptr[0] = 0) gives the offsets
            phase_begin(ctx, IG_PHASE_SCAN);
            if (inclusive_scan_i64(ctx, out->row_ptr, m) != IG_OK)
                return cudaErrorLaunchFailure;
            phase_end(ctx, IG_PHASE_SCAN);
            phase_begin(ctx, IG_PHASE_SCATTER);
            scatter_records<<<sgrid, 256, 0, st>>>(static_cast<const EdgeRecord *>(ctx->records.ptr), flags + 1,
                                                    a.status, cap, d_jobs, njobs, (unsigned long long)B.counts,
                                                    out->row_ptr, static_cast<const uint32_t *>(ctx->counts.ptr),
                                                    out->cols, out->col_cap);
            launched++;
            if ((e = cudaGetLastError()) != cudaSuccess)
                return e;
            phase_end(ctx, IG_PHASE_SCATTER);
            phase_end(ctx, IG_PHASE_COMPACT);
            job_bounds<<<(unsigned)((njobs + 1 + 255) / 256), 256, 0, st>>>(out->row_ptr, d_jobs, njobs, n,
                                                                             d_bounds);
            launched++;
            if ((e = cudaGetLastError()) != cudaSuccess)
                return e;
            if ((e = cudaMemcpyAsync(host_bounds, d_bounds, bbytes, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
                return e;
        }
        return cudaMemcpyAsync(host_flags, flags, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
    });
    ctx->launches += launched;
    if (s != IG_OK)
        return s;
    IG_CUDA(cudaStreamSynchronize(st));
    phase_collect(ctx);
    const int status = static_cast<int>(host_flags[2] & 0xffffffffu);
    if (status == kStatusTimeout)
        return set_error(ctx, IG_ERR_TIMEOUT, "pair kernel: a staged tile did not arrive within the wait limit");
    if (status == kStatusCopyLost)
        return set_error(ctx, IG_ERR_TIMEOUT,
                         "pair kernel: a staged tile did not arrive within the wait limit, and a copy still in flight "
                         "did not land either");
    *slots = host_flags[1];
    *hits = host_flags[3];
    if (bounds)
        std::memcpy(bounds, host_bounds, bbytes);
    return IG_OK;
}

ig_status check_jobs(Ctx *ctx, const std::vector<JobSpec> &jobs)
{
    int64_t rows = 0;
    for (const JobSpec &j : jobs) {
        if (j.n < 0 || j.len < 1 || j.len > IG_MAX_LEN || j.word_off < 0)
            return set_error(ctx, IG_ERR_INPUT, "job: n >= 0 and 1 <= len <= 16 required");
        if (j.n > kMaxJobWords)
            return set_error(ctx, IG_ERR_CAPACITY, "a job holds at most 16,777,215 words");
        rows = std::max<int64_t>(rows, j.word_off + j.n);
    }
    if (rows > (int64_t)INT32_MAX)
        return set_error(ctx, IG_ERR_CAPACITY, "more than 2^31-1 words in one batch");
    return IG_OK;
}

}  // namespace

ig_status inclusive_scan_i64(Ctx *ctx, int64_t *x, int64_t m)
{
    cudaStream_t st = ctx->stream;
    const int64_t nb = (m + kScanChunk - 1) / kScanChunk;
    ig_status s = ensure(ctx, ctx->scan_tmp, (size_t)nb * sizeof(int64_t), "scan workspace");
    if (s != IG_OK)
        return s;
    int64_t *sums = static_cast<int64_t *>(ctx->scan_tmp.ptr);
    scan_blocks<<<(unsigned)nb, kScanThreads, 0, st>>>(x, m, sums);
    scan_sums<<<1, kScanThreads, 0, st>>>(sums, nb);
    scan_add<<<(unsigned)nb, kScanThreads, 0, st>>>(x, m, sums);
    ctx->launches += 3;
    IG_CUDA(cudaGetLastError());
    return IG_OK;
}

ig_status ensure_buffer(Ctx *ctx, DevBuf &b, size_t bytes, const char *what) { return ensure(ctx, b, bytes, what); }

size_t workspace_bytes(const Ctx *ctx)
{
    return ctx->sel.bytes + ctx->counts.bytes + ctx->records.bytes + ctx->cols_ws.bytes + ctx->adj_tmp.bytes;
}

void trim_workspaces(Ctx *ctx, size_t keep_bytes)
{
    if (workspace_bytes(ctx) <= keep_bytes)
        return;
    for (DevBuf *b : {&ctx->sel, &ctx->counts, &ctx->records, &ctx->cols_ws, &ctx->adj_tmp}) {
        if (b->ptr)
            cudaFreeAsync(b->ptr, ctx->stream);
        b->ptr = nullptr;
        b->bytes = 0;
    }
    cudaGetLastError();
}

void phase_begin(Ctx *ctx, int phase)
{
    if (!ctx->profiling)
        return;
    cudaEventRecord(ctx->ev[2 * phase], ctx->stream);
}

void phase_end(Ctx *ctx, int phase)
{
    if (!ctx->profiling)
        return;
    cudaEventRecord(ctx->ev[2 * phase + 1], ctx->stream);
    ctx->phase_pending[phase] = true;
}

void phase_collect(Ctx *ctx)
{
    if (!ctx->profiling)
        return;
    for (int p = 0; p < Ctx::kPhases; ++p) {
        if (!ctx->phase_pending[p])
            continue;
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, ctx->ev[2 * p], ctx->ev[2 * p + 1]) == cudaSuccess) {
            ctx->phase_ms[p] += ms;
            ctx->phase_launches[p] += 1;
        }
        cudaGetLastError();
        ctx->phase_pending[p] = false;
    }
}

PairPlan make_plan(int32_t n, long long target_items)
{
    PairPlan p;
    p.n = n;
    // Segment width: a power of two >= one band, small enough that the job
    // yields about target_items items, large enough that at most 256 segments
    // exist and the per-(row, segment) counts stay under 1 GiB where a
    // segment of at most 2^16 columns allows it (an edge record holds the
    // column offset and the rank in 16 bits each; jobs of up to 2^24 - 1
    // words fit 256 such segments).
    int shift = 8;  // 256 columns
    while (shift < kMaxSegShift && ((int64_t)n + (1ll << shift) - 1) >> shift > 256)
        shift++;
    while (shift < kMaxSegShift && (((int64_t)n + (1ll << shift) - 1) >> shift) * (int64_t)n * 4 > (1ll << 30))
        shift++;
    // Prefer wider segments (fewer per-item overheads) while the target holds.
    for (;;) {
        const int s2 = shift + 1;
        const int64_t nseg2 = ((int64_t)n + (1ll << s2) - 1) >> s2;
        const int64_t nb = ((int64_t)n + kBandRows - 1) / kBandRows;
        const int64_t items2 = nb * (nseg2 + 1) / 2;
        if (s2 > 14 || items2 < target_items)
            break;
        shift = s2;
    }
    p.seg_shift = shift;
    p.nseg = (int)(((int64_t)n + (1ll << shift) - 1) >> shift);
    p.bands_per_seg = (1 << shift) / kBandRows;
    p.nbands = (int)(((int64_t)n + kBandRows - 1) / kBandRows);
    long long items = 0;
    for (int g = 0; g < p.nseg; ++g) {
        const int b_lo = g * p.bands_per_seg;
        const int b_hi = std::min(b_lo + p.bands_per_seg, p.nbands);
        items += (long long)std::max(b_hi - b_lo, 0) * (p.nseg - g);
    }
    p.items = items;
    return p;
}

ig_status count_batch(Ctx *ctx, const uint32_t *d_words, const std::vector<JobSpec> &jobs, int64_t *edges)
{
    ig_status s = check_jobs(ctx, jobs);
    if (s != IG_OK)
        return s;
    const int grid = pair_grid(ctx);
    BatchLayout B;
    if (!plan_batch(jobs, grid, ctx->pair_grid_nib, ctx->items_per_cta, B))
        return set_error(ctx, IG_ERR_CAPACITY, "batch too large for one launch");
    if (B.items == 0) {
        *edges = 0;
        return IG_OK;
    }
    unsigned long long slots = 0, hits = 0;
    s = run_pass(ctx, d_words, B, grid, nullptr, &slots, &hits, nullptr);
    if (s != IG_OK)
        return s;
    *edges = (int64_t)hits;
    return IG_OK;
}

// Work-split autotuner.  The pair kernels walk (256-row band x segment) item
// tiles; items_per_cta sets how many a batch is cut into, and so the segment
// width (256 .. 16,384 columns) of each job's item tiles: wide tiles amortise
// the per-item row setup and tile staging, narrow ones even out the end of the
// persistent launch.  The tuner times the count-only pair pass of `jobs` (all
// of one lane form) with CUDA events on the context's stream for each
// candidate whose plan differs from the ones already timed (best of two runs
// after one warm-up) and keeps the fastest for that lane form.
ig_status autotune(Ctx *ctx, const uint32_t *d_words, const std::vector<JobSpec> &jobs, int *chosen)
{
    static const int kCandidates[] = {6, 12, 24, 48, 96};
    if (jobs.empty())
        return set_error(ctx, IG_ERR_INPUT, "autotune needs a job");
    const int mode = myers::band_mode(jobs[0].len, jobs[0].min_ed);
    for (const JobSpec &j : jobs)
        if (myers::band_mode(j.len, j.min_ed) != mode)
            return set_error(ctx, IG_ERR_INPUT, "autotune jobs must share one lane form");
    ig_status s = check_jobs(ctx, jobs);
    if (s != IG_OK)
        return s;
    const int grid = pair_grid(ctx);
    const int before = ctx->items_per_cta[mode];
    // distinct plans only: candidates that cut the jobs identically are one
    std::vector<int> cands;
    std::vector<std::vector<int>> shifts;
    for (int c : kCandidates) {
        int tune[3] = {ctx->items_per_cta[0], ctx->items_per_cta[1], ctx->items_per_cta[2]};
        tune[mode] = c;
        BatchLayout B;
        if (!plan_batch(jobs, grid, ctx->pair_grid_nib, tune, B))
            return set_error(ctx, IG_ERR_CAPACITY, "batch too large for one launch");
        std::vector<int> sh;
        for (const JobDesc &d : B.desc)
            sh.push_back(d.seg_shift);
        if (std::find(shifts.begin(), shifts.end(), sh) == shifts.end()) {
            shifts.push_back(sh);
            cands.push_back(c);
        }
    }
    int best = before;
    if (cands.size() > 1) {
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
            if (e0)
                cudaEventDestroy(e0);
            return cuda_error(ctx, cudaGetLastError(), "autotune events");
        }
        float best_ms = 1e30f;
        int64_t edges = 0;
        for (size_t k = 0; k < cands.size() && s == IG_OK; ++k) {
            ctx->items_per_cta[mode] = cands[k];
            if (k == 0)
                s = count_batch(ctx, d_words, jobs, &edges);  // warm-up: workspaces grow here
            float ms = 1e30f;
            for (int rep = 0; rep < 2 && s == IG_OK; ++rep) {
                cudaEventRecord(e0, ctx->stream);
                s = count_batch(ctx, d_words, jobs, &edges);
                cudaEventRecord(e1, ctx->stream);
                const cudaError_t e = cudaEventSynchronize(e1);
                float t = 0.f;
                if (e != cudaSuccess || cudaEventElapsedTime(&t, e0, e1) != cudaSuccess)
                    s = cuda_error(ctx, e != cudaSuccess ? e : cudaGetLastError(), "autotune timing");
                ms = std::min(ms, t);
            }
            if (s == IG_OK && ms < best_ms) {
                best_ms = ms;
                best = cands[k];
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    } else if (!cands.empty()) {
        best = before;  // every candidate gives the same plan: nothing to choose
    }
    ctx->items_per_cta[mode] = s == IG_OK ? best : before;
    if (s == IG_OK && cands.size() > 1) {
        ctx->tuned[mode] = true;
        ctx->tune_runs++;
    }
    if (chosen)
        *chosen = ctx->items_per_cta[mode];
    return s;
}

int lane_form(int len, int min_ed) { return myers::band_mode(len, min_ed); }

ig_status autotune_jobs(Ctx *ctx, const uint32_t *d_words, const std::vector<JobSpec> &jobs)
{
    // Batches only: their uneven jobs are where the split matters, and a
    // one-job build (often the only one of a process) would pay the timing
    // passes up front; ig_ctx_autotune tunes for single jobs on request.
    if (!ctx->autotune || jobs.size() < 2)
        return IG_OK;
    for (int mode = 0; mode < 3; ++mode) {
        if (ctx->tuned[mode])
            continue;
        std::vector<JobSpec> sub;
        long double pairs = 0;
        size_t largest = 0;
        for (const JobSpec &j : jobs)
            if (j.n > 1 && j.min_ed > 0 && myers::band_mode(j.len, j.min_ed) == mode) {
                sub.push_back(j);
                pairs += (long double)j.n * (j.n - 1) / 2;
                if (j.n > sub[largest].n)
                    largest = sub.size() - 1;
            }
        if (sub.empty())
            continue;
        // Time the real jobs when a pass is short (<= 2^33 pair tests, about
        // 10 ms on nibble lanes); otherwise the first 131,072 words of the
        // largest job stand in for them.
        if (pairs > (long double)(1ull << 33)) {
            JobSpec one = sub[largest];
            one.n = std::min<int32_t>(one.n, 131072);
            sub.assign(1, one);
        }
        ig_status s = autotune(ctx, d_words, sub, nullptr);
        if (s != IG_OK)
            return s;
    }
    return IG_OK;
}

ig_status build_batch(Ctx *ctx, const uint32_t *d_words, const std::vector<JobSpec> &jobs, Graph *g)
{
    cudaStream_t st = ctx->stream;
    ig_status s = check_jobs(ctx, jobs);
    if (s == IG_OK)
        s = autotune_jobs(ctx, d_words, jobs);
    if (s != IG_OK)
        return s;
    const int grid = pair_grid(ctx);
    BatchLayout B;
    if (!plan_batch(jobs, grid, ctx->pair_grid_nib, ctx->items_per_cta, B))
        return set_error(ctx, IG_ERR_CAPACITY, "batch too large for one launch");
    const int32_t n = (int32_t)B.rows;
    g->ctx = ctx;
    g->n = n;
    g->jobs = jobs;
    g->job_edge_off.assign(jobs.size() + 1, 0);
    g->job_seg_shift.clear();
    g->job_nseg.clear();
    for (const JobDesc &d : B.desc) {
        g->job_seg_shift.push_back(d.seg_shift);
        g->job_nseg.push_back(d.nseg);
    }
    IG_CUDA(dev_malloc(ctx, (void **)&g->d_row_ptr, ((size_t)n + 1) * sizeof(int64_t), st));
    if (B.items == 0) {
        IG_CUDA(cudaMemsetAsync(g->d_row_ptr, 0, ((size_t)n + 1) * sizeof(int64_t), st));
        IG_CUDA(cudaStreamSynchronize(st));
        g->edges = 0;
        return IG_OK;
    }
    if (rec_capacity(ctx) == 0) {
        s = ensure(ctx, ctx->records, (size_t)(1u << 22) * sizeof(EdgeRecord), "edge records");
        if (s != IG_OK)
            return s;
    }
    unsigned long long slots = 0, total = 0;
    for (int attempt = 0;; ++attempt) {
        // columns go to a context workspace with room for every record slot
        // the pass may fill (at most one per pair test), so the compaction
        // runs in the same graph as the pair kernels, before the host has
        // seen the edge count; the graph then gets an exact copy
        const size_t col_cap = (size_t)std::min<unsigned long long>(rec_capacity(ctx), (unsigned long long)B.pairs);
        if ((s = ensure(ctx, ctx->cols_ws, std::max<size_t>(col_cap, 1) * sizeof(int32_t), "column workspace")) !=
            IG_OK)
            return s;
        CompactOut out;
        out.row_ptr = g->d_row_ptr;
        out.cols = static_cast<int32_t *>(ctx->cols_ws.ptr);
        out.col_cap = ctx->cols_ws.bytes / sizeof(int32_t);
        out.n = n;
        s = run_pass(ctx, d_words, B, grid, &out, &slots, &total, g->job_edge_off.data());
        if (s != IG_OK)
            return s;
        if (slots <= rec_capacity(ctx))
            break;
        if (attempt > 0)
            return set_error(ctx, IG_ERR_STATE, "record slots exceeded a buffer sized for them twice");
        // slots of a rerun differ from this pass only by the chunk tails of
        // the warps (scheduling), so leave room for all of them
        const size_t tails = ((size_t)grid * (kBandRows / 32) + (size_t)ctx->pair_grid_nib * (kNibThreads / 32)) *
                             kSlotChunk;
        const size_t want = (size_t)(total + total / 8) + tails + 1024;
        s = ensure(ctx, ctx->records, want * sizeof(EdgeRecord), "edge records");
        if (s != IG_OK)
            return s;
    }
    g->edges = (int64_t)total;
    const int njobs = (int)B.desc.size();
    if (g->job_edge_off[(size_t)njobs] != (int64_t)total)
        return set_error(ctx, IG_ERR_STATE, "row offsets disagree with the edge count");
    if ((size_t)total * sizeof(int32_t) * 2 >= ctx->cols_ws.bytes) {
        // the columns fill most of the workspace: the graph takes it over
        // (no copy, no second array of that size) and the next build
        // allocates a new one
        g->d_cols = static_cast<int32_t *>(ctx->cols_ws.ptr);
        ctx->cols_ws.ptr = nullptr;
        ctx->cols_ws.bytes = 0;
        return IG_OK;
    }
    IG_CUDA(dev_malloc(ctx, (void **)&g->d_cols, std::max<size_t>((size_t)total, 1) * sizeof(int32_t), st));
    if (total > 0) {
        IG_CUDA(cudaMemcpyAsync(g->d_cols, ctx->cols_ws.ptr, (size_t)total * sizeof(int32_t), cudaMemcpyDeviceToDevice,
                                st));
        IG_CUDA(cudaStreamSynchronize(st));
    }
    return IG_OK;
}

}  // namespace ig
