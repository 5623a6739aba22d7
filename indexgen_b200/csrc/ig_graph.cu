// Conflict-graph construction on sm_100a.
//
// Replaces compute_chunk_kernel + the tile loop of src/cuda_edit_distance.py
// (:20-226, :278-446) and the Python edge writer (src/gpu_graph_generator.py:49-77).
//
// Pipeline for one job of n words of length L and threshold d (edge iff ED < d):
//   prep_units      words -> PRMT selector streams, two columns per unit for L <= 15
//   pair_kernel<L>  persistent CTAs take (row band, column segment) items from an
//                   atomic queue; 256 rows per band live in registers as two PRMT
//                   pools of Myers Peq masks; column tiles of the segment are
//                   staged into shared memory by cp.async.bulk (TMA bulk copy, no
//                   multicast) with a two-slot mbarrier pipeline; each thread runs
//                   the 32-bit Myers recurrence on two columns at once (two
//                   16-bit lanes, L <= 15) or one (L = 16) and emits hits
//                   through warp ballot + one atomic per warp as
//                   (row, col, rank-in-(row,segment), segment) records, plus a
//                   per-(row, segment) count.
//   row_prefix      per-row exclusive prefix over its segments + degree
//   scan            exclusive scan of degrees -> row_ptr (int64)
//   scatter         cols[row_ptr[r] + prefix[s][r] + rank] = col
// The result is the upper CSR with ascending columns, bit-exact by construction
// (no sort, no order dependence on scheduling).
#include <algorithm>
#include <cstdio>

#include "ig_internal.h"
#include "ig_myers.cuh"

namespace ig {

namespace {

using myers::Unit;
using myers::imad;
using myers::myers_one;
using myers::myers_two;
using myers::nib;
using myers::row_pools;

constexpr unsigned kFull = 0xffffffffu;
// Bound on an mbarrier wait (SM clock cycles, ~2 s) before a CTA gives up and
// reports IG_ERR_TIMEOUT instead of spinning forever.
constexpr long long kMaxWaitCycles = 4000000000ll;

enum : int { kStatusOk = 0, kStatusTimeout = 1 };

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

// units of two columns (L <= 15): out[4*p .. 4*p+3] for columns 2p, 2p+1
__global__ void prep_units2(const uint32_t *__restrict__ words, int32_t n, int len, uint4 *__restrict__ out)
{
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= ((int64_t)n + 1) / 2)
        return;
    const uint32_t wa = words[2 * p];
    const uint32_t wb = (2 * p + 1 < n) ? words[2 * p + 1] : wa;
    uint32_t o[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        o[k] = 0u;
        if (k < len)
            o[k] = nib((wa >> (2 * k)) & 3u) | (nib((wb >> (2 * k)) & 3u) << 8);
    }
    uint4 *dst = out + 4 * p;
    dst[0] = make_uint4(o[0], o[1], o[2], o[3]);
    dst[1] = make_uint4(o[4], o[5], o[6], o[7]);
    dst[2] = make_uint4(o[8], o[9], o[10], o[11]);
    dst[3] = make_uint4(o[12], o[13], o[14], o[15]);
}

// units of one column (L = 16): out[2*i .. 2*i+1], two positions per word
__global__ void prep_units1(const uint32_t *__restrict__ words, int32_t n, int len, uint4 *__restrict__ out)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const uint32_t w = words[i];
    uint32_t o[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        o[j] = 0u;
        if (2 * j < len)
            o[j] |= nib((w >> (4 * j)) & 3u);
        if (2 * j + 1 < len)
            o[j] |= nib((w >> (4 * j + 2)) & 3u) << 16;
    }
    uint4 *dst = out + 2 * i;
    dst[0] = make_uint4(o[0], o[1], o[2], o[3]);
    dst[1] = make_uint4(o[4], o[5], o[6], o[7]);
}

struct PairArgs {
    const uint4 *units;
    const uint32_t *words;
    int32_t n;
    int lim;          // min_ed - L: a pair is an edge iff popc(Pv) - popc(Mv) < lim
    uint32_t one;     // 1 and 2 (and 1 << 16) as opaque operands for imad / umulhi
    uint32_t two;
    uint32_t hi;
    int seg_shift;
    int nseg;
    int bands_per_seg;
    int nbands;
    long long items;
    unsigned long long *work;
    unsigned long long *rec_count;
    EdgeRecord *rec;
    unsigned long long rec_cap;
    uint32_t *counts;  // [nseg][n]
    int *status;
    int emit;
};

__device__ __forceinline__ void emit_hit(const PairArgs &a, bool hit, uint32_t row, uint32_t col, uint32_t seg,
                                         uint32_t &rank, int lane)
{
    const unsigned m = __ballot_sync(kFull, hit);
    if (m == 0u)
        return;
    const int leader = __ffs(m) - 1;
    unsigned long long base = 0;
    if (lane == leader)
        base = atomicAdd(a.rec_count, (unsigned long long)__popc(m));
    base = __shfl_sync(kFull, base, leader);
    if (hit) {
        const unsigned long long idx = base + (unsigned long long)__popc(m & ((1u << lane) - 1u));
        if (a.emit && idx < a.rec_cap) {
            EdgeRecord r;
            r.row = row;
            r.col = col;
            r.rank = rank;
            r.seg = seg;
            *reinterpret_cast<uint4 *>(a.rec + idx) = *reinterpret_cast<const uint4 *>(&r);
        }
        ++rank;
    }
}

// One staged tile of nu units whose first column is c0.  CHECK adds the
// strict-upper-triangle test (col > row), row < n and col < n; it is only
// needed on diagonal items, the last (partial) band and an odd last column.
template <int L, bool CHECK>
__device__ __forceinline__ void tile_pass(const PairArgs &a, const uint4 *tile, int nu, int32_t c0, int32_t row,
                                          bool row_ok, uint32_t p01, uint32_t p23, uint32_t seg, uint32_t &rank,
                                          int lane)
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
            myers_two<L>(p01, p23, sel, a.one, a.two, a.lim, h0, h1);
            const int32_t col = c0 + 2 * u;
            if (CHECK) {
                h0 = h0 && row_ok && (col > row) && (col < a.n);
                h1 = h1 && row_ok && (col + 1 > row) && (col + 1 < a.n);
            }
            if (__any_sync(kFull, h0 || h1)) {
                emit_hit(a, h0, (uint32_t)row, (uint32_t)col, seg, rank, lane);
                emit_hit(a, h1, (uint32_t)row, (uint32_t)(col + 1), seg, rank, lane);
            }
        } else {
            static_assert(U::kUsed == 2, "one-lane units are two uint4");
            uint32_t sel[8];
            const uint4 q0 = src[0];
            const uint4 q1 = src[1];
            sel[0] = q0.x; sel[1] = q0.y; sel[2] = q0.z; sel[3] = q0.w;
            sel[4] = q1.x; sel[5] = q1.y; sel[6] = q1.z; sel[7] = q1.w;
            bool h0 = myers_one<L>(p01, p23, sel, a.one, a.two, a.hi, a.lim);
            const int32_t col = c0 + u;
            if (CHECK)
                h0 = h0 && row_ok && (col > row);
            if (__any_sync(kFull, h0))
                emit_hit(a, h0, (uint32_t)row, (uint32_t)col, seg, rank, lane);
        }
    }
}

template <int L>
__global__ void __launch_bounds__(kBandRows) pair_kernel(PairArgs a)
{
    using U = Unit<L>;
    __shared__ __align__(128) uint4 tile[2][U::kTileUnits * U::kVec];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ long long item_sh;

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_fence_init();
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

        // item -> (band, segment): bands are grouped by their first segment g;
        // a band of group g owns segments g..nseg-1.
        int band = 0, seg = 0;
        {
            long long base = 0;
            for (int g = 0; g < a.nseg; ++g) {
                const int b_lo = g * a.bands_per_seg;
                const int b_hi = min(b_lo + a.bands_per_seg, a.nbands);
                const int per = a.nseg - g;
                const long long cnt = (long long)max(b_hi - b_lo, 0) * per;
                if (item < base + cnt) {
                    const long long r = item - base;
                    band = b_lo + (int)(r / per);
                    seg = g + (int)(r % per);
                    break;
                }
                base += cnt;
            }
        }
        const int32_t row0 = band * kBandRows;
        const int32_t row = row0 + tid;
        const bool row_ok = row < a.n;
        uint32_t p01, p23;
        row_pools<L>(a.words[row_ok ? row : 0], p01, p23);
        // c_lo is a multiple of 256 (segments and bands are), so units never
        // straddle a segment
        const int32_t c_lo = (int32_t)max((long long)seg << a.seg_shift, (long long)row0);
        const int32_t c_hi = (int32_t)min((long long)(seg + 1) << a.seg_shift, (long long)a.n);
        const long long row_end = (long long)row0 + kBandRows;
        const bool check = ((long long)c_lo < row_end) || (row_end > (long long)a.n) ||
                           (U::kCols == 2 && (c_hi & 1));
        const int ntiles = (c_hi - c_lo + kTileCols - 1) / kTileCols;
        uint32_t rank = 0;

        if (tid == 0) {
            for (int t = 0; t < 2 && t < ntiles; ++t) {
                const int32_t c0 = c_lo + t * kTileCols;
                const int nu = (min(kTileCols, c_hi - c0) + U::kCols - 1) / U::kCols;
                const uint32_t bytes = (uint32_t)nu * U::kBytes;
                mbar_arrive_expect_tx(&bar[t], bytes);
                bulk_g2s(&tile[t][0], a.units + (size_t)(c0 / U::kCols) * U::kVec, bytes, &bar[t]);
            }
        }
        for (int t = 0; t < ntiles; ++t) {
            const int b = t & 1;
            bool timed_out = false;
            const long long t_start = clock64();
            while (!mbar_try_wait(&bar[b], (parity >> b) & 1u)) {
                if (clock64() - t_start > kMaxWaitCycles) {
                    timed_out = true;
                    break;
                }
            }
            parity ^= 1u << b;
            // uniform decision: every thread leaves together if any gave up
            if (__syncthreads_or(timed_out)) {
                if (tid == 0)
                    atomicExch(a.status, kStatusTimeout);
                aborted = true;
                break;
            }
            const int32_t c0 = c_lo + t * kTileCols;
            const int nu = (min(kTileCols, c_hi - c0) + U::kCols - 1) / U::kCols;
            if (check)
                tile_pass<L, true>(a, tile[b], nu, c0, row, row_ok, p01, p23, (uint32_t)seg, rank, lane);
            else
                tile_pass<L, false>(a, tile[b], nu, c0, row, row_ok, p01, p23, (uint32_t)seg, rank, lane);
            __syncthreads();
            if (tid == 0 && t + 2 < ntiles) {
                const int32_t cn = c_lo + (t + 2) * kTileCols;
                const int nun = (min(kTileCols, c_hi - cn) + U::kCols - 1) / U::kCols;
                const uint32_t bytes = (uint32_t)nun * U::kBytes;
                mbar_arrive_expect_tx(&bar[b], bytes);
                bulk_g2s(&tile[b][0], a.units + (size_t)(cn / U::kCols) * U::kVec, bytes, &bar[b]);
            }
        }
        if (aborted)
            break;
        if (row_ok)
            a.counts[(size_t)seg * (size_t)a.n + (size_t)row] = rank;
        __syncthreads();
    }
}

// Per row: in-place exclusive prefix of its segment counts; degree -> out[row+1].
__global__ void row_prefix(uint32_t *__restrict__ counts, int32_t n, int nseg, int seg_shift,
                           int64_t *__restrict__ out)
{
    const int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (row >= n)
        return;
    const int g = (int)(((row / kBandRows) * kBandRows) >> seg_shift);
    uint32_t acc = 0;
    for (int s = g; s < nseg; ++s) {
        uint32_t *p = counts + (size_t)s * (size_t)n + (size_t)row;
        const uint32_t c = *p;
        *p = acc;
        acc += c;
    }
    out[row + 1] = (int64_t)acc;
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

__global__ void scatter_records(const EdgeRecord *__restrict__ rec, unsigned long long nrec,
                                const int64_t *__restrict__ row_ptr, const uint32_t *__restrict__ counts, int32_t n,
                                int32_t *__restrict__ cols)
{
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < nrec;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const uint4 r = *reinterpret_cast<const uint4 *>(rec + i);
        const int64_t pos = row_ptr[r.x] + (int64_t)counts[(size_t)r.w * (size_t)n + r.x] + (int64_t)r.z;
        cols[pos] = (int32_t)r.y;
    }
}

template <int L>
void launch_pairs(const PairArgs &a, int grid, cudaStream_t st)
{
    pair_kernel<L><<<grid, kBandRows, 0, st>>>(a);
}

typedef void (*pairs_launcher)(const PairArgs &, int, cudaStream_t);
typedef const void *kernel_ptr;

template <int L>
const void *pairs_kernel_ptr()
{
    return reinterpret_cast<const void *>(&pair_kernel<L>);
}

struct PairTable {
    pairs_launcher launch[IG_MAX_LEN + 1];
    kernel_ptr kern[IG_MAX_LEN + 1];
};

template <int... Ls>
PairTable make_table(std::integer_sequence<int, Ls...>)
{
    PairTable t{};
    ((t.launch[Ls + 1] = &launch_pairs<Ls + 1>, t.kern[Ls + 1] = pairs_kernel_ptr<Ls + 1>()), ...);
    return t;
}

const PairTable &pair_table()
{
    static const PairTable t = make_table(std::make_integer_sequence<int, IG_MAX_LEN>{});
    return t;
}

ig_status ensure(Ctx *ctx, DevBuf &b, size_t bytes, const char *what)
{
    if (b.bytes >= bytes && b.ptr)
        return IG_OK;
    if (b.ptr) {
        cudaFreeAsync(b.ptr, ctx->stream);
        b.ptr = nullptr;
        b.bytes = 0;
    }
    size_t want = std::max<size_t>(bytes, 256);
    cudaError_t e = cudaMallocAsync(&b.ptr, want, ctx->stream);
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

int pair_grid(Ctx *ctx, int len)
{
    int bps = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, pair_table().kern[len], kBandRows, 0);
    if (bps < 1)
        bps = 1;
    return bps * ctx->sm_count;
}

// Runs prep + the pair kernel.  On return *total holds the number of edges;
// records are complete iff *total <= capacity.
ig_status run_pairs(Ctx *ctx, const uint32_t *d_words, int32_t n, int len, int min_ed, const PairPlan &plan,
                    int grid, int emit, unsigned long long *total)
{
    cudaStream_t st = ctx->stream;
    ig_status s;
    const bool two = len <= 15;
    const size_t unit_bytes = two ? 64 : 32;
    const size_t units = two ? ((size_t)n + 1) / 2 : (size_t)n;
    if ((s = ensure(ctx, ctx->sel, units * unit_bytes, "column streams")) != IG_OK)
        return s;
    if ((s = ensure(ctx, ctx->counts, (size_t)plan.nseg * (size_t)n * sizeof(uint32_t), "segment counts")) !=
        IG_OK)
        return s;
    if ((s = ensure(ctx, ctx->flags, 4 * sizeof(unsigned long long), "flags")) != IG_OK)
        return s;
    phase_begin(ctx, IG_PHASE_PREP);
    if (two)
        prep_units2<<<(unsigned)((units + 255) / 256), 256, 0, st>>>(d_words, n, len,
                                                                     static_cast<uint4 *>(ctx->sel.ptr));
    else
        prep_units1<<<(unsigned)((units + 255) / 256), 256, 0, st>>>(d_words, n, len,
                                                                     static_cast<uint4 *>(ctx->sel.ptr));
    phase_end(ctx, IG_PHASE_PREP);
    ctx->launches++;
    IG_CUDA(cudaGetLastError());
    unsigned long long *flags = static_cast<unsigned long long *>(ctx->flags.ptr);
    IG_CUDA(cudaMemsetAsync(flags, 0, 4 * sizeof(unsigned long long), st));
    PairArgs a;
    a.units = static_cast<const uint4 *>(ctx->sel.ptr);
    a.words = d_words;
    a.n = n;
    // min_ed <= 0: no pair can be an edge; min_ed > L: every pair is one
    a.lim = (int)std::max(-64, std::min(64, min_ed - len));
    a.one = 1u;
    a.two = 2u;
    a.hi = 1u << 16;
    a.seg_shift = plan.seg_shift;
    a.nseg = plan.nseg;
    a.bands_per_seg = plan.bands_per_seg;
    a.nbands = plan.nbands;
    a.items = plan.items;
    a.work = flags + 0;
    a.rec_count = flags + 1;
    a.status = reinterpret_cast<int *>(flags + 2);
    a.rec = static_cast<EdgeRecord *>(ctx->records.ptr);
    a.rec_cap = emit ? ctx->rec_capacity : 0;
    a.counts = static_cast<uint32_t *>(ctx->counts.ptr);
    a.emit = emit;
    phase_begin(ctx, IG_PHASE_PAIRS);
    pair_table().launch[len](a, grid, st);
    phase_end(ctx, IG_PHASE_PAIRS);
    ctx->launches++;
    IG_CUDA(cudaGetLastError());
    unsigned long long host_flags[4];
    IG_CUDA(cudaMemcpyAsync(host_flags, flags, sizeof(host_flags), cudaMemcpyDeviceToHost, st));
    IG_CUDA(cudaStreamSynchronize(st));
    phase_collect(ctx);
    if (static_cast<int>(host_flags[2] & 0xffffffffu) == kStatusTimeout)
        return set_error(ctx, IG_ERR_TIMEOUT, "pair kernel: staged tile never arrived (bounded wait expired)");
    *total = host_flags[1];
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
    for (int p = 0; p < 3; ++p) {
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

PairPlan make_plan(int32_t n, int grid_ctas)
{
    PairPlan p;
    p.n = n;
    // Segment width: a power of two >= one band, small enough that the queue
    // holds many items per CTA, large enough that at most 256 segments exist
    // and the per-(row, segment) counts stay under 1 GiB.
    int shift = 8;  // 256 columns
    while (((int64_t)n + (1ll << shift) - 1) >> shift > 256)
        shift++;
    while ((((int64_t)n + (1ll << shift) - 1) >> shift) * (int64_t)n * 4 > (1ll << 30))
        shift++;
    // Prefer wider segments (fewer per-item overheads) while the queue keeps
    // at least 24 items per CTA.
    for (;;) {
        const int s2 = shift + 1;
        const int64_t nseg2 = ((int64_t)n + (1ll << s2) - 1) >> s2;
        const int64_t nb = ((int64_t)n + kBandRows - 1) / kBandRows;
        const int64_t items2 = nb * (nseg2 + 1) / 2;
        if (s2 > 14 || items2 < 24ll * grid_ctas)
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

ig_status count_edges(Ctx *ctx, const uint32_t *d_words, int32_t n, int len, int min_ed, int64_t *edges)
{
    if (n < 2) {
        *edges = 0;
        return IG_OK;
    }
    const int grid = pair_grid(ctx, len);
    const PairPlan plan = make_plan(n, grid);
    unsigned long long total = 0;
    ig_status s = run_pairs(ctx, d_words, n, len, min_ed, plan, grid, 0, &total);
    if (s != IG_OK)
        return s;
    *edges = (int64_t)total;
    return IG_OK;
}

ig_status build_graph(Ctx *ctx, const uint32_t *d_words, int32_t n, int len, int min_ed, Graph *g)
{
    cudaStream_t st = ctx->stream;
    g->ctx = ctx;
    g->n = n;
    g->len = len;
    g->min_ed = min_ed;
    IG_CUDA(cudaMallocAsync((void **)&g->d_row_ptr, ((size_t)n + 1) * sizeof(int64_t), st));
    if (n < 2) {
        IG_CUDA(cudaMemsetAsync(g->d_row_ptr, 0, ((size_t)n + 1) * sizeof(int64_t), st));
        IG_CUDA(cudaStreamSynchronize(st));
        g->edges = 0;
        return IG_OK;
    }
    const int grid = pair_grid(ctx, len);
    const PairPlan plan = make_plan(n, grid);
    if (ctx->rec_capacity == 0) {
        ig_status s = ensure(ctx, ctx->records, (size_t)(1u << 22) * sizeof(EdgeRecord), "edge records");
        if (s != IG_OK)
            return s;
        ctx->rec_capacity = ctx->records.bytes / sizeof(EdgeRecord);
    }
    unsigned long long total = 0;
    for (int attempt = 0;; ++attempt) {
        ig_status s = run_pairs(ctx, d_words, n, len, min_ed, plan, grid, 1, &total);
        if (s != IG_OK)
            return s;
        if (total <= ctx->rec_capacity)
            break;
        if (attempt > 0)
            return set_error(ctx, IG_ERR_STATE, "edge count changed between identical passes");
        const size_t want = (size_t)(total + total / 8 + 1024);
        s = ensure(ctx, ctx->records, want * sizeof(EdgeRecord), "edge records");
        if (s != IG_OK)
            return s;
        ctx->rec_capacity = ctx->records.bytes / sizeof(EdgeRecord);
    }
    g->edges = (int64_t)total;
    IG_CUDA(cudaMallocAsync((void **)&g->d_cols, std::max<size_t>((size_t)total, 1) * sizeof(int32_t), st));
    IG_CUDA(cudaMemsetAsync(g->d_row_ptr, 0, sizeof(int64_t), st));
    phase_begin(ctx, IG_PHASE_COMPACT);
    row_prefix<<<(n + 255) / 256, 256, 0, st>>>(static_cast<uint32_t *>(ctx->counts.ptr), n, plan.nseg,
                                                  plan.seg_shift, g->d_row_ptr);
    ctx->launches++;
    IG_CUDA(cudaGetLastError());
    // inclusive scan over row_ptr[0..n] (row_ptr[0] = 0) gives the offsets
    ig_status s = inclusive_scan_i64(ctx, g->d_row_ptr, (int64_t)n + 1);
    if (s != IG_OK)
        return s;
    if (total > 0) {
        const int sgrid = (int)std::min<unsigned long long>((total + 255) / 256, (unsigned long long)ctx->sm_count * 16);
        scatter_records<<<sgrid, 256, 0, st>>>(static_cast<const EdgeRecord *>(ctx->records.ptr), total,
                                                g->d_row_ptr, static_cast<const uint32_t *>(ctx->counts.ptr), n,
                                                g->d_cols);
        ctx->launches++;
        IG_CUDA(cudaGetLastError());
    }
    phase_end(ctx, IG_PHASE_COMPACT);
    int64_t last = -1;
    IG_CUDA(cudaMemcpyAsync(&last, g->d_row_ptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    IG_CUDA(cudaStreamSynchronize(st));
    phase_collect(ctx);
    if (last != (int64_t)total)
        return set_error(ctx, IG_ERR_STATE, "row offsets disagree with the edge count");
    return IG_OK;
}

}  // namespace ig
