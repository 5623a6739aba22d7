// Nearest-centre assignment for random_cluster on sm_100a.
//
// Replaces compute_distance_matrix_kernel + the host argmin of
// src/gpu_cluster.py (:16-193, :239-300), which RandomCluster::fit runs through
// system() (src/clustering/impl/random_cluster/RandomCluster.cpp:42-136): the
// reference fills a dense K x N uint8 distance matrix per 32768-word batch,
// copies it to the host and takes np.argmin over the centres.  Here one kernel
// computes each word's Levenshtein distance to every centre and keeps the
// running minimum in registers; only the N int32 assignments leave the device.
// Ties go to the lowest centre index, as np.argmin's first occurrence does.
//
// Layout: centres are the Myers patterns (their Peq pools are staged in
// shared memory, 2048 per pass), words the texts: each thread holds the
// selector stream of two words (two 16-bit lanes, L <= 15) or one (L = 16) in
// registers and walks all centres with the full Myers recurrence of
// ig_myers.cuh, reading the exact distance at the end.
#include <algorithm>
#include <climits>

#include "ig_internal.h"
#include "ig_myers.cuh"

namespace ig {
namespace {

using myers::Unit;
using myers::nib;
using myers::row_pools;

constexpr int kAssignThreads = 256;
constexpr int kCentreChunk = 2048;  // centre pools per shared-memory pass (16 KiB)

// The running minimum of the two-lane form as one key per word: distance in
// bits 26..30, centre index in bits 0..25, so one unsigned min keeps the
// nearest centre and, among equals, the lowest index (np.argmin's first
// occurrence).  The key is formed by two IMADs on the FMA pipe from the two
// popcounts, with the multipliers 2^26 and -2^26 passed in as arguments so
// that they stay multiplies; the ALU pipe, which the recurrence saturates,
// then spends one min per distance instead of an add, a compare and two
// selects.
constexpr int kKeyShift = 26;
constexpr uint32_t kKeyIndexMask = (1u << kKeyShift) - 1u;

template <int L, bool kKeyed>
__global__ void __launch_bounds__(kAssignThreads) assign_kernel(const uint32_t *__restrict__ words, long long n,
                                                               const uint32_t *__restrict__ centres, int k,
                                                               int32_t *__restrict__ out, uint32_t one,
                                                               uint32_t two, uint32_t hi, uint32_t unit,
                                                               uint32_t neg_unit)
{
    __shared__ uint2 pools[kCentreChunk];
    using U = Unit<L>;
    const long long first = (blockIdx.x * (long long)blockDim.x + threadIdx.x) * U::kCols;
    const uint32_t wa = first < n ? words[first] : 0u;
    const uint32_t wb = (U::kTwo && first + 1 < n) ? words[first + 1] : wa;
    // this thread's selector stream, in the column-unit layout of ig_myers.cuh
    uint32_t sel[16];
    if constexpr (U::kTwo) {
#pragma unroll
        for (int p = 0; p < 16; ++p)
            sel[p] = (p < L) ? (nib((wa >> (2 * p)) & 3u) | (nib((wb >> (2 * p)) & 3u) << 8)) : 0u;
    } else {
#pragma unroll
        for (int j = 0; j < 8; ++j)
            sel[j] = nib((wa >> (4 * j)) & 3u) | (nib((wa >> (4 * j + 2)) & 3u) << 16);
#pragma unroll
        for (int j = 8; j < 16; ++j)
            sel[j] = 0u;
    }
    int best0 = INT_MAX, best1 = INT_MAX, arg0 = 0, arg1 = 0;
    uint32_t key0 = 0xffffffffu, key1 = 0xffffffffu;  // kKeyed: two-lane form, k <= 2^26
    for (int c0 = 0; c0 < k; c0 += kCentreChunk) {
        const int cn = min(kCentreChunk, k - c0);
        __syncthreads();  // the previous pass is done with the pools
        for (int i = threadIdx.x; i < cn; i += blockDim.x) {
            uint32_t p01, p23;
            row_pools<L>(centres[c0 + i], p01, p23);
            pools[i] = make_uint2(p01, p23);
        }
        __syncthreads();
        for (int i = 0; i < cn; ++i) {
            const uint2 p = pools[i];
            if constexpr (U::kTwo) {
                if constexpr (kKeyed) {
                    uint32_t pv, mv;
                    myers::myers_two_vectors<L>(p.x, p.y, sel, one, two, pv, mv);
                    constexpr uint32_t M0 = (1u << L) - 1u;
                    constexpr uint32_t M1 = M0 << 16;
                    // (L + popc(Pv) - popc(Mv)) << 26 | index, modulo 2^32
                    const uint32_t base = ((uint32_t)L << kKeyShift) + (uint32_t)(c0 + i);
                    const uint32_t k0 = myers::imad((uint32_t)__popc(mv & M0), neg_unit,
                                                    myers::imad((uint32_t)__popc(pv & M0), unit, base));
                    const uint32_t k1 = myers::imad((uint32_t)__popc(mv & M1), neg_unit,
                                                    myers::imad((uint32_t)__popc(pv & M1), unit, base));
                    key0 = min(key0, k0);
                    key1 = min(key1, k1);
                } else {
                    int d0, d1;
                    myers::myers_two_dist<L>(p.x, p.y, sel, one, two, d0, d1);
                    if (d0 < best0) {
                        best0 = d0;
                        arg0 = c0 + i;
                    }
                    if (d1 < best1) {
                        best1 = d1;
                        arg1 = c0 + i;
                    }
                }
            } else {
                uint32_t s8[8];
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    s8[j] = sel[j];
                const int d0 = myers::myers_one_dist<L>(p.x, p.y, s8, one, two, hi);
                if (d0 < best0) {
                    best0 = d0;
                    arg0 = c0 + i;
                }
            }
        }
    }
    if constexpr (kKeyed) {
        arg0 = (int)(key0 & kKeyIndexMask);
        arg1 = (int)(key1 & kKeyIndexMask);
    }
    if (first < n)
        out[first] = arg0;
    if (U::kTwo && first + 1 < n)
        out[first + 1] = arg1;
}

// The keyed minimum for the two-lane lengths (L <= 15) with at most 2^26
// centres; the compare-and-select form otherwise.
template <int L>
void launch_assign_len(int grid, cudaStream_t st, const uint32_t *words, long long n, const uint32_t *centres, int k,
                       int32_t *out)
{
    constexpr uint32_t unit = 1u << kKeyShift;
    if constexpr (Unit<L>::kTwo) {
        if (k <= (int)kKeyIndexMask + 1) {
            assign_kernel<L, true><<<grid, kAssignThreads, 0, st>>>(words, n, centres, k, out, 1u, 2u, 1u << 16,
                                                                    unit, 0u - unit);
            return;
        }
    }
    assign_kernel<L, false><<<grid, kAssignThreads, 0, st>>>(words, n, centres, k, out, 1u, 2u, 1u << 16, unit,
                                                             0u - unit);
}

template <int... Ls>
void launch_assign(int L, int grid, cudaStream_t st, const uint32_t *words, long long n, const uint32_t *centres,
                   int k, int32_t *out, std::integer_sequence<int, Ls...>)
{
    ((L == Ls + 1 ? launch_assign_len<Ls + 1>(grid, st, words, n, centres, k, out) : void()), ...);
}

__global__ void gather_words_kernel(const uint32_t *__restrict__ src, const int32_t *__restrict__ idx, long long n,
                                    uint32_t *__restrict__ dst)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = src[idx[i]];
}

}  // namespace

ig_status gather_words(Ctx *ctx, const uint32_t *d_src, const int32_t *d_idx, int64_t n, uint32_t *d_dst)
{
    if (n == 0)
        return IG_OK;
    const long long blocks = std::min<long long>((n + 255) / 256, (long long)ctx->sm_count * 8);
    gather_words_kernel<<<(int)blocks, 256, 0, ctx->stream>>>(d_src, d_idx, n, d_dst);
    ctx->launches++;
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? IG_OK : cuda_error(ctx, e, "gather_words launch");
}

ig_status assign_centers(Ctx *ctx, const uint32_t *d_words, int64_t n, const uint32_t *d_centres, int32_t k, int len,
                         int32_t *d_out)
{
    if (n == 0)
        return IG_OK;
    const int per_thread = len <= 15 ? 2 : 1;
    const long long threads = (n + per_thread - 1) / per_thread;
    const long long grid = (threads + kAssignThreads - 1) / kAssignThreads;
    if (grid > INT32_MAX)
        return set_error(ctx, IG_ERR_CAPACITY, "too many words for one assignment launch");
    launch_assign(len, (int)grid, ctx->stream, d_words, n, d_centres, k, d_out,
                  std::make_integer_sequence<int, IG_MAX_LEN>{});
    ctx->launches++;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return cuda_error(ctx, e, "assign_kernel launch");
    return IG_OK;
}

}  // namespace ig
