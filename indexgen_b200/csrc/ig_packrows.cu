// Neighbour lists bit-packed for the trip to the host greedy.
//
// The greedy reads every neighbour list once, front to back, and a list of
// the canonical adjacency is strictly ascending (lower neighbours < x < upper
// neighbours, each part ascending).  So each row x of degree D >= 1 ships as
//   word 0      w, the bit width of the largest gap (0..32)
//   word 1      the first neighbour (global id)
//   then        the D - 1 gaps a[k] - a[k-1] - 1, w bits each, packed
//               little-endian across 32-bit words
// and a row of degree 0 ships nothing.  Dense rows (gaps of tens) take about
// 10 bits per neighbour instead of 32, sparse rows about 15: the copy over
// PCIe and the host memory the graphs hold while their greedies run shrink
// by 2-3x, which is what bounds a stream of dense jobs.  The host decodes a
// row into a buffer just before the greedy walks it (ig_host.cpp).
//
//   pack_width   one warp per row: w from the largest gap, row size in words
//   (scan)       row word offsets
//   pack_write   one warp per row: header, then each lane composes whole
//                output words from the gaps whose bits fall in them
#include <algorithm>

#include "ig_internal.h"

namespace ig {
namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ uint32_t gap_at(const int32_t *__restrict__ a, int64_t k)
{
    return (uint32_t)(a[k] - a[k - 1] - 1);
}

__global__ void pack_width(const int64_t *__restrict__ adj_ptr, const int32_t *__restrict__ adj, int32_t n,
                           uint8_t *__restrict__ width, int64_t *__restrict__ words)
{
    const int64_t x = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (x >= n)
        return;
    const int64_t b = adj_ptr[x], e = adj_ptr[x + 1];
    uint32_t mx = 0;
    for (int64_t k = b + 1 + lane; k < e; k += 32)
        mx = max(mx, gap_at(adj, k));
    mx = __reduce_max_sync(kFull, mx);
    if (lane == 0) {
        const int w = mx == 0 ? 0 : 32 - __clz(mx);
        const int64_t d = e - b;
        width[x] = (uint8_t)w;
        words[x + 1] = d == 0 ? 0 : 2 + ((d - 1) * w + 31) / 32;
    }
}

__global__ void pack_write(const int64_t *__restrict__ adj_ptr, const int32_t *__restrict__ adj, int32_t n,
                           const uint8_t *__restrict__ width, const int64_t *__restrict__ off,
                           uint32_t *__restrict__ out)
{
    const int64_t x = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (x >= n)
        return;
    const int64_t b = adj_ptr[x], e = adj_ptr[x + 1];
    if (e == b)
        return;
    const int w = width[x];
    uint32_t *row = out + off[x];
    if (lane == 0) {
        row[0] = (uint32_t)w;
        row[1] = (uint32_t)adj[b];
    }
    if (w == 0)
        return;
    const int64_t gaps = e - b - 1;  // gap j (j = 0..gaps-1) sits at bits [j*w, j*w + w)
    const int64_t nwords = (gaps * w + 31) / 32;
    for (int64_t q = lane; q < nwords; q += 32) {
        const int64_t lo = 32 * q;  // the word covers bits [lo, lo + 32)
        int64_t j = lo / w;
        uint32_t v = 0;
        for (; j < gaps && j * w < lo + 32; ++j) {
            const uint32_t g = gap_at(adj, b + 1 + j);
            const int64_t sh = j * w - lo;
            v |= sh >= 0 ? g << sh : g >> -sh;
        }
        row[2 + q] = v;
    }
}

}  // namespace

ig_status build_packed_rows(Ctx *ctx, Graph *g)
{
    if (g->d_pk_off)
        return IG_OK;
    ig_status s = build_adjacency(ctx, g);
    if (s != IG_OK)
        return s;
    cudaStream_t st = ctx->stream;
    const int32_t n = g->n;
    int64_t *off = nullptr;
    uint32_t *pk = nullptr;
    uint8_t *width = nullptr;
    auto fail = [&](ig_status r) {
        if (off)
            cudaFreeAsync(off, st);
        if (pk)
            cudaFreeAsync(pk, st);
        if (width)
            cudaFreeAsync(width, st);
        cudaStreamSynchronize(st);
        cudaGetLastError();
        return r;
    };
    cudaError_t e = dev_malloc(ctx, (void **)&off, ((size_t)n + 1) * sizeof(int64_t), st);
    if (e == cudaSuccess)
        e = dev_malloc(ctx, (void **)&width, std::max<size_t>((size_t)n, 1), st);
    if (e != cudaSuccess)
        return fail(cuda_error(ctx, e, "packed row offsets"));
    int64_t total = 0;
    if (n > 0) {
        e = cudaMemsetAsync(off, 0, sizeof(int64_t), st);
        const unsigned grid = (unsigned)(((int64_t)n * 32 + 255) / 256);
        if (e == cudaSuccess) {
            pack_width<<<grid, 256, 0, st>>>(g->d_adj_ptr, g->d_adj, n, width, off);
            ctx->launches++;
            e = cudaGetLastError();
        }
        if (e != cudaSuccess)
            return fail(cuda_error(ctx, e, "pack_width"));
        if ((s = inclusive_scan_i64(ctx, off, (int64_t)n + 1)) != IG_OK)
            return fail(s);
        e = cudaMemcpyAsync(&total, off + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(st);
        if (e != cudaSuccess)
            return fail(cuda_error(ctx, e, "packed size"));
    }
    // one spare word at the end: the host decoder reads 64 bits at a time
    e = dev_malloc(ctx, (void **)&pk, ((size_t)total + 2) * sizeof(uint32_t), st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(pk + total, 0, 2 * sizeof(uint32_t), st);
    if (e != cudaSuccess)
        return fail(cuda_error(ctx, e, "packed rows"));
    if (n > 0) {
        pack_write<<<(unsigned)(((int64_t)n * 32 + 255) / 256), 256, 0, st>>>(g->d_adj_ptr, g->d_adj, n, width, off,
                                                                               pk);
        ctx->launches++;
        if ((e = cudaGetLastError()) != cudaSuccess)
            return fail(cuda_error(ctx, e, "pack_write"));
    }
    cudaFreeAsync(width, st);
    width = nullptr;
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess)
        return fail(cuda_error(ctx, e, "packed rows"));
    g->d_pk_off = off;
    g->d_pk = pk;
    g->pk_words = total;
    return IG_OK;
}

}  // namespace ig
