// Symmetric adjacency of a conflict graph in the reference's canonical
// neighbour order: m[x] = [lower neighbours ascending] ++ [upper neighbours
// ascending].  That is the order AdjList::FromBinaryFile builds from a
// row-sorted edge file (src/SparseMat.cpp:338-390) and the order FillAdjList
// builds with one thread (src/SparseMat.cpp:599-609); the greedy then runs on
// it without any host-side list assembly.
//
//   lower_degree       ldeg[x] = #{w < x : x in upper(w)}        (atomics, one per edge)
//   full_degree        deg[x]  = ldeg[x] + udeg[x]; scan -> adj_ptr
//   fill_rows          upper part copied in place; lower part scattered with a
//                      per-row atomic cursor (arbitrary order)
//   sort_lower_small   rows with <= 1024 lower entries: warp bitonic sort in
//                      shared memory
//   sort_lower_big     longer rows: one CTA per row, value bitmap over
//                      [0, x) in 512 Ki-value chunks, emitted in order by a
//                      block prefix sum of popcounts
#include <algorithm>
#include <climits>

#include "ig_internal.h"

namespace ig {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kSmallMax = 1024;           // lower entries sorted by one warp
constexpr int kBigThreads = 1024;
constexpr int kBitmapWords = 16384;       // 64 KiB of shared memory
constexpr int kChunkValues = kBitmapWords * 32;

__global__ void lower_degree(const int32_t *__restrict__ cols, int64_t nnz, int32_t *__restrict__ ldeg)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(&ldeg[cols[k]], 1);
}

__global__ void full_degree(const int64_t *__restrict__ row_ptr, const int32_t *__restrict__ ldeg, int32_t n,
                            int64_t *__restrict__ adj_ptr)
{
    const int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (x == 0)
        adj_ptr[0] = 0;
    if (x < n)
        adj_ptr[x + 1] = (row_ptr[x + 1] - row_ptr[x]) + ldeg[x];
}

// One warp per source row w.
__global__ void fill_rows(const int64_t *__restrict__ row_ptr, const int32_t *__restrict__ cols, int32_t n,
                          const int64_t *__restrict__ adj_ptr, const int32_t *__restrict__ ldeg,
                          int32_t *__restrict__ cursor, int32_t *__restrict__ adj)
{
    const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= n)
        return;
    const int64_t b = row_ptr[w], e = row_ptr[w + 1];
    const int64_t up = adj_ptr[w] + ldeg[w];
    for (int64_t k = b + lane; k < e; k += 32) {
        const int32_t x = cols[k];
        adj[up + (k - b)] = x;
        const int32_t slot = atomicAdd(&cursor[x], 1);
        adj[adj_ptr[x] + slot] = (int32_t)w;
    }
}

// One warp per row; rows with more than kSmallMax lower entries are queued.
__global__ void sort_lower_small(const int64_t *__restrict__ adj_ptr, const int32_t *__restrict__ ldeg, int32_t n,
                                 int32_t *__restrict__ adj, int32_t *__restrict__ big, int32_t *__restrict__ nbig)
{
    __shared__ int32_t buf[8][kSmallMax];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int64_t x = (int64_t)blockIdx.x * 8 + warp;
    if (x >= n)
        return;
    const int m = ldeg[x];
    if (m <= 1)
        return;
    if (m > kSmallMax) {
        if (lane == 0)
            big[atomicAdd(nbig, 1)] = (int32_t)x;
        return;
    }
    int P = 32;
    while (P < m)
        P <<= 1;
    int32_t *s = buf[warp];
    const int64_t base = adj_ptr[x];
    for (int i = lane; i < P; i += 32)
        s[i] = (i < m) ? adj[base + i] : INT_MAX;
    __syncwarp();
    for (int k = 2; k <= P; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = lane; i < P; i += 32) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const int32_t a = s[i], c = s[ixj];
                    const bool up = (i & k) == 0;
                    if ((a > c) == up) {
                        s[i] = c;
                        s[ixj] = a;
                    }
                }
            }
            __syncwarp();
        }
    }
    for (int i = lane; i < m; i += 32)
        adj[base + i] = s[i];
}

// Exclusive block scan of one value per thread (kBigThreads threads).
__device__ __forceinline__ int32_t block_excl_scan(int32_t v, int32_t *warp_tot, int32_t *total)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t t = __shfl_up_sync(kFull, incl, o);
        if (lane >= o)
            incl += t;
    }
    if (lane == 31)
        warp_tot[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        int32_t w = warp_tot[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t t = __shfl_up_sync(kFull, w, o);
            if (lane >= o)
                w += t;
        }
        warp_tot[lane] = w;
        if (lane == 31)
            *total = w;
    }
    __syncthreads();
    return incl - v + (wid > 0 ? warp_tot[wid - 1] : 0);
}

// One CTA per long row x.  Its lower entries are distinct values in [0, x);
// they are copied to `scratch` (same offsets as adj) and re-emitted in order,
// one 512 Ki-value window of a shared-memory bitmap at a time.
__global__ void __launch_bounds__(kBigThreads) sort_lower_big(const int64_t *__restrict__ adj_ptr,
                                                              const int32_t *__restrict__ ldeg,
                                                              const int32_t *__restrict__ big,
                                                              int32_t *__restrict__ adj,
                                                              int32_t *__restrict__ scratch)
{
    extern __shared__ uint32_t bm[];  // kBitmapWords
    __shared__ int32_t warp_tot[32];
    __shared__ int32_t total;
    const int32_t x = big[blockIdx.x];
    const int m = ldeg[x];
    const int64_t base = adj_ptr[x];
    for (int i = threadIdx.x; i < m; i += kBigThreads)
        scratch[base + i] = adj[base + i];
    __syncthreads();
    constexpr int kPer = kBitmapWords / kBigThreads;  // words per thread
    int64_t out = 0;
    for (int64_t c0 = 0; c0 < x; c0 += kChunkValues) {
        for (int w = threadIdx.x; w < kBitmapWords; w += kBigThreads)
            bm[w] = 0u;
        __syncthreads();
        for (int i = threadIdx.x; i < m; i += kBigThreads) {
            const int64_t v = (int64_t)scratch[base + i] - c0;
            if (v >= 0 && v < kChunkValues)
                atomicOr(&bm[v >> 5], 1u << (v & 31));
        }
        __syncthreads();
        int32_t mine = 0;
#pragma unroll
        for (int q = 0; q < kPer; ++q)
            mine += __popc(bm[threadIdx.x * kPer + q]);
        const int32_t excl = block_excl_scan(mine, warp_tot, &total);
        int64_t o = base + out + excl;
#pragma unroll 1
        for (int q = 0; q < kPer; ++q) {
            uint32_t word = bm[threadIdx.x * kPer + q];
            const int64_t v0 = c0 + (int64_t)(threadIdx.x * kPer + q) * 32;
            while (word) {
                const int bit = __ffs(word) - 1;
                word &= word - 1;
                adj[o++] = (int32_t)(v0 + bit);
            }
        }
        out += total;
        __syncthreads();
    }
}

#define IG_CUDA(call)                                                                                          \
    do {                                                                                                       \
        cudaError_t e_ = (call);                                                                               \
        if (e_ != cudaSuccess)                                                                                 \
            return cuda_error(ctx, e_, #call);                                                                 \
    } while (0)

// The adjacency goes to fresh arrays that the graph takes only when every
// step succeeded: a failed build (an allocation, a launch) frees them, so a
// later request never sees a half-built adjacency.
ig_status build_adjacency_into(Ctx *ctx, const Graph *g, int64_t *adj_ptr, int32_t *adj)
{
    cudaStream_t st = ctx->stream;
    const int32_t n = g->n;
    const int64_t nnz = g->edges;
    if (n == 0 || nnz == 0) {
        IG_CUDA(cudaMemsetAsync(adj_ptr, 0, ((size_t)n + 1) * sizeof(int64_t), st));
        IG_CUDA(cudaStreamSynchronize(st));
        return IG_OK;
    }
    // ldeg, cursor (n each) + big-row queue (n + 1)
    ig_status s = ensure_buffer(ctx, ctx->adj_tmp, (size_t)(3 * (size_t)n + 1) * sizeof(int32_t), "adjacency workspace");
    if (s != IG_OK)
        return s;
    int32_t *ldeg = static_cast<int32_t *>(ctx->adj_tmp.ptr);
    int32_t *cursor = ldeg + n;
    int32_t *big = cursor + n;
    int32_t *nbig = big + n;
    IG_CUDA(cudaMemsetAsync(ldeg, 0, (size_t)2 * n * sizeof(int32_t), st));
    IG_CUDA(cudaMemsetAsync(nbig, 0, sizeof(int32_t), st));
    const int grid = ctx->sm_count * 8;
    lower_degree<<<grid, 256, 0, st>>>(g->d_cols, nnz, ldeg);
    full_degree<<<(n + 256) / 256, 256, 0, st>>>(g->d_row_ptr, ldeg, n, adj_ptr);
    ctx->launches += 2;
    IG_CUDA(cudaGetLastError());
    s = inclusive_scan_i64(ctx, adj_ptr, (int64_t)n + 1);
    if (s != IG_OK)
        return s;
    fill_rows<<<(unsigned)(((int64_t)n * 32 + 255) / 256), 256, 0, st>>>(g->d_row_ptr, g->d_cols, n, adj_ptr, ldeg,
                                                                          cursor, adj);
    sort_lower_small<<<(n + 7) / 8, 256, 0, st>>>(adj_ptr, ldeg, n, adj, big, nbig);
    ctx->launches += 2;
    IG_CUDA(cudaGetLastError());
    int32_t host_nbig = 0;
    IG_CUDA(cudaMemcpyAsync(&host_nbig, nbig, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    IG_CUDA(cudaStreamSynchronize(st));
    if (host_nbig > 0) {
        // scratch for the long rows: same offsets as adj, so 2*nnz ints
        s = ensure_buffer(ctx, ctx->records, (size_t)(2 * nnz) * sizeof(int32_t), "sort scratch");
        if (s != IG_OK)
            return s;
        const size_t smem = kBitmapWords * sizeof(uint32_t);
        IG_CUDA(cudaFuncSetAttribute(sort_lower_big, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        sort_lower_big<<<host_nbig, kBigThreads, smem, st>>>(adj_ptr, ldeg, big, adj,
                                                              static_cast<int32_t *>(ctx->records.ptr));
        ctx->launches++;
        IG_CUDA(cudaGetLastError());
    }
    IG_CUDA(cudaStreamSynchronize(st));
    return IG_OK;
}

}  // namespace

ig_status build_adjacency(Ctx *ctx, Graph *g)
{
    if (g->d_adj_ptr)
        return IG_OK;
    cudaStream_t st = ctx->stream;
    int64_t *adj_ptr = nullptr;
    int32_t *adj = nullptr;
    cudaError_t e = dev_malloc(ctx, (void **)&adj_ptr, ((size_t)g->n + 1) * sizeof(int64_t), st);
    if (e == cudaSuccess)
        e = dev_malloc(ctx, (void **)&adj, std::max<size_t>((size_t)(2 * g->edges), 1) * sizeof(int32_t), st);
    ig_status s = e == cudaSuccess ? build_adjacency_into(ctx, g, adj_ptr, adj) : cuda_error(ctx, e, "adjacency arrays");
    if (s != IG_OK) {
        if (adj_ptr)
            cudaFreeAsync(adj_ptr, st);
        if (adj)
            cudaFreeAsync(adj, st);
        cudaStreamSynchronize(st);
        cudaGetLastError();
        return s;
    }
    g->d_adj_ptr = adj_ptr;
    g->d_adj = adj;
    return IG_OK;
}

}  // namespace ig
