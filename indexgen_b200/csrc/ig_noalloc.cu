// Conflict count that allocates no memory.
//
// Who needs it: hosts that own all device memory themselves and forbid a
// library from calling the CUDA allocator -- for example a JVM / Go / Rust
// process that hands out slices of one preallocated arena, a service running
// under a hard per-process memory budget, or code that must not touch the
// allocator at a point where an allocation could block or fail (while other
// work holds the device).  Those callers cannot use ig_count_conflicts, whose
// context grows workspace with cudaMalloc.
//
// How: the scratch this count needs (the column selector streams and two
// counters) lives in one file-scope __device__ array of fixed size, so it is
// part of the library image that every GPU which loads the library holds until
// the process exits.  Host code never uses the array's name as a device
// address (there it is only a host-side stand-in): the first call on each
// device, with that device current, looks the address up once with
// cudaGetSymbolAddress and caches it.  Make that first call before any stream
// capture begins.  The cache lives as long as the process: after a
// cudaDeviceReset the module may come back at another address, so a host that
// resets a device must not call this entry point on it again.
//
// Limits and sharing: at most IG_NOALLOC_MAX_WORDS words per call.  Every call
// uses the same array and leaves its contents behind; each call clears the two
// counters it accumulates into before its kernels run.  Two calls whose work
// overlaps on the GPU (different streams, or different host threads on one
// device) race on the array and give wrong counts: serialise them.
#include <mutex>

#include "ig_internal.h"
#include "ig_myers.cuh"

namespace ig {
namespace {

using myers::nib;
using myers::row_pools;
using myers::Unit;

constexpr unsigned kFull = 0xffffffffu;
constexpr int kRows = 256;   // rows per CTA (one per thread)
constexpr int kCols = 256;   // columns per CTA tile
constexpr int kMaxUnitsVec = IG_NOALLOC_MAX_WORDS * 2;  // uint4 of the unit streams (32 B per word)

// [0, kMaxUnitsVec) selector units; then one uint4 holding the edge counter.
static __device__ __align__(256) uint4 g_noalloc_scratch[kMaxUnitsVec + 1];

__global__ void noalloc_prep(const uint32_t *__restrict__ words, int32_t n, int len, uint4 *__restrict__ units)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (len <= 15) {
        if (i >= ((int64_t)n + 1) / 2)
            return;
        const uint32_t wa = words[2 * i];
        const uint32_t wb = (2 * i + 1 < n) ? words[2 * i + 1] : wa;
        uint32_t o[16];
#pragma unroll
        for (int k = 0; k < 16; ++k)
            o[k] = (k < len) ? (nib((wa >> (2 * k)) & 3u) | (nib((wb >> (2 * k)) & 3u) << 8)) : 0u;
#pragma unroll
        for (int v = 0; v < 4; ++v)
            units[4 * i + v] = make_uint4(o[4 * v], o[4 * v + 1], o[4 * v + 2], o[4 * v + 3]);
    } else {
        if (i >= n)
            return;
        const uint32_t w = words[i];
        uint32_t o[8];
#pragma unroll
        for (int j = 0; j < 8; ++j)
            o[j] = nib((w >> (4 * j)) & 3u) | (nib((w >> (4 * j + 2)) & 3u) << 16);
        units[2 * i] = make_uint4(o[0], o[1], o[2], o[3]);
        units[2 * i + 1] = make_uint4(o[4], o[5], o[6], o[7]);
    }
}

// One CTA per (row band, column tile) of the upper triangle: the tile's units
// are staged in shared memory, each thread tests its row against them and the
// CTA adds its hits to the counter.
template <int L>
__global__ void __launch_bounds__(kRows) noalloc_count(const uint32_t *__restrict__ words,
                                                       const uint4 *__restrict__ units, int32_t n, int lim,
                                                       uint32_t one, uint32_t two, uint32_t hi,
                                                       unsigned long long *__restrict__ counter)
{
    using U = Unit<L>;
    __shared__ uint4 tile[kCols / U::kCols * U::kVec];
    const int32_t row0 = blockIdx.y * kRows;
    const int32_t c0 = blockIdx.x * kCols;
    if (c0 + kCols - 1 <= row0)
        return;  // every column of the tile is <= every row of the band
    const int nunits = (min(kCols, n - c0) + U::kCols - 1) / U::kCols;
    const uint4 *src = units + (size_t)(c0 / U::kCols) * U::kVec;
    for (int i = threadIdx.x; i < nunits * U::kVec; i += kRows)
        tile[i] = src[i];
    __syncthreads();
    const int32_t row = row0 + threadIdx.x;
    const bool row_ok = row < n;
    uint32_t p01, p23;
    row_pools<L>(words[row_ok ? row : 0], p01, p23);
    unsigned hits = 0;
    for (int u = 0; u < nunits; ++u) {
        const uint4 *t = tile + u * U::kVec;
        if constexpr (U::kTwo) {
            uint32_t sel[16];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const uint4 q = (v < U::kUsed) ? t[v] : make_uint4(0u, 0u, 0u, 0u);
                sel[4 * v] = q.x;
                sel[4 * v + 1] = q.y;
                sel[4 * v + 2] = q.z;
                sel[4 * v + 3] = q.w;
            }
            bool h0, h1;
            myers::myers_two<L>(p01, p23, sel, one, two, lim, h0, h1);
            const int32_t col = c0 + 2 * u;
            hits += (h0 && row_ok && col > row && col < n) ? 1u : 0u;
            hits += (h1 && row_ok && col + 1 > row && col + 1 < n) ? 1u : 0u;
        } else {
            const uint4 q0 = t[0], q1 = t[1];
            const uint32_t sel[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
            const bool h = myers::myers_one<L>(p01, p23, sel, one, two, hi, lim);
            const int32_t col = c0 + u;
            hits += (h && row_ok && col > row) ? 1u : 0u;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        hits += __shfl_down_sync(kFull, hits, o);
    if ((threadIdx.x & 31) == 0 && hits)
        atomicAdd(counter, (unsigned long long)hits);
}

template <int L>
void launch_count(dim3 grid, cudaStream_t st, const uint32_t *words, const uint4 *units, int32_t n, int lim,
                  unsigned long long *counter)
{
    noalloc_count<L><<<grid, kRows, 0, st>>>(words, units, n, lim, 1u, 2u, 1u << 16, counter);
}

template <int... Ls>
void dispatch(int len, dim3 grid, cudaStream_t st, const uint32_t *words, const uint4 *units, int32_t n, int lim,
              unsigned long long *counter, std::integer_sequence<int, Ls...>)
{
    ((len == Ls + 1 ? launch_count<Ls + 1>(grid, st, words, units, n, lim, counter) : void()), ...);
}

// Device address of the scratch array, looked up once per device.
std::mutex g_mu;
void *g_addr[256] = {};

}  // namespace
}  // namespace ig

extern "C" ig_status ig_count_conflicts_noalloc(const uint32_t *words, int32_t n, int len, int min_ed,
                                                unsigned long long *count, void *stream)
{
    IG_ABI_TRY
    using namespace ig;
    if (!count || len < 1 || len > IG_MAX_LEN || n < 0 || (n > 0 && !words))
        return IG_ERR_INPUT;
    if (n > IG_NOALLOC_MAX_WORDS)
        return IG_ERR_CAPACITY;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) {
        cudaGetLastError();
        return IG_ERR_CUDA;
    }
    void *base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_addr[dev]) {
            void *p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                cudaGetLastError();
                return IG_ERR_CUDA;
            }
            g_addr[dev] = p;
        }
        base = g_addr[dev];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    uint4 *units = static_cast<uint4 *>(base);
    unsigned long long *counter = reinterpret_cast<unsigned long long *>(units + kMaxUnitsVec);
    if (cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st) != cudaSuccess) {
        cudaGetLastError();
        return IG_ERR_CUDA;
    }
    if (n >= 2) {
        const int64_t work = len <= 15 ? ((int64_t)n + 1) / 2 : (int64_t)n;
        noalloc_prep<<<(unsigned)((work + 255) / 256), 256, 0, st>>>(words, n, len, units);
        const dim3 grid((unsigned)((n + kCols - 1) / kCols), (unsigned)((n + kRows - 1) / kRows));
        const int lim = min_ed - len < -64 ? -64 : (min_ed - len > 64 ? 64 : min_ed - len);
        dispatch(len, grid, st, words, units, n, lim, counter, std::make_integer_sequence<int, IG_MAX_LEN>{});
    }
    if (cudaMemcpyAsync(count, counter, sizeof(unsigned long long), cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
        cudaGetLastError() != cudaSuccess) {
        cudaGetLastError();
        return IG_ERR_CUDA;
    }
    return IG_OK;
    IG_ABI_CATCH
}
