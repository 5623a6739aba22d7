// Checkpoint bridge: the reference's progress_adj_list.txt from and to the
// device graph.
//
// After the GPU build the reference loads the edge file into AdjList and, at
// the start of Codebook, checkpoints it with AdjList::ToFile
// (src/SparseMat.cpp:286-305, called from SaveProgressCodebook :658-663): one
// line "i\tj\n" per neighbour j of every row i, rows ascending, neighbours in
// m-order (lower neighbours ascending, then upper ascending, for a graph that
// came from the GPU edge file).  That is a few hundred MB of text for a
// 20 M-edge graph written by ofstream.  Here the text is formatted on the
// device from the canonical adjacency (per row: byte count, scan, one warp
// writes the row), copied out in row chunks through a pinned buffer and
// written with fwrite.  The reverse direction parses such a file on the
// device (newline compaction, one thread per line) into a graph whose
// adjacency keeps the file's order, as AdjList::FromFile (:306-336) builds it
// with Init(max_node + 1).
#include <algorithm>
#include <cstdio>
#include <memory>

#include "ig_internal.h"

namespace ig {
namespace {

constexpr unsigned kFullMask = 0xffffffffu;

__device__ __forceinline__ int dec_digits(uint32_t v)
{
    int d = 1;
    while (v >= 10u) {
        v /= 10u;
        ++d;
    }
    return d;
}

__device__ __forceinline__ void put_dec(char *p, uint32_t v, int nd)
{
    for (int k = nd - 1; k >= 0; --k) {
        p[k] = (char)('0' + v % 10u);
        v /= 10u;
    }
}

// bytes[i] = text bytes of row i (one warp per row)
__global__ void row_text_bytes(const int64_t *__restrict__ adj_ptr, const int32_t *__restrict__ adj, int32_t n,
                               int64_t *__restrict__ bytes)
{
    const int64_t row = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= n)
        return;
    const int64_t b = adj_ptr[row], e = adj_ptr[row + 1];
    const int ni = dec_digits((uint32_t)row) + 2;
    int64_t acc = 0;
    for (int64_t k = b + lane; k < e; k += 32)
        acc += ni + dec_digits((uint32_t)adj[k]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        acc += __shfl_xor_sync(kFullMask, acc, o);
    if (lane == 0)
        bytes[row + 1] = acc;  // row_off[0] = 0 is set by the caller; scan makes the offsets
}

// Rows [r0, r1): row i's text goes to out + row_off[i] - base (one warp per row).
__global__ void write_row_text(const int64_t *__restrict__ adj_ptr, const int32_t *__restrict__ adj,
                               const int64_t *__restrict__ row_off, int32_t r0, int32_t r1, int64_t base,
                               char *__restrict__ out)
{
    const int64_t row = r0 + ((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= r1)
        return;
    const int64_t b = adj_ptr[row], e = adj_ptr[row + 1];
    const int ni = dec_digits((uint32_t)row);
    int64_t pos = row_off[row] - base;
    for (int64_t k0 = b; k0 < e; k0 += 32) {
        const int64_t k = k0 + lane;
        const bool on = k < e;
        const uint32_t j = on ? (uint32_t)adj[k] : 0u;
        const int nj = dec_digits(j);
        const int len = on ? ni + nj + 2 : 0;
        int incl = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(kFullMask, incl, o);
            if (lane >= o)
                incl += t;
        }
        if (on) {
            char *p = out + pos + (incl - len);
            put_dec(p, (uint32_t)row, ni);
            p[ni] = '\t';
            put_dec(p + ni + 1, j, nj);
            p[ni + 1 + nj] = '\n';
        }
        pos += __shfl_sync(kFullMask, incl, 31);
    }
}

// ---- parsing ----
constexpr int kParseThreads = 256;
constexpr int kParseChunk = kParseThreads * 16;  // bytes per block in the newline pass

__global__ void count_newlines(const char *__restrict__ text, int64_t size, int64_t *__restrict__ per_block)
{
    const int64_t base = (int64_t)blockIdx.x * kParseChunk;
    int c = 0;
    for (int k = threadIdx.x; k < kParseChunk; k += kParseThreads) {
        const int64_t i = base + k;
        if (i < size && text[i] == '\n')
            ++c;
    }
    __shared__ int red[kParseThreads / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        c += __shfl_xor_sync(kFullMask, c, o);
    if ((threadIdx.x & 31) == 0)
        red[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < kParseThreads / 32; ++w)
            t += red[w];
        per_block[blockIdx.x + 1] = t;
    }
}

// Newline positions in file order: block b writes from block_off[b] (inclusive scan of counts, shifted).
__global__ void list_newlines(const char *__restrict__ text, int64_t size, const int64_t *__restrict__ block_off,
                              int64_t *__restrict__ nl)
{
    __shared__ int warp_base[kParseThreads / 32 + 1];
    const int64_t base = (int64_t)blockIdx.x * kParseChunk;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    // each thread owns 16 consecutive bytes; count, scan, write in order
    const int64_t my0 = base + (int64_t)threadIdx.x * 16;
    int c = 0;
    for (int q = 0; q < 16; ++q)
        if (my0 + q < size && text[my0 + q] == '\n')
            ++c;
    int incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(kFullMask, incl, o);
        if (lane >= o)
            incl += t;
    }
    if (lane == 31)
        warp_base[wid + 1] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
        warp_base[0] = 0;
        for (int w = 1; w <= kParseThreads / 32; ++w)
            warp_base[w] += warp_base[w - 1];
    }
    __syncthreads();
    int64_t o = block_off[blockIdx.x] + warp_base[wid] + (incl - c);
    for (int q = 0; q < 16; ++q)
        if (my0 + q < size && text[my0 + q] == '\n')
            nl[o++] = my0 + q;
}

// Line t = text[(t ? nl[t-1] + 1 : 0), nl[t]): "a\tb".  Bad lines set *bad.
__global__ void parse_lines(const char *__restrict__ text, const int64_t *__restrict__ nl, int64_t lines,
                            int32_t *__restrict__ a_out, int32_t *__restrict__ b_out, int *__restrict__ bad)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < lines; t += (int64_t)gridDim.x * blockDim.x) {
        int64_t p = t ? nl[t - 1] + 1 : 0;
        const int64_t end = nl[t];
        uint64_t v[2] = {0, 0};
        int f = 0, nd = 0;
        bool ok = true;
        for (; p < end && ok; ++p) {
            const char ch = text[p];
            if (ch >= '0' && ch <= '9') {
                v[f] = v[f] * 10u + (uint64_t)(ch - '0');
                ok = ++nd <= 10;
            } else if ((ch == '\t' || ch == ' ') && f == 0 && nd > 0) {
                f = 1;
                nd = 0;
            } else if (ch == '\r' && p + 1 == end) {
            } else {
                ok = false;
            }
        }
        ok = ok && f == 1 && nd > 0 && v[0] <= 0x7fffffffull && v[1] <= 0x7fffffffull;
        if (!ok)
            atomicExch(bad, 1);
        a_out[t] = ok ? (int32_t)v[0] : 0;
        b_out[t] = ok ? (int32_t)v[1] : 0;
    }
}

struct DevMem {
    void *p = nullptr;
    cudaStream_t st = nullptr;
    ~DevMem()
    {
        if (p)
            cudaFreeAsync(p, st);
    }
};

#define PG_CUDA(call)                                                                                          \
    do {                                                                                                       \
        cudaError_t e_ = (call);                                                                               \
        if (e_ != cudaSuccess)                                                                                 \
            return cuda_error(ctx, e_, #call);                                                                 \
    } while (0)

}  // namespace

ig_status write_adj_list(Ctx *ctx, Graph *g, const char *path, int64_t *bytes_out)
{
    ig_status s = build_adjacency(ctx, g);
    if (s != IG_OK)
        return s;
    cudaStream_t st = ctx->stream;
    const int32_t n = g->n;
    FILE *f = std::fopen(path, "wb");
    if (!f)
        return set_error(ctx, IG_ERR_INPUT, std::string("cannot open ") + path + " for writing");
    std::unique_ptr<FILE, int (*)(FILE *)> guard(f, std::fclose);
    if (bytes_out)
        *bytes_out = 0;
    if (n == 0)
        return IG_OK;
    DevMem off;
    off.st = st;
    PG_CUDA(dev_malloc(ctx, (void **)&off.p, ((size_t)n + 1) * sizeof(int64_t), st));
    int64_t *d_off = static_cast<int64_t *>(off.p);
    PG_CUDA(cudaMemsetAsync(d_off, 0, sizeof(int64_t), st));
    row_text_bytes<<<(unsigned)(((int64_t)n * 32 + 255) / 256), 256, 0, st>>>(g->d_adj_ptr, g->d_adj, n, d_off);
    ctx->launches++;
    PG_CUDA(cudaGetLastError());
    s = inclusive_scan_i64(ctx, d_off, (int64_t)n + 1);
    if (s != IG_OK)
        return s;
    std::vector<int64_t> h_off((size_t)n + 1);
    PG_CUDA(cudaMemcpyAsync(h_off.data(), d_off, h_off.size() * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    PG_CUDA(cudaStreamSynchronize(st));
    // row chunks of at most kChunk bytes of text (a row longer than that is a chunk of its own)
    constexpr int64_t kChunk = (int64_t)256 << 20;
    int64_t max_chunk = 0;
    for (int32_t r = 0; r < n;) {
        int32_t r1 = r + 1;
        while (r1 < n && h_off[(size_t)r1 + 1] - h_off[(size_t)r] <= kChunk)
            ++r1;
        max_chunk = std::max(max_chunk, h_off[(size_t)r1] - h_off[(size_t)r]);
        r = r1;
    }
    DevMem text;
    text.st = st;
    PG_CUDA(dev_malloc(ctx, (void **)&text.p, (size_t)std::max<int64_t>(max_chunk, 1), st));
    std::shared_ptr<void> pin = ctx->pinned->acquire((size_t)std::max<int64_t>(max_chunk, 1));
    std::unique_ptr<char[]> heap;
    char *host = static_cast<char *>(pin.get());
    if (!host) {
        heap.reset(new (std::nothrow) char[(size_t)std::max<int64_t>(max_chunk, 1)]);
        if (!heap)
            return set_error(ctx, IG_ERR_OOM, "host text buffer");
        host = heap.get();
    }
    for (int32_t r = 0; r < n;) {
        int32_t r1 = r + 1;
        while (r1 < n && h_off[(size_t)r1 + 1] - h_off[(size_t)r] <= kChunk)
            ++r1;
        const int64_t bytes = h_off[(size_t)r1] - h_off[(size_t)r];
        if (bytes > 0) {
            const int64_t threads = (int64_t)(r1 - r) * 32;
            write_row_text<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(
                g->d_adj_ptr, g->d_adj, d_off, r, r1, h_off[(size_t)r], static_cast<char *>(text.p));
            ctx->launches++;
            PG_CUDA(cudaGetLastError());
            PG_CUDA(cudaMemcpyAsync(host, text.p, (size_t)bytes, cudaMemcpyDeviceToHost, st));
            PG_CUDA(cudaStreamSynchronize(st));
            if (std::fwrite(host, 1, (size_t)bytes, f) != (size_t)bytes)
                return set_error(ctx, IG_ERR_INPUT, std::string("write failed: ") + path);
        }
        r = r1;
    }
    if (bytes_out)
        *bytes_out = h_off[(size_t)n];
    return IG_OK;
}

ig_status read_adj_list(Ctx *ctx, const char *path, Graph *g)
{
    cudaStream_t st = ctx->stream;
    FILE *f = std::fopen(path, "rb");
    if (!f)
        return set_error(ctx, IG_ERR_INPUT, std::string("cannot open ") + path);
    std::unique_ptr<FILE, int (*)(FILE *)> guard(f, std::fclose);
    std::fseek(f, 0, SEEK_END);
    const long fsize = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (fsize < 0)
        return set_error(ctx, IG_ERR_INPUT, std::string("cannot size ") + path);
    std::vector<char> buf((size_t)fsize + 1);
    if (fsize > 0 && std::fread(buf.data(), 1, (size_t)fsize, f) != (size_t)fsize)
        return set_error(ctx, IG_ERR_INPUT, std::string("read failed: ") + path);
    int64_t size = fsize;
    if (size > 0 && buf[(size_t)size - 1] != '\n')
        buf[(size_t)size++] = '\n';  // a last line without its newline
    g->ctx = ctx;
    g->jobs.clear();
    g->job_edge_off.assign(2, 0);
    DevMem d_text, d_blocks, d_nl, d_a, d_b, d_bad;
    for (DevMem *m : {&d_text, &d_blocks, &d_nl, &d_a, &d_b, &d_bad})
        m->st = st;
    const int64_t nblk = std::max<int64_t>((size + kParseChunk - 1) / kParseChunk, 1);
    PG_CUDA(dev_malloc(ctx, (void **)&d_text.p, (size_t)std::max<int64_t>(size, 1), st));
    PG_CUDA(dev_malloc(ctx, (void **)&d_blocks.p, (size_t)(nblk + 1) * sizeof(int64_t), st));
    PG_CUDA(dev_malloc(ctx, (void **)&d_bad.p, sizeof(int), st));
    PG_CUDA(cudaMemsetAsync(d_bad.p, 0, sizeof(int), st));
    PG_CUDA(cudaMemsetAsync(d_blocks.p, 0, sizeof(int64_t), st));
    if (size > 0)
        PG_CUDA(cudaMemcpyAsync(d_text.p, buf.data(), (size_t)size, cudaMemcpyHostToDevice, st));
    const char *text = static_cast<const char *>(d_text.p);
    int64_t *blocks = static_cast<int64_t *>(d_blocks.p);
    count_newlines<<<(unsigned)nblk, kParseThreads, 0, st>>>(text, size, blocks);
    ctx->launches++;
    PG_CUDA(cudaGetLastError());
    ig_status s = inclusive_scan_i64(ctx, blocks, nblk + 1);
    if (s != IG_OK)
        return s;
    int64_t lines = 0;
    PG_CUDA(cudaMemcpyAsync(&lines, blocks + nblk, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    PG_CUDA(cudaStreamSynchronize(st));
    PG_CUDA(dev_malloc(ctx, (void **)&d_nl.p, (size_t)std::max<int64_t>(lines, 1) * sizeof(int64_t), st));
    PG_CUDA(dev_malloc(ctx, (void **)&d_a.p, (size_t)std::max<int64_t>(lines, 1) * sizeof(int32_t), st));
    PG_CUDA(dev_malloc(ctx, (void **)&d_b.p, (size_t)std::max<int64_t>(lines, 1) * sizeof(int32_t), st));
    list_newlines<<<(unsigned)nblk, kParseThreads, 0, st>>>(text, size, blocks, static_cast<int64_t *>(d_nl.p));
    ctx->launches++;
    PG_CUDA(cudaGetLastError());
    if (lines > 0) {
        const int grid = (int)std::min<int64_t>((lines + 255) / 256, (int64_t)ctx->sm_count * 16);
        parse_lines<<<grid, 256, 0, st>>>(text, static_cast<const int64_t *>(d_nl.p), lines,
                                         static_cast<int32_t *>(d_a.p), static_cast<int32_t *>(d_b.p),
                                         static_cast<int *>(d_bad.p));
        ctx->launches++;
        PG_CUDA(cudaGetLastError());
    }
    int bad = 0;
    std::vector<int32_t> a((size_t)lines), b((size_t)lines);
    PG_CUDA(cudaMemcpyAsync(&bad, d_bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (lines > 0) {
        PG_CUDA(cudaMemcpyAsync(a.data(), d_a.p, (size_t)lines * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        PG_CUDA(cudaMemcpyAsync(b.data(), d_b.p, (size_t)lines * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    }
    PG_CUDA(cudaStreamSynchronize(st));
    if (bad)
        return set_error(ctx, IG_ERR_INPUT, std::string("not an adjacency list of \"i\\tj\" lines: ") + path);
    // rows: AdjList::FromFile appends b to m[a] in file order over Init(max_node + 1)
    int64_t max_node = -1;
    for (int64_t t = 0; t < lines; ++t)
        max_node = std::max<int64_t>(max_node, std::max(a[(size_t)t], b[(size_t)t]));
    if (max_node >= INT32_MAX)
        return set_error(ctx, IG_ERR_CAPACITY, "vertex id too large");
    const int32_t n = (int32_t)(max_node + 1);
    std::vector<int64_t> ap((size_t)n + 1, 0), up((size_t)n + 1, 0);
    for (int64_t t = 0; t < lines; ++t) {
        ++ap[(size_t)a[(size_t)t] + 1];
        if (b[(size_t)t] > a[(size_t)t])
            ++up[(size_t)a[(size_t)t] + 1];
    }
    for (int32_t r = 0; r < n; ++r) {
        ap[(size_t)r + 1] += ap[(size_t)r];
        up[(size_t)r + 1] += up[(size_t)r];
    }
    // an AdjList file lists every edge from both ends and has no self loops
    int64_t loops = 0;
    for (int64_t t = 0; t < lines; ++t)
        loops += a[(size_t)t] == b[(size_t)t];
    if (loops != 0 || lines != 2 * up[(size_t)n])
        return set_error(ctx, IG_ERR_INPUT, std::string("adjacency list is not symmetric: ") + path);
    std::vector<int32_t> adj((size_t)std::max<int64_t>(lines, 1)), cols((size_t)std::max<int64_t>(up[(size_t)n], 1));
    {
        std::vector<int64_t> ca(ap.begin(), ap.end() - 1), cu(up.begin(), up.end() - 1);
        for (int64_t t = 0; t < lines; ++t) {
            const int32_t r = a[(size_t)t], c = b[(size_t)t];
            adj[(size_t)ca[(size_t)r]++] = c;
            if (c > r)
                cols[(size_t)cu[(size_t)r]++] = c;
        }
    }
    g->n = n;
    g->edges = up[(size_t)n];
    g->jobs.push_back(JobSpec{0, n, 1, 0});
    g->job_edge_off[1] = g->edges;
    PG_CUDA(dev_malloc(ctx, (void **)&g->d_row_ptr, ((size_t)n + 1) * sizeof(int64_t), st));
    PG_CUDA(dev_malloc(ctx, (void **)&g->d_cols, (size_t)std::max<int64_t>(g->edges, 1) * sizeof(int32_t), st));
    PG_CUDA(dev_malloc(ctx, (void **)&g->d_adj_ptr, ((size_t)n + 1) * sizeof(int64_t), st));
    PG_CUDA(dev_malloc(ctx, (void **)&g->d_adj, (size_t)std::max<int64_t>(lines, 1) * sizeof(int32_t), st));
    PG_CUDA(cudaMemcpyAsync(g->d_row_ptr, up.data(), up.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    PG_CUDA(cudaMemcpyAsync(g->d_adj_ptr, ap.data(), ap.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    if (g->edges > 0)
        PG_CUDA(cudaMemcpyAsync(g->d_cols, cols.data(), (size_t)g->edges * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    if (lines > 0)
        PG_CUDA(cudaMemcpyAsync(g->d_adj, adj.data(), (size_t)lines * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    PG_CUDA(cudaStreamSynchronize(st));
    return IG_OK;
}

}  // namespace ig
