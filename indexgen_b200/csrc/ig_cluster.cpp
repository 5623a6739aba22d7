// Iterative clustered solve with random_cluster, words resident in HBM.
//
// The reference (src/SparseMat.cpp:920-1095) repeats, until the codebook size
// is the same for `convergenceIterations` iterations in a row:
//   cluster the current candidates with random_cluster (RandomCluster::fit,
//     src/clustering/impl/random_cluster/RandomCluster.cpp:42-136: k random
//     candidates are the centres, each candidate joins its nearest centre, a
//     cluster keeps candidate order, empty clusters are dropped; k is raised to
//     ceil(N / 200000) when clusters would exceed 200,000 candidates),
//   solve every cluster (SolveIndependentSet, GPU neighbour order),
//   concatenate the clusters' codebooks in cluster order -> next candidates.
// Each step there is a process or a file round trip; here the words are
// uploaded once and every iteration is: gather the current candidates' words
// on the device, one assignment launch, a stable partition of the (small)
// assignment array on the host, a gather into cluster order, one batch build
// for all clusters (one persistent pair launch), and the clusters' greedies on
// host threads.
//
// Centres: the reference seeds std::shuffle from std::random_device, so its
// runs do not repeat.  Here iteration t takes the first k entries of a partial
// Fisher-Yates shuffle of [0, N) driven by splitmix64 seeded with
// seed ^ (t * 0xD1B54A32D192ED03); the test oracle restates the same picker.
#include <algorithm>
#include <memory>
#include <new>
#include <numeric>
#include <thread>
#include <vector>

#include "ig_internal.h"

namespace ig {
namespace {

constexpr int kMaxClusterSize = 200000;

uint64_t splitmix64(uint64_t &x)
{
    x += 0x9E3779B97F4A7C15ull;
    uint64_t z = x;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

std::vector<int32_t> pick_centres(int32_t n, int32_t k, uint64_t seed, int iteration)
{
    std::vector<int32_t> idx((size_t)n);
    std::iota(idx.begin(), idx.end(), 0);
    uint64_t x = seed ^ ((uint64_t)iteration * 0xD1B54A32D192ED03ull);
    for (int32_t i = 0; i < k; ++i) {
        const int32_t j = i + (int32_t)(splitmix64(x) % (uint64_t)(n - i));
        std::swap(idx[(size_t)i], idx[(size_t)j]);
    }
    idx.resize((size_t)k);
    return idx;
}

struct DevArray {
    Ctx *ctx = nullptr;
    void *p = nullptr;
    ~DevArray()
    {
        if (p) {
            DeviceGuard dg(ctx->device);
            cudaFreeAsync(p, ctx->stream);
            cudaStreamSynchronize(ctx->stream);
        }
    }
    ig_status alloc(Ctx *c, size_t bytes)
    {
        ctx = c;
        const cudaError_t e = dev_malloc(c, &p, std::max<size_t>(bytes, 256), c->stream);
        return e == cudaSuccess ? IG_OK : cuda_error(c, e, "cluster-solve workspace");
    }
};

}  // namespace
}  // namespace ig

extern "C" ig_status ig_cluster_solve(ig_ctx *ctx, const uint32_t *words, int32_t n, int len, int min_ed, int32_t k,
                                      int32_t converge_iters, uint64_t seed, int32_t max_iters, int host_threads,
                                      int32_t *codebook, int32_t *count, int32_t *iterations, int64_t *sizes)
{
    IG_ABI_TRY
    using namespace ig;
    if (!ctx || n < 0 || len < 1 || len > IG_MAX_LEN || max_iters < 1 || !count || (n > 0 && (!words || !codebook)))
        return IG_ERR_INPUT;
    *count = 0;
    if (iterations)
        *iterations = 0;
    if (n == 0)
        return IG_OK;
    if (host_threads <= 0)
        host_threads = (int)std::max(1u, std::thread::hardware_concurrency());
    // device words (all candidates, uploaded once), current candidates' words,
    // the same in cluster order, ids, centres and assignments
    DevArray d_all, d_cur, d_part, d_ids, d_cen, d_asg;
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        DeviceGuard dg(ctx->device);
        if (!dg.ok)
            return set_error(ctx, IG_ERR_CUDA, "cannot select the context's device");
        ig_status s;
        const size_t wb = (size_t)n * sizeof(uint32_t);
        if ((s = d_all.alloc(ctx, wb)) != IG_OK || (s = d_cur.alloc(ctx, wb)) != IG_OK ||
            (s = d_part.alloc(ctx, wb)) != IG_OK || (s = d_ids.alloc(ctx, (size_t)n * sizeof(int32_t))) != IG_OK ||
            (s = d_asg.alloc(ctx, (size_t)n * sizeof(int32_t))) != IG_OK || (s = d_cen.alloc(ctx, wb)) != IG_OK)
            return s;
        const cudaError_t e = cudaMemcpyAsync(d_all.p, words, wb, cudaMemcpyHostToDevice, ctx->stream);
        if (e != cudaSuccess)
            return cuda_error(ctx, e, "word upload");
    }
    std::vector<int32_t> cur((size_t)n), next;
    std::iota(cur.begin(), cur.end(), 0);
    std::vector<int64_t> history;
    int iteration = 0;
    for (;;) {
        if (cur.empty() || iteration >= max_iters)
            break;
        ++iteration;
        const int32_t N = (int32_t)cur.size();
        int32_t eff_k = k;
        if (eff_k > 0 && N / eff_k > kMaxClusterSize)
            eff_k = std::max(2, (N + kMaxClusterSize - 1) / kMaxClusterSize);
        // cluster: assignment of every current candidate to its nearest centre
        std::vector<int32_t> asg((size_t)N, 0);
        int32_t kk = 1;
        {
            std::lock_guard<std::mutex> lk(ctx->mu);
            DeviceGuard dg(ctx->device);
            cudaError_t e = cudaMemcpyAsync(d_ids.p, cur.data(), (size_t)N * sizeof(int32_t), cudaMemcpyHostToDevice,
                                            ctx->stream);
            if (e != cudaSuccess)
                return cuda_error(ctx, e, "candidate id upload");
            ig_status s = gather_words(ctx, static_cast<const uint32_t *>(d_all.p), static_cast<const int32_t *>(d_ids.p),
                                       N, static_cast<uint32_t *>(d_cur.p));
            if (s != IG_OK)
                return s;
            if (eff_k > 0) {
                kk = std::min(eff_k, N);
                const std::vector<int32_t> pick = pick_centres(N, kk, seed, iteration);
                std::vector<uint32_t> cw((size_t)kk);
                for (int32_t c = 0; c < kk; ++c)
                    cw[(size_t)c] = words[cur[(size_t)pick[(size_t)c]]];
                e = cudaMemcpyAsync(d_cen.p, cw.data(), (size_t)kk * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                    ctx->stream);
                if (e != cudaSuccess)
                    return cuda_error(ctx, e, "centre upload");
                s = assign_centers(ctx, static_cast<const uint32_t *>(d_cur.p), N,
                                   static_cast<const uint32_t *>(d_cen.p), kk, len, static_cast<int32_t *>(d_asg.p));
                if (s != IG_OK)
                    return s;
                e = cudaMemcpyAsync(asg.data(), d_asg.p, (size_t)N * sizeof(int32_t), cudaMemcpyDeviceToHost,
                                    ctx->stream);
                if (e == cudaSuccess)
                    e = cudaStreamSynchronize(ctx->stream);
                if (e != cudaSuccess)
                    return cuda_error(ctx, e, "assignment download");
            }
        }
        // stable partition by cluster; empty clusters vanish
        std::vector<int64_t> start((size_t)kk + 1, 0);
        for (int32_t i = 0; i < N; ++i)
            ++start[(size_t)asg[(size_t)i] + 1];
        std::vector<int64_t> offs{0};
        std::vector<int32_t> cl_of;  // cluster index of each non-empty cluster
        for (int32_t c = 0; c < kk; ++c)
            if (start[(size_t)c + 1] > 0) {
                cl_of.push_back(c);
                offs.push_back(offs.back() + start[(size_t)c + 1]);
            }
        for (int32_t c = 0; c < kk; ++c)
            start[(size_t)c + 1] += start[(size_t)c];
        std::vector<int32_t> part((size_t)N);  // global ids in cluster order
        for (int32_t i = 0; i < N; ++i)
            part[(size_t)start[(size_t)asg[(size_t)i]]++] = cur[(size_t)i];
        const int32_t jobs = (int32_t)cl_of.size();
        {
            std::lock_guard<std::mutex> lk(ctx->mu);
            DeviceGuard dg(ctx->device);
            cudaError_t e = cudaMemcpyAsync(d_ids.p, part.data(), (size_t)N * sizeof(int32_t), cudaMemcpyHostToDevice,
                                            ctx->stream);
            if (e != cudaSuccess)
                return cuda_error(ctx, e, "partition upload");
            ig_status s = gather_words(ctx, static_cast<const uint32_t *>(d_all.p),
                                       static_cast<const int32_t *>(d_ids.p), N, static_cast<uint32_t *>(d_part.p));
            if (s != IG_OK)
                return s;
        }
        // all clusters as one pipelined batch: groups built on the device
        // while host threads run the greedies of the groups already built
        std::vector<int32_t> lens((size_t)jobs, len), eds((size_t)jobs, min_ed), counts((size_t)jobs, 0);
        std::vector<int32_t> order((size_t)N, 0);
        ig_status s = solve_groups(ctx, static_cast<const uint32_t *>(d_part.p), 1, offs.data(), jobs, lens.data(),
                                   eds.data(), 1, host_threads, order.data(), counts.data(), nullptr);
        if (s != IG_OK)
            return s;
        next.clear();
        for (int32_t j = 0; j < jobs; ++j)
            for (int32_t q = 0; q < counts[(size_t)j]; ++q)
                next.push_back(part[(size_t)(offs[(size_t)j] + order[(size_t)(offs[(size_t)j] + q)])]);
        history.push_back((int64_t)next.size());
        if (sizes)
            sizes[iteration - 1] = (int64_t)next.size();
        // the reference's test: the last convergenceIterations sizes agree
        // (a value <= 1 stops after the first iteration; < 0 never does)
        bool converged = converge_iters >= 0 && (int64_t)history.size() >= (int64_t)converge_iters;
        for (int32_t c = 1; converged && c < converge_iters; ++c)
            converged = history[history.size() - 1] == history[history.size() - 1 - (size_t)c];
        cur.swap(next);
        if (converged)
            break;
    }
    std::copy(cur.begin(), cur.end(), codebook);
    *count = (int32_t)cur.size();
    if (iterations)
        *iterations = iteration;
    return IG_OK;
    IG_ABI_CATCH
}
