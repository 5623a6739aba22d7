// C ABI of libindexgen_cuda (declarations and reference citations in
// include/indexgen_cuda.h).
#include <algorithm>
#include <atomic>
#include <memory>
#include <cstdlib>
#include <cstring>
#include <new>
#include <numeric>
#include <string>
#include <thread>

#include <unistd.h>

#include "ig_internal.h"


namespace ig {

ig_status set_error(Ctx *ctx, ig_status s, const std::string &msg)
{
    if (ctx) {
        std::lock_guard<std::mutex> lk(ctx->err_mu);
        ctx->last_error = msg;
    }
    return s;
}

std::shared_ptr<void> HostBudget::acquire(int64_t bytes)
{
    std::unique_lock<std::mutex> lk(mu_);
    cv_.wait(lk, [&] { return used_ == 0 || used_ + bytes <= limit_; });
    used_ += bytes;
    auto self = shared_from_this();
    return std::shared_ptr<void>(reinterpret_cast<void *>(1), [self, bytes](void *) {
        std::lock_guard<std::mutex> g(self->mu_);
        self->used_ -= bytes;
        self->cv_.notify_all();
    });
}

void HostBudget::set_limit(int64_t limit)
{
    std::lock_guard<std::mutex> lk(mu_);
    limit_ = limit;
    cv_.notify_all();
}

int64_t HostBudget::limit()
{
    std::lock_guard<std::mutex> lk(mu_);
    return limit_;
}

int64_t HostBudget::used()
{
    std::lock_guard<std::mutex> lk(mu_);
    return used_;
}

int64_t default_host_budget()
{
    const long pages = sysconf(_SC_PHYS_PAGES), page = sysconf(_SC_PAGE_SIZE);
    if (pages <= 0 || page <= 0)
        return (int64_t)16 << 30;
    return (int64_t)pages * page / 2;
}

cudaError_t dev_malloc(Ctx *ctx, void **p, size_t bytes, cudaStream_t st)
{
    ctx->device_allocs++;
    int64_t left = ctx->fail_alloc_in.load();
    while (left > 0 && !ctx->fail_alloc_in.compare_exchange_weak(left, left - 1)) {
    }
    if (left == 1) {  // this is the allocation chosen to fail (injected, once)
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    return cudaMallocAsync(p, bytes, st);
}

ig_status cuda_error(Ctx *ctx, cudaError_t e, const char *what)
{
    cudaGetLastError();
    return set_error(ctx, e == cudaErrorMemoryAllocation ? IG_ERR_OOM : IG_ERR_CUDA,
                     std::string(what) + ": " + cudaGetErrorString(e));
}

namespace {

ig_status check_job(const uint32_t *words, int32_t n, int len)
{
    if (n < 0 || len < 1 || len > IG_MAX_LEN || (n > 0 && !words))
        return IG_ERR_INPUT;
    return IG_OK;
}

// Device copy of the words (host input) or the caller's device pointer.
ig_status stage_words(Ctx *ctx, const uint32_t *words, int32_t n, int on_device, const uint32_t **d_words)
{
    if (on_device || n == 0) {
        *d_words = words;
        return IG_OK;
    }
    const size_t bytes = (size_t)n * sizeof(uint32_t);
    if (ctx->words.bytes < bytes) {
        if (ctx->words.ptr)
            cudaFreeAsync(ctx->words.ptr, ctx->stream);
        ctx->words.ptr = nullptr;
        ctx->words.bytes = 0;
        cudaError_t e = dev_malloc(ctx, &ctx->words.ptr, bytes, ctx->stream);
        if (e != cudaSuccess)
            return cuda_error(ctx, e, "word buffer allocation");
        ctx->words.bytes = bytes;
    }
    cudaError_t e = cudaMemcpyAsync(ctx->words.ptr, words, bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess)
        return cuda_error(ctx, e, "word upload");
    *d_words = static_cast<const uint32_t *>(ctx->words.ptr);
    return IG_OK;
}

void release_graph(ig_graph *g, bool caller_holds_lock = false)
{
    if (!g)
        return;
    if (g->ctx) {
        // the frees go on the context stream: under the context lock, so that
        // they never land inside another thread's graph capture of that stream
        std::unique_lock<std::mutex> lk(g->ctx->mu, std::defer_lock);
        if (!caller_holds_lock)
            lk.lock();
        DeviceGuard dg(g->ctx->device);
        if (g->d_row_ptr)
            cudaFreeAsync(g->d_row_ptr, g->ctx->stream);
        if (g->d_cols)
            cudaFreeAsync(g->d_cols, g->ctx->stream);
        if (g->d_adj_ptr)
            cudaFreeAsync(g->d_adj_ptr, g->ctx->stream);
        if (g->d_adj)
            cudaFreeAsync(g->d_adj, g->ctx->stream);
        if (g->d_pk_off)
            cudaFreeAsync(g->d_pk_off, g->ctx->stream);
        if (g->d_pk)
            cudaFreeAsync(g->d_pk, g->ctx->stream);
        cudaStreamSynchronize(g->ctx->stream);
    }
    delete g;
}

ig_status fetch_host(ig_graph *g)
{
    if (g->host_valid)
        return IG_OK;
    ig::Ctx *ctx = g->ctx;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    try {
        g->h_row_ptr.resize((size_t)g->n + 1);
        g->h_cols.resize((size_t)std::max<int64_t>(g->edges, 1));
    } catch (...) {
        return set_error(ctx, IG_ERR_OOM, "host CSR allocation failed");
    }
    cudaError_t e = cudaMemcpyAsync(g->h_row_ptr.data(), g->d_row_ptr, ((size_t)g->n + 1) * sizeof(int64_t),
                                    cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess && g->edges > 0)
        e = cudaMemcpyAsync(g->h_cols.data(), g->d_cols, (size_t)g->edges * sizeof(int32_t),
                            cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess)
        return cuda_error(ctx, e, "CSR download");
    g->host_valid = true;
    return IG_OK;
}

// One host block of `bytes` for a graph download (pinned when the pool has
// room, else plain memory), holding `token` -- its share of the host budget,
// taken by the caller before the context lock -- until the block is released.
std::shared_ptr<void> host_block(Ctx *ctx, size_t bytes, std::shared_ptr<void> token)
{
    std::shared_ptr<void> block = ctx->pinned->acquire(bytes);
    if (!block) {
        void *p = std::malloc(bytes);  // uninitialised: the copy fills it
        if (!p)
            return nullptr;
        block = std::shared_ptr<void>(p, std::free);
    }
    void *raw = block.get();
    return std::shared_ptr<void>(raw, [block, token](void *) mutable {
        block.reset();
        token.reset();
    });
}

// A graph goes to the host greedy as its canonical adjacency (offsets and
// 4-byte neighbour ids) or, when that would take at least kPackRowsMinBytes,
// with its rows bit-packed (ig_packrows.cu): the packing cuts the copy and
// the host memory a dense graph holds while its greedy runs by 2-3x, and the
// decoding adds about 1 ns per neighbour to the greedy, which a small graph's
// download does not win back.
constexpr size_t kPackRowsMinBytes = (size_t)512 << 20;

bool pack_for_host(const Graph *g)
{
    const int form = g->ctx->host_lists.load();
    if (form != IG_LISTS_AUTO)
        return form == IG_LISTS_PACKED;
    return ((size_t)g->n + 1) * sizeof(int64_t) + (size_t)g->edges * 8 >= kPackRowsMinBytes;
}

// Host bytes of a graph's download for the greedy.
size_t download_bytes(const Graph *g, bool packed)
{
    const size_t ptr_bytes = ((size_t)g->n + 1) * sizeof(int64_t);
    if (packed)
        return 2 * ptr_bytes + ((size_t)g->pk_words + 2) * sizeof(uint32_t);
    return ptr_bytes + (size_t)std::max<int64_t>(2 * g->edges, 1) * sizeof(int32_t);
}

// Decides the download's form and takes its share of the host budget with the
// context lock released, so that a caller whose greedy would free host room is
// never kept waiting for the device.  Packed rows are built first (their size
// is known only then); the plain adjacency is built by the copy.
ig_status reserve_download(ig_graph *g, bool &packed, std::shared_ptr<void> &token)
{
    ig::Ctx *ctx = g->ctx;
    packed = pack_for_host(g);
    if (packed) {
        std::lock_guard<std::mutex> lk(ctx->mu);
        DeviceGuard dg(ctx->device);
        ig_status s = build_packed_rows(ctx, g);
        if (s != IG_OK)
            return s;
    }
    token = ctx->host_budget->acquire((int64_t)download_bytes(g, packed));
    return IG_OK;
}

// Caller holds ctx->mu: the graph's greedy form into one new host block,
// copied on `st`.
ig_status queue_download(ig_graph *g, bool packed, std::shared_ptr<void> token, cudaStream_t st, HostGraph &hg)
{
    ig::Ctx *ctx = g->ctx;
    if (!packed) {
        ig_status s = build_adjacency(ctx, g);  // ends with the context stream idle
        if (s != IG_OK)
            return s;
    }
    const size_t ptr_bytes = ((size_t)g->n + 1) * sizeof(int64_t);
    std::shared_ptr<void> block = host_block(ctx, download_bytes(g, packed), std::move(token));
    if (!block)
        return set_error(ctx, IG_ERR_OOM, "host adjacency allocation failed");
    char *base = static_cast<char *>(block.get());
    int64_t *ap = reinterpret_cast<int64_t *>(base);
    cudaError_t e = cudaMemcpyAsync(ap, g->d_adj_ptr, ptr_bytes, cudaMemcpyDeviceToHost, st);
    hg.ptr = ap;
    if (packed) {
        int64_t *po = reinterpret_cast<int64_t *>(base + ptr_bytes);
        uint32_t *pk = reinterpret_cast<uint32_t *>(base + 2 * ptr_bytes);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(po, g->d_pk_off, ptr_bytes, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(pk, g->d_pk, ((size_t)g->pk_words + 2) * sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
        hg.idx = nullptr;
        hg.pk_off = po;
        hg.pk = pk;
    } else {
        int32_t *adj = reinterpret_cast<int32_t *>(base + ptr_bytes);
        if (e == cudaSuccess && g->edges > 0)
            e = cudaMemcpyAsync(adj, g->d_adj, (size_t)(2 * g->edges) * sizeof(int32_t), cudaMemcpyDeviceToHost, st);
        hg.idx = adj;
        hg.pk_off = nullptr;
        hg.pk = nullptr;
    }
    hg.storage = std::move(block);
    if (e != cudaSuccess) {
        cudaStreamSynchronize(st);
        hg.storage.reset();
        return cuda_error(ctx, e, "adjacency download");
    }
    return IG_OK;
}

// The graph's greedy form on the host (blocking).
ig_status fetch_adjacency(ig_graph *g, HostGraph &hg)
{
    ig::Ctx *ctx = g->ctx;
    bool packed = false;
    std::shared_ptr<void> token;
    ig_status s = reserve_download(g, packed, token);
    if (s != IG_OK)
        return s;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    if ((s = queue_download(g, packed, std::move(token), ctx->stream, hg)) != IG_OK)
        return s;
    const cudaError_t e = cudaStreamSynchronize(ctx->stream);
    return e == cudaSuccess ? IG_OK : cuda_error(ctx, e, "adjacency download");
}

// Validated job list from an offsets array.
ig_status make_jobs(Ctx *ctx, const int64_t *offsets, int32_t k, const int32_t *lens, const int32_t *min_eds,
                    std::vector<JobSpec> &jobs)
{
    if (k < 0 || (k > 0 && (!offsets || !lens || !min_eds)))
        return set_error(ctx, IG_ERR_INPUT, "jobs: offsets[k+1], lens[k] and min_eds[k] are required");
    if (k > 0 && offsets[0] != 0)
        return set_error(ctx, IG_ERR_INPUT, "jobs: offsets[0] must be 0");
    jobs.clear();
    for (int32_t j = 0; j < k; ++j) {
        const int64_t n = offsets[j + 1] - offsets[j];
        if (n < 0 || n > INT32_MAX || lens[j] < 1 || lens[j] > IG_MAX_LEN)
            return set_error(ctx, IG_ERR_INPUT, "jobs: offsets must not decrease and 1 <= len <= 16");
        jobs.push_back(JobSpec{offsets[j], (int32_t)n, lens[j], min_eds[j]});
    }
    if (k > 0 && offsets[k] > INT32_MAX)
        return set_error(ctx, IG_ERR_CAPACITY, "more than 2^31-1 words in one batch");
    return IG_OK;
}

}  // namespace

// fetch_adjacency with the copy on the context's download stream: returns
// once the copy is queued, followed by the host function `then(arg)` (run by
// the CUDA runtime when the copy has landed; it must not call CUDA) and the
// event *done.  The caller may queue more work on the context stream
// meanwhile (the next batch group's build overlaps the copy) and must wait on
// *done before it frees g.  On an error nothing of `then` runs.
ig_status fetch_adjacency_async(ig_graph *g, HostGraph &hg, cudaEvent_t *done, cudaHostFn_t then, void *arg)
{
    ig::Ctx *ctx = g->ctx;
    bool packed = false;
    std::shared_ptr<void> token;
    ig_status s = reserve_download(g, packed, token);
    if (s != IG_OK)
        return s;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    cudaError_t e = cudaSuccess;
    if (!ctx->dl_stream && (e = cudaStreamCreateWithFlags(&ctx->dl_stream, cudaStreamNonBlocking)) != cudaSuccess) {
        ctx->dl_stream = nullptr;
        return cuda_error(ctx, e, "download stream");
    }
    cudaEvent_t fin = nullptr;
    if ((e = cudaEventCreateWithFlags(&fin, cudaEventDisableTiming)) != cudaSuccess)
        return cuda_error(ctx, e, "download event");
    hg.order_threads = 1;
    hg.jobs = g->jobs;
    hg.job_edge_off = g->job_edge_off;
    if ((s = queue_download(g, packed, std::move(token), ctx->dl_stream, hg)) != IG_OK) {
        cudaEventDestroy(fin);
        return s;
    }
    if (then && (e = cudaLaunchHostFunc(ctx->dl_stream, then, arg)) != cudaSuccess) {
        cudaStreamSynchronize(ctx->dl_stream);
        cudaEventDestroy(fin);
        return cuda_error(ctx, e, "download callback");
    }
    if ((e = cudaEventRecord(fin, ctx->dl_stream)) != cudaSuccess) {
        cudaStreamSynchronize(ctx->dl_stream);  // `then` has run
        cudaEventDestroy(fin);
        *done = nullptr;
        return IG_OK;
    }
    *done = fin;
    return IG_OK;
}


bool reserve_pool(Ctx *ctx, size_t bytes)
{
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    void *p = nullptr;
    cudaError_t e = dev_malloc(ctx, &p, bytes, ctx->stream);
    if (e == cudaSuccess)
        e = cudaFreeAsync(p, ctx->stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(ctx->stream);
    cudaGetLastError();
    return e == cudaSuccess;
}

std::shared_ptr<void> PinnedPool::acquire(size_t bytes)
{
    // size classes: powers of two up to 1 GiB, whole GiB above
    constexpr size_t kGiB = (size_t)1 << 30;
    size_t cls = (size_t)1 << 20;
    while (cls < bytes && cls < kGiB)
        cls <<= 1;
    if (cls < bytes)
        cls = (bytes + kGiB - 1) / kGiB * kGiB;
    const size_t slack = cls < kGiB ? 3 * cls : 2 * kGiB;  // a cached block this much larger still serves
    void *p = nullptr;
    {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = free_.lower_bound(cls);
        if (it != free_.end() && it->first <= cls + slack) {
            cls = it->first;
            p = it->second;
            free_.erase(it);
        } else {
            // make room by unpinning cached blocks that serve no one now
            while (total_ + cls > kCap && !free_.empty()) {
                auto big = std::prev(free_.end());
                cudaFreeHost(big->second);
                total_ -= big->first;
                free_.erase(big);
            }
            cudaGetLastError();
            if (total_ + cls > kCap)
                return nullptr;
            total_ += cls;  // reserved before the (slow) pinning, outside the lock
        }
    }
    if (!p && cudaHostAlloc(&p, cls, cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        std::lock_guard<std::mutex> lk(mu_);
        total_ -= cls;
        return nullptr;
    }
    std::shared_ptr<PinnedPool> self = shared_from_this();
    return std::shared_ptr<void>(p, [self, cls](void *q) {
        std::lock_guard<std::mutex> lk(self->mu_);
        self->free_.emplace(cls, q);
    });
}

PinnedPool::~PinnedPool()
{
    for (auto &b : free_)
        cudaFreeHost(b.second);
    cudaGetLastError();
}

// What the host greedy needs of a graph, downloaded once: the canonical
// adjacency (order_threads = 1) or the upper CSR (other orders), plus the jobs.
ig_status download_for_greedy(Graph *gg, int order_threads, HostGraph &hg)
{
    ig_graph *g = static_cast<ig_graph *>(gg);
    hg.order_threads = order_threads;
    hg.jobs = g->jobs;
    hg.job_edge_off = g->job_edge_off;
    if (order_threads == 1)
        return fetch_adjacency(g, hg);
    std::shared_ptr<void> token = g->ctx->host_budget->acquire(
        (int64_t)(((size_t)g->n + 1) * sizeof(int64_t) + (size_t)g->edges * sizeof(int32_t)));
    ig_status s = fetch_host(g);
    if (s != IG_OK)
        return s;
    try {
        auto csr = std::make_shared<std::pair<std::vector<int64_t>, std::vector<int32_t>>>(g->h_row_ptr, g->h_cols);
        hg.ptr = csr->first.data();
        hg.idx = csr->second.data();
        hg.storage = std::shared_ptr<void>(csr.get(), [csr, token](void *) mutable {
            csr.reset();
            token.reset();
        });
    } catch (...) {
        return set_error(g->ctx, IG_ERR_OOM, "host CSR copy failed");
    }
    return IG_OK;
}

// Greedy of every job on `host_threads` host threads (pure host work),
// largest job first.  Job j's selection (job-local ids) goes to
// order + word_off_j - order_base; counts[j] its size.
int32_t greedy_one(const HostGraph &hg, int job, int32_t *out)
{
    const JobSpec &J = hg.jobs[(size_t)job];
    if (hg.pk)
        return greedy_from_packed(hg.ptr + J.word_off, hg.pk_off + J.word_off, hg.pk, J.n, J.word_off, out);
    if (hg.order_threads == 1)
        return greedy_from_adjacency(hg.ptr + J.word_off, hg.idx, J.n, J.word_off, out);
    return greedy_from_upper(hg.ptr + J.word_off, hg.idx, J.n, J.word_off, hg.order_threads, out);
}

bool run_greedies(const HostGraph &hg, int host_threads, int64_t order_base, int32_t *order, int32_t *counts)
{
    const int k = (int)hg.jobs.size();
    std::vector<int> seq((size_t)k);
    std::iota(seq.begin(), seq.end(), 0);
    std::stable_sort(seq.begin(), seq.end(), [&](int a, int b) {
        return hg.job_edge_off[(size_t)a + 1] - hg.job_edge_off[(size_t)a] >
               hg.job_edge_off[(size_t)b + 1] - hg.job_edge_off[(size_t)b];
    });
    std::atomic<int> next{0};
    std::atomic<bool> failed{false};
    int T = host_threads > 0 ? host_threads : (int)std::max(1u, std::thread::hardware_concurrency());
    T = std::max(1, std::min(T, k));
    // several threads: a pool, one greedy per thread; one: the caller's own
    // greedies, one after another
    const bool pooled = T > 1;
    auto worker = [&]() {
        for (;;) {
            const int q = next++;
            if (q >= k)
                return;
            const JobSpec &J = hg.jobs[(size_t)seq[(size_t)q]];
            try {
                PooledGreedyScope scope(pooled);
                counts[seq[(size_t)q]] = greedy_one(hg, seq[(size_t)q], order + (J.word_off - order_base));
            } catch (...) {
                failed = true;
            }
        }
    };
    if (T == 1) {
        worker();
    } else {
        std::vector<std::thread> pool;
        for (int t = 0; t < T; ++t)
            pool.emplace_back(worker);
        for (auto &th : pool)
            th.join();
    }
    return !failed;
}

GreedyPool::GreedyPool(int threads)
{
    const int T = threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency());
    for (int t = 0; t < T; ++t)
        threads_.emplace_back([this]() { work(); });
}

GreedyPool::~GreedyPool()
{
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_ = true;
    }
    cv_.notify_all();
    for (auto &th : threads_)
        th.join();
}

void GreedyPool::submit(std::shared_ptr<const HostGraph> hg, int64_t order_base, int32_t *order, int32_t *counts,
                        const std::shared_ptr<Ticket> &ticket)
{
    {
        std::lock_guard<std::mutex> lk(mu_);
        for (int j = 0; j < (int)hg->jobs.size(); ++j) {
            Task t;
            t.edges = hg->job_edge_off[(size_t)j + 1] - hg->job_edge_off[(size_t)j];
            t.seq = seq_++;
            t.hg = hg;
            t.job = j;
            t.out = order + (hg->jobs[(size_t)j].word_off - order_base);
            t.count = counts + j;
            t.ticket = ticket;
            ticket->left++;
            q_.push(std::move(t));
        }
    }
    cv_.notify_all();
}

bool GreedyPool::wait(const std::shared_ptr<Ticket> &ticket)
{
    // the waiting thread is done driving the device: it runs queued
    // greedies too (the largest first, whoever queued them) until its own
    // jobs have finished
    std::unique_lock<std::mutex> lk(mu_);
    while (ticket->left > 0) {
        if (!q_.empty())
            run_one(lk);
        else
            done_.wait(lk);
    }
    return !ticket->failed;
}

void GreedyPool::run_one(std::unique_lock<std::mutex> &lk)
{
    Task t = q_.top();
    q_.pop();
    lk.unlock();
    bool ok = true;
    try {
        PooledGreedyScope pooled;
        *t.count = greedy_one(*t.hg, t.job, t.out);
    } catch (...) {
        ok = false;
    }
    t.hg.reset();  // the last task of a graph frees its host copy here
    lk.lock();
    if (!ok)
        t.ticket->failed = true;
    if (--t.ticket->left == 0)
        done_.notify_all();
}

void GreedyPool::work()
{
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
        cv_.wait(lk, [this]() { return stop_ || !q_.empty(); });
        if (q_.empty())
            return;  // stop_ and nothing left
        run_one(lk);
    }
}

// Concurrent ig_solve calls on one context, built together.  The reference
// host solves clusters from a pool of worker threads, each calling its GPU
// path on its own (src/SparseMat.cpp:978-1010); here a call that finds the
// device busy leaves its job in `pending`, and whichever waiting caller gets
// the device next builds every pending job as one batch (one persistent
// pair launch, block-diagonal graph).  Each caller then runs its own job's
// greedy on its own thread.  Nothing waits for company: a lone call is built
// at once.
struct SolveRequest {
    const uint32_t *words = nullptr;
    int32_t n = 0;
    int len = 1, min_ed = 0;
    std::shared_ptr<HostGraph> hg;  // the batch's adjacency on the host
    int job = -1;                   // this request's job in it
    int64_t edges = 0;
    ig_status status = IG_OK;
    bool ready = false;
};

struct SolveCombiner {
    std::mutex mu;
    std::condition_variable cv;
    std::vector<SolveRequest *> pending;
    bool building = false;
    int64_t batches = 0, requests = 0;
};

std::shared_ptr<SolveCombiner> solve_combiner(Ctx *ctx)
{
    std::lock_guard<std::mutex> lk(ctx->greedy_mu);
    if (!ctx->combiner)
        ctx->combiner = std::make_shared<SolveCombiner>();
    return ctx->combiner;
}

// The waiting requests one coalesced build takes, in arrival order: the
// first always, more while the batch stays within 2^36 pair tests (about
// 0.1 s of device work) and 2^26 words; the rest wait for the next build.
void take_coalesced(std::vector<SolveRequest *> &pending, std::vector<SolveRequest *> &batch)
{
    long double pairs = 0;
    int64_t words = 0;
    size_t k = 0;
    for (; k < pending.size(); ++k) {
        const SolveRequest *r = pending[k];
        const long double p = (long double)r->n * (r->n > 0 ? r->n - 1 : 0) / 2;
        if (k > 0 && (pairs + p > (long double)(1ull << 36) || words + r->n > ((int64_t)1 << 26)))
            break;
        pairs += p;
        words += r->n;
    }
    batch.assign(pending.begin(), pending.begin() + (long)k);
    pending.erase(pending.begin(), pending.begin() + (long)k);
}

void build_requests(ig_ctx *ctx, const std::vector<SolveRequest *> &reqs);

// A merged build can fail where each request alone would not (its summed
// workspace or a per-launch limit): those requests are then built one by
// one, and each keeps its own outcome.
void build_requests_or_split(ig_ctx *ctx, const std::vector<SolveRequest *> &reqs)
{
    build_requests(ctx, reqs);
    if (reqs.size() < 2 || (reqs[0]->status != IG_ERR_OOM && reqs[0]->status != IG_ERR_CAPACITY))
        return;
    for (SolveRequest *r : reqs)
        build_requests(ctx, {r});
}

// Builds the requests as one batch and downloads its canonical adjacency.
void build_requests(ig_ctx *ctx, const std::vector<SolveRequest *> &reqs)
{
    ig_status s = IG_OK;
    try {
        std::vector<uint32_t> words;
        std::vector<int64_t> off{0};
        std::vector<int32_t> lens, eds;
        for (SolveRequest *r : reqs) {
            words.insert(words.end(), r->words, r->words + r->n);
            off.push_back(off.back() + r->n);
            lens.push_back(r->len);
            eds.push_back(r->min_ed);
        }
        ig_graph *g = nullptr;
        s = ig_batch_build(ctx, words.data(), off.data(), (int32_t)reqs.size(), lens.data(), eds.data(), 0, &g);
        if (s == IG_OK) {
            auto hg = std::make_shared<HostGraph>();
            s = download_for_greedy(g, 1, *hg);
            if (s == IG_OK)
                for (size_t j = 0; j < reqs.size(); ++j) {
                    reqs[j]->hg = hg;
                    reqs[j]->job = (int)j;
                    reqs[j]->edges = g->job_edge_off[j + 1] - g->job_edge_off[j];
                }
            release_graph(g);
        }
    } catch (const std::bad_alloc &) {
        s = IG_ERR_OOM;
    } catch (...) {  // the waiting callers must hear back whatever happens
        s = IG_ERR_STATE;
    }
    for (SolveRequest *r : reqs)
        r->status = s;
}

std::shared_ptr<GreedyPool> shared_greedy_pool(Ctx *ctx)
{
    std::lock_guard<std::mutex> lk(ctx->greedy_mu);
    if (!ctx->greedy_pool) {
        const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
        ctx->greedy_pool = std::make_shared<GreedyPool>(std::max(1, hw - 1));
    }
    return ctx->greedy_pool;
}

// Host callback of a group's adjacency copy: queues the group's greedies.
struct SubmitWhenCopied {
    GreedyPool *pool;
    std::shared_ptr<HostGraph> hg;
    int32_t *order;
    int32_t *counts;
    std::shared_ptr<GreedyPool::Ticket> ticket;
    static void CUDART_CB run(void *p)
    {
        std::unique_ptr<SubmitWhenCopied> c(static_cast<SubmitWhenCopied *>(p));
        c->pool->submit(c->hg, 0, c->order, c->counts, c->ticket);
    }
};

// Pipeline: the batch is cut into up to eight contiguous groups of about
// equal pair count (at least 2^30 pair tests each); as soon as a group's graph is downloaded its jobs join the
// greedy pool's queue (largest first), so host threads run the greedies of
// every finished group while the device builds the next.
ig_status solve_groups(ig_ctx *ctx, const uint32_t *words, int words_on_device, const int64_t *offsets, int32_t jobs,
                       const int32_t *lens, const int32_t *min_eds, int order_threads, int host_threads,
                       int32_t *order, int32_t *counts, int64_t *edges)
{
    long double total = 0;
    for (int32_t j = 0; j < jobs; ++j)
        total += (long double)(offsets[j + 1] - offsets[j]) * (offsets[j + 1] - offsets[j]);
    // a group costs a few hundred microseconds of host round trips besides
    // its device work, so each one gets at least 2^30 pair tests (about
    // 1.4 ms on nibble lanes): small batches stay one launch
    const long double min_group = (long double)(1ull << 31);  // total counts n^2, not n(n-1)/2
    const int groups = (int)std::max<long double>(1, std::min<long double>({8.0L, (long double)jobs, total / min_group}));
    std::vector<int> cut{0};
    long double acc = 0;
    for (int32_t j = 0; j < jobs; ++j) {
        acc += (long double)(offsets[j + 1] - offsets[j]) * (offsets[j + 1] - offsets[j]);
        if ((int)cut.size() < groups && acc >= total * cut.size() / groups && j + 1 < jobs)
            cut.push_back(j + 1);
    }
    cut.push_back(jobs);
    ig_status s = IG_OK;
    // The greedies run on the context's pool (one thread fewer than the
    // cores: this thread drives the device, and a build that waits for a
    // core behind the greedies stalls the whole pipeline), or on a pool of
    // their own when the caller asks for fewer threads than that.
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    const int cap = std::max(1, hw - 1);
    std::shared_ptr<GreedyPool> pool_ref;
    if (host_threads > 0 && host_threads < cap)
        pool_ref = std::make_shared<GreedyPool>(std::max(1, std::min<int>(host_threads, jobs)));
    else
        pool_ref = shared_greedy_pool(ctx);
    GreedyPool &pool = *pool_ref;
    const auto ticket = std::make_shared<GreedyPool::Ticket>();
    // A group whose adjacency copy runs on the download stream while the
    // next group builds; the copy's host callback queues its greedies the
    // moment it lands, and the group's device buffers are freed after the
    // next build.
    struct Pending {
        ig_graph *g = nullptr;
        cudaEvent_t done = nullptr;
    } pend;
    auto finish = [&]() -> ig_status {
        if (!pend.g)
            return IG_OK;
        ig_status r = IG_OK;
        if (pend.done) {
            const cudaError_t e = cudaEventSynchronize(pend.done);
            cudaEventDestroy(pend.done);
            if (e != cudaSuccess)
                r = cuda_error(ctx, e, "adjacency download");
        }
        release_graph(pend.g);
        pend = Pending();
        return r;
    };
    for (size_t gi = 0; gi + 1 < cut.size(); ++gi) {
        const int lo = cut[gi], hi = cut[gi + 1];
        if (lo >= hi)
            continue;
        std::vector<int64_t> sub((size_t)(hi - lo) + 1);
        for (int j = lo; j <= hi; ++j)
            sub[(size_t)(j - lo)] = offsets[j] - offsets[lo];
        ig_graph *g = nullptr;
        s = ig_batch_build(ctx, words + offsets[lo], sub.data(), hi - lo, lens + lo, min_eds + lo, words_on_device,
                           &g);
        const ig_status f = finish();  // the previous group's copy ran during this build
        if (s == IG_OK)
            s = f;
        if (s != IG_OK) {
            release_graph(g);
            break;
        }
        if (edges)
            for (int j = lo; j < hi; ++j)
                edges[j] = g->job_edge_off[(size_t)(j - lo) + 1] - g->job_edge_off[(size_t)(j - lo)];
        auto hg = std::make_shared<HostGraph>();
        if (order_threads == 1) {
            cudaEvent_t done = nullptr;
            auto *sub_ctx = new SubmitWhenCopied{&pool, hg, order + offsets[lo], counts + lo, ticket};
            s = fetch_adjacency_async(g, *hg, &done, SubmitWhenCopied::run, sub_ctx);
            if (s != IG_OK) {
                delete sub_ctx;
                release_graph(g);
                break;
            }
            pend.g = g;
            pend.done = done;
        } else {
            s = download_for_greedy(g, order_threads, *hg);
            release_graph(g);
            if (s != IG_OK)
                break;
            pool.submit(hg, 0, order + offsets[lo], counts + lo, ticket);
        }
    }
    const ig_status f = finish();
    if (s == IG_OK)
        s = f;
    const bool host_ok = pool.wait(ticket);
    if (s == IG_OK && !host_ok)
        s = set_error(ctx, IG_ERR_OOM, "host greedy allocation failed");
    return s;
}

namespace {

ig_status job_codebooks_impl(ig_graph *g, int order_threads, int host_threads, int32_t *order, int32_t *counts)
{
    HostGraph hg;
    ig_status s = download_for_greedy(g, order_threads, hg);
    if (s != IG_OK)
        return s;
    if (!run_greedies(hg, host_threads, 0, order, counts))
        return set_error(g->ctx, IG_ERR_OOM, "host greedy allocation failed");
    return IG_OK;
}

}  // namespace
}  // namespace ig

namespace ig {

ig_status estimate_edges(Ctx *ctx, const std::vector<SampleJob> &jobs, std::vector<long double> &edges)
{
    edges.assign(jobs.size(), 0.0L);
    std::vector<uint32_t> words;
    std::vector<JobSpec> spec;
    std::vector<long double> scale;
    for (const SampleJob &j : jobs) {
        const int32_t S = std::min<int32_t>(j.n, kSampleWords);
        spec.push_back(JobSpec{(int64_t)words.size(), S, j.len, j.min_ed});
        for (int32_t i = 0; i < S; ++i)
            words.push_back(j.words[(int64_t)i * j.n / S]);
        scale.push_back(S == j.n || S < 2 ? 1.0L
                                          : (long double)j.n * (j.n - 1) / ((long double)S * (S - 1)));
    }
    if (words.empty())
        return IG_OK;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    if (!dg.ok)
        return set_error(ctx, IG_ERR_CUDA, "cannot select the context's device");
    ig_graph *g = new (std::nothrow) ig_graph();
    if (!g)
        return IG_ERR_OOM;
    const uint32_t *d_words = nullptr;
    ig_status s = stage_words(ctx, words.data(), (int32_t)words.size(), 0, &d_words);
    const bool tune = ctx->autotune;
    ctx->autotune = false;  // samples must not pick the work split of real batches
    if (s == IG_OK)
        s = build_batch(ctx, d_words, spec, g);
    ctx->autotune = tune;
    if (s == IG_OK)
        for (size_t k = 0; k < jobs.size(); ++k)
            edges[k] = (long double)(g->job_edge_off[k + 1] - g->job_edge_off[k]) * scale[k];
    release_graph(g, true);
    return s;
}

}  // namespace ig

extern "C" {

const char *ig_version(void) { return "indexgen_b200 0.1 (sm_100a)"; }

const char *ig_status_string(ig_status s)
{
    switch (s) {
    case IG_OK: return "ok";
    case IG_ERR_INPUT: return "invalid input";
    case IG_ERR_CAPACITY: return "capacity exceeded";
    case IG_ERR_OOM: return "out of memory";
    case IG_ERR_CUDA: return "CUDA error";
    case IG_ERR_TIMEOUT: return "device wait timed out";
    case IG_ERR_CANCELLED: return "cancelled";
    case IG_ERR_STATE: return "invalid state";
    }
    return "unknown status";
}

ig_status ig_ctx_create(ig_ctx **out, int device)
{
    IG_ABI_TRY
    if (!out)
        return IG_ERR_INPUT;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return device < 0 ? IG_ERR_INPUT : IG_ERR_CUDA;
    }
    ig_ctx *c = new (std::nothrow) ig_ctx();
    if (!c)
        return IG_ERR_OOM;
    c->device = device;
    ig::DeviceGuard dg(device);
    cudaDeviceProp prop;
    if (!dg.ok || cudaGetDeviceProperties(&prop, device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete c;
        return IG_ERR_CUDA;
    }
    c->sm_count = prop.multiProcessorCount;
    // Keep freed stream-ordered allocations cached in the device pool so that
    // repeated jobs do not go back to the driver.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
    *out = c;
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_ctx_destroy(ig_ctx *ctx)
{
    IG_ABI_TRY
    if (!ctx)
        return IG_ERR_INPUT;
    {
        ig::DeviceGuard dg(ctx->device);
        for (ig::DevBuf *b :
             {&ctx->words, &ctx->sel, &ctx->counts, &ctx->records, &ctx->scan_tmp, &ctx->flags, &ctx->adj_tmp,
              &ctx->jobs, &ctx->aux, &ctx->cols_ws})
            if (b->ptr)
                cudaFreeAsync(b->ptr, ctx->stream);
        cudaStreamSynchronize(ctx->stream);
        cudaStreamDestroy(ctx->stream);
        for (cudaEvent_t e : ctx->ev)
            if (e)
                cudaEventDestroy(e);
        ctx->greedy_pool.reset();  // joins its threads (no call is running on a context being destroyed)
        for (cudaGraphExec_t x : ctx->graph_exec)
            if (x)
                cudaGraphExecDestroy(x);
        if (ctx->dl_stream) {
            cudaStreamSynchronize(ctx->dl_stream);
            cudaStreamDestroy(ctx->dl_stream);
        }
        if (ctx->stage)
            cudaFreeHost(ctx->stage);
        cudaGetLastError();
    }
    delete ctx;
    return IG_OK;
    IG_ABI_CATCH
}

const char *ig_last_error(const ig_ctx *ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

ig_status ig_ctx_stream(ig_ctx *ctx, void **stream)
{
    IG_ABI_TRY
    if (!ctx || !stream)
        return IG_ERR_INPUT;
    *stream = (void *)ctx->stream;
    return IG_OK;
    IG_ABI_CATCH
}

int64_t ig_ctx_launches(const ig_ctx *ctx) { return ctx ? ctx->launches : -1; }

ig_status ig_ctx_set_profiling(ig_ctx *ctx, int enable)
{
    IG_ABI_TRY
    if (!ctx)
        return IG_ERR_INPUT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ig::DeviceGuard dg(ctx->device);
    if (enable && !ctx->ev[0]) {
        for (cudaEvent_t &e : ctx->ev)
            if (cudaEventCreate(&e) != cudaSuccess)
                return ig::cuda_error(ctx, cudaGetLastError(), "cudaEventCreate");
    }
    ctx->profiling = enable != 0;
    for (int p = 0; p < ig::Ctx::kPhases; ++p) {
        ctx->phase_ms[p] = 0;
        ctx->phase_launches[p] = 0;
        ctx->phase_pending[p] = false;
    }
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_ctx_phase_time(const ig_ctx *ctx, int phase, double *ms, int64_t *launches)
{
    IG_ABI_TRY
    if (!ctx || phase < 0 || phase >= ig::Ctx::kPhases)
        return IG_ERR_INPUT;
    if (ms)
        *ms = ctx->phase_ms[phase];
    if (launches)
        *launches = ctx->phase_launches[phase];
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_ctx_reserve(ig_ctx *ctx, int64_t edges)
{
    IG_ABI_TRY
    if (!ctx || edges < 0)
        return IG_ERR_INPUT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ig::DeviceGuard dg(ctx->device);
    if ((unsigned long long)edges <= ig::rec_capacity(ctx))
        return IG_OK;
    if (ctx->records.ptr)
        cudaFreeAsync(ctx->records.ptr, ctx->stream);
    ctx->records.ptr = nullptr;
    ctx->records.bytes = 0;
    const size_t bytes = (size_t)edges * sizeof(ig::EdgeRecord);
    cudaError_t e = ig::dev_malloc(ctx, &ctx->records.ptr, bytes, ctx->stream);
    if (e != cudaSuccess) {
        ctx->records.ptr = nullptr;
        return ig::cuda_error(ctx, e, "edge record reservation");
    }
    ctx->records.bytes = bytes;
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_graph_build(ig_ctx *ctx, const uint32_t *words, int32_t n, int len, int min_ed, int words_on_device,
                         ig_graph **out)
{
    IG_ABI_TRY
    if (!ctx || !out)
        return IG_ERR_INPUT;
    *out = nullptr;
    if (ig::check_job(words, n, len) != IG_OK)
        return ig::set_error(ctx, IG_ERR_INPUT, "words must be non-null, n >= 0 and 1 <= len <= 16");
    std::lock_guard<std::mutex> lk(ctx->mu);
    ig::DeviceGuard dg(ctx->device);
    if (!dg.ok)
        return ig::set_error(ctx, IG_ERR_CUDA, "cannot select the context's device");
    ig_graph *g = new (std::nothrow) ig_graph();
    if (!g)
        return IG_ERR_OOM;
    const uint32_t *d_words = nullptr;
    ig_status s = ig::stage_words(ctx, words, n, words_on_device, &d_words);
    if (s == IG_OK)
        s = ig::build_batch(ctx, d_words, {ig::JobSpec{0, n, len, min_ed}}, g);
    if (s != IG_OK) {
        ig::release_graph(g, true);
        return s;
    }
    *out = g;
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_graph_free(ig_graph *g)
{
    IG_ABI_TRY
    if (!g)
        return IG_ERR_INPUT;
    ig::release_graph(g);
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_graph_stats(const ig_graph *g, int32_t *n, int64_t *edges)
{
    IG_ABI_TRY
    if (!g)
        return IG_ERR_INPUT;
    if (n)
        *n = g->n;
    if (edges)
        *edges = g->edges;
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_graph_upper_csr(const ig_graph *g, int64_t *row_ptr, int32_t *cols)
{
    IG_ABI_TRY
    if (!g || !row_ptr || (g->edges > 0 && !cols))
        return IG_ERR_INPUT;
    ig::Ctx *ctx = g->ctx;
    if (g->host_valid) {
        std::memcpy(row_ptr, g->h_row_ptr.data(), ((size_t)g->n + 1) * sizeof(int64_t));
        if (g->edges > 0)
            std::memcpy(cols, g->h_cols.data(), (size_t)g->edges * sizeof(int32_t));
        return IG_OK;
    }
    // straight from HBM into the caller's buffers (a DMA when they are pinned)
    std::lock_guard<std::mutex> lk(ctx->mu);
    ig::DeviceGuard dg(ctx->device);
    cudaError_t e = cudaMemcpyAsync(row_ptr, g->d_row_ptr, ((size_t)g->n + 1) * sizeof(int64_t),
                                    cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess && g->edges > 0)
        e = cudaMemcpyAsync(cols, g->d_cols, (size_t)g->edges * sizeof(int32_t), cudaMemcpyDeviceToHost,
                            ctx->stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess)
        return ig::cuda_error(ctx, e, "CSR download");
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_graph_pairs(const ig_graph *gc, int32_t *pairs)
{
    IG_ABI_TRY
    ig_graph *g = const_cast<ig_graph *>(gc);
    if (!g || (g->edges > 0 && !pairs))
        return IG_ERR_INPUT;
    ig_status s = ig::fetch_host(g);
    if (s != IG_OK)
        return s;
    int64_t k = 0;
    for (int32_t r = 0; r < g->n; ++r)
        for (int64_t e = g->h_row_ptr[(size_t)r]; e < g->h_row_ptr[(size_t)r + 1]; ++e) {
            pairs[2 * k] = r;
            pairs[2 * k + 1] = g->h_cols[(size_t)e];
            ++k;
        }
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_graph_device_csr(const ig_graph *g, const int64_t **row_ptr, const int32_t **cols)
{
    IG_ABI_TRY
    if (!g || !row_ptr || !cols)
        return IG_ERR_INPUT;
    *row_ptr = g->d_row_ptr;
    *cols = g->d_cols;
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_graph_adjacency(ig_graph *g, int64_t *adj_ptr, int32_t *adj)
{
    IG_ABI_TRY
    if (!g || !adj_ptr || (g->edges > 0 && !adj))
        return IG_ERR_INPUT;
    ig::Ctx *ctx = g->ctx;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ig::DeviceGuard dg(ctx->device);
    ig_status s = ig::build_adjacency(ctx, g);
    if (s != IG_OK)
        return s;
    cudaError_t e = cudaMemcpyAsync(adj_ptr, g->d_adj_ptr, ((size_t)g->n + 1) * sizeof(int64_t),
                                    cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess && g->edges > 0)
        e = cudaMemcpyAsync(adj, g->d_adj, (size_t)(2 * g->edges) * sizeof(int32_t), cudaMemcpyDeviceToHost,
                            ctx->stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess)
        return ig::cuda_error(ctx, e, "adjacency download");
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_graph_device_adjacency(ig_graph *g, const int64_t **adj_ptr, const int32_t **adj)
{
    IG_ABI_TRY
    if (!g || !adj_ptr || !adj)
        return IG_ERR_INPUT;
    ig::Ctx *ctx = g->ctx;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ig::DeviceGuard dg(ctx->device);
    ig_status s = ig::build_adjacency(ctx, g);
    if (s != IG_OK)
        return s;
    *adj_ptr = g->d_adj_ptr;
    *adj = g->d_adj;
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_graph_codebook(ig_graph *g, int order_threads, int32_t *order, int32_t *count)
{
    IG_ABI_TRY
    if (!g || !count || order_threads < 1 || (g->n > 0 && !order))
        return IG_ERR_INPUT;
    if (g->jobs.size() != 1)
        return ig::set_error(g->ctx, IG_ERR_STATE, "graph holds several jobs: use ig_graph_job_codebooks");
    int32_t c = 0;
    ig_status s = ig::job_codebooks_impl(g, order_threads, 1, order, &c);
    if (s == IG_OK)
        *count = c;
    return s;
    IG_ABI_CATCH
}

ig_status ig_graph_job_count(const ig_graph *g, int32_t *jobs)
{
    IG_ABI_TRY
    if (!g || !jobs)
        return IG_ERR_INPUT;
    *jobs = (int32_t)g->jobs.size();
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_graph_job_stats(const ig_graph *g, int32_t job, int64_t *first_word, int32_t *n, int64_t *edges)
{
    IG_ABI_TRY
    if (!g || job < 0 || job >= (int32_t)g->jobs.size())
        return IG_ERR_INPUT;
    if (first_word)
        *first_word = g->jobs[(size_t)job].word_off;
    if (n)
        *n = g->jobs[(size_t)job].n;
    if (edges)
        *edges = g->job_edge_off[(size_t)job + 1] - g->job_edge_off[(size_t)job];
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_graph_job_tiling(const ig_graph *g, int32_t job, int32_t *segment_width, int32_t *segments)
{
    IG_ABI_TRY
    if (!g || job < 0 || job >= (int32_t)g->jobs.size())
        return IG_ERR_INPUT;
    const bool known = (size_t)job < g->job_nseg.size();
    if (segment_width)
        *segment_width = known && g->job_nseg[(size_t)job] > 0 ? 1 << g->job_seg_shift[(size_t)job] : 0;
    if (segments)
        *segments = known ? g->job_nseg[(size_t)job] : 0;
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_graph_job_codebooks(ig_graph *g, int order_threads, int host_threads, int32_t *order, int32_t *counts)
{
    IG_ABI_TRY
    if (!g || order_threads < 1 || (g->n > 0 && !order) || (!g->jobs.empty() && !counts))
        return IG_ERR_INPUT;
    return ig::job_codebooks_impl(g, order_threads, host_threads, order, counts);
    IG_ABI_CATCH
}

ig_status ig_batch_build(ig_ctx *ctx, const uint32_t *words, const int64_t *offsets, int32_t jobs,
                         const int32_t *lens, const int32_t *min_eds, int words_on_device, ig_graph **out)
{
    IG_ABI_TRY
    if (!ctx || !out)
        return IG_ERR_INPUT;
    *out = nullptr;
    std::vector<ig::JobSpec> spec;
    ig_status s = ig::make_jobs(ctx, offsets, jobs, lens, min_eds, spec);
    if (s != IG_OK)
        return s;
    const int64_t total = jobs > 0 ? offsets[jobs] : 0;
    if (total > 0 && !words)
        return ig::set_error(ctx, IG_ERR_INPUT, "words must be non-null");
    std::lock_guard<std::mutex> lk(ctx->mu);
    ig::DeviceGuard dg(ctx->device);
    if (!dg.ok)
        return ig::set_error(ctx, IG_ERR_CUDA, "cannot select the context's device");
    ig_graph *g = new (std::nothrow) ig_graph();
    if (!g)
        return IG_ERR_OOM;
    const uint32_t *d_words = nullptr;
    s = ig::stage_words(ctx, words, (int32_t)total, words_on_device, &d_words);
    if (s == IG_OK)
        s = ig::build_batch(ctx, d_words, spec, g);
    if (s != IG_OK) {
        ig::release_graph(g, true);
        return s;
    }
    *out = g;
    return IG_OK;
    IG_ABI_CATCH
}


ig_status ig_solve_batch(ig_ctx *ctx, const uint32_t *words, const int64_t *offsets, int32_t jobs,
                         const int32_t *lens, const int32_t *min_eds, int order_threads, int host_threads,
                         int32_t *order, int32_t *counts, int64_t *edges)
{
    IG_ABI_TRY
    if (!ctx || order_threads < 1 || (jobs > 0 && (!order || !counts)))
        return IG_ERR_INPUT;
    std::vector<ig::JobSpec> spec;
    ig_status s = ig::make_jobs(ctx, offsets, jobs, lens, min_eds, spec);
    if (s != IG_OK)
        return s;
    return ig::solve_groups(ctx, words, 0, offsets, jobs, lens, min_eds, order_threads, host_threads, order, counts,
                            edges);
    IG_ABI_CATCH
}

ig_status ig_graph_write_adj_list(ig_graph *g, const char *path, int64_t *bytes)
{
    IG_ABI_TRY
    if (!g || !path)
        return IG_ERR_INPUT;
    ig::Ctx *ctx = g->ctx;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ig::DeviceGuard dg(ctx->device);
    if (!dg.ok)
        return ig::set_error(ctx, IG_ERR_CUDA, "cannot select the context's device");
    return ig::write_adj_list(ctx, g, path, bytes);
    IG_ABI_CATCH
}

ig_status ig_graph_read_adj_list(ig_ctx *ctx, const char *path, ig_graph **out)
{
    IG_ABI_TRY
    if (!ctx || !path || !out)
        return IG_ERR_INPUT;
    *out = nullptr;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ig::DeviceGuard dg(ctx->device);
    if (!dg.ok)
        return ig::set_error(ctx, IG_ERR_CUDA, "cannot select the context's device");
    ig_graph *g = new (std::nothrow) ig_graph();
    if (!g)
        return IG_ERR_OOM;
    const ig_status s = ig::read_adj_list(ctx, path, g);
    if (s != IG_OK) {
        ig::release_graph(g, true);
        return s;
    }
    *out = g;
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_assign_centers(ig_ctx *ctx, const uint32_t *words, int64_t n, const uint32_t *centers, int32_t k,
                            int len, int on_device, int32_t *assignment)
{
    IG_ABI_TRY
    if (!ctx || n < 0 || k < 0 || len < 1 || len > IG_MAX_LEN)
        return IG_ERR_INPUT;
    if (n == 0)
        return IG_OK;
    if (!words || !assignment || k < 1 || !centers)
        return ig::set_error(ctx, IG_ERR_INPUT, "assign: words, centers (k >= 1) and assignment are required");
    if (n > INT32_MAX)
        return ig::set_error(ctx, IG_ERR_CAPACITY, "assign: more than 2^31-1 words");
    std::lock_guard<std::mutex> lk(ctx->mu);
    ig::DeviceGuard dg(ctx->device);
    if (!dg.ok)
        return ig::set_error(ctx, IG_ERR_CUDA, "cannot select the context's device");
    cudaStream_t st = ctx->stream;
    if (on_device) {
        ig_status s = ig::assign_centers(ctx, words, n, centers, k, len, assignment);
        if (s != IG_OK)
            return s;
        const cudaError_t e = cudaStreamSynchronize(st);
        return e == cudaSuccess ? IG_OK : ig::cuda_error(ctx, e, "assign");
    }
    const uint32_t *d_words = nullptr;
    ig_status s = ig::stage_words(ctx, words, (int32_t)n, 0, &d_words);
    if (s != IG_OK)
        return s;
    const size_t cbytes = ((size_t)k * sizeof(uint32_t) + 255) & ~(size_t)255;
    s = ig::ensure_buffer(ctx, ctx->aux, cbytes + (size_t)n * sizeof(int32_t), "assignment workspace");
    if (s != IG_OK)
        return s;
    uint32_t *d_centres = static_cast<uint32_t *>(ctx->aux.ptr);
    int32_t *d_out = reinterpret_cast<int32_t *>(static_cast<char *>(ctx->aux.ptr) + cbytes);
    cudaError_t e = cudaMemcpyAsync(d_centres, centers, (size_t)k * sizeof(uint32_t), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess)
        return ig::cuda_error(ctx, e, "centre upload");
    s = ig::assign_centers(ctx, d_words, n, d_centres, k, len, d_out);
    if (s != IG_OK)
        return s;
    e = cudaMemcpyAsync(assignment, d_out, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    return e == cudaSuccess ? IG_OK : ig::cuda_error(ctx, e, "assignment download");
    IG_ABI_CATCH
}

ig_status ig_solve(ig_ctx *ctx, const uint32_t *words, int32_t n, int len, int min_ed, int order_threads,
                   int32_t *order, int32_t *count, int64_t *edges)
{
    IG_ABI_TRY
    if (!ctx || !count || order_threads < 1 || (n > 0 && !order))
        return IG_ERR_INPUT;
    if (ctx->coalesce && order_threads == 1) {
        if (ig::check_job(words, n, len) != IG_OK)
            return ig::set_error(ctx, IG_ERR_INPUT, "words must be non-null, n >= 0 and 1 <= len <= 16");
        ig::SolveRequest req;
        req.words = words;
        req.n = n;
        req.len = len;
        req.min_ed = min_ed;
        const auto C = ig::solve_combiner(ctx);
        {
            std::unique_lock<std::mutex> lk(C->mu);
            C->pending.push_back(&req);
            while (!req.ready) {
                if (!C->building) {  // the device is free: build what waits, up to a cap
                    C->building = true;
                    std::vector<ig::SolveRequest *> batch;
                    ig::take_coalesced(C->pending, batch);
                    lk.unlock();
                    ig::build_requests_or_split(ctx, batch);
                    lk.lock();
                    for (ig::SolveRequest *r : batch)
                        r->ready = true;
                    C->building = false;
                    C->batches++;
                    C->requests += (int64_t)batch.size();
                    C->cv.notify_all();
                } else {
                    C->cv.wait(lk);
                }
            }
        }
        if (req.status != IG_OK)
            return req.status;
        if (edges)
            *edges = req.edges;
        *count = ig::greedy_one(*req.hg, req.job, order);
        return IG_OK;
    }
    // one caller at a time from its build until its device graph is freed;
    // the greedy runs after that, so concurrent callers hold host copies
    // only, within the context's host budget
    ig::HostGraph hg;
    {
        std::lock_guard<std::mutex> slot(ctx->solve_slot);
        ig_graph *g = nullptr;
        ig_status s = ig_graph_build(ctx, words, n, len, min_ed, 0, &g);
        if (s != IG_OK)
            return s;
        if (edges)
            *edges = g->edges;
        s = ig::download_for_greedy(g, order_threads, hg);
        ig::release_graph(g);
        if (s != IG_OK)
            return s;
    }
    *count = ig::greedy_one(hg, 0, order);
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_count_conflicts(ig_ctx *ctx, const uint32_t *words, int32_t n, int len, int min_ed, int64_t *edges)
{
    IG_ABI_TRY
    if (!ctx || !edges)
        return IG_ERR_INPUT;
    if (ig::check_job(words, n, len) != IG_OK)
        return ig::set_error(ctx, IG_ERR_INPUT, "words must be non-null, n >= 0 and 1 <= len <= 16");
    std::lock_guard<std::mutex> lk(ctx->mu);
    ig::DeviceGuard dg(ctx->device);
    const uint32_t *d_words = nullptr;
    ig_status s = ig::stage_words(ctx, words, n, 0, &d_words);
    if (s != IG_OK)
        return s;
    return ig::count_batch(ctx, d_words, {ig::JobSpec{0, n, len, min_ed}}, edges);
    IG_ABI_CATCH
}

int ig_lane_form(int len, int min_ed)
{
    if (len < 1 || len > IG_MAX_LEN)
        return -1;
    return ig::lane_form(len, min_ed);
}

ig_status ig_ctx_autotune(ig_ctx *ctx, const uint32_t *words, int32_t n, int len, int min_ed, int words_on_device,
                          int32_t *items_per_cta)
{
    IG_ABI_TRY
    if (!ctx)
        return IG_ERR_INPUT;
    if (ig::check_job(words, n, len) != IG_OK || n < 2 || min_ed < 1)
        return ig::set_error(ctx, IG_ERR_INPUT, "autotune needs n >= 2 words of 1 <= len <= 16 and min_ed >= 1");
    std::lock_guard<std::mutex> lk(ctx->mu);
    ig::DeviceGuard dg(ctx->device);
    if (!dg.ok)
        return ig::set_error(ctx, IG_ERR_CUDA, "cannot select the context's device");
    const uint32_t *d_words = nullptr;
    ig_status s = ig::stage_words(ctx, words, n, words_on_device, &d_words);
    int chosen = 0;
    if (s == IG_OK)
        s = ig::autotune(ctx, d_words, {ig::JobSpec{0, n, len, min_ed}}, &chosen);
    if (s == IG_OK && items_per_cta)
        *items_per_cta = chosen;
    return s;
    IG_ABI_CATCH
}

ig_status ig_ctx_set_work_split(ig_ctx *ctx, int lane_form, int32_t items_per_cta)
{
    IG_ABI_TRY
    if (!ctx || lane_form < 0 || lane_form > 2 || items_per_cta < 1 || items_per_cta > 4096)
        return IG_ERR_INPUT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->items_per_cta[lane_form] = items_per_cta;
    ctx->tuned[lane_form] = true;
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_ctx_work_split(ig_ctx *ctx, int lane_form, int32_t *items_per_cta, int *tuned)
{
    IG_ABI_TRY
    if (!ctx || lane_form < 0 || lane_form > 2)
        return IG_ERR_INPUT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (items_per_cta)
        *items_per_cta = ctx->items_per_cta[lane_form];
    if (tuned)
        *tuned = ctx->tuned[lane_form] ? 1 : 0;
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_ctx_set_graphs(ig_ctx *ctx, int enable)
{
    IG_ABI_TRY
    if (!ctx)
        return IG_ERR_INPUT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->use_graphs = enable != 0;
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_ctx_graph_stats(const ig_ctx *ctx, int64_t *launches, int64_t *instantiations, int64_t *updates)
{
    IG_ABI_TRY
    if (!ctx)
        return IG_ERR_INPUT;
    if (launches)
        *launches = ctx->graph_launches;
    if (instantiations)
        *instantiations = ctx->graph_instantiations;
    if (updates)
        *updates = ctx->graph_updates;
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_ctx_set_host_lists(ig_ctx *ctx, int form)
{
    IG_ABI_TRY
    if (!ctx || (form != IG_LISTS_AUTO && form != IG_LISTS_PLAIN && form != IG_LISTS_PACKED))
        return IG_ERR_INPUT;
    ctx->host_lists = form;
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_ctx_alloc_stats(ig_ctx *ctx, int64_t *device_allocs)
{
    IG_ABI_TRY
    if (!ctx || !device_allocs)
        return IG_ERR_INPUT;
    *device_allocs = ctx->device_allocs.load();
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_ctx_set_host_budget(ig_ctx *ctx, int64_t bytes)
{
    IG_ABI_TRY
    if (!ctx || bytes < 0)
        return IG_ERR_INPUT;
    ctx->host_budget->set_limit(bytes == 0 ? ig::default_host_budget() : bytes);
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_ctx_host_budget(ig_ctx *ctx, int64_t *limit, int64_t *used)
{
    IG_ABI_TRY
    if (!ctx)
        return IG_ERR_INPUT;
    if (limit)
        *limit = ctx->host_budget->limit();
    if (used)
        *used = ctx->host_budget->used();
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_ctx_set_wait_limit(ig_ctx *ctx, int64_t cycles)
{
    IG_ABI_TRY
    if (!ctx || cycles < 0)
        return IG_ERR_INPUT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->wait_cycles = cycles == 0 ? ig::kDefaultWaitCycles : (long long)cycles;
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_ctx_inject_fault(ig_ctx *ctx, int kind, int64_t arg)
{
    IG_ABI_TRY
    if (!ctx)
        return IG_ERR_INPUT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    switch (kind) {
    case IG_FAULT_NONE:
        ctx->fail_alloc_in.store(0);
        ctx->fault_tile_copy = false;
        return IG_OK;
    case IG_FAULT_DEVICE_ALLOC:
        if (arg < 1)
            return IG_ERR_INPUT;
        ctx->fail_alloc_in.store(arg);
        return IG_OK;
    case IG_FAULT_TILE_COPY:
        ctx->fault_tile_copy = true;
        return IG_OK;
    default:
        return IG_ERR_INPUT;
    }
    IG_ABI_CATCH
}

ig_status ig_ctx_set_coalescing(ig_ctx *ctx, int enable)
{
    IG_ABI_TRY
    if (!ctx)
        return IG_ERR_INPUT;
    ctx->coalesce = enable != 0;
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_ctx_coalesce_stats(ig_ctx *ctx, int64_t *batches, int64_t *requests)
{
    IG_ABI_TRY
    if (!ctx)
        return IG_ERR_INPUT;
    const auto C = ig::solve_combiner(ctx);
    std::lock_guard<std::mutex> lk(C->mu);
    if (batches)
        *batches = C->batches;
    if (requests)
        *requests = C->requests;
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_ctx_set_autotune(ig_ctx *ctx, int enable)
{
    IG_ABI_TRY
    if (!ctx)
        return IG_ERR_INPUT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->autotune = enable != 0;
    return IG_OK;
    IG_ABI_CATCH
}

}  // extern "C"
