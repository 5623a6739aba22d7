// Serving loop: continuous batching of codebook jobs of mixed (n, L, d).
//
// The reference solves one job per process invocation (src/SparseMat.cpp:878)
// and, in the clustered mode, one python3 GPU process per cluster
// (src/SparseMat.cpp:805-814).  Here a long-lived server owns a context and
// two stages that overlap:
//   scheduler thread  takes the jobs that have arrived, in arrival order, as
//                     long as the batch stays within the HBM budget (footprint
//                     estimated per job) and the per-launch pair budget; builds
//                     all their graphs with one device pipeline (one persistent
//                     pair-test launch); queues the canonical adjacency's copy
//                     to the host on a second stream, behind which a host
//                     callback hands the jobs to the greedy pool; and
//                     immediately admits the jobs that arrived meanwhile, whose
//                     build overlaps that copy.
//   greedy pool       host threads run each job's greedy while the device works
//                     on the next batch; a job is done when its greedy is.
// A job's result does not depend on what it was batched with: its graph is a
// diagonal block of the batch graph and its greedy runs on that block alone.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <new>
#include <thread>
#include <unordered_map>

#include "ig_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

enum JobState { kQueued = 0, kOnDevice = 1, kGreedy = 2, kDone = 3, kCancelled = 4, kFailed = 5 };

struct ServerJob {
    int64_t ticket = 0;
    std::vector<uint32_t> words;
    int32_t n = 0, len = 1, min_ed = 0;
    bool estimated = false;   // est_edges and footprint are known
    bool solo = false;        // build alone (a merged build that held it failed)
    long double est_edges = 0;
    int64_t footprint = 0;
    long double pairs = 0;
    JobState state = kQueued;
    ig_status status = IG_OK;
    Clock::time_point t_submit, t_done;
    std::vector<int32_t> order;
    int32_t count = 0;
    int64_t edges = 0;
};

struct GreedyTask {
    std::shared_ptr<ig::HostGraph> hg;
    int job_in_batch = 0;
    std::shared_ptr<ServerJob> job;
};

// Device memory a job needs at its peak, from its (estimated) edge count:
// words, column units and count cells (at most 256 segments per row), CSR
// offsets and canonical adjacency offsets; then per edge 8 B of edge record
// and 4 B of column while it builds, and the columns plus 8 B of canonical
// adjacency (4 B each way) while its adjacency is built -- the record buffer
// doubles as the sort scratch of long adjacency rows.  The estimate gets a
// fifth more room, and the record-chunk tails of the launch a fixed allowance.
int64_t device_footprint(int32_t n, long double edges)
{
    const long double nseg = std::min<long double>(256, std::max<long double>(1, n / 256.0L));
    const long double e = edges * 1.2L + 65536;
    return (int64_t)(4.0L * n + 32.0L * n + 4.0L * n * nseg + 24.0L * ((long double)n + 1) + 20.0L * e);
}

// Device memory a built graph holds until it is freed: CSR offsets and
// columns, adjacency offsets and lists.
int64_t graph_bytes(const ig_graph *g)
{
    return 16 * ((int64_t)g->n + 1) + 12 * g->edges;
}

}  // namespace

struct ig_server {
    ig_ctx *ctx = nullptr;
    ig_server_opts opts{};
    std::mutex mu;
    std::condition_variable cv_queue, cv_done, cv_tasks;
    std::deque<std::shared_ptr<ServerJob>> queue;
    std::unordered_map<int64_t, std::shared_ptr<ServerJob>> jobs;
    std::deque<GreedyTask> tasks;
    int64_t next_ticket = 1;
    bool stopping = false;
    bool scheduler_done = false;
    std::thread scheduler;
    std::vector<std::thread> pool;
    // counters
    int64_t batches = 0, completed = 0, failed = 0, cancelled = 0, max_batch = 0;

    void schedule_loop();
    void greedy_loop();
    void trim();
};

// Host callback behind a batch's adjacency copy: the batch's jobs go to the
// greedy pool the moment their adjacency has landed (no CUDA calls here).
struct BatchDelivery {
    ig_server *sv;
    std::shared_ptr<ig::HostGraph> hg;
    std::vector<std::shared_ptr<ServerJob>> batch;
    static void CUDART_CB run(void *p)
    {
        std::unique_ptr<BatchDelivery> d(static_cast<BatchDelivery *>(p));
        std::lock_guard<std::mutex> lk(d->sv->mu);
        for (size_t b = 0; b < d->batch.size(); ++b) {
            d->batch[b]->state = kGreedy;
            d->sv->tasks.push_back(GreedyTask{d->hg, (int)b, d->batch[b]});
        }
        d->sv->cv_tasks.notify_all();
    }
};

void ig_server::schedule_loop()
{
    // the previous batch: its adjacency copy overlaps this batch's build, and
    // its device graph is freed once the copy is done
    ig_graph *pend_g = nullptr;
    cudaEvent_t pend_done = nullptr;
    auto finish_pending = [&]() {
        if (!pend_g)
            return;
        if (pend_done) {
            cudaEventSynchronize(pend_done);
            cudaEventDestroy(pend_done);
        }
        ig_graph_free(pend_g);
        pend_g = nullptr;
        pend_done = nullptr;
    };
    auto fail_job = [&](const std::shared_ptr<ServerJob> &j, ig_status s) {  // mu held
        j->state = kFailed;
        j->status = s;
        j->t_done = Clock::now();
        ++failed;
    };
    for (;;) {
        std::vector<std::shared_ptr<ServerJob>> batch;
        std::vector<std::shared_ptr<ServerJob>> fresh;  // not estimated yet
        bool settle = false;
        {
            std::unique_lock<std::mutex> lk(mu);
            if (queue.empty() && pend_g) {  // nothing to overlap with: settle the last batch
                lk.unlock();
                finish_pending();
                lk.lock();
            }
            cv_queue.wait(lk, [&] { return stopping || !queue.empty(); });
            if (stopping && queue.empty()) {
                lk.unlock();
                finish_pending();
                return;
            }
            for (auto &j : queue)
                if (!j->estimated && j->state == kQueued && fresh.size() < 512)
                    fresh.push_back(j);
        }
        // Admission needs each job's HBM footprint, which depends on its edge
        // count: one count pass over strided samples of the new jobs gives it
        // (exact for jobs of at most 4,096 words).
        if (!fresh.empty()) {
            std::vector<ig::SampleJob> smp;
            for (auto &j : fresh)
                smp.push_back(ig::SampleJob{j->words.data(), j->n, j->len, j->min_ed});
            std::vector<long double> est;
            const ig_status s = ig::estimate_edges(ctx, smp, est);
            std::lock_guard<std::mutex> lk(mu);
            for (size_t k = 0; k < fresh.size(); ++k) {
                auto &j = fresh[k];
                if (s != IG_OK) {
                    if (j->state == kQueued)
                        fail_job(j, s);
                    continue;
                }
                j->est_edges = est[k];
                j->footprint = device_footprint(j->n, est[k]);
                j->estimated = true;
                if (j->state == kQueued && j->footprint > opts.hbm_budget_bytes)
                    fail_job(j, IG_ERR_OOM);  // this job alone does not fit the HBM budget
            }
            cv_done.notify_all();
        }
        {
            std::unique_lock<std::mutex> lk(mu);
            const int64_t pend_mem = pend_g ? graph_bytes(pend_g) : 0;
            int64_t mem = 0;
            long double pairs = 0;
            while (!queue.empty()) {
                std::shared_ptr<ServerJob> j = queue.front();
                if (j->state != kQueued) {  // cancelled or failed while queued
                    queue.pop_front();
                    continue;
                }
                if (!j->estimated)
                    break;  // arrived during the estimate: next round
                const bool first = batch.empty();
                const bool fits = mem + j->footprint + pend_mem <= opts.hbm_budget_bytes;
                if (first && !fits && pend_mem > 0) {
                    settle = true;  // room comes back once the previous batch is freed
                    break;
                }
                if (!first && ((int)batch.size() >= opts.max_batch_jobs || !fits || j->solo ||
                               pairs + j->pairs > (long double)opts.max_batch_pairs))
                    break;
                queue.pop_front();
                j->state = kOnDevice;
                mem += j->footprint;
                pairs += j->pairs;
                batch.push_back(j);
                if (j->solo)
                    break;
            }
        }
        if (settle) {
            finish_pending();
            continue;
        }
        if (batch.empty())
            continue;
        // one device pipeline for the whole batch
        std::vector<uint32_t> words;
        std::vector<int64_t> off{0};
        std::vector<int32_t> lens, eds;
        long double want_records = 0;
        for (auto &j : batch) {
            words.insert(words.end(), j->words.begin(), j->words.end());
            off.push_back(off.back() + j->n);
            lens.push_back(j->len);
            eds.push_back(j->min_ed);
            want_records += j->est_edges;
        }
        // room for the estimated records up front (a short estimate costs a
        // rerun of the pass, never a wrong result)
        ig_status s = IG_OK;
        {
            const long double need = want_records * 1.2L + (1 << 20);
            int64_t cap = 0;
            {
                std::lock_guard<std::mutex> lk(ctx->mu);
                cap = (int64_t)ig::rec_capacity(ctx);
            }
            if ((long double)cap < need)
                s = ig_ctx_reserve(ctx, (int64_t)need);
        }
        ig_graph *g = nullptr;
        if (s == IG_OK)
            s = ig_batch_build(ctx, words.data(), off.data(), (int32_t)batch.size(), lens.data(), eds.data(), 0, &g);
        finish_pending();  // the previous batch's copy ran during this build
        if ((s == IG_ERR_OOM || s == IG_ERR_CAPACITY) && batch.size() > 1) {
            // the merged build failed where each job alone may not: they go
            // back to the head of the queue and are built one by one
            std::lock_guard<std::mutex> lk(mu);
            for (auto it = batch.rbegin(); it != batch.rend(); ++it) {
                (*it)->state = kQueued;
                (*it)->solo = true;
                queue.push_front(*it);
            }
            continue;
        }
        auto hg = std::make_shared<ig::HostGraph>();
        if (s == IG_OK && opts.order_threads == 1) {
            for (size_t b = 0; b < batch.size(); ++b)
                batch[b]->edges = g->job_edge_off[b + 1] - g->job_edge_off[b];
            auto *d = new BatchDelivery{this, hg, batch};
            cudaEvent_t done = nullptr;
            s = ig::fetch_adjacency_async(g, *hg, &done, BatchDelivery::run, d);
            if (s == IG_OK) {
                pend_g = g;
                pend_done = done;
                trim();
                std::lock_guard<std::mutex> lk(mu);
                ++batches;
                max_batch = std::max<int64_t>(max_batch, (int64_t)batch.size());
                continue;  // the callback hands the jobs to the greedy pool
            }
            delete d;
            ig_graph_free(g);
        } else if (s == IG_OK) {
            s = ig::download_for_greedy(g, opts.order_threads, *hg);
            ig_graph_free(g);
        }
        trim();
        std::unique_lock<std::mutex> lk(mu);
        ++batches;
        max_batch = std::max<int64_t>(max_batch, (int64_t)batch.size());
        if (s != IG_OK) {
            for (auto &j : batch)
                fail_job(j, s);
            cv_done.notify_all();
            continue;
        }
        for (size_t b = 0; b < batch.size(); ++b) {
            batch[b]->edges = hg->job_edge_off[b + 1] - hg->job_edge_off[b];
            batch[b]->state = kGreedy;
            tasks.push_back(GreedyTask{hg, (int)b, batch[b]});
        }
        cv_tasks.notify_all();
    }
}

// After a batch: the context's pair-pass workspaces (grown to the largest
// batch so far) go back to the device pool when they hold more than a quarter
// of the HBM budget, so that one dense job does not keep its record buffer
// for the rest of the stream.
void ig_server::trim()
{
    std::lock_guard<std::mutex> lk(ctx->mu);
    ig::DeviceGuard dg(ctx->device);
    ig::trim_workspaces(ctx, (size_t)(opts.hbm_budget_bytes / 4));
}

void ig_server::greedy_loop()
{
    for (;;) {
        GreedyTask t;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_tasks.wait(lk, [&] { return scheduler_done || !tasks.empty(); });
            if (tasks.empty())
                return;  // the scheduler has stopped and nothing is left
            t = std::move(tasks.front());
            tasks.pop_front();
        }
        ig_status s = IG_OK;
        int32_t c = 0;
        try {
            t.job->order.resize((size_t)std::max(t.job->n, 1));
            ig::PooledGreedyScope pooled;
            c = ig::greedy_one(*t.hg, t.job_in_batch, t.job->order.data());
        } catch (...) {
            s = IG_ERR_OOM;
        }
        t.hg.reset();
        std::unique_lock<std::mutex> lk(mu);
        t.job->count = c;
        t.job->order.resize((size_t)c);
        t.job->status = s;
        t.job->state = s == IG_OK ? kDone : kFailed;
        t.job->t_done = Clock::now();
        if (s == IG_OK)
            ++completed;
        else
            ++failed;
        cv_done.notify_all();
    }
}

extern "C" {

ig_status ig_server_create(ig_ctx *ctx, const ig_server_opts *opts, ig_server **out)
{
    IG_ABI_TRY
    if (!ctx || !out)
        return IG_ERR_INPUT;
    *out = nullptr;
    ig_server *sv = new (std::nothrow) ig_server();
    if (!sv)
        return IG_ERR_OOM;
    sv->ctx = ctx;
    ig_server_opts o{};
    if (opts)
        o = *opts;
    // greedy threads leave one core to the scheduler thread, which drives the
    // device: a build that waits for a core stalls every job behind it
    const int cores = (int)std::max(1u, std::thread::hardware_concurrency());
    if (o.host_threads <= 0)
        o.host_threads = cores;
    o.host_threads = std::max(1, std::min(o.host_threads, cores - 1));
    if (o.max_batch_jobs <= 0)
        o.max_batch_jobs = 256;
    if (o.max_batch_pairs <= 0)
        o.max_batch_pairs = 20000000000ll;  // ~0.1 s of device work per launch
    if (o.order_threads <= 0)
        o.order_threads = 1;
    if (o.hbm_budget_bytes <= 0) {
        size_t free_b = 0, total_b = 0;
        int prev = -1;
        cudaGetDevice(&prev);
        cudaSetDevice(ctx->device);
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess)
            free_b = (size_t)8 << 30;
        cudaGetLastError();
        if (prev >= 0)
            cudaSetDevice(prev);
        o.hbm_budget_bytes = (int64_t)(free_b / 10 * 8);
    }
    if (o.pool_reserve_bytes == 0)
        o.pool_reserve_bytes = std::min<int64_t>((int64_t)4 << 30, o.hbm_budget_bytes / 4);
    if (o.pool_reserve_bytes > 0)
        ig::reserve_pool(ctx, (size_t)o.pool_reserve_bytes);  // best effort
    sv->opts = o;
    try {
        sv->scheduler = std::thread([sv] { sv->schedule_loop(); });
        for (int i = 0; i < o.host_threads; ++i)
            sv->pool.emplace_back([sv] { sv->greedy_loop(); });
    } catch (...) {  // a thread could not start: stop the ones that did
        ig_server_destroy(sv);
        return IG_ERR_OOM;
    }
    *out = sv;
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_server_submit(ig_server *sv, const uint32_t *words, int32_t n, int len, int min_ed, int64_t *ticket)
{
    IG_ABI_TRY
    if (!sv || !ticket || n < 0 || len < 1 || len > IG_MAX_LEN || (n > 0 && !words))
        return IG_ERR_INPUT;
    auto j = std::make_shared<ServerJob>();
    try {
        j->words.assign(words, words + n);
    } catch (...) {
        return IG_ERR_OOM;
    }
    j->n = n;
    j->len = len;
    j->min_ed = min_ed;
    j->pairs = (long double)n * (n > 0 ? n - 1 : 0) / 2;
    j->t_submit = Clock::now();
    std::unique_lock<std::mutex> lk(sv->mu);
    if (sv->stopping)
        return IG_ERR_STATE;
    j->ticket = sv->next_ticket++;
    sv->jobs[j->ticket] = j;
    sv->queue.push_back(j);
    *ticket = j->ticket;
    sv->cv_queue.notify_one();
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_server_poll(ig_server *sv, int64_t ticket, int *state)
{
    IG_ABI_TRY
    if (!sv || !state)
        return IG_ERR_INPUT;
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->jobs.find(ticket);
    if (it == sv->jobs.end())
        return IG_ERR_INPUT;
    *state = (int)it->second->state;
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_server_wait(ig_server *sv, int64_t ticket, int32_t *order, int32_t *count, int64_t *edges,
                         double *latency_ms)
{
    IG_ABI_TRY
    if (!sv || !count)
        return IG_ERR_INPUT;
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->jobs.find(ticket);
    if (it == sv->jobs.end())
        return IG_ERR_INPUT;
    std::shared_ptr<ServerJob> j = it->second;
    sv->cv_done.wait(lk, [&] { return j->state >= kDone; });
    sv->jobs.erase(it);
    if (latency_ms)
        *latency_ms = std::chrono::duration<double, std::milli>(j->t_done - j->t_submit).count();
    if (j->state == kCancelled)
        return IG_ERR_CANCELLED;
    if (j->state == kFailed)
        return j->status;
    if (j->count > 0 && !order)
        return IG_ERR_INPUT;
    if (j->count > 0)
        std::copy(j->order.begin(), j->order.end(), order);
    *count = j->count;
    if (edges)
        *edges = j->edges;
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_server_cancel(ig_server *sv, int64_t ticket)
{
    IG_ABI_TRY
    if (!sv)
        return IG_ERR_INPUT;
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->jobs.find(ticket);
    if (it == sv->jobs.end())
        return IG_ERR_INPUT;
    if (it->second->state != kQueued)
        return IG_ERR_STATE;  // already on the device or finished
    it->second->state = kCancelled;
    it->second->t_done = Clock::now();
    ++sv->cancelled;
    sv->cv_done.notify_all();
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_server_stats(ig_server *sv, int64_t *batches, int64_t *completed, int64_t *max_batch_jobs)
{
    IG_ABI_TRY
    if (!sv)
        return IG_ERR_INPUT;
    std::unique_lock<std::mutex> lk(sv->mu);
    if (batches)
        *batches = sv->batches;
    if (completed)
        *completed = sv->completed;
    if (max_batch_jobs)
        *max_batch_jobs = sv->max_batch;
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_server_destroy(ig_server *sv)
{
    IG_ABI_TRY
    if (!sv)
        return IG_ERR_INPUT;
    {
        std::unique_lock<std::mutex> lk(sv->mu);
        sv->stopping = true;
        for (auto &j : sv->queue)
            if (j->state == kQueued) {
                j->state = kCancelled;
                j->t_done = Clock::now();
            }
        sv->queue.clear();
        sv->cv_queue.notify_all();
        sv->cv_tasks.notify_all();
        sv->cv_done.notify_all();
    }
    if (sv->scheduler.joinable())
        sv->scheduler.join();
    {
        std::unique_lock<std::mutex> lk(sv->mu);
        sv->scheduler_done = true;
        sv->cv_tasks.notify_all();
    }
    for (auto &t : sv->pool)
        t.join();
    delete sv;
    return IG_OK;
    IG_ABI_CATCH
}

}  // extern "C"
