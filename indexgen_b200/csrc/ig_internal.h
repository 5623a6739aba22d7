// Internal declarations shared by the libindexgen_cuda translation units.
#pragma once

#include <atomic>
#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <queue>
#include <condition_variable>
#include <thread>
#include <string>
#include <vector>

#include <new>

#include <cuda_runtime.h>

#include "indexgen_cuda.h"

// Every ig_status entry point runs its body between IG_ABI_TRY and
// IG_ABI_CATCH, so no C++ exception crosses the C ABI: an allocation failure
// in host code becomes IG_ERR_OOM, anything else IG_ERR_STATE.
#define IG_ABI_TRY try {
#define IG_ABI_CATCH                        \
    }                                       \
    catch (const std::bad_alloc &)          \
    {                                       \
        return IG_ERR_OOM;                  \
    }                                       \
    catch (...)                             \
    {                                       \
        return IG_ERR_STATE;                \
    }

namespace ig {

// Rows of one band = threads of one pair-test CTA; columns of one staged tile.
constexpr int kBandRows = 256;
constexpr int kTileCols = 256;

// One emitted edge, 8 bytes: the index of its (row, segment) count cell, and
// pos = (column offset within the segment) << 16 | rank of the column among
// the row's hits in that cell.  The cell gives the job, row and segment
// (cell = count_off + segment * n + row), so the row and the global column
// are recovered in the scatter; ranks make it order-exact without a sort.
// Segments are at most 2^16 columns wide, so offset and rank fit 16 bits each.
struct EdgeRecord {
    uint32_t cell, pos;
};
constexpr int kMaxSegShift = 16;
constexpr long long kDefaultWaitCycles = 4000000000ll;
// Largest job: its count cells (at most 256 segments x n) must be indexable
// by 32 bits.
constexpr int32_t kMaxJobWords = (1 << 24) - 1;

// One job of a batch as the device sees it.  Rows and columns of a job are
// local (0..n-1); word_off maps them to the concatenated word array.
struct JobDesc {
    int64_t word_off;    // first word of the job (global row/column base)
    int64_t unit_off;    // first uint4 of the job's column-unit stream
    int64_t unit_start;  // first unit (prefix over jobs, in units)
    int64_t item_off;    // first (band, segment) work item (prefix over jobs)
    int64_t count_off;   // first per-(segment, row) count ([nseg][n] block)
    int32_t n, L, lim;   // words, length, min_ed - L
    int32_t seg_shift, nseg, bands_per_seg, nbands;
    int32_t mode, w;     // lane form (full Myers / banded nibble / banded byte), band half-width
    uint32_t vp0, bm, cmask, kthr;  // banded-mode constants
};

// Host description of a job.
struct JobSpec {
    int64_t word_off = 0;
    int32_t n = 0;
    int32_t len = 1;
    int32_t min_ed = 0;
};

// Grow-only device buffer owned by a context.
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
};

// Page-locked host blocks for graph downloads, recycled across calls: a
// pageable download of a few hundred MB runs at a few GB/s and first touches
// fresh pages, a pinned one at tens of GB/s.  Blocks come in power-of-two
// sizes up to 1 GiB and whole GiB above; the pool holds at most kCap bytes,
// unpins cached blocks that no download holds to make room for a new size,
// and callers fall back to pageable memory beyond that (ig_api.cu).
class PinnedPool : public std::enable_shared_from_this<PinnedPool> {
public:
    static constexpr size_t kCap = (size_t)32 << 30;
    // A block of at least `bytes`, returned to the pool when the last copy of
    // the pointer goes; nullptr when the pool is full or pinning fails.
    std::shared_ptr<void> acquire(size_t bytes);
    ~PinnedPool();

private:
    std::mutex mu_;
    std::multimap<size_t, void *> free_;
    size_t total_ = 0;
};

// Host memory held by graphs downloaded for the greedy (canonical adjacency
// or upper CSR), from the download until the last greedy that reads them has
// finished.  A download waits until it fits the limit, so that concurrent
// callers, batch groups and served batches of dense graphs cannot take more
// host memory than the limit together; one request larger than the limit
// waits until nothing else is held and then goes ahead alone (ig_api.cu).
class HostBudget : public std::enable_shared_from_this<HostBudget> {
  public:
    explicit HostBudget(int64_t limit) : limit_(limit) {}
    // Blocks until `bytes` fit; the token releases them when its last copy goes.
    std::shared_ptr<void> acquire(int64_t bytes);
    void set_limit(int64_t limit);
    int64_t limit();
    int64_t used();

  private:
    std::mutex mu_;
    std::condition_variable cv_;
    int64_t limit_ = 0, used_ = 0;
};
// Default limit: half of the machine's physical memory.
int64_t default_host_budget();

struct Ctx {
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    std::mutex mu;
    std::mutex err_mu;  // guards last_error (set_error runs with or without mu held)
    std::string last_error;
    int64_t launches = 0;
    // workspace
    DevBuf words, sel, counts, records, scan_tmp, flags, adj_tmp, jobs, aux, cols_ws;
    int pair_grid = 0;                    // persistent CTAs of the pair kernel
    int pair_grid_nib = 0;                // ... of the nibble-lane pair kernel
    // work split per lane form (full Myers, nibble, byte lanes): target items
    // per CTA, chosen by the autotuner (ig_ctx_autotune) or left at 24
    int items_per_cta[3] = {24, 24, 24};
    bool tuned[3] = {false, false, false};
    bool autotune = true;  // tune a lane form on its first batch worth tuning
    int64_t tune_runs = 0; // tuner runs that chose among several plans
    // optional per-phase timing (IG_PHASE_*)
    bool profiling = false;
    static constexpr int kPhases = 6;
    cudaEvent_t ev[2 * kPhases] = {};
    double phase_ms[kPhases] = {};
    int64_t phase_launches[kPhases] = {};
    bool phase_pending[kPhases] = {};
    std::shared_ptr<PinnedPool> pinned = std::make_shared<PinnedPool>();
    // CUDA graphs of the batch pipeline: [0] a build pass (job table upload,
    // selector streams, pair kernels, row offsets, scan, scatter into CSR,
    // job bounds, readback), [1] a count-only pass.  A pass whose arguments
    // equal the cached graph's relaunches it; otherwise it is captured and
    // applied to the cached executable graph with cudaGraphExecUpdate (a new
    // instantiation only when the topology changed).
    bool use_graphs = true;
    cudaGraphExec_t graph_exec[2] = {};
    std::vector<uint64_t> graph_sig[2];  // arguments baked into each cached graph
    int64_t graph_launches = 0, graph_instantiations = 0, graph_updates = 0;
    // second stream for device-to-host copies that overlap the next build
    cudaStream_t dl_stream = nullptr;
    // host threads for batch greedies, shared by the calls on this context
    std::mutex greedy_mu;
    std::shared_ptr<class GreedyPool> greedy_pool;
    // concurrent ig_solve calls built together (ig_api.cu)
    std::atomic<bool> coalesce{true};
    // uncoalesced ig_solve calls hold this from their build until their device
    // graph is freed: callers waiting for host room never hold device graphs
    std::mutex solve_slot;
    // form of the neighbour lists sent to the host greedy (IG_LISTS_*)
    std::atomic<int> host_lists{IG_LISTS_AUTO};
    std::shared_ptr<struct SolveCombiner> combiner;
    // page-locked staging of the graphs' host copies
    void *stage = nullptr;
    size_t stage_bytes = 0;
    // bound on every mbarrier wait of the pair kernels (SM clock cycles,
    // about 2 s at 1.965 GHz unless ig_ctx_set_wait_limit lowers it)
    long long wait_cycles = kDefaultWaitCycles;
    // fault injection for failure-path tests (ig_ctx_inject_fault): the
    // number of device allocations left before one fails (0 = off), and a
    // pair pass that withholds the copy of one staged tile (both one-shot)
    std::atomic<int64_t> fail_alloc_in{0};
    std::atomic<int64_t> device_allocs{0};  // dev_malloc calls on this context
    bool fault_tile_copy = false;
    std::shared_ptr<HostBudget> host_budget = std::make_shared<HostBudget>(default_host_budget());
};

// Edge records that fit the context's record buffer.  Derived from the
// buffer itself, so that a failed (re)allocation, which leaves the buffer
// empty, can never leave a stale capacity behind.
inline unsigned long long rec_capacity(const Ctx *ctx) { return ctx->records.bytes / sizeof(EdgeRecord); }

// Records an event pair around a phase when profiling is on.
void phase_begin(Ctx *ctx, int phase);
void phase_end(Ctx *ctx, int phase);
void phase_collect(Ctx *ctx);  // after a stream sync: fold finished pairs in

struct Graph {
    Ctx *ctx = nullptr;
    int32_t n = 0;                      // rows over all jobs
    int64_t edges = 0;
    std::vector<JobSpec> jobs;          // one entry for a single-job graph
    std::vector<int64_t> job_edge_off;  // [jobs+1] row_ptr at job boundaries
    std::vector<int32_t> job_seg_shift, job_nseg;  // pair-pass tiling per job (0 when not built here)
    int64_t *d_row_ptr = nullptr;       // [n+1]
    int32_t *d_cols = nullptr;          // [edges], global column ids
    // host copies, filled on first use
    std::vector<int64_t> h_row_ptr;
    std::vector<int32_t> h_cols;
    bool host_valid = false;
    // symmetric adjacency in canonical order (built on first request)
    int64_t *d_adj_ptr = nullptr;  // [n+1]
    int32_t *d_adj = nullptr;      // [2*edges]
    // that adjacency bit-packed per row for the host (built on first request)
    int64_t *d_pk_off = nullptr;   // [n+1] first word of each row
    uint32_t *d_pk = nullptr;      // [pk_words + 2]
    int64_t pk_words = 0;
};

// Geometry of the upper-triangle work decomposition for one job.
struct PairPlan {
    int32_t n = 0;
    int seg_shift = 0;     // segment width = 1 << seg_shift columns (multiple of kBandRows)
    int nseg = 0;          // segments covering [0, n)
    int bands_per_seg = 0; // segment width / kBandRows
    int nbands = 0;
    long long items = 0;   // (band, segment) work items in the upper triangle
};

// Plan for a job of n words that should yield about `target_items` items.
PairPlan make_plan(int32_t n, long long target_items);

// Device pipeline stages (ig_graph.cu).  Jobs index into d_words.
ig_status build_batch(Ctx *ctx, const uint32_t *d_words, const std::vector<JobSpec> &jobs, Graph *g);
ig_status count_batch(Ctx *ctx, const uint32_t *d_words, const std::vector<JobSpec> &jobs, int64_t *edges);
// Lane form of the pair kernel for (len, min_ed): kModeFull 0, kModeNib 1,
// kModeByte 2 (ig_graph.cu).
int lane_form(int len, int min_ed);
// Times the work-split candidates on `jobs` (one lane form) and keeps the
// fastest for that lane form (ig_graph.cu).
ig_status autotune(Ctx *ctx, const uint32_t *d_words, const std::vector<JobSpec> &jobs, int *chosen);
// With ctx->autotune set and a batch of two or more jobs, tunes every lane
// form of `jobs` not tuned yet on this context (on the jobs themselves, or on
// a 131,072-word sample of the largest when they hold more than 2^33 pair
// tests).  Caller holds ctx->mu.
ig_status autotune_jobs(Ctx *ctx, const uint32_t *d_words, const std::vector<JobSpec> &jobs);

// In-place inclusive scan of m int64 on the context stream (ig_graph.cu).
ig_status inclusive_scan_i64(Ctx *ctx, int64_t *x, int64_t m);
ig_status ensure_buffer(Ctx *ctx, DevBuf &b, size_t bytes, const char *what);
// Takes `bytes` into the device's stream-ordered pool (allocated and freed
// once; the pool keeps freed memory) so that later workspace and output
// allocations are served from it instead of new driver mappings (ig_api.cu).
bool reserve_pool(Ctx *ctx, size_t bytes);
// Symmetric CSR in the canonical neighbour order (ig_adjacency.cu).
ig_status build_adjacency(Ctx *ctx, Graph *g);
// That adjacency bit-packed per row -- gap width, first neighbour, gaps
// minus one in that width -- for the host greedy (ig_packrows.cu).
ig_status build_packed_rows(Ctx *ctx, Graph *g);
// Nearest-centre index of every word, device pointers, on the context stream
// (ig_assign.cu).
ig_status assign_centers(Ctx *ctx, const uint32_t *d_words, int64_t n, const uint32_t *d_centres, int32_t k, int len,
                         int32_t *d_out);
// progress_adj_list.txt (AdjList::ToFile format) from / to a graph (ig_progress.cu).
ig_status write_adj_list(Ctx *ctx, Graph *g, const char *path, int64_t *bytes);
ig_status read_adj_list(Ctx *ctx, const char *path, Graph *g);
// d_dst[i] = d_src[d_idx[i]], i < n, on the context stream (ig_assign.cu).
ig_status gather_words(Ctx *ctx, const uint32_t *d_src, const int32_t *d_idx, int64_t n, uint32_t *d_dst);

// Host greedy (ig_host.cpp).  Vertex ids in cols / adj are global; `base`
// is subtracted to get the job-local ids the greedy works with and returns.
int32_t greedy_from_upper(const int64_t *row_ptr, const int32_t *cols, int32_t n, int64_t base, int order_threads,
                          int32_t *order);
// Greedy directly over neighbour lists already in m-order.
int32_t greedy_from_adjacency(const int64_t *adj_ptr, const int32_t *adj, int32_t n, int64_t base,
                              int32_t *order);
// The same over bit-packed rows (ig_packrows.cu's format); adj_ptr gives the
// degrees.
int32_t greedy_from_packed(const int64_t *adj_ptr, const int64_t *pk_off, const uint32_t *pk, int32_t n, int64_t base,
                           int32_t *order);

// What the host greedy needs of a graph, downloaded once: the canonical
// adjacency (order_threads = 1) or the upper CSR (other orders), plus the jobs.
struct HostGraph {
    int order_threads = 1;
    const int64_t *ptr = nullptr;   // adjacency or row offsets, [n+1]
    const int32_t *idx = nullptr;   // neighbour / column ids (global), or
    const int64_t *pk_off = nullptr;  // ... the adjacency rows bit-packed
    const uint32_t *pk = nullptr;
    std::shared_ptr<void> storage;  // owns ptr and idx (pinned block or heap)
    std::vector<JobSpec> jobs;
    std::vector<int64_t> job_edge_off;
};
// Device -> host (ig_api.cu); the graph stays valid.
ig_status download_for_greedy(Graph *g, int order_threads, HostGraph &hg);
// The canonical adjacency (order_threads = 1) built on the device and copied
// on the context's download stream, followed by the host function then(arg)
// (run when the copy has landed; it must not call CUDA) and the event *done
// (null when the copy has already completed).  The caller waits on *done
// before it frees g (ig_api.cu).
ig_status fetch_adjacency_async(ig_graph *g, HostGraph &hg, cudaEvent_t *done, cudaHostFn_t then, void *arg);
// Greedy of every job on host threads, largest first; job j's selection goes
// to order + word_off_j - order_base.  False on allocation failure.
bool run_greedies(const HostGraph &hg, int host_threads, int64_t order_base, int32_t *order, int32_t *counts);
// Greedy of one job of a downloaded graph into out (job-local ids).
int32_t greedy_one(const HostGraph &hg, int job, int32_t *out);
// While one is alive on a thread, the greedies run there stay on that thread:
// the library's greedy pools (batches, the clustered solve, the server)
// already run one greedy per core, and a helper thread would only compete
// with them.
struct PooledGreedyScope {
    explicit PooledGreedyScope(bool on = true);
    ~PooledGreedyScope();
    PooledGreedyScope(const PooledGreedyScope &) = delete;
    PooledGreedyScope &operator=(const PooledGreedyScope &) = delete;

  private:
    bool on_;
};

// Builds the jobs (words [offsets[j], offsets[j+1]), host or device pointer)
// in up to eight groups and runs their greedies on host_threads threads as
// each group arrives; job j's selection goes to order + offsets[j], its size
// to counts[j], its edge count to edges[j] (optional).  Jobs must be valid
// (ig_api.cu).
ig_status solve_groups(ig_ctx *ctx, const uint32_t *words, int words_on_device, const int64_t *offsets, int32_t jobs,
                       const int32_t *lens, const int32_t *min_eds, int order_threads, int host_threads,
                       int32_t *order, int32_t *counts, int64_t *edges);

// Host threads that run job greedies as downloaded graphs arrive: tasks of
// all submitted graphs share one queue, largest (most edges) first, so the
// greedies of a batch group start while the device builds the next group and
// idle threads take jobs of any group (ig_api.cu).
class GreedyPool {
  public:
    // One caller's jobs: how many are unfinished, and whether one failed.
    struct Ticket {
        int left = 0;
        bool failed = false;
    };
    explicit GreedyPool(int threads);
    ~GreedyPool();  // callers have waited for their tickets
    // Queues every job of hg under `ticket`: job j's selection goes to
    // order + word_off_j - order_base, its size to counts[j].
    void submit(std::shared_ptr<const HostGraph> hg, int64_t order_base, int32_t *order, int32_t *counts,
                const std::shared_ptr<Ticket> &ticket);
    // Runs queued greedies on the calling thread too until every job of
    // `ticket` has finished; false if one of them failed to allocate.
    bool wait(const std::shared_ptr<Ticket> &ticket);

  private:
    struct Task {
        int64_t edges;
        int64_t seq;
        std::shared_ptr<const HostGraph> hg;
        int job;
        int32_t *out;
        int32_t *count;
        std::shared_ptr<Ticket> ticket;
        bool operator<(const Task &o) const { return edges != o.edges ? edges < o.edges : seq > o.seq; }
    };
    void work();
    void run_one(std::unique_lock<std::mutex> &lk);  // pops the top task; lk held on entry and exit
    std::mutex mu_;
    std::condition_variable cv_, done_;
    std::priority_queue<Task> q_;
    std::vector<std::thread> threads_;
    int64_t seq_ = 0;
    bool stop_ = false;
};

// The context's greedy pool (cores - 1 threads), started on first use.
std::shared_ptr<GreedyPool> shared_greedy_pool(Ctx *ctx);

// Makes a device current for the duration of a call and restores the
// caller's device afterwards.
struct DeviceGuard {
    int prev = -1;
    bool ok = false;
    explicit DeviceGuard(int dev)
    {
        if (cudaGetDevice(&prev) != cudaSuccess)
            prev = -1;
        ok = cudaSetDevice(dev) == cudaSuccess;
    }
    ~DeviceGuard()
    {
        if (prev >= 0)
            cudaSetDevice(prev);
    }
};

ig_status set_error(Ctx *ctx, ig_status s, const std::string &msg);

// Edge counts of jobs estimated from one batch build over a strided sample of
// at most kSampleWords words of each job: exact for jobs no larger than the
// sample, otherwise the sample's edges scaled by the pair ratio (the sample
// pairs are a uniform draw from the job's pairs).  Used where memory must be
// sized before a build, such as the server's admission (ig_api.cu).
constexpr int32_t kSampleWords = 4096;
struct SampleJob {
    const uint32_t *words = nullptr;  // host
    int32_t n = 0;
    int32_t len = 1, min_ed = 0;
};
ig_status estimate_edges(Ctx *ctx, const std::vector<SampleJob> &jobs, std::vector<long double> &edges);
// Frees the context's pair-pass workspaces (column streams, count cells, edge
// records, column workspace, adjacency scratch) when together they hold more
// than keep_bytes; the freed memory stays in the device pool for the next
// allocations, and the workspaces grow again on demand (ig_graph.cu).
void trim_workspaces(Ctx *ctx, size_t keep_bytes);
size_t workspace_bytes(const Ctx *ctx);
// Every device allocation of the library goes through here (stream-ordered),
// so that ig_ctx_inject_fault can make a chosen one fail as out of memory.
cudaError_t dev_malloc(Ctx *ctx, void **p, size_t bytes, cudaStream_t st);
ig_status cuda_error(Ctx *ctx, cudaError_t e, const char *what);

}  // namespace ig

// The opaque ABI handles are the internal objects.
struct ig_ctx : ig::Ctx {
};
struct ig_graph : ig::Graph {
};
