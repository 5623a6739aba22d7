/* libindexgen_cuda -- B200 (sm_100a) conflict-graph + greedy codebook library.
 *
 * C ABI that replaces the reference's GPU boundary: the C++ host of IndexGen
 * calls these entry points where it shells out to
 *     python3 src/gpu_graph_generator.py <cands.txt> <edges.bin> <minED> <maxGB>
 * (src/SparseMat.cpp:454-534, FillAdjListGPU) and where it runs the
 * independent-set solve (src/SparseMat.cpp:679-851).  Plain pointers and sizes
 * only; no exceptions cross this boundary; every call returns an ig_status.
 *
 * Words: one uint32 per candidate of length len (1..16) over {0,1,2,3}
 * (A=0, C=1, G=2, T=3); character p is stored in bits 2p..2p+1.  Bits above
 * 2*len are ignored.
 *
 * Edge predicate: i<j is an edge iff Levenshtein(c_i, c_j) < min_ed, the
 * negation of EditDistanceBandedAtLeast(c_j, MakePattern(c_i), min_ed)
 * (include/EditDistance.hpp:368-372) used by FillAdjListTH
 * (src/SparseMat.cpp:536-565) and of `score < threshold` in
 * src/cuda_edit_distance.py:195.
 */
#ifndef INDEXGEN_CUDA_H
#define INDEXGEN_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IG_MAX_LEN 16

typedef enum ig_status {
    IG_OK = 0,
    IG_ERR_INPUT = 1,     /* bad argument: length, symbol, size, null pointer   */
    IG_ERR_CAPACITY = 2,  /* a caller buffer or a fixed limit is too small       */
    IG_ERR_OOM = 3,       /* device or host allocation failed / over budget     */
    IG_ERR_CUDA = 4,      /* a CUDA runtime call failed                         */
    IG_ERR_TIMEOUT = 5,   /* a bounded device wait gave up                      */
    IG_ERR_CANCELLED = 6, /* a queued job was cancelled                         */
    IG_ERR_STATE = 7      /* call made on an object in the wrong state          */
} ig_status;

typedef struct ig_ctx ig_ctx;     /* device, stream and reusable workspace       */
typedef struct ig_graph ig_graph; /* one conflict graph, CSR resident in HBM     */

/* ---- library / context ------------------------------------------------- */

const char *ig_version(void);
const char *ig_status_string(ig_status s);

/* Creates a context on `device`.  A context owns one CUDA stream and a
 * workspace that grows to the largest job seen; calls on one context are
 * serialised internally (safe to share between host threads). */
ig_status ig_ctx_create(ig_ctx **out, int device);
ig_status ig_ctx_destroy(ig_ctx *ctx);
/* Message of the last failure on this context (thread-unsafe snapshot). */
const char *ig_last_error(const ig_ctx *ctx);
/* The context's cudaStream_t, for callers that time or order device work. */
ig_status ig_ctx_stream(ig_ctx *ctx, void **stream);
/* Pre-size the edge workspace (optional; it otherwise grows on demand). */
ig_status ig_ctx_reserve(ig_ctx *ctx, int64_t edges);
/* Number of device kernels this context has launched so far. */
int64_t ig_ctx_launches(const ig_ctx *ctx);
/* Per-phase device timing with CUDA events on the context's stream (off by
 * default).  Phases: IG_PHASE_PAIRS (the pair-test kernel), IG_PHASE_COMPACT
 * (row prefix + scan + scatter into CSR), IG_PHASE_PREP (selector streams),
 * and the three parts of IG_PHASE_COMPACT: IG_PHASE_PREFIX (per-row prefix
 * of the segment counts), IG_PHASE_SCAN (row offsets), IG_PHASE_SCATTER
 * (records into columns).  ig_ctx_phase_time returns the accumulated
 * milliseconds and launch count since profiling was last enabled. */
#define IG_PHASE_PAIRS 0
#define IG_PHASE_COMPACT 1
#define IG_PHASE_PREP 2
#define IG_PHASE_PREFIX 3
#define IG_PHASE_SCAN 4
#define IG_PHASE_SCATTER 5
ig_status ig_ctx_set_profiling(ig_ctx *ctx, int enable);
ig_status ig_ctx_phase_time(const ig_ctx *ctx, int phase, double *ms, int64_t *launches);

/* ---- work split and its autotuner -------------------------------------- */
/* No counterpart in the reference, whose tiling is fixed: 16,384 x 16,384
 * pair tiles, one launch each with 16 x 16-thread blocks
 * (src/cuda_edit_distance.py:278, :335-338, :384-425).  The
 * pair kernels are persistent: each CTA claims (256-row band x segment) item
 * tiles of the pair triangle from a device counter.  The work split -- target
 * items per CTA of the grid -- sets how many items a batch is cut into and so
 * each job's segment width (256 .. 16,384 columns): wide tiles amortise the
 * per-item setup, narrow ones even out the end of the launch.  It is kept per
 * lane form of the pair kernel, which (len, min_ed) selects: */
#define IG_LANES_FULL 0   /* full Myers lanes (min_ed > 8)                   */
#define IG_LANES_NIBBLE 1 /* 8 banded nibble lanes per word (min_ed <= 4)    */
#define IG_LANES_BYTE 2   /* 4 banded byte lanes per word (5 <= min_ed <= 8) */
/* Lane form for (len, min_ed); -1 when len is out of range. */
int ig_lane_form(int len, int min_ed);
/* Times the count-only pair pass of a representative job (host or device
 * words, as ig_graph_build) for each candidate split whose plan differs
 * (6, 12, 24, 48, 96 items per CTA; CUDA events on the context's stream,
 * best of two after a warm-up) and keeps the fastest for the job's lane
 * form; *items_per_cta (optional) = the choice.  Results never depend on
 * the split.  With autotuning on (the default) a context tunes each lane
 * form by itself on the first batch build (two or more jobs) whose
 * candidates cut differently: on the batch's jobs of that form, or on a
 * 131,072-word sample of the largest of them when they hold more than 2^33
 * pair tests.  Single-job builds keep the current split (24 until tuned),
 * so a process that builds once pays no timing passes. */
ig_status ig_ctx_autotune(ig_ctx *ctx, const uint32_t *words, int32_t n, int len, int min_ed, int words_on_device,
                          int32_t *items_per_cta);
/* Pins a lane form's split (1..4096 items per CTA; the untuned default is
 * 24); the automatic tuner then leaves that form alone. */
ig_status ig_ctx_set_work_split(ig_ctx *ctx, int lane_form, int32_t items_per_cta);
/* The current split of a lane form and whether it was tuned or pinned. */
ig_status ig_ctx_work_split(ig_ctx *ctx, int lane_form, int32_t *items_per_cta, int *tuned);
/* Automatic tuning on (1, default) or off (0). */
ig_status ig_ctx_set_autotune(ig_ctx *ctx, int enable);
/* Host memory that graphs downloaded for the greedy may hold at once on this
 * context (0 restores the default, half of physical memory): a download
 * waits until the graphs whose greedies are still running leave room, so
 * concurrent callers, batch groups and served batches of dense graphs stay
 * within it together (one graph larger than the limit goes ahead alone once
 * nothing else is held).  ig_ctx_host_budget reports the limit and the bytes
 * held now. */
ig_status ig_ctx_set_host_budget(ig_ctx *ctx, int64_t bytes);
ig_status ig_ctx_host_budget(ig_ctx *ctx, int64_t *limit, int64_t *used);
/* Bound on every device-side wait of the pair kernels, in SM clock cycles
 * (0 restores the default, about 2 s at 1.965 GHz).  A wait that runs out ends
 * the build with IG_ERR_TIMEOUT after the CTA's copies in flight have landed;
 * the context stays usable.  Replaces the reference's unbounded waits on its
 * python3 subprocess (src/SparseMat.cpp:500-513). */
ig_status ig_ctx_set_wait_limit(ig_ctx *ctx, int64_t cycles);
/* Fault injection for tests of the failure paths; nothing here faults the
 * GPU, each kind fires once:
 *   IG_FAULT_NONE          clears any pending injection;
 *   IG_FAULT_DEVICE_ALLOC  the arg-th device allocation this context makes
 *                          from now on (arg >= 1) fails as out of memory;
 *   IG_FAULT_TILE_COPY     the next pair pass does not issue the copy of the
 *                          first staged tile of each pair kernel's first work
 *                          item, so that tile's bounded wait runs out. */
/* Form of the neighbour lists a graph is sent in to the host greedy:
 *   IG_LISTS_AUTO    packed when the plain lists would take 512 MB or more
 *                    (the default);
 *   IG_LISTS_PLAIN   offsets and 4-byte neighbour ids;
 *   IG_LISTS_PACKED  each row bit-packed on the device (gap width, first
 *                    neighbour, gaps in that width): 2-3x less PCIe traffic
 *                    and host memory per graph, about 1 ns more greedy time
 *                    per neighbour.
 * The codebooks do not depend on it. */
#define IG_LISTS_AUTO 0
#define IG_LISTS_PLAIN 1
#define IG_LISTS_PACKED 2
ig_status ig_ctx_set_host_lists(ig_ctx *ctx, int form);
/* Device allocations this context has asked for so far (workspaces grow
 * rarely and are reused, so a steady stream of builds adds only the graphs'
 * own arrays); with IG_FAULT_DEVICE_ALLOC it tells a test which one to fail. */
ig_status ig_ctx_alloc_stats(ig_ctx *ctx, int64_t *device_allocs);
#define IG_FAULT_NONE 0
#define IG_FAULT_DEVICE_ALLOC 1
#define IG_FAULT_TILE_COPY 2
ig_status ig_ctx_inject_fault(ig_ctx *ctx, int kind, int64_t arg);
/* Concurrent ig_solve calls built together (1, default) or one by one (0),
 * and how many batches and calls have gone through the combiner. */
ig_status ig_ctx_set_coalescing(ig_ctx *ctx, int enable);
ig_status ig_ctx_coalesce_stats(ig_ctx *ctx, int64_t *batches, int64_t *requests);

/* ---- CUDA graphs of the batch pipeline ---------------------------------- */
/* Each build (single job or batch) is one CUDA graph launch on the
 * context's stream -- job table upload, selector streams, the persistent pair
 * kernel(s), then the compaction into CSR (row offsets, scan, scatter, job
 * bounds) and the status readback -- with one host wait at the end.  A build
 * whose arguments equal the cached graph's relaunches it; otherwise the calls
 * are captured and applied to the cached executable graph with
 * cudaGraphExecUpdate, so a batch of a known shape costs no instantiation.
 * On by default; per-phase timing (ig_ctx_set_profiling) runs the same calls
 * without graphs.  Results never depend on it. */
ig_status ig_ctx_set_graphs(ig_ctx *ctx, int enable);
/* Graph launches, instantiations and in-place updates on this context. */
ig_status ig_ctx_graph_stats(const ig_ctx *ctx, int64_t *launches, int64_t *instantiations, int64_t *updates);

/* ---- host-side input preparation (no device work) ---------------------- */

/* '0'..'3' text rows, `stride` bytes apart, to packed words.  Replaces the
 * text load + pack of src/gpu_graph_generator.py:11-15 and
 * src/cuda_edit_distance.py:246-255.  On a bad symbol returns IG_ERR_INPUT and
 * stores the failing row in *bad_row (if non-null). */
ig_status ig_pack(const char *text, int64_t n, int len, int64_t stride, uint32_t *out, int64_t *bad_row);

/* Homopolymer-run and GC-content filters of CandidateGenerator::applyFilters
 * (src/CandidateGenerator.cpp:24-50; MaxRun / TestGCCont, src/Utils.cpp:420-462,
 * same double comparisons).  keep[i] = 1 when word i passes. */
ig_status ig_filter(const uint32_t *words, int64_t n, int len, int max_run, double min_gc, double max_gc,
                    uint8_t *keep);

/* ---- conflict graph (FillAdjListGPU, src/SparseMat.cpp:454-534) -------- */

/* Builds the graph of all pairs i<j with ED < min_ed.  `words` is a host
 * pointer, or a device pointer when words_on_device != 0 (it must then be
 * ready on the context's stream).  The result stays in HBM as an upper CSR
 * with ascending columns.  Blocks until the graph is complete. */
ig_status ig_graph_build(ig_ctx *ctx, const uint32_t *words, int32_t n, int len, int min_ed, int words_on_device,
                         ig_graph **out);
ig_status ig_graph_free(ig_graph *g);
/* n and the number of edges (u<v); matrixOnesNum of the reference = 2*edges. */
ig_status ig_graph_stats(const ig_graph *g, int32_t *n, int64_t *edges);
/* Upper CSR to host buffers: row_ptr[n+1], cols[edges] (ascending per row). */
ig_status ig_graph_upper_csr(const ig_graph *g, int64_t *row_ptr, int32_t *cols);
/* Edges as int32 (u, v) pairs, u<v, rows ascending, columns ascending: the
 * binary edge-file layout that AdjList::FromBinaryFile reads
 * (src/gpu_graph_generator.py:49-77, src/SparseMat.cpp:338-390). */
ig_status ig_graph_pairs(const ig_graph *g, int32_t *pairs);
/* Device pointers of the resident upper CSR (valid until ig_graph_free). */
ig_status ig_graph_device_csr(const ig_graph *g, const int64_t **row_ptr, const int32_t **cols);
/* Symmetric adjacency in the canonical neighbour order m[x] = lower neighbours
 * ascending, then upper neighbours ascending -- the lists AdjList holds after
 * FromBinaryFile on the pair file (src/SparseMat.cpp:338-390) or after
 * FillAdjList with one thread (src/SparseMat.cpp:599-609).  Built on the device
 * on first request.  adj_ptr[n+1], adj[2*edges] host buffers. */
ig_status ig_graph_adjacency(ig_graph *g, int64_t *adj_ptr, int32_t *adj);
/* Device pointers of that adjacency (built on first request). */
ig_status ig_graph_device_adjacency(ig_graph *g, const int64_t **adj_ptr, const int32_t **adj);
/* Greedy minimum-degree independent set over a single-job graph, reproducing AdjList's
 * selection order (src/SparseMat.cpp:81-266, :679-731) for neighbour lists
 * assembled as FillAdjList(order_threads) does (src/SparseMat.cpp:599-609);
 * order_threads = 1 is the sorted order the GPU-path loader builds.
 * order[] receives up to n vertex ids in selection order; *count their number. */
ig_status ig_graph_codebook(ig_graph *g, int order_threads, int32_t *order, int32_t *count);

/* ---- batches of independent jobs --------------------------------------- */
/* The clustered solve runs SolveIndependentSet once per cluster from a pool of
 * host threads (src/SparseMat.cpp:927-1095, :784-851), one python3 process
 * per cluster on the GPU path.  Here a whole batch of jobs is one device
 * pipeline with ONE persistent pair-test launch; job j is words
 * [offsets[j], offsets[j+1]) of length lens[j] with threshold min_eds[j].
 * The result is one graph whose CSR is block diagonal over the jobs (global
 * word ids); jobs never share an edge. */
ig_status ig_batch_build(ig_ctx *ctx, const uint32_t *words, const int64_t *offsets, int32_t jobs,
                         const int32_t *lens, const int32_t *min_eds, int words_on_device, ig_graph **out);
ig_status ig_graph_job_count(const ig_graph *g, int32_t *jobs);
ig_status ig_graph_job_stats(const ig_graph *g, int32_t job, int64_t *first_word, int32_t *n, int64_t *edges);
/* Tiling the pair pass used for job j: column segments of segment_width
 * columns (a power of two, at most 65,536) and their number; each (row,
 * segment) pair had one count cell.  Zero for jobs without pair tests and for
 * graphs read from a file.  The replacement of the reference's fixed
 * 16384 x 16384 tiles (src/cuda_edit_distance.py:380-390). */
ig_status ig_graph_job_tiling(const ig_graph *g, int32_t job, int32_t *segment_width, int32_t *segments);
/* Greedy of every job on host_threads host threads (0 = all cores), largest
 * job first.  Job j's codebook, as job-local vertex ids in selection order,
 * is written to order + offsets[j]; counts[j] is its size.  order_threads as
 * in ig_graph_codebook. */
ig_status ig_graph_job_codebooks(ig_graph *g, int order_threads, int host_threads, int32_t *order, int32_t *counts);
/* Build + job codebooks in one call; edges[j] (optional) = edges of job j.
 * The jobs are built in up to eight groups (at least 2^30 pair tests each);
 * each group's greedies start on the host as soon as its adjacency has been
 * copied, while the device builds the next group.  Greedy threads: at most
 * host_threads (0 = all cores), and always one fewer than the cores, so the
 * thread that drives the device is never starved. */
ig_status ig_solve_batch(ig_ctx *ctx, const uint32_t *words, const int64_t *offsets, int32_t jobs,
                         const int32_t *lens, const int32_t *min_eds, int order_threads, int host_threads,
                         int32_t *order, int32_t *counts, int64_t *edges);

/* ---- serving: continuous batching of codebook jobs --------------------- */
/* A server owns a scheduler thread and a pool of greedy threads on top of a
 * context.  Jobs of any (n, len, min_ed) are submitted from any thread; the
 * scheduler admits the jobs that have arrived, in arrival order, while the
 * batch stays within hbm_budget_bytes (estimated footprint) and
 * max_batch_pairs, builds them with one device pipeline, and admits the next
 * arrivals while the greedy threads finish the previous batch.  A job's
 * codebook is the same as ig_solve's for it alone.  There is no counterpart
 * in the reference, which solves one job per program run. */
typedef struct ig_server ig_server;
typedef struct ig_server_opts {
    int host_threads;          /* greedy threads (0 = all cores; at most cores - 1,
                                * leaving one to the scheduler)                  */
    int max_batch_jobs;        /* jobs per launch (0 = 256)                       */
    int order_threads;         /* neighbour order (0 or 1 = canonical sorted)     */
    int reserved;
    int64_t max_batch_pairs;   /* pair tests per launch (0 = 2e10, ~0.1 s)        */
    int64_t hbm_budget_bytes;  /* estimated HBM per launch (0 = half the free HBM) */
    int64_t pool_reserve_bytes; /* device memory taken into the context's stream-
                                 * ordered pool at start, so that the first large
                                 * jobs do not wait on the driver to map memory
                                 * (0 = min(4 GiB, budget / 4); < 0 = none)      */
} ig_server_opts;
/* Job states reported by ig_server_poll. */
#define IG_JOB_QUEUED 0
#define IG_JOB_ON_DEVICE 1
#define IG_JOB_GREEDY 2
#define IG_JOB_DONE 3
#define IG_JOB_CANCELLED 4
#define IG_JOB_FAILED 5
ig_status ig_server_create(ig_ctx *ctx, const ig_server_opts *opts, ig_server **out);
/* Copies the words; returns at once with a ticket. */
ig_status ig_server_submit(ig_server *sv, const uint32_t *words, int32_t n, int len, int min_ed, int64_t *ticket);
ig_status ig_server_poll(ig_server *sv, int64_t ticket, int *state);
/* Blocks until the job is done; writes its codebook (order[n] job-local ids in
 * selection order), size, edge count and submit-to-done latency, then forgets
 * the ticket.  IG_ERR_CANCELLED / the failure status otherwise. */
ig_status ig_server_wait(ig_server *sv, int64_t ticket, int32_t *order, int32_t *count, int64_t *edges,
                         double *latency_ms);
/* Cancels a job that is still queued (IG_ERR_STATE once it has started). */
ig_status ig_server_cancel(ig_server *sv, int64_t ticket);
ig_status ig_server_stats(ig_server *sv, int64_t *batches, int64_t *completed, int64_t *max_batch_jobs);
/* Cancels queued jobs, finishes the running batch, joins the threads. */
ig_status ig_server_destroy(ig_server *sv);

/* ---- checkpoint bridge --------------------------------------------------- */
/* Writes the graph as the reference's progress_adj_list.txt: AdjList::ToFile
 * (src/SparseMat.cpp:286-305, SaveProgressCodebook :658-663) of the AdjList
 * the GPU edge file loads into (FromBinaryFile, :338-390), i.e. "i\tj\n" for
 * every neighbour j of every row i, rows ascending, lower neighbours then
 * upper neighbours ascending.  The text is formatted on the device.  bytes
 * (optional) = file size. */
ig_status ig_graph_write_adj_list(ig_graph *g, const char *path, int64_t *bytes);
/* Reads such a file (also one written part-way through the greedy, with the
 * deleted rows gone) into a graph, as AdjList::FromFile (:306-336) does: n =
 * largest id + 1, each row's neighbours in file order, which the codebook
 * greedy then walks (ig_graph_codebook with order_threads = 1). */
ig_status ig_graph_read_adj_list(ig_ctx *ctx, const char *path, ig_graph **out);

/* ---- clustering: nearest-centre assignment ------------------------------ */
/* For each of the n words, the index of the nearest of the k centres
 * (Levenshtein distance, ties to the lowest index), written to
 * assignment[0..n).  Replaces solve_assignments_cuda (src/gpu_cluster.py:
 * 239-300: dense K x N uint8 distance matrix + host np.argmin), which
 * RandomCluster::fit runs through system()
 * (src/clustering/impl/random_cluster/RandomCluster.cpp:68-111).  words and
 * centres are packed like ig_graph_build's input, all of length len;
 * on_device = 1: words, centers and assignment are device pointers (cuda:
 * device of ctx), 0: host pointers.  k >= 1 when n > 0; n <= 2^31 - 1. */
ig_status ig_assign_centers(ig_ctx *ctx, const uint32_t *words, int64_t n, const uint32_t *centers, int32_t k,
                            int len, int on_device, int32_t *assignment);

/* Iterative clustered solve with random_cluster, the words resident on the
 * device (src/SparseMat.cpp:920-1095 with RandomCluster::fit,
 * src/clustering/impl/random_cluster/RandomCluster.cpp:42-136): repeat
 * {k random centres among the current candidates (k raised to
 * ceil(N / 200000) when N / k > 200000; k <= 0: one cluster), nearest-centre
 * clusters in candidate order, every cluster solved (greedy in the sorted
 * neighbour order), codebooks concatenated in cluster order} until the last
 * converge_iters codebook sizes agree (<= 1: after one iteration, < 0: never)
 * or max_iters iterations ran.  codebook[0..*count) receives ids into words
 * (room for n); sizes (optional, room for max_iters) the size after each
 * iteration.  Centres come from a seeded splitmix64 partial Fisher-Yates
 * shuffle (iteration t: seed ^ t * 0xD1B54A32D192ED03) where the reference
 * draws from std::random_device. */
ig_status ig_cluster_solve(ig_ctx *ctx, const uint32_t *words, int32_t n, int len, int min_ed, int32_t k,
                           int32_t converge_iters, uint64_t seed, int32_t max_iters, int host_threads,
                           int32_t *codebook, int32_t *count, int32_t *iterations, int64_t *sizes);

/* ---- one-call conveniences --------------------------------------------- */

/* SolveIndependentSet (src/SparseMat.cpp:784-851): graph + greedy.
 * edges may be null.  With order_threads = 1, calls made on one context from
 * several host threads at once (the reference's cluster worker pool,
 * src/SparseMat.cpp:978-1010) are built together: a call that finds the
 * device busy leaves its job waiting, and the next caller to get the device
 * builds every waiting job as one batch; each caller then runs its own
 * greedy.  A lone call is built at once.  Results are the same either way. */
ig_status ig_solve(ig_ctx *ctx, const uint32_t *words, int32_t n, int len, int min_ed, int order_threads,
                   int32_t *order, int32_t *count, int64_t *edges);
/* Number of conflicting pairs only (VerifyDist's GPU branch passes when it is
 * zero, src/Utils.cpp:203-288). */
ig_status ig_count_conflicts(ig_ctx *ctx, const uint32_t *words, int32_t n, int len, int min_ed, int64_t *edges);
/* Greedy over caller-supplied neighbour lists in host memory, taken in the
 * order given -- AdjList::m as the reference holds it before RowsBySum
 * (src/SparseMat.cpp:81-120), e.g. the lists of ig_graph_adjacency; each
 * undirected edge appears in both lists (no device work). */
ig_status ig_codebook_from_adjacency(const int64_t *adj_ptr, const int32_t *adj, int32_t n, int32_t *order,
                                     int32_t *count);
/* Greedy over a caller-supplied upper CSR in host memory (no device work). */
ig_status ig_codebook_from_upper_csr(const int64_t *row_ptr, const int32_t *cols, int32_t n, int order_threads,
                                     int32_t *order, int32_t *count);
/* No counterpart in the reference (its greedy is single-threaded).  A greedy
 * run by a caller's thread (ig_solve, ig_graph_codebook, the two calls above)
 * over a graph with at least min_entries neighbour-list entries (twice its
 * edges) runs on two threads -- the caller walks the balls and keeps the
 * degrees, a helper thread keeps the degree buckets -- when it is the only
 * greedy running in the process, fewer than max_helpers helper threads are
 * in use and the greedies plus the helpers stay below the hardware threads.
 * In the library's greedy pools (batches, the clustered solve, the server:
 * one greedy per core already) only graphs with at least 64 * min_entries
 * entries do so, under the same helper rule.  Otherwise a greedy runs on one
 * thread.  Both forms give the same codebook.
 * Process-wide.  max_helpers < 0: (hardware threads - 1) / 2; 0: never.
 * min_entries < 0: 2^20. */
ig_status ig_set_greedy_threads(int max_helpers, int64_t min_entries);
/* Greedies run so far in this process, two-threaded and single-threaded
 * (either pointer may be null). */
ig_status ig_greedy_stats(int64_t *pipelined, int64_t *sequential);

/* ---- allocation-free variant ------------------------------------------- */

/* No counterpart in the reference.  Counts the pairs i<j with ED < min_ed
 * like ig_count_conflicts, but never allocates device memory: for hosts that
 * manage every device byte themselves (a fixed arena handed out by a JVM, Go
 * or Rust runtime, a hard per-process memory budget) or that must not enter
 * the allocator where it could block or fail.  `words` (n packed words) and
 * `count` (one unsigned 64-bit integer) are device pointers owned by the
 * caller; the work is queued on `stream` (a cudaStream_t; NULL = the default
 * stream) of the current device and the call returns without waiting.  The
 * scratch is a fixed array inside the library image, at most
 * IG_NOALLOC_MAX_WORDS words per call (larger n: IG_ERR_CAPACITY).  The first
 * call on each device looks up that array's device address; make it before
 * any stream capture.  The address is kept for the life of the process: a
 * host that resets a device (cudaDeviceReset) must not call this entry point
 * on that device again in the same process.  All calls share the array:
 * calls that overlap on the GPU race and must be serialised by the caller. */
#define IG_NOALLOC_MAX_WORDS 65536
ig_status ig_count_conflicts_noalloc(const uint32_t *words, int32_t n, int len, int min_ed,
                                     unsigned long long *count, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* INDEXGEN_CUDA_H */
