// Host-side parts of libindexgen_cuda: input packing, candidate filters and
// the greedy independent set.
//
// The greedy is a sequential bucket-queue walk whose every step depends on the
// previous one (a chain of dependent loads and stores per removed edge); it is
// latency-bound pointer chasing, so it runs on the host next to the device CSR
// it consumes, as the reference's AdjList does.  Large graphs split each step
// over two threads (PipelinedGreedy): one walks the balls and keeps the
// degrees, the other keeps the degree buckets.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <memory>
#include <system_error>
#include <thread>
#include <vector>
#if defined(__x86_64__)
#include <immintrin.h>
#endif

#include "ig_internal.h"

namespace ig {

namespace {

// Greedies running and helper threads of pipelined greedies in use in this
// process, and the limits set by ig_set_greedy_threads (negative = default).
std::atomic<int> g_greedies_running{0};
std::atomic<int> g_helpers_busy{0};
std::atomic<int> g_helpers_max{-1};
std::atomic<int64_t> g_pipeline_min{-1};
std::atomic<int64_t> g_runs_pipelined{0};
std::atomic<int64_t> g_runs_sequential{0};
constexpr int64_t kPipelineMinEntries = int64_t(1) << 20;
thread_local int t_pooled = 0;  // PooledGreedyScope depth on this thread

inline void cpu_relax()
{
#if defined(__x86_64__)
    _mm_pause();
#endif
}

// The two threads of a pipelined greedy wait on each other once per ball
// (the mover's backlog then drains in a few microseconds): spin briefly, then
// yield so that a busy host still runs the other thread.
struct Backoff {
    int spins = 0;
    void pause()
    {
        if (++spins < 256)
            cpu_relax();
        else
            std::this_thread::yield();
    }
};

int helper_cap()
{
    const int m = g_helpers_max.load();
    if (m >= 0)
        return m;
    const int hc = (int)std::thread::hardware_concurrency();
    return std::max(0, (hc - 1) / 2);
}

// A helper is taken only while the cap allows it and the greedies running
// plus the helpers stay below the hardware threads: a batch or a server that
// already runs a greedy per core gets none, so no pipelined pair ever waits
// on a partner that is not running.
bool take_helper()
{
    const int cap = helper_cap();
    const int hc = std::max(1, (int)std::thread::hardware_concurrency());
    int cur = g_helpers_busy.load();
    while (cur < cap && g_greedies_running.load() + cur < hc)
        if (g_helpers_busy.compare_exchange_weak(cur, cur + 1))
            return true;
    return false;
}

// Neighbour lists in the order FillAdjList(T) assembles them
// (src/SparseMat.cpp:599-609): thread t holds pairs (i, j) with i = t (mod T),
// sorted by (i, j); for each pair m[i] gets j and m[j] gets i.  For vertex x
// this yields, for t = 0..T-1: the lower neighbours w = t (mod T) ascending,
// followed -- when t = x mod T -- by all upper neighbours ascending.  T = 1 is
// the fully sorted order AdjList::FromBinaryFile builds from a row-sorted
// edge file (src/SparseMat.cpp:338-390).
// row_ptr covers the job's n rows (its values index cols); column ids are
// global and `base` maps them to job-local ids.  The output is job-local.
void assemble(const int64_t *row_ptr, const int32_t *cols_in, int32_t n, int64_t base, int T,
              std::vector<int64_t> &ap, std::vector<int32_t> &adj)
{
    const int64_t first = row_ptr[0];
    const int64_t nnz = row_ptr[n] - first;
    std::vector<int32_t> local((size_t)std::max<int64_t>(nnz, 1));
    for (int64_t k = 0; k < nnz; ++k)
        local[(size_t)k] = (int32_t)(cols_in[first + k] - base);
    std::vector<int64_t> rp((size_t)n + 1);
    for (int32_t i = 0; i <= n; ++i)
        rp[(size_t)i] = row_ptr[i] - first;
    const int32_t *cols = local.data();
    row_ptr = rp.data();
    std::vector<int64_t> lp((size_t)n + 1, 0);
    for (int64_t k = 0; k < nnz; ++k)
        lp[(size_t)cols[k] + 1]++;
    for (int32_t i = 0; i < n; ++i)
        lp[(size_t)i + 1] += lp[(size_t)i];
    std::vector<int32_t> lo((size_t)std::max<int64_t>(nnz, 1));
    {
        std::vector<int64_t> fill(lp.begin(), lp.end() - 1);
        for (int32_t w = 0; w < n; ++w)
            for (int64_t k = row_ptr[w]; k < row_ptr[w + 1]; ++k)
                lo[(size_t)fill[(size_t)cols[k]]++] = w;
    }
    ap.assign((size_t)n + 1, 0);
    adj.resize((size_t)std::max<int64_t>(2 * nnz, 1));
    std::vector<int32_t> tmp;
    std::vector<int64_t> rc((size_t)std::max(T, 1) + 1);
    int64_t o = 0;
    for (int32_t x = 0; x < n; ++x) {
        const int32_t *lb = lo.data() + lp[(size_t)x];
        const int64_t nl = lp[(size_t)x + 1] - lp[(size_t)x];
        const int32_t *ub = cols + row_ptr[x];
        const int64_t nu = row_ptr[x + 1] - row_ptr[x];
        if (T <= 1) {
            std::memcpy(adj.data() + o, lb, (size_t)nl * sizeof(int32_t));
            o += nl;
            std::memcpy(adj.data() + o, ub, (size_t)nu * sizeof(int32_t));
            o += nu;
        } else {
            // stable counting pass by residue w mod T keeps w ascending per group
            std::fill(rc.begin(), rc.end(), 0);
            for (int64_t k = 0; k < nl; ++k)
                rc[(size_t)(lb[k] % T) + 1]++;
            for (int t = 0; t < T; ++t)
                rc[(size_t)t + 1] += rc[(size_t)t];
            const int rx = x % T;
            // upper neighbours follow the lower ones of residue <= x mod T
            const int64_t head = rc[(size_t)rx + 1];
            tmp.resize((size_t)nl);
            for (int64_t k = 0; k < nl; ++k)
                tmp[(size_t)rc[(size_t)(lb[k] % T)]++] = lb[k];
            std::memcpy(adj.data() + o, tmp.data(), (size_t)head * sizeof(int32_t));
            o += head;
            std::memcpy(adj.data() + o, ub, (size_t)nu * sizeof(int32_t));
            o += nu;
            std::memcpy(adj.data() + o, tmp.data() + head, (size_t)(nl - head) * sizeof(int32_t));
            o += nl - head;
        }
        ap[(size_t)x + 1] = o;
    }
}

// The AdjList degree-bucket structure (include/SparseMat.hpp:42-194) with the
// exact semantics of its members (src/SparseMat.cpp:81-266): LIFO buckets,
// swap-with-last removal, moved rows appended to the lower bucket, and a
// minimum tracker that only advances when the tracked bucket empties.
//
// Layout: the degree doubles as the deletion mark (-1 = deleted; the
// reference skips deleted neighbours and neighbours of degree 0 alike) and
// sits next to the bucket position of the same vertex; and
// all buckets share one flat array: bucket b gets a fixed slice of
// #{v : initial degree >= b} slots, which bounds its size at any time because
// degrees only fall.  The slice array is left uninitialised so only the slots
// actually used are ever touched.
// Neighbour lists as the canonical adjacency in memory: row i is a slice of adj.
struct PlainRows {
    const int64_t *ap;
    const int32_t *adj;
    const int32_t *get(int32_t i, int32_t *) const { return adj + ap[i]; }
    void prefetch(int32_t i) const { __builtin_prefetch(adj + ap[i]); }
};

// Neighbour lists bit-packed per row (ig_packrows.cu): a header word with the
// gap width w, the first neighbour, then the gaps a[k] - a[k-1] - 1 in w bits
// each; decoded into the caller's buffer just before the row is walked.
struct PackedRows {
    const int64_t *ap;   // degrees: ap[i+1] - ap[i]
    const int64_t *off;  // first word of each row
    const uint32_t *pk;  // the words (two spare words at the end)
    const int32_t *get(int32_t i, int32_t *buf) const
    {
        const int64_t d = ap[i + 1] - ap[i];
        if (d == 0)
            return buf;
        const uint32_t *row = pk + off[i];
        const uint32_t w = row[0];
        const uint32_t *g = row + 2;
        const uint64_t mask = w >= 32 ? 0xffffffffull : ((1ull << w) - 1);
        int32_t a = (int32_t)row[1];
        buf[0] = a;
        uint64_t pos = 0;
        for (int64_t k = 1; k < d; ++k, pos += w) {
            const uint64_t word = pos >> 5;
            uint64_t v;
            std::memcpy(&v, g + word, sizeof(v));
            a += (int32_t)((v >> (pos & 31)) & mask) + 1;
            buf[k] = a;
        }
        return buf;
    }
    void prefetch(int32_t i) const { __builtin_prefetch(pk + off[i]); }
};

template <class Rows>
class BucketGreedy {
  public:
    // ap covers the n job rows (its differences are the degrees); neighbour
    // ids in the rows are global and `base` maps them to job-local ids.
    BucketGreedy(const int64_t *ap, Rows rows, int32_t n, int64_t base)
        : ap_(ap), rows_(rows), base_(base), v_((size_t)n)
    {
        int32_t maxd = 0;
        for (int32_t i = 0; i < n; ++i) {
            v_[(size_t)i].deg = (int32_t)(ap[i + 1] - ap[i]);
            maxd = std::max(maxd, v_[(size_t)i].deg);
        }
        nb_ = maxd + 1;
        std::vector<int64_t> hist((size_t)nb_ + 1, 0);
        for (int32_t i = 0; i < n; ++i)
            hist[(size_t)v_[(size_t)i].deg]++;
        // cap_b = #{v : deg >= b}
        start_.resize((size_t)nb_ + 1);
        size_.assign((size_t)nb_, 0);
        int64_t ge = n, off = 0;
        for (int32_t b = 0; b < nb_; ++b) {
            start_[(size_t)b] = off;
            off += ge;
            ge -= hist[(size_t)b];
        }
        start_[(size_t)nb_] = off;
        data_.reset(new int32_t[(size_t)std::max<int64_t>(off, 1)]);
        tracker_ = maxd + 1;
        for (int32_t i = 0; i < n; ++i) {  // RowsBySum: ascending vertex id
            const int32_t d = v_[(size_t)i].deg;
            v_[(size_t)i].pos = size_[(size_t)d];
            data_[(size_t)(start_[(size_t)d] + size_[(size_t)d]++)] = i;
            tracker_ = std::min(tracker_, d);
        }
        active_ = n;
        todel_.reserve((size_t)maxd + 1);
        bufx_.resize((size_t)maxd + 1);
        bufi_.resize((size_t)maxd + 1);
    }

    int32_t run(int32_t *order)
    {
        int32_t cnt = 0;
        while (active_ > 0) {
            // MinSumRow: back of the minimum bucket
            const int32_t x = data_[(size_t)(start_[(size_t)tracker_] + size_[(size_t)tracker_] - 1)];
            order[cnt++] = x;
            // DelBall: active neighbours in m-order, then the vertex itself
            const int32_t *row = rows_.get(x, bufx_.data());
            const int64_t len = ap_[x + 1] - ap_[x];
            todel_.resize((size_t)len + 1);
            int32_t nt = 0;
            for (int64_t k = 0; k < len; ++k) {  // branch-free compaction
                const int32_t j = (int32_t)(row[k] - base_);
                todel_[(size_t)nt] = j;
                nt += v_[(size_t)j].deg >= 0;
            }
            todel_[(size_t)nt++] = x;
            // the neighbour lists of the ball's vertices are read next: fetch
            // their heads a few vertices ahead
            for (int32_t t = 0; t < nt && t < 4; ++t)
                rows_.prefetch(todel_[(size_t)t]);
            for (int32_t t = 0; t < nt; ++t) {
                if (t + 4 < nt)
                    rows_.prefetch(todel_[(size_t)t + 4]);
                del_row_col(todel_[(size_t)t]);
            }
        }
        return cnt;
    }

  private:
    void delete_row(int32_t cur, int32_t row)
    {
        const int64_t base = start_[(size_t)cur];
        const int32_t sz = --size_[(size_t)cur];
        const int32_t p = v_[(size_t)row].pos;
        const int32_t last = data_[(size_t)(base + sz)];
        data_[(size_t)(base + p)] = last;
        v_[(size_t)last].pos = p;
        if (cur == tracker_ && sz == 0)
            while (tracker_ < nb_ && size_[(size_t)tracker_] == 0)
                ++tracker_;
    }

    void decrease_sum(int32_t cur, int32_t row)
    {
        delete_row(cur, row);
        const int32_t b = cur - 1;
        const int32_t s = size_[(size_t)b]++;
        data_[(size_t)(start_[(size_t)b] + s)] = row;
        v_[(size_t)row].deg = b;
        v_[(size_t)row].pos = s;
        if (b < tracker_)
            tracker_ = b;
    }

    // Neighbours are visited in blocks of 8: their degrees are loaded together
    // (independent loads overlap, the next block's are prefetched) and only
    // the live ones (degree > 0) are walked through a bitmask.  Exact: within one pass over m[i] the
    // neighbours are distinct and decrease_sum(j) changes only deg[j].
    void del_row_col(int32_t i)
    {
        const int32_t di = v_[(size_t)i].deg;
        if (di < 0)
            return;
        const int32_t *row = rows_.get(i, bufi_.data());
        const int64_t e = ap_[i + 1] - ap_[i];
        for (int64_t k = 0; k < e; k += 8) {
            const int m = (int)std::min<int64_t>(8, e - k);
            for (int64_t q = k + 8; q < std::min<int64_t>(k + 16, e); ++q)  // next block's degrees
                __builtin_prefetch(&v_[(size_t)(row[q] - base_)]);
            int32_t jj[8], dd[8];
            unsigned live = 0;
            for (int t = 0; t < m; ++t) {
                jj[t] = (int32_t)(row[k + t] - base_);
                dd[t] = v_[(size_t)jj[t]].deg;
            }
            for (int t = 0; t < m; ++t)
                live |= (unsigned)(dd[t] > 0) << t;
            while (live) {
                const int t = __builtin_ctz(live);
                live &= live - 1;
                decrease_sum(dd[t], jj[t]);
            }
        }
        delete_row(v_[(size_t)i].deg, i);
        v_[(size_t)i].deg = -1;
        --active_;
    }

    struct Vtx {
        int32_t deg;  // current degree, -1 once deleted
        int32_t pos;  // slot inside its degree bucket
    };
    const int64_t *ap_;
    Rows rows_;
    int64_t base_;
    std::vector<Vtx> v_;
    std::vector<int32_t> size_;
    std::vector<int64_t> start_;
    std::unique_ptr<int32_t[]> data_;
    std::vector<int32_t> todel_, bufx_, bufi_;
    int32_t nb_ = 0;
    int32_t tracker_ = 0;
    int32_t active_ = 0;
};

// BucketGreedy's walk split over two threads, with the same result.
//
// With the live-neighbour test made branch-free, the sequential walk spends
// its time in two halves of similar cost: loading and lowering the degrees of
// the neighbours, and moving those neighbours between degree buckets.  Here
// the calling thread (the walker) selects the vertices, collects each ball and
// keeps the degrees: for every neighbour it loads the degree, lowers it if
// positive, and writes the bucket move (vertex, old degree) into a ring whose
// cursor advances only for live neighbours, followed by the deletion
// (vertex, final degree) of each ball vertex.  A helper thread (the mover)
// applies the ring in order to the buckets with BucketGreedy's own
// delete_row / decrease_sum steps and keeps the minimum tracker.  Every
// bucket therefore sees exactly the sequential sequence of appends and
// swap-removals.  Before each selection the walker waits until the mover has
// applied everything written, then reads the back of the minimum bucket.
//
// Degrees (walker) and bucket positions (mover) live in separate arrays so
// neither thread writes a cache line the other one is using.
template <class Rows>
class PipelinedGreedy {
  public:
    PipelinedGreedy(const int64_t *ap, Rows rows, int32_t n, int64_t base)
        : ap_(ap), rows_(rows), base_(base), n_(n), deg_((size_t)n), pos_((size_t)n)
    {
        int32_t maxd = 0;
        for (int32_t i = 0; i < n; ++i) {
            deg_[(size_t)i] = (int32_t)(ap[i + 1] - ap[i]);
            maxd = std::max(maxd, deg_[(size_t)i]);
        }
        nb_ = maxd + 1;
        std::vector<int64_t> hist((size_t)nb_ + 1, 0);
        for (int32_t i = 0; i < n; ++i)
            hist[(size_t)deg_[(size_t)i]]++;
        start_.resize((size_t)nb_ + 1);
        size_.assign((size_t)nb_, 0);
        int64_t ge = n, off = 0;
        for (int32_t b = 0; b < nb_; ++b) {
            start_[(size_t)b] = off;
            off += ge;
            ge -= hist[(size_t)b];
        }
        start_[(size_t)nb_] = off;
        data_.reset(new int32_t[(size_t)std::max<int64_t>(off, 1)]);
        int32_t tracker = maxd + 1;
        for (int32_t i = 0; i < n; ++i) {
            const int32_t d = deg_[(size_t)i];
            pos_[(size_t)i] = size_[(size_t)d];
            data_[(size_t)(start_[(size_t)d] + size_[(size_t)d]++)] = i;
            tracker = std::min(tracker, d);
        }
        tracker_.store(tracker);
        todel_.resize((size_t)maxd + 1);
        bufx_.resize((size_t)maxd + 1);
        bufi_.resize((size_t)maxd + 1);
        ring_.reset(new uint64_t[(size_t)kRing]);
    }

    // The selection's size, or -1 when the mover thread could not be started
    // (nothing has been changed then; the caller runs BucketGreedy).
    int32_t run(int32_t *order)
    {
        std::thread mover;
        try {
            mover = std::thread([this]() { move_loop(); });
        } catch (const std::system_error &) {
            return -1;
        }
        int32_t *deg = deg_.data();
        uint64_t *ring = ring_.get();
        int64_t p = 0;  // ring entries written
        int32_t cnt = 0, active = n_;
        while (active > 0) {
            // MinSumRow once every move so far is in the buckets
            pub_.store(p, std::memory_order_release);
            for (Backoff bo; cons_.load(std::memory_order_acquire) < p;)
                bo.pause();
            const int32_t t = tracker_.load(std::memory_order_relaxed);
            const int32_t x = data_[(size_t)(start_[(size_t)t] + size_[(size_t)t] - 1)];
            order[cnt++] = x;
            // DelBall: active neighbours in m-order, then the vertex itself
            const int32_t *row = rows_.get(x, bufx_.data());
            const int64_t len = ap_[x + 1] - ap_[x];
            int32_t nt = 0;
            for (int64_t k = 0; k < len; ++k) {
                const int32_t j = (int32_t)(row[k] - base_);
                todel_[(size_t)nt] = j;
                nt += deg[j] >= 0;
            }
            todel_[(size_t)nt++] = x;
            for (int32_t q = 0; q < nt && q < 4; ++q)
                rows_.prefetch(todel_[(size_t)q]);
            for (int32_t q = 0; q < nt; ++q) {
                if (q + 4 < nt)
                    rows_.prefetch(todel_[(size_t)q + 4]);
                const int32_t i = todel_[(size_t)q];
                if (deg[i] < 0)
                    continue;
                const int32_t *ri = rows_.get(i, bufi_.data());
                const int64_t e = ap_[i + 1] - ap_[i];
                // chunks of at most kChunk neighbours; room for the chunk and
                // the deletion that may follow it is waited for first
                for (int64_t k0 = 0;; k0 += kChunk) {
                    const int64_t k1 = std::min<int64_t>(e, k0 + kChunk);
                    pub_.store(p, std::memory_order_release);
                    for (Backoff bo; p + kChunk + 1 - cons_.load(std::memory_order_acquire) > kRing;)
                        bo.pause();
                    for (int64_t k = k0; k < k1; ++k) {
                        if (k + 16 < e)
                            __builtin_prefetch(deg + (ri[k + 16] - base_));
                        const int32_t j = (int32_t)(ri[k] - base_);
                        const int32_t d = deg[j];
                        ring[p & (kRing - 1)] = ((uint64_t)(uint32_t)d << 32) | (uint32_t)j;
                        deg[j] = d - (d > 0);
                        p += d > 0;
                    }
                    if (k1 >= e)
                        break;
                }
                ring[p & (kRing - 1)] = ((uint64_t)(uint32_t)deg[i] << 32) | (uint32_t)i | kDelete;
                ++p;
                deg[i] = -1;
                --active;
            }
        }
        pub_.store(p, std::memory_order_release);
        done_.store(true, std::memory_order_release);
        mover.join();
        return cnt;
    }

  private:
    static constexpr int64_t kRing = int64_t(1) << 16;  // entries (512 KB)
    static constexpr int64_t kChunk = 4096;
    static constexpr uint64_t kDelete = uint64_t(1) << 31;

    void move_loop()
    {
        int32_t *pos = pos_.data();
        int32_t *sz = size_.data();
        const int64_t *start = start_.data();
        int32_t *data = data_.get();
        const uint64_t *ring = ring_.get();
        int32_t tracker = tracker_.load(std::memory_order_relaxed);
        int64_t c = 0;
        for (Backoff bo;;) {
            const int64_t p = pub_.load(std::memory_order_acquire);
            if (c == p) {
                if (done_.load(std::memory_order_acquire) && pub_.load(std::memory_order_acquire) == c)
                    return;
                bo.pause();
                continue;
            }
            bo.spins = 0;
            for (; c < p; ++c) {
                if (c + 16 < p)
                    __builtin_prefetch(pos + ((uint32_t)ring[(c + 16) & (kRing - 1)] & 0x7fffffffu));
                const uint64_t op = ring[c & (kRing - 1)];
                const int32_t v = (int32_t)((uint32_t)op & 0x7fffffffu);
                const int32_t cur = (int32_t)(op >> 32);
                // delete_row(cur, v)
                const int64_t base = start[cur];
                const int32_t s = --sz[cur];
                const int32_t q = pos[v];
                const int32_t last = data[base + s];
                data[base + q] = last;
                pos[last] = q;
                if (cur == tracker && s == 0)
                    while (tracker < nb_ && sz[tracker] == 0)
                        ++tracker;
                if (!(op & kDelete)) {  // decrease_sum: append to the bucket below
                    const int32_t b = cur - 1;
                    const int32_t s1 = sz[b]++;
                    data[start[b] + s1] = v;
                    pos[v] = s1;
                    if (b < tracker)
                        tracker = b;
                }
                if ((c & 1023) == 1023) {
                    tracker_.store(tracker, std::memory_order_relaxed);
                    cons_.store(c + 1, std::memory_order_release);
                }
            }
            tracker_.store(tracker, std::memory_order_relaxed);
            cons_.store(c, std::memory_order_release);
        }
    }

    const int64_t *ap_;
    Rows rows_;
    int64_t base_;
    int32_t n_;
    std::vector<int32_t> deg_;  // walker: current degree, -1 once deleted
    std::vector<int32_t> pos_;  // mover: slot inside the degree bucket
    std::vector<int32_t> size_;
    std::vector<int64_t> start_;
    std::unique_ptr<int32_t[]> data_;
    std::unique_ptr<uint64_t[]> ring_;
    std::vector<int32_t> todel_, bufx_, bufi_;
    int32_t nb_ = 0;
    alignas(64) std::atomic<int64_t> pub_{0};   // entries the walker has published
    alignas(64) std::atomic<int64_t> cons_{0};  // entries the mover has applied
    alignas(64) std::atomic<int32_t> tracker_{0};
    alignas(64) std::atomic<bool> done_{false};
};

// A greedy over n rows: pipelined over two threads when a helper thread is
// free and either it is the only greedy running in the process, outside the
// library's greedy pools, on a graph with at least the configured number of
// neighbour-list entries, or it runs in a pool on a graph with 64 times that
// (2^26 entries by default: the densest jobs of a stream, whose greedies run
// for seconds to minutes while the small jobs' greedies come and go; the
// helper rule keeps the greedies plus helpers below the hardware threads);
// else sequential on the calling thread.
template <class Rows>
int32_t run_greedy(const int64_t *ap, Rows rows, int32_t n, int64_t base, int32_t *order)
{
    if (n <= 0)
        return 0;
    struct Running {
        Running() { g_greedies_running.fetch_add(1); }
        ~Running() { g_greedies_running.fetch_sub(1); }
    } running;
    int64_t min_entries = g_pipeline_min.load();
    if (min_entries < 0)
        min_entries = kPipelineMinEntries;
    const int64_t entries = ap[n] - ap[0];
    const bool lone = t_pooled == 0 && g_greedies_running.load() == 1 && entries >= min_entries;
    const bool large_pooled = t_pooled > 0 && entries / 64 >= min_entries;
    if ((lone || large_pooled) && take_helper()) {
        struct Give {
            ~Give() { g_helpers_busy.fetch_sub(1); }
        } give;
        PipelinedGreedy<Rows> g(ap, rows, n, base);
        const int32_t cnt = g.run(order);
        if (cnt >= 0) {
            g_runs_pipelined++;
            return cnt;
        }
    }
    g_runs_sequential++;
    BucketGreedy<Rows> g(ap, rows, n, base);
    return g.run(order);
}

}  // namespace

PooledGreedyScope::PooledGreedyScope(bool on) : on_(on)
{
    if (on_)
        ++t_pooled;
}

PooledGreedyScope::~PooledGreedyScope()
{
    if (on_)
        --t_pooled;
}

int32_t greedy_from_upper(const int64_t *row_ptr, const int32_t *cols, int32_t n, int64_t base, int order_threads,
                          int32_t *order)
{
    if (n <= 0)
        return 0;
    std::vector<int64_t> ap;
    std::vector<int32_t> adj;
    assemble(row_ptr, cols, n, base, order_threads, ap, adj);
    return run_greedy(ap.data(), PlainRows{ap.data(), adj.data()}, n, 0, order);
}

int32_t greedy_from_adjacency(const int64_t *adj_ptr, const int32_t *adj, int32_t n, int64_t base, int32_t *order)
{
    return run_greedy(adj_ptr, PlainRows{adj_ptr, adj}, n, base, order);
}

int32_t greedy_from_packed(const int64_t *adj_ptr, const int64_t *pk_off, const uint32_t *pk, int32_t n, int64_t base,
                           int32_t *order)
{
    return run_greedy(adj_ptr, PackedRows{adj_ptr, pk_off, pk}, n, base, order);
}

}  // namespace ig

extern "C" {

ig_status ig_pack(const char *text, int64_t n, int len, int64_t stride, uint32_t *out, int64_t *bad_row)
{
    IG_ABI_TRY
    if (n < 0 || len < 1 || len > IG_MAX_LEN || stride < len || (n > 0 && (!text || !out)))
        return IG_ERR_INPUT;
    for (int64_t i = 0; i < n; ++i) {
        const char *s = text + i * stride;
        uint32_t w = 0;
        for (int p = 0; p < len; ++p) {
            const int c = s[p] - '0';
            if (c < 0 || c > 3) {
                if (bad_row)
                    *bad_row = i;
                return IG_ERR_INPUT;
            }
            w |= (uint32_t)c << (2 * p);
        }
        out[i] = w;
    }
    if (bad_row)
        *bad_row = -1;
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_filter(const uint32_t *words, int64_t n, int len, int max_run, double min_gc, double max_gc,
                    uint8_t *keep)
{
    IG_ABI_TRY
    if (n < 0 || len < 1 || len > IG_MAX_LEN || (n > 0 && (!words || !keep)))
        return IG_ERR_INPUT;
    const bool use_run = max_run > 0;
    const bool use_gc = (min_gc > 0 || max_gc > 0);
    for (int64_t i = 0; i < n; ++i) {
        const uint32_t w = words[i];
        bool ok = true;
        if (use_run) {
            int best = 0, run = 1;
            for (int p = 1; p < len; ++p) {
                if (((w >> (2 * p)) & 3u) == ((w >> (2 * p - 2)) & 3u)) {
                    ++run;
                } else {
                    best = std::max(best, run);
                    run = 1;
                }
            }
            best = std::max(best, run);
            ok = best <= max_run;
        }
        if (ok && use_gc) {
            int gc = 0;
            for (int p = 0; p < len; ++p) {
                const uint32_t c = (w >> (2 * p)) & 3u;
                gc += (c == 1u || c == 2u);
            }
            const double frac = double(gc) / double(len);
            ok = (frac >= min_gc) && (frac <= max_gc);
        }
        keep[i] = ok ? 1 : 0;
    }
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_codebook_from_adjacency(const int64_t *adj_ptr, const int32_t *adj, int32_t n, int32_t *order,
                                     int32_t *count)
{
    IG_ABI_TRY
    if (n < 0 || !count || (n > 0 && (!adj_ptr || !order)) || (n > 0 && adj_ptr[n] > 0 && !adj) ||
        (n > 0 && adj_ptr[0] != 0))
        return IG_ERR_INPUT;
    for (int32_t i = 0; i < n; ++i)
        if (adj_ptr[i + 1] < adj_ptr[i])
            return IG_ERR_INPUT;
    for (int64_t k = 0; n > 0 && k < adj_ptr[n]; ++k)
        if (adj[k] < 0 || adj[k] >= n)
            return IG_ERR_INPUT;
    try {
        *count = ig::greedy_from_adjacency(adj_ptr, adj, n, 0, order);
    } catch (...) {
        return IG_ERR_OOM;
    }
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_set_greedy_threads(int max_helpers, int64_t min_entries)
{
    IG_ABI_TRY
    ig::g_helpers_max.store(max_helpers < 0 ? -1 : max_helpers);
    ig::g_pipeline_min.store(min_entries < 0 ? -1 : min_entries);
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_greedy_stats(int64_t *pipelined, int64_t *sequential)
{
    IG_ABI_TRY
    if (pipelined)
        *pipelined = ig::g_runs_pipelined.load();
    if (sequential)
        *sequential = ig::g_runs_sequential.load();
    return IG_OK;
    IG_ABI_CATCH
}

ig_status ig_codebook_from_upper_csr(const int64_t *row_ptr, const int32_t *cols, int32_t n, int order_threads,
                                     int32_t *order, int32_t *count)
{
    IG_ABI_TRY
    if (n < 0 || !count || (n > 0 && (!row_ptr || !order)) || (n > 0 && row_ptr[n] > 0 && !cols))
        return IG_ERR_INPUT;
    if (order_threads < 1)
        return IG_ERR_INPUT;
    for (int32_t i = 0; i < n; ++i)
        if (row_ptr[i + 1] < row_ptr[i])
            return IG_ERR_INPUT;
    for (int64_t k = 0; n > 0 && k < row_ptr[n]; ++k)
        if (cols[k] < 0 || cols[k] >= n)
            return IG_ERR_INPUT;
    try {
        *count = ig::greedy_from_upper(row_ptr, cols, n, 0, order_threads, order);
    } catch (...) {
        return IG_ERR_OOM;
    }
    return IG_OK;
    IG_ABI_CATCH
}

}  // extern "C"
