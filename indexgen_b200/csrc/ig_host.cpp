// Host-side parts of libindexgen_cuda: input packing, candidate filters and
// the sequential greedy independent set.
//
// The greedy is a sequential bucket-queue walk whose every step depends on the
// previous one (a chain of dependent loads and stores per removed edge); it is
// latency-bound pointer chasing, so it runs on the host next to the device CSR
// it consumes, as the reference's AdjList does.
#include <algorithm>
#include <cstring>
#include <vector>

#include "ig_internal.h"

namespace ig {

namespace {

// Neighbour lists in the order FillAdjList(T) assembles them
// (src/SparseMat.cpp:599-609): thread t holds pairs (i, j) with i = t (mod T),
// sorted by (i, j); for each pair m[i] gets j and m[j] gets i.  For vertex x
// this yields, for t = 0..T-1: the lower neighbours w = t (mod T) ascending,
// followed -- when t = x mod T -- by all upper neighbours ascending.  T = 1 is
// the fully sorted order AdjList::FromBinaryFile builds from a row-sorted
// edge file (src/SparseMat.cpp:338-390).
void assemble(const int64_t *row_ptr, const int32_t *cols, int32_t n, int T, std::vector<int64_t> &ap,
              std::vector<int32_t> &adj)
{
    const int64_t nnz = row_ptr[n];
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
            tmp.assign(lb, lb + nl);
            std::stable_sort(tmp.begin(), tmp.end(), [T](int32_t a, int32_t b) { return a % T < b % T; });
            const int rx = x % T;
            auto split = std::upper_bound(tmp.begin(), tmp.end(), rx,
                                          [T](int r, int32_t w) { return r < w % T; });
            const int64_t head = split - tmp.begin();
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
class BucketGreedy {
  public:
    BucketGreedy(const int64_t *ap, const int32_t *adj, int32_t n) : ap_(ap), adj_(adj), n_(n)
    {
        deg_.resize((size_t)n);
        pos_.resize((size_t)n);
        deleted_.assign((size_t)n, 0);
        int32_t maxd = 0;
        for (int32_t i = 0; i < n; ++i) {
            deg_[(size_t)i] = (int32_t)(ap[i + 1] - ap[i]);
            maxd = std::max(maxd, deg_[(size_t)i]);
        }
        buckets_.resize((size_t)maxd + 1);
        tracker_ = maxd + 1;
        for (int32_t i = 0; i < n; ++i) {  // RowsBySum
            auto &b = buckets_[(size_t)deg_[(size_t)i]];
            pos_[(size_t)i] = (int32_t)b.size();
            b.push_back(i);
            tracker_ = std::min(tracker_, deg_[(size_t)i]);
        }
        active_ = n;
        todel_.reserve((size_t)maxd + 1);
    }

    int32_t run(int32_t *order)
    {
        int32_t cnt = 0;
        while (active_ > 0) {
            const int32_t x = buckets_[(size_t)tracker_].back();  // MinSumRow
            order[cnt++] = x;
            todel_.clear();  // DelBall
            for (int64_t k = ap_[x]; k < ap_[x + 1]; ++k)
                if (!deleted_[(size_t)adj_[k]])
                    todel_.push_back(adj_[k]);
            todel_.push_back(x);
            for (int32_t y : todel_)
                del_row_col(y);
        }
        return cnt;
    }

  private:
    void delete_row(int32_t cur, int32_t row)
    {
        auto &b = buckets_[(size_t)cur];
        const int32_t p = pos_[(size_t)row];
        const int32_t last = b.back();
        b[(size_t)p] = last;
        pos_[(size_t)last] = p;
        b.pop_back();
        if (cur == tracker_ && b.empty())
            while (tracker_ < (int32_t)buckets_.size() && buckets_[(size_t)tracker_].empty())
                ++tracker_;
    }

    void decrease_sum(int32_t cur, int32_t row)
    {
        delete_row(cur, row);
        deg_[(size_t)row] = cur - 1;
        auto &b = buckets_[(size_t)cur - 1];
        pos_[(size_t)row] = (int32_t)b.size();
        b.push_back(row);
        if (cur - 1 < tracker_)
            tracker_ = cur - 1;
    }

    void del_row_col(int32_t i)
    {
        if (deleted_[(size_t)i])
            return;
        for (int64_t k = ap_[i]; k < ap_[i + 1]; ++k) {
            const int32_t j = adj_[k];
            if (deleted_[(size_t)j])
                continue;
            const int32_t dj = deg_[(size_t)j];
            if (dj > 0)
                decrease_sum(dj, j);
        }
        delete_row(deg_[(size_t)i], i);
        deleted_[(size_t)i] = 1;
        --active_;
    }

    const int64_t *ap_;
    const int32_t *adj_;
    int32_t n_;
    std::vector<int32_t> deg_, pos_;
    std::vector<uint8_t> deleted_;
    std::vector<std::vector<int32_t>> buckets_;
    std::vector<int32_t> todel_;
    int32_t tracker_ = 0;
    int32_t active_ = 0;
};

}  // namespace

int32_t greedy_from_upper(const int64_t *row_ptr, const int32_t *cols, int32_t n, int order_threads,
                          int32_t *order)
{
    if (n <= 0)
        return 0;
    std::vector<int64_t> ap;
    std::vector<int32_t> adj;
    assemble(row_ptr, cols, n, order_threads, ap, adj);
    BucketGreedy g(ap.data(), adj.data(), n);
    return g.run(order);
}

}  // namespace ig

extern "C" {

ig_status ig_pack(const char *text, int64_t n, int len, int64_t stride, uint32_t *out, int64_t *bad_row)
{
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
}

ig_status ig_filter(const uint32_t *words, int64_t n, int len, int max_run, double min_gc, double max_gc,
                    uint8_t *keep)
{
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
}

ig_status ig_codebook_from_upper_csr(const int64_t *row_ptr, const int32_t *cols, int32_t n, int order_threads,
                                     int32_t *order, int32_t *count)
{
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
        *count = ig::greedy_from_upper(row_ptr, cols, n, order_threads, order);
    } catch (...) {
        return IG_ERR_OOM;
    }
    return IG_OK;
}

}  // extern "C"
