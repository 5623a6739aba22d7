/* CPU oracle for the IndexGen conflict-graph + greedy path.
 *
 * TEST INFRASTRUCTURE ONLY (see ig_oracle.h).  Plain C restatement of:
 *   - the edge predicate  !EditDistanceBandedAtLeast(c[j], MakePattern(c[i]), minED)
 *     i.e. Levenshtein(c[i], c[j]) < minED   (include/EditDistance.hpp:368-372,
 *     exact Myers at :78-105), used by FillAdjListTH (src/SparseMat.cpp:536-565);
 *   - the neighbour-list order FillAdjList assembles (src/SparseMat.cpp:599-609);
 *   - the AdjList degree-bucket greedy (src/SparseMat.cpp:81-266, :679-731);
 *   - the homopolymer / GC filters (src/CandidateGenerator.cpp:24-50,
 *     src/Utils.cpp:420-462).
 * The score is tracked at the top pattern bit exactly as MyersSingleWord does,
 * so it is an independent formulation from the CUDA kernel's end-of-text count.
 */
#include "ig_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

static inline int sym(uint32_t w, int p) { return (int)((w >> (2 * p)) & 3u); }

int64_t igo_pack(const char *text, int64_t n, int len, int64_t stride, uint32_t *out)
{
    for (int64_t i = 0; i < n; i++) {
        const char *s = text + i * stride;
        uint32_t w = 0;
        for (int p = 0; p < len; p++) {
            int c = s[p] - '0';
            if (c < 0 || c > 3)
                return i;
            w |= (uint32_t)c << (2 * p);
        }
        out[i] = w;
    }
    return -1;
}

int igo_lev_dp(uint32_t a, uint32_t b, int len)
{
    int prev[17], cur[17];
    for (int j = 0; j <= len; j++)
        prev[j] = j;
    for (int i = 1; i <= len; i++) {
        cur[0] = i;
        for (int j = 1; j <= len; j++) {
            int sub = prev[j - 1] + (sym(a, i - 1) != sym(b, j - 1));
            int del = prev[j] + 1;
            int ins = cur[j - 1] + 1;
            int m = sub < del ? sub : del;
            cur[j] = m < ins ? m : ins;
        }
        memcpy(prev, cur, sizeof(int) * (size_t)(len + 1));
    }
    return prev[len];
}

/* Myers bit-vector recurrence, pattern a (bits), text b streamed; score kept
 * at pattern row len-1 (include/EditDistance.hpp:85-103). */
int igo_lev_myers(uint32_t a, uint32_t b, int len)
{
    if (len == 0)
        return 0;
    uint64_t peq[4] = {0, 0, 0, 0};
    for (int p = 0; p < len; p++)
        peq[sym(a, p)] |= 1ull << p;
    uint64_t pv = ~0ull, mv = 0;
    int score = len;
    const int top = len - 1;
    for (int j = 0; j < len; j++) {
        uint64_t eq = peq[sym(b, j)];
        uint64_t x = eq | mv;
        uint64_t d0 = (((x & pv) + pv) ^ pv) | x;
        uint64_t hn = pv & d0;
        uint64_t hp = mv | ~(pv | d0);
        uint64_t x2 = (hp << 1) | 1ull;
        mv = x2 & d0;
        pv = (hn << 1) | ~(x2 | d0);
        score += (int)((hp >> top) & 1u) - (int)((hn >> top) & 1u);
    }
    return score;
}

void igo_filter(const uint32_t *words, int64_t n, int len, int max_run, double min_gc, double max_gc,
                uint8_t *keep)
{
    const int use_run = max_run > 0;
    const int use_gc = (min_gc > 0 || max_gc > 0);
    for (int64_t i = 0; i < n; i++) {
        uint32_t w = words[i];
        int ok = 1;
        if (use_run) {
            int best = 0, run = 1;
            for (int p = 1; p < len; p++) {
                if (sym(w, p) == sym(w, p - 1))
                    run++;
                else {
                    if (run > best)
                        best = run;
                    run = 1;
                }
            }
            if (run > best)
                best = run;
            ok = best <= max_run;
        }
        if (ok && use_gc) {
            int gc = 0;
            for (int p = 0; p < len; p++) {
                int c = sym(w, p);
                gc += (c == 1 || c == 2);
            }
            double frac = (double)gc / (double)len;
            ok = (frac >= min_gc) && (frac <= max_gc);
        }
        keep[i] = (uint8_t)ok;
    }
}

/* ---------------- all-pairs upper CSR (threads own rows i = t mod T) ---------------- */

typedef struct {
    const uint32_t *words;
    int32_t n;
    int len, min_ed, t, nthreads;
    int64_t *row_cnt;   /* per row */
    int32_t *buf;       /* this thread's columns, rows in ascending order */
    int64_t used, cap;
    int fail;
} upper_job;

static void *upper_worker(void *arg)
{
    upper_job *jb = (upper_job *)arg;
    for (int32_t i = jb->t; i < jb->n; i += jb->nthreads) {
        int64_t c0 = jb->used;
        for (int32_t j = i + 1; j < jb->n; j++) {
            if (igo_lev_myers(jb->words[i], jb->words[j], jb->len) < jb->min_ed) {
                if (jb->used == jb->cap) {
                    int64_t nc = jb->cap ? jb->cap * 2 : 4096;
                    int32_t *nb = (int32_t *)realloc(jb->buf, (size_t)nc * sizeof(int32_t));
                    if (!nb) {
                        jb->fail = 1;
                        return NULL;
                    }
                    jb->buf = nb;
                    jb->cap = nc;
                }
                jb->buf[jb->used++] = j;
            }
        }
        jb->row_cnt[i] = jb->used - c0;
    }
    return NULL;
}

static int conflict_upper_impl(const uint32_t *words, int32_t n, int len, int min_ed, int threads,
                               int64_t *row_ptr, int32_t *cols, int32_t **cols_alloc);

int igo_conflict_upper(const uint32_t *words, int32_t n, int len, int min_ed, int threads, int64_t *row_ptr,
                       int32_t *cols)
{
    return conflict_upper_impl(words, n, len, min_ed, threads, row_ptr, cols, NULL);
}

int igo_conflict_upper_alloc(const uint32_t *words, int32_t n, int len, int min_ed, int threads, int64_t *row_ptr,
                             int32_t **cols)
{
    *cols = NULL;
    return conflict_upper_impl(words, n, len, min_ed, threads, row_ptr, NULL, cols);
}

void igo_free(void *p) { free(p); }

static int conflict_upper_impl(const uint32_t *words, int32_t n, int len, int min_ed, int threads,
                               int64_t *row_ptr, int32_t *cols, int32_t **cols_alloc)
{
    if (threads < 1)
        threads = 1;
    int64_t *cnt = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t));
    upper_job *jobs = (upper_job *)calloc((size_t)threads, sizeof(upper_job));
    pthread_t *tid = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
    if (!cnt || !jobs || !tid)
        return -1;
    for (int t = 0; t < threads; t++) {
        jobs[t] = (upper_job){words, n, len, min_ed, t, threads, cnt, NULL, 0, 0, 0};
        pthread_create(&tid[t], NULL, upper_worker, &jobs[t]);
    }
    int fail = 0;
    for (int t = 0; t < threads; t++) {
        pthread_join(tid[t], NULL);
        fail |= jobs[t].fail;
    }
    row_ptr[0] = 0;
    for (int32_t i = 0; i < n; i++)
        row_ptr[i + 1] = row_ptr[i] + cnt[i];
    if (cols_alloc && !fail) {
        cols = (int32_t *)malloc((size_t)(row_ptr[n] ? row_ptr[n] : 1) * sizeof(int32_t));
        *cols_alloc = cols;
        fail = cols == NULL;
    }
    if (cols && !fail) {
        int64_t *off = (int64_t *)calloc((size_t)threads, sizeof(int64_t));
        for (int32_t i = 0; i < n; i++) {
            int t = i % threads;
            memcpy(cols + row_ptr[i], jobs[t].buf + off[t], (size_t)cnt[i] * sizeof(int32_t));
            off[t] += cnt[i];
        }
        free(off);
    }
    for (int t = 0; t < threads; t++)
        free(jobs[t].buf);
    free(jobs);
    free(tid);
    free(cnt);
    return fail ? -1 : 0;
}

/* ---------------- nearest-centre assignment ---------------- */
/* solve_assignments_cuda (src/gpu_cluster.py:239-300): for each word the
 * index of the centre at minimal Levenshtein distance, np.argmin order (the
 * first, i.e. lowest, index on ties).  Distances by igo_lev_myers with the
 * centre as the pattern, as the reference kernel builds Peq from the centres. */
typedef struct {
    const uint32_t *words, *centers;
    int64_t n;
    int32_t k;
    int len, t, nthreads;
    int32_t *out;
} assign_job;

static void *assign_worker(void *arg)
{
    assign_job *jb = (assign_job *)arg;
    for (int64_t i = jb->t; i < jb->n; i += jb->nthreads) {
        int best = 1 << 30;
        int32_t arg_best = 0;
        for (int32_t c = 0; c < jb->k; c++) {
            const int d = igo_lev_myers(jb->centers[c], jb->words[i], jb->len);
            if (d < best) {
                best = d;
                arg_best = c;
            }
        }
        jb->out[i] = arg_best;
    }
    return NULL;
}

int igo_assign_centers(const uint32_t *words, int64_t n, const uint32_t *centers, int32_t k, int len, int threads,
                       int32_t *out)
{
    if (threads < 1)
        threads = 1;
    if (k < 1)
        return n > 0 ? -1 : 0;
    assign_job *jobs = (assign_job *)calloc((size_t)threads, sizeof(assign_job));
    pthread_t *tid = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
    if (!jobs || !tid) {
        free(jobs);
        free(tid);
        return -1;
    }
    for (int t = 0; t < threads; t++) {
        jobs[t] = (assign_job){words, centers, n, k, len, t, threads, out};
        pthread_create(&tid[t], NULL, assign_worker, &jobs[t]);
    }
    for (int t = 0; t < threads; t++)
        pthread_join(tid[t], NULL);
    free(jobs);
    free(tid);
    return 0;
}

/* ---------------- full neighbour rows of sampled vertices ---------------- */
/* For spot checks of graphs too large for the all-pairs oracle: for each
 * sampled row r, every c != r with ED(w_r, w_c) < min_ed, ascending (the
 * symmetric neighbour set, FillAdjList's edge predicate of
 * include/EditDistance.hpp:368-372 restated as igo_lev_myers). */
typedef struct {
    const uint32_t *words;
    int32_t n;
    int len, min_ed;
    const int32_t *rows;
    int32_t nrows;
    int t, nthreads;
    int32_t **out;
    int64_t *cnt;
    int fail;
} row_job;

static void *row_worker(void *arg)
{
    row_job *jb = (row_job *)arg;
    for (int32_t k = jb->t; k < jb->nrows; k += jb->nthreads) {
        const int32_t r = jb->rows[k];
        int64_t cap = 1024, used = 0;
        int32_t *buf = (int32_t *)malloc((size_t)cap * sizeof(int32_t));
        if (!buf) {
            jb->fail = 1;
            return NULL;
        }
        for (int32_t c = 0; c < jb->n; c++) {
            if (c == r || igo_lev_myers(jb->words[r], jb->words[c], jb->len) >= jb->min_ed)
                continue;
            if (used == cap) {
                cap *= 2;
                int32_t *nb = (int32_t *)realloc(buf, (size_t)cap * sizeof(int32_t));
                if (!nb) {
                    free(buf);
                    jb->fail = 1;
                    return NULL;
                }
                buf = nb;
            }
            buf[used++] = c;
        }
        jb->out[k] = buf;
        jb->cnt[k] = used;
    }
    return NULL;
}

int igo_row_neighbours(const uint32_t *words, int32_t n, int len, int min_ed, const int32_t *rows, int32_t nrows,
                       int threads, int64_t *ptr, int32_t **cols)
{
    *cols = NULL;
    if (threads < 1)
        threads = 1;
    int32_t **out = (int32_t **)calloc((size_t)nrows + 1, sizeof(int32_t *));
    int64_t *cnt = (int64_t *)calloc((size_t)nrows + 1, sizeof(int64_t));
    row_job *jobs = (row_job *)calloc((size_t)threads, sizeof(row_job));
    pthread_t *tid = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
    int fail = !out || !cnt || !jobs || !tid;
    if (!fail) {
        for (int t = 0; t < threads; t++) {
            jobs[t] = (row_job){words, n, len, min_ed, rows, nrows, t, threads, out, cnt, 0};
            pthread_create(&tid[t], NULL, row_worker, &jobs[t]);
        }
        for (int t = 0; t < threads; t++) {
            pthread_join(tid[t], NULL);
            fail |= jobs[t].fail;
        }
    }
    if (!fail) {
        ptr[0] = 0;
        for (int32_t k = 0; k < nrows; k++)
            ptr[k + 1] = ptr[k] + cnt[k];
        *cols = (int32_t *)malloc((size_t)(ptr[nrows] ? ptr[nrows] : 1) * sizeof(int32_t));
        fail = *cols == NULL;
        for (int32_t k = 0; k < nrows && !fail; k++)
            memcpy(*cols + ptr[k], out[k], (size_t)cnt[k] * sizeof(int32_t));
    }
    if (out)
        for (int32_t k = 0; k < nrows; k++)
            free(out[k]);
    free(out);
    free(cnt);
    free(jobs);
    free(tid);
    return fail ? -1 : 0;
}

/* ---------------- neighbour order of FillAdjList(T) ---------------- */

void igo_adjacency(const int64_t *row_ptr, const int32_t *cols, int32_t n, int order_threads, int64_t *adj_ptr,
                   int32_t *adj)
{
    const int T = order_threads < 1 ? 1 : order_threads;
    int64_t nnz = row_ptr[n];
    /* lower lists by sequential transposition: sources visited in ascending order */
    int64_t *lo_ptr = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t));
    int32_t *lo = (int32_t *)malloc((size_t)(nnz ? nnz : 1) * sizeof(int32_t));
    int64_t *fill = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t));
    for (int64_t k = 0; k < nnz; k++)
        lo_ptr[cols[k] + 1]++;
    for (int32_t i = 0; i < n; i++)
        lo_ptr[i + 1] += lo_ptr[i];
    for (int32_t w = 0; w < n; w++)
        for (int64_t k = row_ptr[w]; k < row_ptr[w + 1]; k++) {
            int32_t x = cols[k];
            lo[lo_ptr[x] + fill[x]++] = w;
        }
    adj_ptr[0] = 0;
    for (int32_t x = 0; x < n; x++) {
        int64_t o = adj_ptr[x];
        int64_t lb = lo_ptr[x], le = lo_ptr[x + 1];
        if (T == 1) {
            for (int64_t k = lb; k < le; k++)
                adj[o++] = lo[k];
            for (int64_t k = row_ptr[x]; k < row_ptr[x + 1]; k++)
                adj[o++] = cols[k];
        } else {
            for (int t = 0; t < T; t++) {
                for (int64_t k = lb; k < le; k++)
                    if (lo[k] % T == t)
                        adj[o++] = lo[k];
                if (t == x % T)
                    for (int64_t k = row_ptr[x]; k < row_ptr[x + 1]; k++)
                        adj[o++] = cols[k];
            }
        }
        adj_ptr[x + 1] = o;
    }
    free(lo_ptr);
    free(lo);
    free(fill);
}

/* ---------------- degree-bucket greedy (AdjList) ---------------- */

typedef struct {
    int32_t *v;
    int64_t size, cap;
} ivec;

static void ivec_push(ivec *b, int32_t x)
{
    if (b->size == b->cap) {
        b->cap = b->cap ? b->cap * 2 : 8;
        b->v = (int32_t *)realloc(b->v, (size_t)b->cap * sizeof(int32_t));
    }
    b->v[b->size++] = x;
}

typedef struct {
    ivec *bucket;
    int64_t nb;
    int32_t *deg, *pos;
    uint8_t *deleted;
    int64_t tracker;
    int32_t active;
} gstate;

/* AdjList::DeleteRow (src/SparseMat.cpp:139-154) */
static void delete_row(gstate *g, int32_t cur, int32_t row)
{
    ivec *b = &g->bucket[cur];
    int32_t p = g->pos[row];
    int32_t last = b->v[b->size - 1];
    b->v[p] = last;
    g->pos[last] = p;
    b->size--;
    if (cur == g->tracker && b->size == 0)
        while (g->tracker < g->nb && g->bucket[g->tracker].size == 0)
            g->tracker++;
}

/* AdjList::DecreaseSum (src/SparseMat.cpp:156-167) */
static void decrease_sum(gstate *g, int32_t cur, int32_t row)
{
    delete_row(g, cur, row);
    g->deg[row] = cur - 1;
    g->pos[row] = (int32_t)g->bucket[cur - 1].size;
    ivec_push(&g->bucket[cur - 1], row);
    if (cur - 1 < g->tracker)
        g->tracker = cur - 1;
}

/* AdjList::DelRowCol (src/SparseMat.cpp:207-227) */
static void del_row_col(gstate *g, const int64_t *ap, const int32_t *adj, int32_t i)
{
    if (g->deleted[i])
        return;
    for (int64_t k = ap[i]; k < ap[i + 1]; k++) {
        int32_t j = adj[k];
        if (g->deleted[j])
            continue;
        if (g->deg[j] > 0)
            decrease_sum(g, g->deg[j], j);
    }
    delete_row(g, g->deg[i], i);
    g->deleted[i] = 1;
    g->active--;
}

int32_t igo_greedy(const int64_t *ap, const int32_t *adj, int32_t n, int32_t *order)
{
    gstate g;
    memset(&g, 0, sizeof g);
    g.deg = (int32_t *)malloc((size_t)(n ? n : 1) * sizeof(int32_t));
    g.pos = (int32_t *)malloc((size_t)(n ? n : 1) * sizeof(int32_t));
    g.deleted = (uint8_t *)calloc((size_t)(n ? n : 1), 1);
    int64_t maxd = 0;
    for (int32_t i = 0; i < n; i++) {
        g.deg[i] = (int32_t)(ap[i + 1] - ap[i]);
        if (g.deg[i] > maxd)
            maxd = g.deg[i];
    }
    /* AdjList::RowsBySum (src/SparseMat.cpp:92-120) */
    g.nb = maxd + 1;
    g.bucket = (ivec *)calloc((size_t)g.nb, sizeof(ivec));
    g.tracker = maxd + 1;
    for (int32_t i = 0; i < n; i++) {
        g.pos[i] = (int32_t)g.bucket[g.deg[i]].size;
        ivec_push(&g.bucket[g.deg[i]], i);
        if (g.deg[i] < g.tracker)
            g.tracker = g.deg[i];
    }
    g.active = n;
    int32_t cnt = 0;
    int32_t *todel = (int32_t *)malloc((size_t)(maxd + 1) * sizeof(int32_t));
    while (g.active > 0) {
        /* FindMinDel -> MinSumRow (:122-127) -> DelBall (:229-251) */
        ivec *b = &g.bucket[g.tracker];
        int32_t x = b->v[b->size - 1];
        order[cnt++] = x;
        int32_t nt = 0;
        for (int64_t k = ap[x]; k < ap[x + 1]; k++)
            if (!g.deleted[adj[k]])
                todel[nt++] = adj[k];
        todel[nt++] = x;
        for (int32_t k = 0; k < nt; k++)
            del_row_col(&g, ap, adj, todel[k]);
    }
    for (int64_t d = 0; d < g.nb; d++)
        free(g.bucket[d].v);
    free(g.bucket);
    free(g.deg);
    free(g.pos);
    free(g.deleted);
    free(todel);
    return cnt;
}
