/* CPU oracle for the IndexGen conflict-graph + greedy path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithm used to check the CUDA library; only tests/, the smoke check and
 * the CPU-baseline leg of bench.py may load it.  The product never calls it.
 *
 * Parity pin: checked against golden vectors produced by the reference's own
 * C++ code (tests/golden/, generated by tests/golden/make_golden.py).
 *
 * Packing: word w holds a length-L string over {0,1,2,3}; character p sits in
 * bits 2p..2p+1 (L <= 16).
 */
#ifndef IG_ORACLE_H
#define IG_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* '0'..'3' text rows (stride bytes apart) -> packed words.  Returns the index
 * of the first invalid row, or -1 when every row is valid. */
int64_t igo_pack(const char *text, int64_t n, int len, int64_t stride, uint32_t *out);

/* Levenshtein distance by the textbook dynamic program (small-case check). */
int igo_lev_dp(uint32_t a, uint32_t b, int len);

/* Levenshtein distance by bit-parallel Myers (global, one 32-bit word). */
int igo_lev_myers(uint32_t a, uint32_t b, int len);

/* Homopolymer-run / GC filter of src/CandidateGenerator.cpp:24-50. keep[i] = 0/1. */
void igo_filter(const uint32_t *words, int64_t n, int len, int max_run, double min_gc, double max_gc,
                uint8_t *keep);

/* All pairs i<j with ED < min_ed as an upper CSR with ascending columns.
 * Pass cols = NULL to only fill row_ptr (int64[n+1]).  threads >= 1. */
int igo_conflict_upper(const uint32_t *words, int32_t n, int len, int min_ed, int threads, int64_t *row_ptr,
                       int32_t *cols);

/* Same, in one pass: *cols receives a malloc'ed array of row_ptr[n] entries
 * (release with igo_free). */
int igo_conflict_upper_alloc(const uint32_t *words, int32_t n, int len, int min_ed, int threads, int64_t *row_ptr,
                             int32_t **cols);
void igo_free(void *p);

/* Nearest centre of every word (Levenshtein; lowest index on ties). */
int igo_assign_centers(const uint32_t *words, int64_t n, const uint32_t *centers, int32_t k, int len, int threads,
                       int32_t *out);

/* Symmetric neighbour rows of the sampled vertices rows[0..nrows): row k's
 * neighbours (ascending) are (*cols)[ptr[k] .. ptr[k+1]) (release with igo_free). */
int igo_row_neighbours(const uint32_t *words, int32_t n, int len, int min_ed, const int32_t *rows, int32_t nrows,
                       int threads, int64_t *ptr, int32_t **cols);

/* Neighbour lists in the order src/SparseMat.cpp:599-609 builds them for a
 * FillAdjList run with `order_threads` threads (1 = fully sorted, which is also
 * the order AdjList::FromBinaryFile builds from a row-sorted edge file).
 * adj_ptr int64[n+1], adj int32[2*nnz]. */
void igo_adjacency(const int64_t *row_ptr, const int32_t *cols, int32_t n, int order_threads, int64_t *adj_ptr,
                   int32_t *adj);

/* Min-degree greedy of src/SparseMat.cpp:679-731 over adjacency lists; writes
 * the selected vertex ids in selection order and returns how many. */
int32_t igo_greedy(const int64_t *adj_ptr, const int32_t *adj, int32_t n, int32_t *order);

#ifdef __cplusplus
}
#endif
#endif
