/*
 * oracle.h -- CPU restatement of the reference's all-pairs similarity search,
 * used ONLY as test infrastructure (the checker) and as the timed CPU
 * baseline. The product path never links or calls it.
 *
 * What each function follows in the reference (fengyilin118/APSS-CUDA):
 *  - oracle_apss_fp64 / oracle_join_fp64: the definition in README.md:2 (all
 *    pairs with cosine similarity >= t) and the intended accept rule of
 *    similarity_apss_rest / similarity_join_rest (similarity_search.cu:498,
 *    907: "acc + dot >= t"; self-join pairs are unordered, m > n at 704/888),
 *    accumulated like InvertedIndex_search (main.cu:104-141: for every
 *    feature of the query, walk that feature's inverted list and add
 *    x_q * x_c to the candidate's accumulator), but in FP64 and without the
 *    reference's dropped work (B3/B4: half the candidates of a chunk and
 *    entries 512..1023 of long rows are skipped there; B5: its prune uses
 *    <= t). Accumulation order for a pair is ascending feature id, which the
 *    GPU's FP64 rescore reproduces bit for bit.
 *  - oracle_index_ref: generate_index_ptr4 (similarity_search.cu:105-191:
 *    count postings of features >= p), the host exclusive scan (1168-1186)
 *    and construct_Index2 (221-274: scatter (row, value) at an atomic
 *    cursor). The reference's lists come out in nondeterministic order; this
 *    restatement emits them sorted by row, the canonical form compared.
 *  - oracle_feature_remap: no counterpart (the reference fixes the head to
 *    ids < 4096, similarity_search.cu:130 etc.); the frequency order is
 *    (count descending, id ascending).
 *  - cpu_hybrid_apss: the reference's hybrid method on the host, FP32, with
 *    OpenMP: tail features (rank >= p) accumulated through inverted lists
 *    (similarity_apss1, similarity_search.cu:642-735), the Cauchy-Schwarz
 *    prune on head norms (filter_pair_apss, 833-852, with >= instead of
 *    B5's <=), then the head dot per surviving pair against a dense copy of
 *    the query's head (similarity_apss_rest, 854-915) and the threshold.
 *    This is the timed CPU baseline, not a parity oracle.
 */
#ifndef CUAPSS_ORACLE_H_
#define CUAPSS_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Self-join in FP64. Writes up to cap pairs (i < j) sorted by (i, j) into
 * oi/oj/os; returns the total number found (may exceed cap: then only the
 * first cap are written). Returns -1 on malformed input. */
int64_t oracle_apss_fp64(int64_t n, int64_t d, const int64_t* rowptr,
                         const int32_t* col, const float* val, double t,
                         int64_t cap, int32_t* oi, int32_t* oj, double* os);

/* Cross-join A x B in FP64; (i in A, j in B), sorted by (i, j). */
int64_t oracle_join_fp64(int64_t na, const int64_t* arp, const int32_t* acol,
                         const float* aval, int64_t nb, const int64_t* brp,
                         const int32_t* bcol, const float* bval, int64_t d,
                         double t, int64_t cap, int32_t* oi, int32_t* oj,
                         double* os);

/* FP64 similarity of given pairs, merge of the two sorted rows in ascending
 * feature order (same arithmetic as oracle_apss_fp64). */
void oracle_pair_sims(const int64_t* rowptr, const int32_t* col,
                      const float* val, int64_t m, const int32_t* pi,
                      const int32_t* pj, double* out);

/* For each query row q in rows[0..m): every other row j (j != q) with FP64
 * similarity >= t. Output pairs (min, max) sorted by (i, j), deduplicated
 * when both ends are query rows. Scales to large n for sampled checks. */
int64_t oracle_rows_fp64(int64_t n, int64_t d, const int64_t* rowptr,
                         const int32_t* col, const float* val, double t,
                         int64_t m, const int32_t* rows, int64_t cap,
                         int32_t* oi, int32_t* oj, double* os);

/* Reference-semantics tail index (see header comment). dim_ptr[d+1];
 * idx_row/idx_val sized >= number of entries with col >= p. Returns that
 * number, or -1. */
int64_t oracle_index_ref(int64_t n, int64_t d, const int64_t* rowptr,
                         const int32_t* col, const float* val, int32_t p,
                         int32_t* dim_ptr, int32_t* idx_row, float* idx_val);

/* counts[f] = postings of f; perm[f] = rank of f in (count desc, id asc). */
void oracle_feature_remap(int64_t n, int64_t d, const int64_t* rowptr,
                          const int32_t* col, int32_t* perm, int32_t* counts);

/* OpenMP FP32 hybrid baseline over query rows [q0, q1) against all j > i.
 * p = head width after the frequency remap. Returns the number of pairs with
 * FP32 similarity >= t (pairs are counted, not stored). threads <= 0: all.
 * sec_prep / sec_query (may be NULL) receive the wall seconds of the
 * preprocessing (remap, re-sort, inverted lists) and of the query loop. */
int64_t cpu_hybrid_apss(int64_t n, int64_t d, const int64_t* rowptr,
                        const int32_t* col, const float* val, float t,
                        int32_t p, int64_t q0, int64_t q1, int threads,
                        double* sec_prep, double* sec_query);

/* The same baseline split in two: the preprocessing once (the handle keeps
 * pointers to rowptr, which must outlive it), then queries over any rows:
 * qrows[0..m) when qrows is non-NULL, else rows q0 .. q0 + m - 1. */
typedef struct cpu_hybrid cpu_hybrid_t;
cpu_hybrid_t* cpu_hybrid_prepare(int64_t n, int64_t d, const int64_t* rowptr,
                                 const int32_t* col, const float* val,
                                 int32_t p, int threads, double* sec_prep);
int64_t cpu_hybrid_query(const cpu_hybrid_t* h, float t, int64_t m,
                         const int64_t* qrows, int64_t q0, int threads,
                         double* sec_query);
void cpu_hybrid_free(cpu_hybrid_t* h);

/* Threads OpenMP will use for threads <= 0. */
int oracle_max_threads(void);

#ifdef __cplusplus
}
#endif

#endif
