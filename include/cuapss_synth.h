/*
 * cuapss_synth.h -- seeded synthetic sparse-vector generator (host, C ABI).
 *
 * The reference's input file (main.cu:270) is a pre-processed text corpus
 * that is not distributed; these generators produce seeded stand-ins with the
 * shapes and value distributions of the benchmark configurations:
 *   - nnz per row ~ lognormal with arithmetic mean m and log-sigma s
 *     (mu = ln m - s^2/2), rounded, clipped to [1, min(nnz_max, d)];
 *   - feature ids: Zipf(zipf_s) ranks drawn without replacement per row,
 *     mapped through a seeded permutation of [0, d), sorted ascending;
 *   - values 1 + ln(tf), tf ~ Geometric(tf_p) on {1, 2, ...}, each row
 *     L2-normalised in FP64 and stored as float32;
 *   - planted near-duplicates: a dup_frac share of rows are copies of a
 *     random earlier row with dup_drop of its entries dropped and each value
 *     scaled by U(dup_scale_lo, dup_scale_hi), then renormalised.
 * Every row is generated from its own counter-based random stream, so the
 * output does not depend on the number of host threads.
 */
#ifndef CUAPSS_SYNTH_H_
#define CUAPSS_SYNTH_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int64_t n;
  int64_t d;
  double nnz_mean;
  double nnz_sigma;
  int64_t nnz_max;
  double zipf_s;
  double tf_p;
  double dup_frac;
  double dup_drop;
  double dup_scale_lo;
  double dup_scale_hi;
  uint64_t seed;
  int64_t row_offset;  /* generate rows [row_offset, row_offset + n) of the
                          stream defined by seed (for appends / shards) */
  uint64_t stream;     /* 0: the rows of seed's stream; else an independent
                          row stream over the same feature permutation (one
                          per instance of a batch: same vocabulary, own rows
                          and own planted duplicates) */
} cuapss_synth_params;

/* Fill rowptr[0..n] (rowptr[0] = 0). Returns 0, or -1 on bad parameters. */
int cuapss_synth_rowptr(const cuapss_synth_params* p, int64_t* rowptr);

/* Fill col/val for the rows described by rowptr (from cuapss_synth_rowptr
 * with the same parameters). Returns 0, or -1 on bad parameters. */
int cuapss_synth_fill(const cuapss_synth_params* p, const int64_t* rowptr,
                      int32_t* col, float* val);

/* Number of host threads the generator uses (OpenMP). */
int cuapss_synth_threads(void);

#ifdef __cplusplus
}
#endif

#endif /* CUAPSS_SYNTH_H_ */
