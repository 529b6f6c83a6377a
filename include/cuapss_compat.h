/*
 * cuapss_compat.h -- the reference's entry point, kept as a compatibility
 * shim over the C ABI of cuapss.h.
 *
 * similarity_join_device has the exact signature of fengyilin118/APSS-CUDA
 * similarity_search.h:3-14 (C++ linkage, as there), so a caller of the
 * reference relinks against libcuapss.so unchanged. It reads the eight
 * partitions in the reference's tile-ELL layout (main.cu:269-340: vectors in
 * tiles of 32, entry j of vector v at tile_start[v / 32] + v % 32 + 32 j,
 * tile width (tile_start[k + 1] - tile_start[k]) / 32, unused slots holding
 * feature id -1), converts them to one CSR matrix (partition X's vector v is
 * row offset_X + v), runs one exact self-join at the reference's threshold
 * (the constant threhold = 0.3, similarity_search.cu:18) and prints the pair
 * count of every partition pair in the reference's format
 * ("par_A join par_B: sum pair=%d", similarity_search.cu:1342 ...;
 * "par_A apss: sum pair=%d", similarity_search.cu:2687 ...).
 *
 * Differences, by design: the counts are exact (the reference emits no pairs
 * and skips candidates); pre_norm_*, b_id_a, apss_block_seg and
 * apss_seg_start are accepted and ignored (the library computes its own head
 * norms and schedule); rows are taken as given (no normalisation check, the
 * similarity is the dot product, as in the reference).
 */
#ifndef CUAPSS_COMPAT_H_
#define CUAPSS_COMPAT_H_

#include <stdint.h>

#ifdef __cplusplus
void similarity_join_device(int* dim_A, float* feature_A, int* tile_start_A, int* dim_B,
                            float* feature_B, int* tile_start_B, int* dim_C, float* feature_C,
                            int* tile_start_C, int* dim_D, float* feature_D, int* tile_start_D,
                            int* dim_E, float* feature_E, int* tile_start_E, int* dim_F,
                            float* feature_F, int* tile_start_F, int* dim_G, float* feature_G,
                            int* tile_start_G, int* dim_H, float* feature_H, int* tile_start_H,
                            float* pre_norm_A1, float* pre_norm_B1, float* pre_norm_C1,
                            float* pre_norm_D1, float* pre_norm_E1, float* pre_norm_F1,
                            float* pre_norm_G1, float* pre_norm_H1, int sum_vec_A, int sum_feat_A,
                            int sum_tile_A, int sum_vec_B, int sum_feat_B, int sum_tile_B,
                            int sum_vec_C, int sum_feat_C, int sum_tile_C, int sum_vec_D,
                            int sum_feat_D, int sum_tile_D, int sum_vec_E, int sum_feat_E,
                            int sum_tile_E, int sum_vec_F, int sum_feat_F, int sum_tile_F,
                            int sum_vec_G, int sum_feat_G, int sum_tile_G, int sum_vec_H,
                            int sum_feat_H, int sum_tile_H, int* b_id_a, int* apss_block_seg,
                            int* apss_seg_start);
extern "C" {
#endif

/* Threshold of later similarity_join_device calls (default 0.3). No
 * counterpart in the reference (a compile-time constant there). */
void cuapss_compat_set_threshold(float t);

/* Pair counts of the last successful similarity_join_device call:
 * counts[8 * X + Y] for partitions X <= Y (X == Y: within X). Returns 0, or
 * -1 when no call has succeeded. No counterpart in the reference. */
int cuapss_compat_counts(int64_t counts[64]);

/* One partition in tile-ELL layout -> CSR with ascending feature ids (host).
 * rowptr has sum_vec + 1 entries; col/val need room for the partition's
 * non-padding entries (at most tile_start[sum_tile]). Returns nnz, or -1 on a
 * malformed layout (tile bounds, negative width, repeated feature id in one
 * vector). Restates the reference loader's layout (main.cu:269-340). */
int64_t cuapss_compat_tile_ell_to_csr(const int* dim, const float* feature, const int* tile_start,
                                      int sum_vec, int sum_tile, int64_t* rowptr, int32_t* col,
                                      float* val);

/* The reference's input text format (main.cu:301-323): one vector per line.
 * A line is empty (an empty vector) or one separator character followed by
 * "d v" pairs (feature id, value; any whitespace between them), each pair
 * followed by one character: a separator, or the line's newline. The
 * reference reads it with `input.get(ch); while (ch != '\n') { input >> d >> v;
 * ...; input.get(ch); }` for each vector.
 *
 * cuapss_compat_text_size scans the file: *n_rows = vectors (at most
 * max_rows when max_rows >= 0), *nnz = their entries, *d = largest feature id
 * + 1. cuapss_compat_read_text then fills a CSR of those vectors (rowptr
 * n_rows + 1, col/val nnz), each row sorted by feature id. Both return 0, or
 * -1 when the file cannot be read or a line is malformed (a token that is
 * not a number, a negative id, an id repeated within a vector, a missing
 * value). No counterpart in the reference, which parses inline in main(). */
int cuapss_compat_text_size(const char* path, int64_t max_rows, int64_t* n_rows, int64_t* nnz,
                            int64_t* d);
int cuapss_compat_read_text(const char* path, int64_t max_rows, int64_t* rowptr, int32_t* col,
                            float* val);

/* Writes n CSR rows in that text format (separator ' ', values printed with
 * 9 significant digits, which round-trip FP32 exactly). Returns 0, or -1 on
 * an I/O error. */
int cuapss_compat_write_text(const char* path, int64_t n, const int64_t* rowptr,
                             const int32_t* col, const float* val);

#ifdef __cplusplus
}
#endif

#endif /* CUAPSS_COMPAT_H_ */
