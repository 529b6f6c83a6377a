// The reference's entry point as a compatibility shim (cuapss_compat.h):
// tile-ELL partitions in, one exact self-join over their union, pair counts
// per partition pair printed in the reference's format.
#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <numeric>
#include <utility>
#include <vector>

#include "cuapss.h"
#include "cuapss_compat.h"

namespace {

std::mutex g_mu;
float g_threshold = 0.3f;  // the reference's constant (similarity_search.cu:18)
bool g_have_counts = false;
int64_t g_counts[64] = {};

struct Part {
  const int* dim;
  const float* feature;
  const int* tile_start;
  int sum_vec, sum_feat, sum_tile;
};

}  // namespace

extern "C" int64_t cuapss_compat_tile_ell_to_csr(const int* dim, const float* feature,
                                                 const int* tile_start, int sum_vec,
                                                 int sum_tile, int64_t* rowptr, int32_t* col,
                                                 float* val) {
  if (sum_vec < 0 || sum_tile < 0 || !rowptr) return -1;
  if (sum_vec > 0 && (!dim || !feature || !tile_start || sum_tile < (sum_vec + 31) / 32)) return -1;
  rowptr[0] = 0;
  int64_t nnz = 0;
  std::vector<std::pair<int32_t, float>> row;
  for (int v = 0; v < sum_vec; ++v) {
    const int k = v / 32, lane = v % 32;
    const int64_t t0 = tile_start[k], t1 = tile_start[k + 1];
    if (t1 < t0 || (t1 - t0) % 32 != 0) return -1;
    const int64_t width = (t1 - t0) / 32;
    row.clear();
    for (int64_t j = 0; j < width; ++j) {
      const int d = dim[t0 + lane + 32 * j];
      if (d == -1) continue;  // padding of a shorter vector in the tile
      if (d < 0) return -1;
      row.emplace_back(d, feature[t0 + lane + 32 * j]);
    }
    std::sort(row.begin(), row.end(),
              [](const std::pair<int32_t, float>& a, const std::pair<int32_t, float>& b) {
                return a.first < b.first;
              });
    for (size_t m = 0; m < row.size(); ++m) {
      if (m > 0 && row[m].first == row[m - 1].first) return -1;
      if (col) col[nnz] = row[m].first;
      if (val) val[nnz] = row[m].second;
      ++nnz;
    }
    rowptr[v + 1] = nnz;
  }
  return nnz;
}

namespace {

// Parses the reference's text format (one vector per line, see
// cuapss_compat.h). For each vector calls row(entries); stops after
// max_rows vectors when max_rows >= 0. Returns false on a malformed line.
template <typename Row>
bool parse_text(const char* path, int64_t max_rows, Row row) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  std::vector<char> line;
  std::vector<std::pair<int32_t, float>> ent;
  bool ok = true;
  int64_t rows = 0;
  for (;;) {
    if (max_rows >= 0 && rows >= max_rows) break;
    line.clear();
    int c;
    while ((c = std::fgetc(f)) != EOF && c != '\n') line.push_back((char)c);
    if (c == EOF && line.empty()) break;  // end of file (no partial last vector)
    line.push_back('\0');
    ent.clear();
    // the reference consumes one character, then reads pairs while the
    // character after a pair is not the newline
    const char* q = line.size() > 1 ? line.data() + 1 : line.data() + line.size() - 1;
    while (*q) {
      char* e1 = nullptr;
      errno = 0;
      const long long d = std::strtoll(q, &e1, 10);
      if (e1 == q || errno || d < 0 || d > INT32_MAX) { ok = false; break; }
      char* e2 = nullptr;
      const float v = std::strtof(e1, &e2);
      if (e2 == e1) { ok = false; break; }
      ent.emplace_back((int32_t)d, v);
      q = e2;
      if (*q) ++q;  // the one character after the pair
    }
    if (!ok) break;
    std::sort(ent.begin(), ent.end(),
              [](const std::pair<int32_t, float>& a, const std::pair<int32_t, float>& b) {
                return a.first < b.first;
              });
    for (size_t m = 1; m < ent.size(); ++m)
      if (ent[m].first == ent[m - 1].first) ok = false;
    if (!ok) break;
    row(ent);
    ++rows;
    if (c == EOF) break;
  }
  std::fclose(f);
  return ok;
}

}  // namespace

extern "C" int cuapss_compat_text_size(const char* path, int64_t max_rows, int64_t* n_rows,
                                       int64_t* nnz, int64_t* d) {
  if (!path || !n_rows || !nnz || !d) return -1;
  int64_t n = 0, m = 0, dmax = 0;
  const bool ok = parse_text(path, max_rows, [&](const std::vector<std::pair<int32_t, float>>& e) {
    ++n;
    m += (int64_t)e.size();
    if (!e.empty()) dmax = std::max<int64_t>(dmax, (int64_t)e.back().first + 1);
  });
  if (!ok) return -1;
  *n_rows = n;
  *nnz = m;
  *d = dmax;
  return 0;
}

extern "C" int cuapss_compat_read_text(const char* path, int64_t max_rows, int64_t* rowptr,
                                       int32_t* col, float* val) {
  if (!path || !rowptr) return -1;
  int64_t n = 0, m = 0;
  rowptr[0] = 0;
  const bool ok = parse_text(path, max_rows, [&](const std::vector<std::pair<int32_t, float>>& e) {
    for (const auto& pr : e) {
      col[m] = pr.first;
      val[m] = pr.second;
      ++m;
    }
    rowptr[++n] = m;
  });
  return ok ? 0 : -1;
}

extern "C" int cuapss_compat_write_text(const char* path, int64_t n, const int64_t* rowptr,
                                        const int32_t* col, const float* val) {
  if (!path || n < 0 || (n > 0 && !rowptr)) return -1;
  FILE* f = std::fopen(path, "wb");
  if (!f) return -1;
  bool ok = true;
  for (int64_t r = 0; r < n && ok; ++r) {
    for (int64_t e = rowptr[r]; e < rowptr[r + 1] && ok; ++e)
      ok = std::fprintf(f, " %d %.9g", (int)col[e], (double)val[e]) > 0;
    ok = ok && std::fputc('\n', f) != EOF;
  }
  ok = (std::fclose(f) == 0) && ok;
  return ok ? 0 : -1;
}

extern "C" void cuapss_compat_set_threshold(float t) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_threshold = t;
}

extern "C" int cuapss_compat_counts(int64_t counts[64]) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_have_counts) return -1;
  std::copy(g_counts, g_counts + 64, counts);
  return 0;
}

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
                            int* apss_seg_start) {
  (void)pre_norm_A1, (void)pre_norm_B1, (void)pre_norm_C1, (void)pre_norm_D1;
  (void)pre_norm_E1, (void)pre_norm_F1, (void)pre_norm_G1, (void)pre_norm_H1;
  (void)b_id_a, (void)apss_block_seg, (void)apss_seg_start;
  const Part parts[8] = {{dim_A, feature_A, tile_start_A, sum_vec_A, sum_feat_A, sum_tile_A},
                         {dim_B, feature_B, tile_start_B, sum_vec_B, sum_feat_B, sum_tile_B},
                         {dim_C, feature_C, tile_start_C, sum_vec_C, sum_feat_C, sum_tile_C},
                         {dim_D, feature_D, tile_start_D, sum_vec_D, sum_feat_D, sum_tile_D},
                         {dim_E, feature_E, tile_start_E, sum_vec_E, sum_feat_E, sum_tile_E},
                         {dim_F, feature_F, tile_start_F, sum_vec_F, sum_feat_F, sum_tile_F},
                         {dim_G, feature_G, tile_start_G, sum_vec_G, sum_feat_G, sum_tile_G},
                         {dim_H, feature_H, tile_start_H, sum_vec_H, sum_feat_H, sum_tile_H}};
  float t;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    t = g_threshold;
  }
  // ---- tile-ELL -> one CSR (partition X's rows follow partition X-1's)
  int64_t n = 0, cap = 0;
  int64_t first[9] = {};
  for (int x = 0; x < 8; ++x) {
    first[x] = n;
    n += std::max(parts[x].sum_vec, 0);
    cap += std::max(parts[x].sum_feat, 0);
  }
  first[8] = n;
  std::vector<int64_t> rp((size_t)n + 1, 0);
  std::vector<int32_t> col((size_t)std::max<int64_t>(cap, 1));
  std::vector<float> val((size_t)std::max<int64_t>(cap, 1));
  int64_t nnz = 0;
  for (int x = 0; x < 8; ++x) {
    const Part& P = parts[x];
    if (P.sum_vec <= 0) continue;
    std::vector<int64_t> prp((size_t)P.sum_vec + 1);
    const int64_t m = cuapss_compat_tile_ell_to_csr(P.dim, P.feature, P.tile_start, P.sum_vec,
                                                    P.sum_tile, prp.data(), col.data() + nnz,
                                                    val.data() + nnz);
    if (m < 0 || nnz + m > cap) {
      fprintf(stderr, "similarity_join_device: malformed tile-ELL layout in partition %c\n",
              'A' + x);
      return;
    }
    for (int v = 0; v < P.sum_vec; ++v) rp[first[x] + v + 1] = nnz + prp[v + 1];
    nnz += m;
  }
  int32_t d = 1;
  for (int64_t e = 0; e < nnz; ++e) d = std::max(d, col[e] + 1);
  // ---- one exact self-join
  cuapss_opts o;
  cuapss_default_opts(&o);
  o.precision = CUAPSS_PREC_MIXED;
  o.validate = 0;  // the reference takes the dot product of the rows as given
  cuapss_ctx* ctx = nullptr;
  cuapss_status s = cuapss_create(&ctx, &o);
  if (s != CUAPSS_OK) {
    fprintf(stderr, "similarity_join_device: %s\n", cuapss_status_string(s));
    return;
  }
  cuapss_csr x{n, d, nnz, rp.data(), col.data(), val.data(), 0};
  int64_t pcap = std::max<int64_t>(1 << 16, n);
  std::vector<int32_t> pi, pj;
  std::vector<float> ps;
  cuapss_pairs out{};
  for (int attempt = 0; attempt < 2; ++attempt) {
    pi.resize((size_t)pcap);
    pj.resize((size_t)pcap);
    ps.resize((size_t)pcap);
    out = cuapss_pairs{pi.data(), pj.data(), ps.data(), pcap, 0, 0};
    s = cuapss_run(ctx, &x, t, &out, nullptr);
    if (s != CUAPSS_EOVERFLOW) break;
    pcap = out.count;
  }
  cuapss_destroy(ctx);
  if (s != CUAPSS_OK) {
    fprintf(stderr, "similarity_join_device: %s\n", cuapss_status_string(s));
    return;
  }
  // ---- counts per partition pair, printed as the reference does
  int64_t counts[64] = {};
  auto part_of = [&](int64_t r) {
    return (int)(std::upper_bound(first, first + 9, r) - first) - 1;
  };
  for (int64_t k = 0; k < out.count; ++k) {
    const int a = part_of(pi[k]), b = part_of(pj[k]);
    ++counts[8 * std::min(a, b) + std::max(a, b)];
  }
  for (int a = 0; a < 8; ++a)
    for (int b = a + 1; b < 8; ++b)
      printf("par_%c join par_%c: sum pair=%lld\n\n", 'A' + a, 'A' + b,
             (long long)counts[8 * a + b]);
  for (int a = 0; a < 8; ++a)
    printf("par_%c apss: sum pair=%lld\n\n", 'A' + a, (long long)counts[9 * a]);
  fflush(stdout);
  std::lock_guard<std::mutex> lk(g_mu);
  std::copy(counts, counts + 64, g_counts);
  g_have_counts = true;
}
