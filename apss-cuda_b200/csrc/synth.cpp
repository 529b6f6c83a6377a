// Seeded synthetic CSR generator for the APSS benchmark configurations.
// Host-only C++ with OpenMP; every row draws from its own counter-based
// stream so results are independent of the thread count.
#include "cuapss_synth.h"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace {

constexpr uint64_t kTagPerm = 0x5045524d554c4154ull;
constexpr uint64_t kTagNnz = 0x4e4e5a434f554e54ull;
constexpr uint64_t kTagRow = 0x524f57434f4e5445ull;
constexpr uint64_t kTagDup = 0x4455504c49434154ull;
constexpr uint64_t kTagDupRow = 0x445550524f574f50ull;

inline uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// splitmix64 stream keyed by (seed, tag, index)
struct Rng {
  uint64_t s;
  Rng(uint64_t seed, uint64_t tag, uint64_t idx)
      : s(mix64(seed ^ mix64(tag + 0x9e3779b97f4a7c15ull * (idx + 1)))) {}
  uint64_t next() {
    s += 0x9e3779b97f4a7c15ull;
    return mix64(s);
  }
  double uniform() { return (double)(next() >> 11) * 0x1.0p-53; }  // [0,1)
  double normal() {
    double u1 = 1.0 - uniform();  // (0,1]
    double u2 = uniform();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
};

// Seed of the per-row streams: the table seed itself, or (stream != 0) an
// independent stream over the same feature permutation.
inline uint64_t row_seed(const cuapss_synth_params* p) {
  return p->stream == 0 ? p->seed : mix64(p->seed ^ mix64(0x53545245414dull + p->stream));
}

struct Tables {
  std::vector<double> cdf;     // cdf[r], r = 0..d-1 (rank r+1)
  std::vector<int32_t> guide;  // guide[b] = smallest r with cdf[r] > b/G
  std::vector<int32_t> perm;   // rank -> feature id
};

bool valid(const cuapss_synth_params* p) {
  return p && p->n >= 0 && p->d >= 1 && p->d <= (int64_t)INT32_MAX &&
         p->nnz_mean > 0 && p->nnz_sigma >= 0 && p->nnz_max >= 1 &&
         p->zipf_s >= 0 && p->tf_p > 0 && p->tf_p < 1 && p->dup_frac >= 0 &&
         p->dup_frac <= 1 && p->dup_drop >= 0 && p->dup_drop < 1 &&
         p->dup_scale_lo > 0 && p->dup_scale_hi >= p->dup_scale_lo &&
         p->row_offset >= 0;
}

void build_tables(const cuapss_synth_params* p, Tables* t) {
  const int64_t d = p->d;
  t->cdf.resize(d);
  double acc = 0.0;
  for (int64_t r = 0; r < d; ++r) {
    acc += std::pow((double)(r + 1), -p->zipf_s);
    t->cdf[r] = acc;
  }
  for (int64_t r = 0; r < d; ++r) t->cdf[r] /= acc;
  t->cdf[d - 1] = 1.0;
  const int64_t G = std::max<int64_t>(d, 1024);
  t->guide.resize(G);
  int64_t r = 0;
  for (int64_t b = 0; b < G; ++b) {
    const double lo = (double)b / (double)G;
    while (r < d - 1 && t->cdf[r] <= lo) ++r;
    t->guide[b] = (int32_t)r;
  }
  t->perm.resize(d);
  for (int64_t i = 0; i < d; ++i) t->perm[i] = (int32_t)i;
  Rng rng(p->seed, kTagPerm, 0);
  for (int64_t i = d - 1; i > 0; --i) {
    int64_t j = (int64_t)(rng.uniform() * (double)(i + 1));
    if (j > i) j = i;
    std::swap(t->perm[i], t->perm[j]);
  }
}

inline int32_t zipf_rank(const Tables& t, double u) {
  const int64_t G = (int64_t)t.guide.size();
  int64_t b = (int64_t)(u * (double)G);
  if (b >= G) b = G - 1;
  int64_t r = t.guide[b];
  const int64_t d = (int64_t)t.cdf.size();
  while (r < d - 1 && t.cdf[r] <= u) ++r;
  return (int32_t)r;
}

int64_t orig_nnz(const cuapss_synth_params* p, int64_t row) {
  Rng rng(row_seed(p), kTagNnz, (uint64_t)row);
  const double mu = std::log(p->nnz_mean) - 0.5 * p->nnz_sigma * p->nnz_sigma;
  const double x = std::exp(mu + p->nnz_sigma * rng.normal());
  int64_t k = (int64_t)std::llround(x);
  const int64_t kmax = std::min<int64_t>(p->nnz_max, p->d);
  if (k < 1) k = 1;
  if (k > kmax) k = kmax;
  return k;
}

// Returns base row (>= 0) if `row` is a planted duplicate, else -1.
int64_t dup_base(const cuapss_synth_params* p, int64_t row) {
  if (row <= 0 || p->dup_frac <= 0) return -1;
  Rng rng(row_seed(p), kTagDup, (uint64_t)row);
  if (rng.uniform() >= p->dup_frac) return -1;
  int64_t b = (int64_t)(rng.uniform() * (double)row);
  if (b >= row) b = row - 1;
  return b;
}

inline int64_t dup_keep(const cuapss_synth_params* p, int64_t k) {
  int64_t drop = (int64_t)std::floor(p->dup_drop * (double)k);
  if (k - drop < 1) drop = k - 1;
  return k - drop;
}

struct Scratch {
  std::vector<int32_t> slots;  // open-addressing set of ranks, -1 = empty
  std::vector<int32_t> ids;
  std::vector<double> vals;
  std::vector<int32_t> idx;
};

// Original (non-duplicate) content of `row`: sorted ids and FP64 values with
// unit norm.
void orig_row(const cuapss_synth_params* p, const Tables& t, int64_t row,
              Scratch* s) {
  const int64_t k = orig_nnz(p, row);
  Rng rng(row_seed(p), kTagRow, (uint64_t)row);
  int64_t cap = 16;
  while (cap < 2 * k) cap <<= 1;
  s->slots.assign(cap, -1);
  s->ids.clear();
  const uint64_t mask = (uint64_t)cap - 1;
  while ((int64_t)s->ids.size() < k) {
    const int32_t r = zipf_rank(t, rng.uniform());
    uint64_t h = mix64((uint64_t)r) & mask;
    bool fresh = true;
    while (s->slots[h] != -1) {
      if (s->slots[h] == r) {
        fresh = false;
        break;
      }
      h = (h + 1) & mask;
    }
    if (fresh) {
      s->slots[h] = r;
      s->ids.push_back(t.perm[r]);
    }
  }
  std::sort(s->ids.begin(), s->ids.end());
  s->vals.resize(k);
  const double lq = std::log(1.0 - p->tf_p);
  double ss = 0.0;
  for (int64_t e = 0; e < k; ++e) {
    const double u = rng.uniform();
    const double tf = 1.0 + std::floor(std::log(1.0 - u) / lq);
    const double v = 1.0 + std::log(tf);
    s->vals[e] = v;
    ss += v * v;
  }
  const double inv = 1.0 / std::sqrt(ss);
  for (int64_t e = 0; e < k; ++e) s->vals[e] *= inv;
}

const Tables* get_tables(const cuapss_synth_params* p, Tables* storage) {
  build_tables(p, storage);
  return storage;
}

}  // namespace

extern "C" int cuapss_synth_threads(void) { return omp_get_max_threads(); }

extern "C" int cuapss_synth_rowptr(const cuapss_synth_params* p,
                                   int64_t* rowptr) {
  if (!valid(p) || !rowptr) return -1;
  const int64_t n = p->n;
  std::vector<int64_t> cnt(n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const int64_t row = p->row_offset + i;
    const int64_t b = dup_base(p, row);
    cnt[i] = b >= 0 ? dup_keep(p, orig_nnz(p, b)) : orig_nnz(p, row);
  }
  rowptr[0] = 0;
  for (int64_t i = 0; i < n; ++i) rowptr[i + 1] = rowptr[i] + cnt[i];
  return 0;
}

extern "C" int cuapss_synth_fill(const cuapss_synth_params* p,
                                 const int64_t* rowptr, int32_t* col,
                                 float* val) {
  if (!valid(p) || !rowptr || (p->n > 0 && (!col || !val))) return -1;
  Tables tables;
  const Tables& t = *get_tables(p, &tables);
  const int64_t n = p->n;
  int bad = 0;
#pragma omp parallel
  {
    Scratch s;
#pragma omp for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; ++i) {
      const int64_t row = p->row_offset + i;
      const int64_t b = dup_base(p, row);
      const int64_t off = rowptr[i];
      const int64_t len = rowptr[i + 1] - rowptr[i];
      if (b < 0) {
        orig_row(p, t, row, &s);
        if ((int64_t)s.ids.size() != len) {
#pragma omp atomic write
          bad = 1;
          continue;
        }
        for (int64_t e = 0; e < len; ++e) {
          col[off + e] = s.ids[e];
          val[off + e] = (float)s.vals[e];
        }
      } else {
        orig_row(p, t, b, &s);
        const int64_t k = (int64_t)s.ids.size();
        const int64_t keep = dup_keep(p, k);
        if (keep != len) {
#pragma omp atomic write
          bad = 1;
          continue;
        }
        Rng rng(row_seed(p), kTagDupRow, (uint64_t)row);
        s.idx.resize(k);
        for (int64_t e = 0; e < k; ++e) s.idx[e] = (int32_t)e;
        // partial Fisher-Yates: the first k-keep slots are the dropped ones
        for (int64_t e = 0; e < k - keep; ++e) {
          int64_t j = e + (int64_t)(rng.uniform() * (double)(k - e));
          if (j >= k) j = k - 1;
          std::swap(s.idx[e], s.idx[j]);
        }
        std::sort(s.idx.begin() + (k - keep), s.idx.end());
        double ss = 0.0;
        std::vector<double>& v = s.vals;
        for (int64_t e = 0; e < keep; ++e) {
          const int32_t src = s.idx[k - keep + e];
          const double sc =
              p->dup_scale_lo + (p->dup_scale_hi - p->dup_scale_lo) * rng.uniform();
          const double x = v[src] * sc;
          col[off + e] = s.ids[src];
          v[src] = x;
          ss += x * x;
        }
        const double inv = 1.0 / std::sqrt(ss);
        for (int64_t e = 0; e < keep; ++e) {
          const int32_t src = s.idx[k - keep + e];
          val[off + e] = (float)(v[src] * inv);
        }
      }
    }
  }
  return bad ? -1 : 0;
}
