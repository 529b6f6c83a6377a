// Harness around the reference's own serial CPU search, InvertedIndex_search
// (main.cu:104-141 of fengyilin118/APSS-CUDA). The reference source is
// compiled as-is from its own tree by oracle/Makefile (never copied into this
// repository); this file only fills the reference's globals and calls it.
//
// InvertedIndex_search walks, for every vector of partition B (global `pB`),
// the inverted lists of partition E (global `inverted_index_E`), accumulates
// x_b * x_e per candidate in a std::map<int,float>, and prints
// "sum_pair=<count of candidates with accumulated value >= 0.8>".
//
// usage: ref_cpu_search <B.csr> <E.csr>   (binary CSR files, see read_csr)
// stdout: the reference's own output ("sum_pair=N" is its last line), then
// "search_seconds=S", the wall time of the InvertedIndex_search call alone.
// main.cu relies on nvcc pulling in <cstring>; a host compiler needs it here.
#include <cstring>
#define main cuapss_reference_main_unused
#include "main.cu"
#undef main

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <vector>

namespace {

struct Csr {
  int64_t n = 0, d = 0, nnz = 0;
  std::vector<int64_t> rowptr;
  std::vector<int32_t> col;
  std::vector<float> val;
};

// File layout: int64 n, d, nnz; int64 rowptr[n+1]; int32 col[nnz];
// float32 val[nnz].
bool read_csr(const char* path, Csr* c) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  int64_t h[3];
  bool ok = std::fread(h, sizeof(int64_t), 3, f) == 3;
  if (ok) {
    c->n = h[0];
    c->d = h[1];
    c->nnz = h[2];
    c->rowptr.resize(c->n + 1);
    c->col.resize(c->nnz);
    c->val.resize(c->nnz);
    ok = std::fread(c->rowptr.data(), sizeof(int64_t), c->n + 1, f) == (size_t)(c->n + 1) &&
         std::fread(c->col.data(), sizeof(int32_t), c->nnz, f) == (size_t)c->nnz &&
         std::fread(c->val.data(), sizeof(float), c->nnz, f) == (size_t)c->nnz;
  }
  std::fclose(f);
  return ok;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s B.csr E.csr\n", argv[0]);
    return 2;
  }
  Csr b, e;
  if (!read_csr(argv[1], &b) || !read_csr(argv[2], &e)) {
    std::fprintf(stderr, "cannot read input\n");
    return 2;
  }
  if (b.d > max_dims || e.d > max_dims) {
    std::fprintf(stderr, "d exceeds the reference's max_dims (%d)\n", max_dims);
    return 2;
  }
  initial();  // sizes the reference's inverted lists to max_dims
  for (int64_t r = 0; r < e.n; ++r)
    for (int64_t k = e.rowptr[r]; k < e.rowptr[r + 1]; ++k)
      inverted_index_E[e.col[k]].terms.push_back(new Term((int)r, e.val[k]));
  std::vector<std::pair<int, double> > feats;
  for (int64_t r = 0; r < b.n; ++r) {
    feats.clear();
    double mx = -9999.0, norm1 = 0.0;
    for (int64_t k = b.rowptr[r]; k < b.rowptr[r + 1]; ++k) {
      feats.push_back(std::pair<int, double>(b.col[k], (double)b.val[k]));
      if (b.val[k] > mx) mx = b.val[k];
      norm1 += b.val[k];
    }
    pB.addVector((int)r, (int)feats.size(), mx, norm1,
                 feats.empty() ? nullptr : &feats[0]);
  }
  const auto t0 = std::chrono::steady_clock::now();
  InvertedIndex_search();
  const auto t1 = std::chrono::steady_clock::now();
  std::printf("search_seconds=%.6f\n",
              std::chrono::duration<double>(t1 - t0).count());
  std::fflush(stdout);
  return 0;
}
