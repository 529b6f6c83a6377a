// Harness around the reference's own inverted-index build kernels
// (fengyilin118/APSS-CUDA similarity_search.cu): generate_index_ptr4
// (105-191) counts the postings of every feature >= 4096, the host exclusive
// scan (1168-1186) turns counts into dim_ptr, construct_Index2 (221-274)
// scatters (row, value) at an atomic cursor. The reference source is compiled
// from its own tree by oracle/Makefile (never copied here); this file builds
// the tile-ELL input those kernels read (32-row tiles, element j of row r at
// tile_start + r%32 + 32*j, padded with -1, as main.cu:269-336 lays it out),
// zeroes the counters (the reference leaves them uninitialised, which is its
// bug B1), launches the two kernels with the reference's grid arithmetic
// (1077-1090, 1228-1254) and writes the index with every list sorted by row
// (the reference's list order is nondeterministic).
//
// Inputs must satisfy the kernels' fixed limits: feature ids < max_dim
// (198456); the head split is the reference's constant 4096.
//
// usage: ref_index <in.csr> <out.idx>
// out.idx: int64 d, int64 total; int32 dim_ptr[max_dim+1]; int32 row[total];
//          float32 val[total].
#include "similarity_search.cu"

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <vector>

namespace {

bool read_csr(const char* path, int64_t* n, int64_t* d, std::vector<int64_t>* rp,
              std::vector<int32_t>* col, std::vector<float>* val) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  int64_t h[3];
  bool ok = std::fread(h, sizeof(int64_t), 3, f) == 3;
  if (ok) {
    *n = h[0];
    *d = h[1];
    rp->resize(h[0] + 1);
    col->resize(h[2]);
    val->resize(h[2]);
    ok = std::fread(rp->data(), 8, h[0] + 1, f) == (size_t)(h[0] + 1) &&
         std::fread(col->data(), 4, h[2], f) == (size_t)h[2] &&
         std::fread(val->data(), 4, h[2], f) == (size_t)h[2];
  }
  std::fclose(f);
  return ok;
}

#define CK(x)                                                              \
  do {                                                                     \
    cudaError_t e_ = (x);                                                  \
    if (e_ != cudaSuccess) {                                               \
      std::fprintf(stderr, "%s failed: %s\n", #x, cudaGetErrorString(e_)); \
      return 1;                                                            \
    }                                                                      \
  } while (0)

}  // namespace

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s in.csr out.idx\n", argv[0]);
    return 2;
  }
  int64_t n = 0, d = 0;
  std::vector<int64_t> rp;
  std::vector<int32_t> col;
  std::vector<float> val;
  if (!read_csr(argv[1], &n, &d, &rp, &col, &val)) return 2;
  if (d > max_dim || n <= 0 || n > (1 << 30)) {
    std::fprintf(stderr, "input outside the reference kernels' limits\n");
    return 2;
  }
  for (int32_t c : col)
    if (c < 0 || c >= max_dim) return 2;
  // tile-ELL: tile width = widest row of the tile
  const int64_t ntiles = (n + 31) / 32;
  std::vector<int> tile_start(ntiles + 1, 0);
  for (int64_t t = 0; t < ntiles; ++t) {
    int64_t w = 0;
    for (int64_t r = t * 32; r < std::min<int64_t>(n, t * 32 + 32); ++r)
      w = std::max<int64_t>(w, rp[r + 1] - rp[r]);
    tile_start[t + 1] = tile_start[t] + (int)(32 * w);
  }
  const int64_t slots = tile_start[ntiles];
  std::vector<int> dim(std::max<int64_t>(slots, 1), -1);
  std::vector<float> feat(std::max<int64_t>(slots, 1), 0.0f);
  for (int64_t r = 0; r < n; ++r)
    for (int64_t k = rp[r]; k < rp[r + 1]; ++k) {
      const int64_t j = k - rp[r];
      dim[tile_start[r / 32] + r % 32 + 32 * j] = col[k];
      feat[tile_start[r / 32] + r % 32 + 32 * j] = val[k];
    }
  int *dim_d, *tile_d, *num_d, *ptr_d, *dummy_d;
  float* feat_d;
  CK(cudaMalloc(&dim_d, sizeof(int) * dim.size()));
  CK(cudaMalloc(&feat_d, sizeof(float) * feat.size()));
  CK(cudaMalloc(&tile_d, sizeof(int) * tile_start.size()));
  CK(cudaMalloc(&num_d, sizeof(int) * max_dim));
  CK(cudaMalloc(&ptr_d, sizeof(int) * (max_dim + 1)));
  CK(cudaMalloc(&dummy_d, sizeof(int) * (max_dim + 1)));
  CK(cudaMemcpy(dim_d, dim.data(), sizeof(int) * dim.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(feat_d, feat.data(), sizeof(float) * feat.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(tile_d, tile_start.data(), sizeof(int) * tile_start.size(),
                cudaMemcpyHostToDevice));
  CK(cudaMemset(num_d, 0, sizeof(int) * max_dim));
  CK(cudaMemset(dummy_d, 0, sizeof(int) * (max_dim + 1)));
  const int sum_vec = (int)n;
  // partitions B, C, D are empty: their blocks see vec_id >= 0 == sum_vec
  const int grid1 = sum_vec / BLOCK_SIZE_INDEX + 1 + 3 * (0 / BLOCK_SIZE_INDEX + 1);
  generate_index_ptr4<<<grid1, BLOCK_SIZE_INDEX>>>(
      dim_d, tile_d, dim_d, tile_d, dim_d, tile_d, dim_d, tile_d, num_d, dummy_d,
      dummy_d, dummy_d, sum_vec, 0, 0, 0);
  CK(cudaGetLastError());
  CK(cudaDeviceSynchronize());
  std::vector<int> num(max_dim), dim_ptr(max_dim + 1);
  CK(cudaMemcpy(num.data(), num_d, sizeof(int) * max_dim, cudaMemcpyDeviceToHost));
  int acc = 0;
  dim_ptr[0] = 0;
  for (int i = 1; i <= max_dim; ++i) {
    acc += num[i - 1];
    dim_ptr[i] = acc;
  }
  const int total = acc;
  int* row_d;
  float* rval_d;
  CK(cudaMalloc(&row_d, sizeof(int) * std::max(total, 1)));
  CK(cudaMalloc(&rval_d, sizeof(float) * std::max(total, 1)));
  CK(cudaMemcpy(ptr_d, dim_ptr.data(), sizeof(int) * (max_dim + 1), cudaMemcpyHostToDevice));
  const int grid2 = sum_vec / BLOCK_SIZE_INDEX + 1 + (0 / BLOCK_SIZE_INDEX + 1);
  construct_Index2<<<grid2, BLOCK_SIZE_INDEX>>>(dim_d, feat_d, tile_d, dim_d, feat_d,
                                                tile_d, ptr_d, row_d, rval_d, dummy_d,
                                                row_d, rval_d, sum_vec, 0);
  CK(cudaGetLastError());
  CK(cudaDeviceSynchronize());
  std::vector<int> rows(std::max(total, 1));
  std::vector<float> vals(std::max(total, 1));
  CK(cudaMemcpy(rows.data(), row_d, sizeof(int) * rows.size(), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(vals.data(), rval_d, sizeof(float) * vals.size(), cudaMemcpyDeviceToHost));
  // canonical form: every list sorted by row
  std::vector<std::pair<int, float> > tmp;
  for (int f = 0; f < max_dim; ++f) {
    tmp.clear();
    for (int k = dim_ptr[f]; k < dim_ptr[f + 1]; ++k) tmp.push_back({rows[k], vals[k]});
    std::sort(tmp.begin(), tmp.end(),
              [](const std::pair<int, float>& a, const std::pair<int, float>& b) {
                return a.first < b.first;
              });
    for (size_t q = 0; q < tmp.size(); ++q) {
      rows[dim_ptr[f] + q] = tmp[q].first;
      vals[dim_ptr[f] + q] = tmp[q].second;
    }
  }
  FILE* o = std::fopen(argv[2], "wb");
  if (!o) return 2;
  const int64_t hdr[2] = {d, total};
  std::fwrite(hdr, 8, 2, o);
  std::fwrite(dim_ptr.data(), 4, max_dim + 1, o);
  std::fwrite(rows.data(), 4, total, o);
  std::fwrite(vals.data(), 4, total, o);
  std::fclose(o);
  cudaFree(dim_d);
  cudaFree(feat_d);
  cudaFree(tile_d);
  cudaFree(num_d);
  cudaFree(ptr_d);
  cudaFree(dummy_d);
  cudaFree(row_d);
  cudaFree(rval_d);
  return 0;
}
