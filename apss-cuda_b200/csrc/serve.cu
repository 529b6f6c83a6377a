// Resident index for serving (cuapss_index_*): a matrix kept in HBM in the
// J-side layout of the pair-tile kernels, queried by batches of rows with
// per-row thresholds, grown by appends.
//
// Layout. The index is a list of immutable segments, each a block-aligned
// run of index rows [row0, row0 + n) with its own CSR copy and its prepared
// J side (dense head block, head norms, block nnz maxima, per-J-segment tail
// postings). The frequency remap (and so the head features) is fixed when the
// index is created; appended rows use it too. An append builds a segment for
// the new rows only, then merges trailing segments whose sizes are within a
// factor of two (a merge rebuilds one segment from the two CSRs), so the
// segment count stays logarithmic in the row count.
//
// Query. The query rows are prepared as the I side (staged tail postings in
// shared memory, head block, per-row thresholds); one persistent tile launch
// per segment writes candidates into that segment's region; the finalize of
// each segment maps its rows to index rows; one sort orders the union.
//
// Concurrency. The segment list is changed under a mutex; a query copies the
// list (shared pointers) when it starts and holds it until it returns, so an
// append or merge never frees a segment a running query reads. An append
// builds and publishes its segment (index_append_segment); merges are
// separate steps (index_merge_step) that replace two adjacent segments by
// their union, so the request server runs them on a thread of its own.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "ctx.cuh"
#include "prep.cuh"
#include "serve.h"
#include "prims.cuh"
#include "tiles.cuh"

namespace cuapss {

namespace {

constexpr int kThreads = 256;

inline unsigned grid_for(int64_t work, int threads) {
  const int64_t g = ceil_div(work > 0 ? work : 1, threads);
  return (unsigned)std::min<int64_t>(g, 148 * 16);
}

// Exact-size device allocations owned by one object, stream-ordered: taken
// with cudaMallocAsync on the building stream and returned with
// cudaFreeAsync on the index's own stream, so that neither stalls the other
// streams' work (cudaMalloc / cudaFree can synchronize the whole device).
class DevHeap {
 public:
  explicit DevHeap(cudaStream_t free_stream = nullptr) : free_st_(free_stream) {}
  ~DevHeap() {
    for (void* p : ptrs_) {
      if (free_st_) cudaFreeAsync(p, free_st_);
      else cudaFree(p);
    }
  }
  DevHeap(const DevHeap&) = delete;
  DevHeap& operator=(const DevHeap&) = delete;
  void set_streams(cudaStream_t alloc_stream, cudaStream_t free_stream) {
    alloc_st_ = alloc_stream;
    free_st_ = free_stream;
  }
  template <typename T>
  cuapss_status alloc(size_t count, T** out) {
    void* p = nullptr;
    const size_t bytes = std::max<size_t>(count * sizeof(T), 256);
    const cudaError_t e = alloc_st_ ? cudaMallocAsync(&p, bytes, alloc_st_) : cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return CUAPSS_ENOMEM;
    }
    ptrs_.push_back(p);
    bytes_ += bytes;
    *out = static_cast<T*>(p);
    return CUAPSS_OK;
  }
  // Copies count elements of src (device) into a new allocation.
  template <typename T>
  cuapss_status copy(const T* src, size_t count, T** out, cudaStream_t st) {
    ST_TRY(alloc(count, out));
    if (count > 0 && src)
      CU_TRY(cudaMemcpyAsync(*out, src, sizeof(T) * count, cudaMemcpyDeviceToDevice, st));
    return CUAPSS_OK;
  }
  size_t bytes() const { return bytes_; }

 private:
  std::vector<void*> ptrs_;
  size_t bytes_ = 0;
  cudaStream_t alloc_st_ = nullptr;
  cudaStream_t free_st_ = nullptr;
};

// One immutable run of index rows and its J-side arrays.
struct Segment {
  int64_t row0 = 0, n = 0, nnz = 0;
  int nb = 0;
  int p = 0;
  double nrm = 1.0;
  DevHeap heap;
  // CSR copy (finalize reads the exact rows)
  int64_t* rp = nullptr;
  int32_t* col = nullptr;
  float* val = nullptr;
  // J side
  int32_t* rowperm = nullptr;
  int32_t* nnz_row = nullptr;
  int32_t* blkmax = nullptr;
  float* hnorm = nullptr;
  float* head32 = nullptr;
  void* head16 = nullptr;
  int64_t* hptr = nullptr;
  uint2* rec = nullptr;
  int64_t ntail = 0;
};

using SegList = std::vector<std::shared_ptr<const Segment>>;

__global__ void k_concat_rowptr(const int64_t* __restrict__ a, int64_t na,
                                const int64_t* __restrict__ b, int64_t nb, int64_t* __restrict__ out) {
  const int64_t off = a[na];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= na + nb;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = i <= na ? a[i] : b[i - na] + off;
}

}  // namespace
}  // namespace cuapss

struct cuapss_index {
  ~cuapss_index() {
    segs.clear();  // their memory goes back on free_st
    if (free_st) {
      cudaStreamSynchronize(free_st);
      cudaStreamDestroy(free_st);
    }
  }
  int device = 0;
  cudaStream_t free_st = nullptr;  // stream-ordered frees of dropped segments
  bool mixed = false;
  int p = 0;
  int64_t d = 0;
  float norm_tol = 1e-4f;
  int validate = 1;
  cuapss::DevHeap heap;  // perm
  int32_t* perm = nullptr;
  std::mutex mu;        // guards segs, rows, nrm
  std::mutex append_mu;  // one append at a time
  std::mutex merge_mu;   // one merge at a time
  cuapss::SegList segs;
  int64_t rows = 0;
  double nrm = 0.0;
};

namespace cuapss {
namespace {

// Builds a segment from device CSR x (rows become index rows row0..).
cuapss_status build_segment(cuapss_ctx* ctx, const cuapss_index* idx, const DevCsr& x,
                            int64_t row0, double nrm, std::shared_ptr<Segment>* out) {
  cudaStream_t st = ctx->stream;
  auto seg = std::make_shared<Segment>();
  seg->heap.set_streams(st, idx->free_st);
  seg->row0 = row0;
  seg->n = x.n;
  seg->nnz = x.nnz;
  seg->nrm = nrm;
  DevHeap& H = seg->heap;
  ST_TRY(H.copy(x.rp, (size_t)x.n + 1, &seg->rp, st));
  ST_TRY(H.copy(x.col, (size_t)std::max<int64_t>(x.nnz, 1), &seg->col, st));
  ST_TRY(H.copy(x.val, (size_t)std::max<int64_t>(x.nnz, 1), &seg->val, st));
  PrepOptions po;
  po.p = idx->p;
  po.want_head32 = idx->mixed ? 0 : 1;
  po.want_head16 = idx->mixed ? 1 : 0;
  Side S;
  S.rp0 = seg->rp;
  S.col0 = seg->col;
  S.val0 = seg->val;
  S.n = x.n;
  S.d = idx->d;
  S.nnz = x.nnz;
  S.nrm_max = nrm;
  ST_TRY(build_side(S, po, idx->perm, ctx->ws, "seg", st));
  seg->p = S.p;
  seg->nb = S.nb;
  seg->ntail = S.ntail;
  const int nb = S.nb;
  ST_TRY(H.copy(S.rowperm, (size_t)x.n, &seg->rowperm, st));
  ST_TRY(H.copy(S.nnz_row, (size_t)x.n, &seg->nnz_row, st));
  ST_TRY(H.copy(S.blk_maxnnz, (size_t)nb + 1, &seg->blkmax, st));
  ST_TRY(H.copy(S.hnorm, (size_t)x.n, &seg->hnorm, st));
  if (idx->mixed) {
    __nv_bfloat16* h = nullptr;
    ST_TRY(H.copy(S.head16, (size_t)nb * S.p * kBlockRows, &h, st));
    seg->head16 = h;
  } else {
    ST_TRY(H.copy(S.head32, (size_t)nb * S.p * kBlockRows, &seg->head32, st));
  }
  ST_TRY(H.copy(S.hptr, (size_t)kJSegs * nb + 1, &seg->hptr, st));
  ST_TRY(H.copy(S.bil_rec, (size_t)std::max<int64_t>(S.ntail, 1), &seg->rec, st));
  CU_TRY(cudaStreamSynchronize(st));
  *out = std::move(seg);
  return CUAPSS_OK;
}

// Validates x (device CSR) and returns its largest row norm; counts (d
// entries) receives the posting counts when non-null.
cuapss_status check_rows(cuapss_ctx* ctx, const cuapss_index* idx, const DevCsr& x,
                         int32_t* counts, double* nrm, const std::string& tag) {
  int32_t* c = counts;
  if (!c) ST_TRY(ctx->ws.get(tag + ":counts", (size_t)idx->d, &c));
  CU_TRY(cudaMemsetAsync(c, 0, sizeof(int32_t) * idx->d, ctx->stream));
  ST_TRY(validate_csr(x.rp, x.col, x.val, x.n, idx->d, x.nnz, idx->norm_tol, idx->validate, c,
                      nrm, ctx->ws, tag, ctx->stream));
  return CUAPSS_OK;
}

// Merged CSR of two segments (device), in ctx's workspace.
cuapss_status concat_segments(cuapss_ctx* ctx, const Segment& a, const Segment& b, DevCsr* out) {
  cudaStream_t st = ctx->stream;
  int64_t* rp = nullptr;
  int32_t* col = nullptr;
  float* val = nullptr;
  const int64_t n = a.n + b.n, nnz = a.nnz + b.nnz;
  ST_TRY(ctx->ws.get("merge:rp", (size_t)n + 1, &rp));
  ST_TRY(ctx->ws.get("merge:col", (size_t)std::max<int64_t>(nnz, 1), &col));
  ST_TRY(ctx->ws.get("merge:val", (size_t)std::max<int64_t>(nnz, 1), &val));
  k_concat_rowptr<<<grid_for(n + 1, kThreads), kThreads, 0, st>>>(a.rp, a.n, b.rp, b.n, rp);
  LAUNCH_CHECK();
  if (a.nnz > 0) {
    CU_TRY(cudaMemcpyAsync(col, a.col, sizeof(int32_t) * a.nnz, cudaMemcpyDeviceToDevice, st));
    CU_TRY(cudaMemcpyAsync(val, a.val, sizeof(float) * a.nnz, cudaMemcpyDeviceToDevice, st));
  }
  if (b.nnz > 0) {
    CU_TRY(cudaMemcpyAsync(col + a.nnz, b.col, sizeof(int32_t) * b.nnz, cudaMemcpyDeviceToDevice,
                           st));
    CU_TRY(cudaMemcpyAsync(val + a.nnz, b.val, sizeof(float) * b.nnz, cudaMemcpyDeviceToDevice,
                           st));
  }
  out->n = n;
  out->nnz = nnz;
  out->rp = rp;
  out->col = col;
  out->val = val;
  return CUAPSS_OK;
}

constexpr size_t kMaxSegments = 24;

}  // namespace
}  // namespace cuapss

using namespace cuapss;

extern "C" cuapss_status cuapss_index_create(cuapss_ctx* ctx, const cuapss_csr* x,
                                             cuapss_index** out) {
  if (!ctx || !x || !out) return CUAPSS_EINVAL;
  *out = nullptr;
  CU_TRY(cudaSetDevice(ctx->device));
  DevCsr a;
  ST_TRY(stage_csr(ctx, x, "IX", &a));
  auto idx = std::make_unique<cuapss_index>();
  idx->device = ctx->device;
  CU_TRY(cudaStreamCreateWithFlags(&idx->free_st, cudaStreamNonBlocking));
  {
    // keep freed segment memory in the device's pool for the next segments
    cudaMemPool_t pool = nullptr;
    if (cudaDeviceGetDefaultMemPool(&pool, ctx->device) == cudaSuccess) {
      uint64_t keep = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
  }
  idx->mixed = ctx->opts.precision == CUAPSS_PREC_MIXED;
  idx->d = a.d;
  idx->norm_tol = ctx->opts.norm_tol;
  idx->validate = ctx->opts.validate;
  int32_t* counts = nullptr;
  ST_TRY(ctx->ws.get("IX:counts", (size_t)a.d, &counts));
  double nrm = 1.0;
  ST_TRY(check_rows(ctx, idx.get(), a, counts, &nrm, "IX"));
  if (nrm >= 1.37) return CUAPSS_EINVAL;  // norms^2 < 1.9 for the fixed-point tail
  ST_TRY(idx->heap.alloc((size_t)a.d, &idx->perm));
  ST_TRY(feature_perm(counts, a.d, a.n, ctx->opts.remap, idx->perm, ctx->ws, ctx->stream));
  int p = ctx->opts.head_width;
  if (p <= 0) {
    std::vector<int64_t> prefix;
    if (idx->mixed)
      ST_TRY(rank_count_prefix(counts, a.d, ctx->opts.remap, 8192, ctx->ws, ctx->stream, &prefix));
    p = choose_head_width(ctx->opts.precision, a.n, a.d, a.nnz, prefix);
  }
  const int pq = idx->mixed ? 64 : 32;
  p = (int)std::min<int64_t>(((int64_t)p + pq - 1) / pq * pq, ceil_div(a.d, pq) * pq);
  if (idx->mixed && p < 64) p = 64;
  if (a.d - p > (int64_t)(1u << 20) - 2) return CUAPSS_EINVAL;  // 20-bit tail features
  idx->p = p;
  std::shared_ptr<Segment> seg;
  ST_TRY(build_segment(ctx, idx.get(), a, 0, nrm, &seg));
  idx->p = seg->p;
  ctx->ws.release_prefix("seg:");
  ctx->ws.release_prefix("IX:");
  idx->segs.push_back(seg);
  idx->rows = a.n;
  idx->nrm = nrm;
  *out = idx.release();
  return CUAPSS_OK;
}

namespace cuapss {

cuapss_status index_append_segment(cuapss_ctx* ctx, cuapss_index* idx, const cuapss_csr* x) {
  if (!ctx || !idx || !x) return CUAPSS_EINVAL;
  if (ctx->device != idx->device || x->d != idx->d) return CUAPSS_EINVAL;
  if (x->n == 0) return CUAPSS_OK;
  CU_TRY(cudaSetDevice(ctx->device));
  std::lock_guard<std::mutex> alk(idx->append_mu);
  DevCsr a;
  ST_TRY(stage_csr(ctx, x, "AP", &a));
  double nrm = 1.0;
  ST_TRY(check_rows(ctx, idx, a, nullptr, &nrm, "AP"));
  if (nrm >= 1.37) return CUAPSS_EINVAL;
  int64_t rows = 0;
  {
    std::lock_guard<std::mutex> lk(idx->mu);
    rows = idx->rows;
  }
  std::shared_ptr<Segment> seg;
  ST_TRY(build_segment(ctx, idx, a, rows, nrm, &seg));
  // the build temporaries stay in ctx's grow-only workspace: freeing them
  // here would synchronize the device under running queries
  std::lock_guard<std::mutex> lk(idx->mu);
  idx->segs.push_back(seg);
  idx->rows = rows + a.n;
  idx->nrm = std::max(idx->nrm, nrm);
  return CUAPSS_OK;
}

cuapss_status index_merge_step(cuapss_ctx* ctx, cuapss_index* idx, bool* merged) {
  *merged = false;
  if (!ctx || !idx || ctx->device != idx->device) return CUAPSS_EINVAL;
  CU_TRY(cudaSetDevice(ctx->device));
  std::lock_guard<std::mutex> mlk(idx->merge_mu);  // one merge at a time
  std::shared_ptr<const Segment> A, B;
  {
    // merge the trailing segments when they are of similar size (the newer
    // at least half the older), and the last two whenever there are too many
    std::lock_guard<std::mutex> lk(idx->mu);
    const SegList& segs = idx->segs;
    if (segs.size() < 2) return CUAPSS_OK;
    A = segs[segs.size() - 2];
    B = segs[segs.size() - 1];
    if (!(2 * B->n >= A->n || segs.size() > kMaxSegments)) return CUAPSS_OK;
  }
  DevCsr m;
  ST_TRY(concat_segments(ctx, *A, *B, &m));
  m.d = idx->d;
  std::shared_ptr<Segment> ab;
  ST_TRY(build_segment(ctx, idx, m, A->row0, std::max(A->nrm, B->nrm), &ab));
  std::lock_guard<std::mutex> lk(idx->mu);
  // appends may have added segments behind B meanwhile; only merges remove
  // segments, so A and B are still adjacent
  SegList& segs = idx->segs;
  for (size_t k = 0; k + 1 < segs.size(); ++k) {
    if (segs[k] == A && segs[k + 1] == B) {
      segs[k] = ab;
      segs.erase(segs.begin() + (std::ptrdiff_t)(k + 1));
      *merged = true;
      break;
    }
  }
  return CUAPSS_OK;
}

}  // namespace cuapss

extern "C" cuapss_status cuapss_index_append(cuapss_ctx* ctx, cuapss_index* idx,
                                             const cuapss_csr* x) {
  ST_TRY(cuapss::index_append_segment(ctx, idx, x));
  for (bool merged = true; merged;) ST_TRY(cuapss::index_merge_step(ctx, idx, &merged));
  return CUAPSS_OK;
}

extern "C" cuapss_status cuapss_index_info(const cuapss_index* idx, int64_t* rows,
                                           int32_t* segments, int32_t* head_width,
                                           int64_t* device_bytes) {
  if (!idx) return CUAPSS_EINVAL;
  auto* m = const_cast<cuapss_index*>(idx);
  std::lock_guard<std::mutex> lk(m->mu);
  if (rows) *rows = idx->rows;
  if (segments) *segments = (int32_t)idx->segs.size();
  if (head_width) *head_width = idx->p;
  if (device_bytes) {
    int64_t b = (int64_t)idx->heap.bytes();
    for (auto& s : idx->segs) b += (int64_t)s->heap.bytes();
    *device_bytes = b;
  }
  return CUAPSS_OK;
}

extern "C" cuapss_status cuapss_index_destroy(cuapss_index* idx) {
  if (!idx) return CUAPSS_OK;
  cudaSetDevice(idx->device);
  cudaDeviceSynchronize();
  delete idx;
  return CUAPSS_OK;
}

extern "C" cuapss_status cuapss_index_query(cuapss_ctx* ctx, const cuapss_index* idx,
                                            const cuapss_csr* qx, const float* t,
                                            cuapss_pairs* out, cuapss_stats* stats) {
  return cuapss::index_query_rows(ctx, idx, qx, t, out, stats, nullptr);
}

cuapss_status cuapss::index_query_rows(cuapss_ctx* ctx, const cuapss_index* idx,
                                       const cuapss_csr* qx, const float* t, cuapss_pairs* out,
                                       cuapss_stats* stats, int64_t* rows_seen) {
  if (!ctx || !idx || !qx || !out) return CUAPSS_EINVAL;
  if (ctx->device != idx->device || qx->d != idx->d) return CUAPSS_EINVAL;
  if (out->capacity < 0 || (out->capacity > 0 && (!out->i || !out->j || !out->sim)))
    return CUAPSS_EINVAL;
  if (qx->n > 0 && !t) return CUAPSS_EINVAL;
  for (int64_t i = 0; i < qx->n; ++i)
    if (!(t[i] > 0.0f) || !std::isfinite(t[i])) return CUAPSS_EINVAL;
  CU_TRY(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  Workspace& ws = ctx->ws;
  const int64_t launches0 = g_launches.load();
  cudaEventRecord(ctx->ev[0], st);
  StageRange nvtx("cuapss_index_query:prepare");
  SegList segs;
  int64_t rows = 0;
  double nrm_idx = 1.0;
  {
    auto* m = const_cast<cuapss_index*>(idx);
    std::lock_guard<std::mutex> lk(m->mu);
    segs = idx->segs;
    rows = idx->rows;
    nrm_idx = idx->nrm;
  }
  if (rows_seen) *rows_seen = rows;
  DevCsr q;
  ST_TRY(stage_csr(ctx, qx, "QX", &q));
  double nrm_q = 1.0;
  ST_TRY(check_rows(ctx, idx, q, nullptr, &nrm_q, "QX"));
  const double nrm2 = nrm_q * nrm_idx;
  if (nrm2 >= 1.9) return CUAPSS_EINVAL;
  // ---- query side (I role)
  PrepOptions po;
  po.p = idx->p;
  po.want_head32 = idx->mixed ? 0 : 1;
  po.want_head16 = idx->mixed ? 1 : 0;
  Side SQ;
  SQ.rp0 = q.rp;
  SQ.col0 = q.col;
  SQ.val0 = q.val;
  SQ.n = q.n;
  SQ.d = idx->d;
  SQ.nnz = q.nnz;
  SQ.nrm_max = nrm_q;
  if (q.n > 0) ST_TRY(build_side(SQ, po, idx->perm, ws, "Q", st));
  float* t_row = nullptr;
  ST_TRY(ws.get("Q:trow", (size_t)std::max<int64_t>(q.n, 1), &t_row));
  if (q.n > 0)
    CU_TRY(cudaMemcpyAsync(t_row, t, sizeof(float) * q.n, cudaMemcpyHostToDevice, st));
  ST_TRY(tiles_init(idx->mixed));
  cudaEventRecord(ctx->ev[1], st);
  nvtx.next("cuapss_index_query:tiles");
  // ---- tiles: one launch per segment, candidate region per segment
  const size_t ns = segs.size();
  std::vector<TileArgs> tas(ns);
  std::vector<int> grids(ns, 1);
  std::vector<int64_t> seg_tiles(ns, 0);
  int64_t ntiles = 0;
  int4* d_units = nullptr;
  std::vector<std::vector<int4>> units(ns);
  size_t total_units = 0;
  if (q.n > 0) {
    const double avg = std::max(1.0, (double)SQ.ntail / std::max(1, SQ.nb));
    for (size_t s = 0; s < ns; ++s) {
      const Segment& G = *segs[s];
      auto wI = [&](int I) { return 1.0 + (double)(SQ.h_bptr[I + 1] - SQ.h_bptr[I]) / avg; };
      double total = 0.0;
      for (int I = 0; I < SQ.nb; ++I) total += wI(I) * G.nb;
      const double target = std::max(1.0, total / (ctx->sms * 16.0));
      for (int I = 0; I < SQ.nb; ++I) {
        const int chunk = (int)std::max(1.0, std::floor(target / wI(I)));
        for (int j0 = 0; j0 < G.nb; j0 += chunk)
          units[s].push_back(make_int4(I, j0, std::min(G.nb, j0 + chunk), 0));
      }
      order_units_for_l2(units[s]);
      seg_tiles[s] = (int64_t)SQ.nb * G.nb;
      ntiles += seg_tiles[s];
      total_units += units[s].size();
    }
  }
  ST_TRY(ws.get("Q:units", std::max<size_t>(total_units, 1), &d_units));
  {
    size_t off = 0;
    for (size_t s = 0; s < ns; ++s) {
      if (!units[s].empty())
        CU_TRY(cudaMemcpyAsync(d_units + off, units[s].data(), sizeof(int4) * units[s].size(),
                               cudaMemcpyHostToDevice, st));
      TileArgs& ta = tas[s];
      const Segment& G = *segs[s];
      ta = TileArgs{};
      ta.headI32 = SQ.head32;
      ta.headI16 = SQ.head16;
      ta.nI = SQ.n;
      ta.nbI = SQ.nb;
      ta.blkmaxI = SQ.blk_maxnnz;
      ta.hnormI = SQ.hnorm;
      ta.bptrI = SQ.bptr;
      ta.bilI_key = SQ.bil_key;
      ta.bilI_u = SQ.bil_u;
      ta.bilI_len = SQ.bil_len;
      ta.max_tailI = SQ.max_block_tail;
      ta.headJ32 = G.head32;
      ta.headJ16 = G.head16;
      ta.nJ = G.n;
      ta.nbJ = G.nb;
      ta.blkmaxJ = G.blkmax;
      ta.hnormJ = G.hnorm;
      ta.hptrJ = G.hptr;
      ta.bilJ_rec = G.rec;
      ta.p = idx->p;
      ta.self = 0;
      ta.t = 1.0f;
      ta.t_row = t_row;
      set_tile_margins(ta, nrm2, idx->mixed);
      ta.units = d_units + off;
      ta.nunits = (int)units[s].size();
      grids[s] = std::max(1, std::min(ta.nunits, ctx->sms));
      off += units[s].size();
    }
  }
  int* ucnt = nullptr;
  unsigned long long* ccnt = nullptr;
  int* err = nullptr;
  ST_TRY(ws.get("Q:ucnt", std::max<size_t>(ns, 1), &ucnt));
  ST_TRY(ws.get("Q:ccnt", std::max<size_t>(ns, 1), &ccnt));
  ST_TRY(ws.get("Q:err", 1, &err));
  if (ctx->cand_cap == 0) ctx->cand_cap = 1 << 20;
  std::vector<unsigned long long> hc(std::max<size_t>(ns, 1), 0);
  std::vector<int64_t> cap(ns, 0), coff(ns, 0);
  uint64_t* ckey = nullptr;
  float* csim = nullptr;
  for (int attempt = 0; attempt < 3; ++attempt) {
    int64_t need = 0;
    for (size_t s = 0; s < ns; ++s) {
      const double share = ntiles > 0 ? (double)seg_tiles[s] / ntiles : 0.0;
      cap[s] = std::max<int64_t>((int64_t)(share * ctx->cand_cap), 1 << 14);
      if (attempt > 0) cap[s] = std::max<int64_t>(cap[s], (int64_t)hc[s] + (int64_t)hc[s] / 4);
      coff[s] = need;
      need += cap[s];
    }
    ST_TRY(ws.get("cand:key", (size_t)std::max<int64_t>(need, 1), &ckey));
    ST_TRY(ws.get("cand:sim", (size_t)std::max<int64_t>(need, 1), &csim));
    CU_TRY(cudaMemsetAsync(ucnt, 0, sizeof(int) * std::max<size_t>(ns, 1), st));
    CU_TRY(cudaMemsetAsync(ccnt, 0, sizeof(unsigned long long) * std::max<size_t>(ns, 1), st));
    CU_TRY(cudaMemsetAsync(err, 0, sizeof(int), st));
    // segment launches after the first start on the SMs the previous
    // segment's CTAs leave (programmatic dependent launch; the segments
    // write disjoint candidate regions and counters)
    bool after_tiles = false;
    for (size_t s = 0; s < ns; ++s) {
      TileArgs& ta = tas[s];
      ta.unit_counter = ucnt + s;
      ta.cand_count = ccnt + s;
      ta.err = err;
      ta.cand_key = ckey + coff[s];
      ta.cand_sim = csim + coff[s];
      ta.cand_cap = cap[s];
      if (seg_tiles[s] == 0) continue;
      if (idx->mixed)
        ST_TRY(launch_tiles_mma(ta, SQ.head16, segs[s]->head16, idx->p, grids[s], st,
                                after_tiles));
      else ST_TRY(launch_tiles_fp32(ta, grids[s], st, after_tiles));
      after_tiles = true;
    }
    int herr = 0;
    CU_TRY(cudaMemcpyAsync(hc.data(), ccnt, sizeof(unsigned long long) * std::max<size_t>(ns, 1),
                           cudaMemcpyDeviceToHost, st));
    CU_TRY(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CU_TRY(cudaStreamSynchronize(st));
    if (herr & kErrTimeout) return CUAPSS_ETIMEOUT;
    if (herr) return CUAPSS_ECUDA;
    bool over = false;
    int64_t want = 0;
    for (size_t s = 0; s < ns; ++s) {
      over |= (int64_t)hc[s] > cap[s];
      want += (int64_t)hc[s];
    }
    if (!over) break;
    ctx->cand_cap = std::max<int64_t>(ctx->cand_cap, want + want / 4);
    if (attempt == 2) return CUAPSS_ENOMEM;
  }
  int64_t ncand = 0;
  for (size_t s = 0; s < ns; ++s) ncand += (int64_t)hc[s];
  cudaEventRecord(ctx->ev[2], st);
  nvtx.next("cuapss_index_query:finalize");
  // ---- finalize per segment, one sort
  uint64_t* okey = nullptr;
  uint32_t* oidx = nullptr;
  float* osim = nullptr;
  unsigned long long* ocount = nullptr;
  const int64_t ocap = std::max<int64_t>(ncand, 1);
  ST_TRY(ws.get("out:key", (size_t)ocap, &okey));
  ST_TRY(ws.get("out:idx", (size_t)ocap, &oidx));
  ST_TRY(ws.get("out:sim", (size_t)ocap, &osim));
  ST_TRY(ws.get("out:count", 2, &ocount));
  CU_TRY(cudaMemsetAsync(ocount, 0, 2 * sizeof(unsigned long long), st));
  const int rbitsJ = std::max(1, bits_for((uint64_t)std::max<int64_t>(rows, 1)));
  const int rbitsI = std::max(1, bits_for((uint64_t)std::max<int64_t>(q.n, 1)));
  for (size_t s = 0; s < ns; ++s) {
    if (hc[s] == 0) continue;
    const Segment& G = *segs[s];
    FinalizeArgs fa{};
    fa.cand_key = tas[s].cand_key;
    fa.cand_sim = tas[s].cand_sim;
    fa.ncand = (int64_t)hc[s];
    fa.rowpermI = SQ.rowperm;
    fa.rowpermJ = G.rowperm;
    fa.nnzI = SQ.nnz_row;
    fa.nnzJ = G.nnz_row;
    fa.hnormI = SQ.hnorm;
    fa.hnormJ = G.hnorm;
    fa.rpI = q.rp;
    fa.colI = q.col;
    fa.valI = q.val;
    fa.rpJ = G.rp;
    fa.colJ = G.col;
    fa.valJ = G.val;
    fa.t = 1.0f;
    fa.t_row = t_row;
    fa.j_offset = G.row0;
    fa.eps_c1 = tas[s].eps_c1;
    fa.eps_c0 = tas[s].eps_c0;
    fa.eps_head = tas[s].eps_head;
    fa.self = 0;
    fa.rbits = rbitsJ;
    fa.out_key = okey;
    fa.out_idx = oidx;
    fa.out_sim = osim;
    fa.out_count = ocount;
    fa.out_cap = ocap;
    fa.n_rescored = ocount + 1;
    ST_TRY(launch_finalize(fa, st));
  }
  unsigned long long hcnt[2] = {0, 0};
  CU_TRY(cudaMemcpyAsync(hcnt, ocount, sizeof(hcnt), cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaStreamSynchronize(st));
  const int64_t npairs = (int64_t)hcnt[0];
  ST_TRY(radix_sort_pairs(okey, oidx, npairs, rbitsI + rbitsJ, ws, "out", st));
  out->count = npairs;
  cuapss_status result = CUAPSS_OK;
  if (npairs > out->capacity) {
    result = CUAPSS_EOVERFLOW;
  } else if (npairs > 0) {
    if (out->on_device) {
      ST_TRY(launch_split_pairs(okey, oidx, osim, npairs, rbitsJ, out->i, out->j, out->sim, st));
    } else {
      int32_t *di = nullptr, *dj = nullptr;
      float* ds = nullptr;
      ST_TRY(ws.get("out:i", (size_t)npairs, &di));
      ST_TRY(ws.get("out:j", (size_t)npairs, &dj));
      ST_TRY(ws.get("out:s", (size_t)npairs, &ds));
      ST_TRY(launch_split_pairs(okey, oidx, osim, npairs, rbitsJ, di, dj, ds, st));
      CU_TRY(cudaMemcpyAsync(out->i, di, sizeof(int32_t) * npairs, cudaMemcpyDeviceToHost, st));
      CU_TRY(cudaMemcpyAsync(out->j, dj, sizeof(int32_t) * npairs, cudaMemcpyDeviceToHost, st));
      CU_TRY(cudaMemcpyAsync(out->sim, ds, sizeof(float) * npairs, cudaMemcpyDeviceToHost, st));
    }
  }
  cudaEventRecord(ctx->ev[3], st);
  CU_TRY(cudaStreamSynchronize(st));
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    stats->pairs = npairs;
    stats->candidates = ncand;
    stats->rescored = (int64_t)hcnt[1];
    stats->tiles = ntiles;
    stats->head_width = idx->p;
    stats->tail_entries = SQ.ntail;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
    stats->ms_preprocess = ms;
    cudaEventElapsedTime(&ms, ctx->ev[1], ctx->ev[2]);
    stats->ms_tiles = ms;
    cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]);
    stats->ms_finalize = ms;
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[3]);
    stats->ms_total = ms;
    stats->launches = g_launches.load() - launches0;
  }
  return result;
}
