// Batched self-joins (cuapss_batch_run): k independent APSS instances, each a
// row range of one CSR with its own threshold, in one pass.
//
// Layout: instances are split into size buckets by row count. Each bucket is
// compacted into its own CSR in which every instance starts on a 128-row
// block boundary (the gap rows are empty); the bucket gets its own prepared
// side (remapped rows, head block of its own width p, block-local inverted
// lists). The units of work, (I block, J block range) pairs, only pair blocks
// of the same instance, and each I block carries its instance's threshold.
// One persistent tile launch per bucket, each after the first a programmatic
// dependent launch of the one before: its CTAs start on the SMs the previous
// bucket's CTAs leave, so the buckets run as one continuous pass over the
// SMs. The launches of all buckets are captured in one CUDA graph (updated in
// place when the next batch has the same topology). Finalize runs per bucket
// into one pair list, sorted once.
//
// The autotuner picks p per bucket: the first time a bucket with given
// precision, mean row nnz and d is seen, each candidate width is timed
// (prepare + tiles, device time) on a sample of that bucket's instances and
// the fastest is kept in the context.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "ctx.cuh"
#include "prep.cuh"
#include "prims.cuh"
#include "tiles.cuh"

namespace cuapss {

namespace {

constexpr int kThreads = 256;
constexpr int kNumBuckets = CUAPSS_BATCH_BUCKETS;
constexpr int64_t kTuneRows = 65536;  // rows of a bucket's tuning sample

inline int bucket_of(int64_t n) { return n <= 1024 ? 0 : (n <= 8192 ? 1 : 2); }

inline unsigned grid_for(int64_t work, int threads) {
  const int64_t g = ceil_div(work > 0 ? work : 1, threads);
  return (unsigned)std::min<int64_t>(g, 148 * 16);
}

// tab[4q..4q+3] = {first slot, first caller row, rows, threshold bits} of
// instance q of a bucket; slots [S, S + ceil(n/128)*128) hold its rows, then
// empty rows; every slot gets the instance's threshold.
__global__ void k_slot_rows(const int64_t* __restrict__ tab, int k, const int64_t* __restrict__ rp,
                            int32_t* __restrict__ slot_row, int64_t* __restrict__ len,
                            float* __restrict__ t_row) {
  for (int q = blockIdx.x; q < k; q += gridDim.x) {
    const int64_t S = tab[4 * q], R = tab[4 * q + 1], n = tab[4 * q + 2];
    const float t = __int_as_float((int)tab[4 * q + 3]);
    const int64_t npad = (n + kBlockRows - 1) / kBlockRows * kBlockRows;
    for (int64_t r = threadIdx.x; r < npad; r += blockDim.x) {
      const bool real = r < n;
      slot_row[S + r] = real ? (int32_t)(R + r) : -1;
      len[S + r] = real ? rp[R + r + 1] - rp[R + r] : 0;
      t_row[S + r] = t;
    }
  }
}

// One warp per slot: copies the caller's row into the bucket's CSR.
__global__ void k_gather_rows(const int64_t* __restrict__ rp, const int32_t* __restrict__ col,
                              const float* __restrict__ val, const int32_t* __restrict__ slot_row,
                              const int64_t* __restrict__ rpb, int64_t nslots,
                              int32_t* __restrict__ colb, float* __restrict__ valb) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t s = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; s < nslots;
       s += warps) {
    const int32_t r = slot_row[s];
    if (r < 0) continue;
    const int64_t src = rp[r], dst = rpb[s], len = rp[r + 1] - src;
    for (int64_t e = lane; e < len; e += 32) {
      colb[dst + e] = col[src + e];
      valb[dst + e] = val[src + e];
    }
  }
}

__global__ void k_gather_i64(const int64_t* __restrict__ src, const int64_t* __restrict__ idx,
                             int64_t m, int64_t* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = src[idx[i]];
}

struct Bucket {
  std::vector<int> inst;  // instance ids, ascending
  int p = 0;
  int64_t nslots = 0;
  int nb = 0;
  int64_t nnz = 0;
  Side S;
  int64_t* rp = nullptr;
  int32_t* col = nullptr;
  float* val = nullptr;
  int32_t* slot_row = nullptr;
  float* t_row = nullptr;
  int4* units = nullptr;
  int nunits = 0;
  int grid = 0;
  int64_t ntiles = 0;
  TileArgs ta{};
  // candidate region of this bucket in the shared candidate buffer
  int64_t cand_off = 0, cand_cap = 0;
};

struct BatchIn {
  DevCsr x;
  int k = 0;
  const int64_t* inst_ptr = nullptr;  // host
  const float* t = nullptr;           // host
  const int32_t* perm = nullptr;      // device, frequency remap
  double nrm = 1.0;                   // max row norm
  bool mixed = false;
};

// Compacts the bucket's instances, builds its side and its tile arguments.
cuapss_status prepare_bucket(cuapss_ctx* ctx, const BatchIn& in, Bucket& b, int p,
                             const std::string& tag) {
  cudaStream_t st = ctx->stream;
  Workspace& ws = ctx->ws;
  const std::string t = tag + ":";
  const int kq = (int)b.inst.size();
  std::vector<int64_t> tab(4 * (size_t)std::max(kq, 1));
  int64_t S = 0;
  for (int i = 0; i < kq; ++i) {
    const int q = b.inst[i];
    const int64_t n = in.inst_ptr[q + 1] - in.inst_ptr[q];
    int tbits = 0;
    std::memcpy(&tbits, &in.t[q], sizeof(float));
    tab[4 * i] = S;
    tab[4 * i + 1] = in.inst_ptr[q];
    tab[4 * i + 2] = n;
    tab[4 * i + 3] = tbits;
    S += ceil_div(n, kBlockRows) * kBlockRows;
  }
  b.nslots = S;
  b.nb = (int)(S / kBlockRows);
  if (S >= INT32_MAX) return CUAPSS_EINVAL;
  int64_t* d_tab = nullptr;
  int64_t* len = nullptr;
  ST_TRY(ws.get(t + "tab", tab.size(), &d_tab));
  ST_TRY(ws.get(t + "slot_row", (size_t)S + 1, &b.slot_row));
  ST_TRY(ws.get(t + "len", (size_t)S + 1, &len));
  ST_TRY(ws.get(t + "rp", (size_t)S + 1, &b.rp));
  ST_TRY(ws.get(t + "trow", (size_t)S + 1, &b.t_row));
  CU_TRY(cudaMemcpyAsync(d_tab, tab.data(), sizeof(int64_t) * tab.size(), cudaMemcpyHostToDevice,
                         st));
  k_slot_rows<<<grid_for((int64_t)kq * kThreads, kThreads), kThreads, 0, st>>>(
      d_tab, kq, in.x.rp, b.slot_row, len, b.t_row);
  LAUNCH_CHECK();
  ST_TRY(exclusive_scan<int64_t>(len, b.rp, S, b.rp + S, ws, t + "rpscan", st));
  CU_TRY(cudaMemcpyAsync(&b.nnz, b.rp + S, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaStreamSynchronize(st));
  ST_TRY(ws.get(t + "col", (size_t)std::max<int64_t>(b.nnz, 1), &b.col));
  ST_TRY(ws.get(t + "val", (size_t)std::max<int64_t>(b.nnz, 1), &b.val));
  k_gather_rows<<<grid_for(S * 32, kThreads), kThreads, 0, st>>>(in.x.rp, in.x.col, in.x.val,
                                                                 b.slot_row, b.rp, S, b.col,
                                                                 b.val);
  LAUNCH_CHECK();
  // ---- side
  PrepOptions po;
  po.p = p;
  po.want_head32 = in.mixed ? 0 : 1;
  po.want_head16 = in.mixed ? 1 : 0;
  b.S = Side{};
  b.S.rp0 = b.rp;
  b.S.col0 = b.col;
  b.S.val0 = b.val;
  b.S.n = S;
  b.S.d = in.x.d;
  b.S.nnz = b.nnz;
  b.S.nrm_max = in.nrm;
  ST_TRY(build_side(b.S, po, in.perm, ws, tag, st));
  b.p = b.S.p;
  if (in.x.d - b.p > (int64_t)(1u << 20) - 2) return CUAPSS_EINVAL;  // 20-bit tail keys
  // ---- tile arguments
  TileArgs& ta = b.ta;
  ta = TileArgs{};
  const Side& s = b.S;
  ta.headI32 = ta.headJ32 = s.head32;
  ta.nI = ta.nJ = s.n;
  ta.nbI = ta.nbJ = s.nb;
  ta.blkmaxI = ta.blkmaxJ = s.blk_maxnnz;
  ta.hnormI = ta.hnormJ = s.hnorm;
  ta.bptrI = s.bptr;
  ta.bilI_key = s.bil_key;
  ta.bilI_len = s.bil_len;
  ta.max_tailI = s.max_block_tail;
  ta.bilI_u = s.bil_u;
  ta.hptrJ = s.hptr;
  ta.bilJ_rec = s.bil_rec;
  ta.p = s.p;
  ta.self = 1;
  ta.t = 1.0f;
  ta.t_row = b.t_row;
  set_tile_margins(ta, in.nrm * in.nrm, in.mixed);
  // ---- units: blocks of one instance only, cost-balanced as in a single join
  std::vector<int4> units;
  const double avg = std::max(1.0, (double)s.ntail / std::max(1, s.nb));
  auto weight = [&](int I) { return 1.0 + (double)(s.h_bptr[I + 1] - s.h_bptr[I]) / avg; };
  double total = 0.0;
  b.ntiles = 0;
  for (int i = 0; i < kq; ++i) {
    const int B0 = (int)(tab[4 * i] / kBlockRows);
    const int B1 = B0 + (int)ceil_div(tab[4 * i + 2], kBlockRows);
    for (int I = B0; I < B1; ++I) total += weight(I) * (B1 - I);
    b.ntiles += (int64_t)(B1 - B0) * (B1 - B0 + 1) / 2;
  }
  const double target = std::max(1.0, total / (ctx->sms * 16.0));
  for (int i = 0; i < kq; ++i) {
    const int B0 = (int)(tab[4 * i] / kBlockRows);
    const int B1 = B0 + (int)ceil_div(tab[4 * i + 2], kBlockRows);
    for (int I = B0; I < B1; ++I) {
      const int chunk = (int)std::max(1.0, std::floor(target / weight(I)));
      for (int j0 = I; j0 < B1; j0 += chunk)
        units.push_back(make_int4(I, j0, std::min(B1, j0 + chunk), 0));
    }
  }
  order_units_for_l2(units);
  b.nunits = (int)units.size();
  b.grid = std::max(1, std::min(b.nunits, ctx->sms));
  ST_TRY(ws.get(t + "units", std::max<size_t>(units.size(), 1), &b.units));
  if (!units.empty())
    CU_TRY(cudaMemcpyAsync(b.units, units.data(), sizeof(int4) * units.size(),
                           cudaMemcpyHostToDevice, st));
  ta.units = b.units;
  ta.nunits = b.nunits;
  return CUAPSS_OK;
}

// overlap_prev: this bucket's launch follows another bucket's tile launch
// and may start on the SMs that launch's CTAs leave (the buckets write
// disjoint candidate regions and counters), so the buckets run as one
// continuous persistent pass without an idle tail between launches.
cuapss_status launch_bucket(const Bucket& b, bool mixed, cudaStream_t st, bool overlap_prev) {
  if (b.ntiles == 0) return CUAPSS_OK;
  if (mixed)
    return launch_tiles_mma(b.ta, b.S.head16, b.S.head16, b.p, b.grid, st, overlap_prev);
  return launch_tiles_fp32(b.ta, b.grid, st, overlap_prev);
}

// Counters of one batch launch: per bucket unit counter and candidate count,
// one shared error flag.
struct Counters {
  int* unit = nullptr;                  // [kNumBuckets]
  unsigned long long* cand = nullptr;   // [kNumBuckets]
  int* err = nullptr;
};

// Width candidates of the tuner, and its cache key.
std::vector<int> width_candidates(bool mixed, int64_t d) {
  std::vector<int> c = mixed ? std::vector<int>{256, 512, 1024} : std::vector<int>{64, 128, 256};
  const int g = mixed ? 64 : 32;
  const int64_t cap = ceil_div(d, g) * g;
  std::vector<int> out;
  for (int p : c)
    if (p <= cap) out.push_back(p);
  if (out.empty()) out.push_back((int)cap);
  return out;
}

uint64_t tune_key(bool mixed, int bucket, double mean_nnz, int64_t d) {
  const uint64_t nz = (uint64_t)std::lround(std::log2(std::max(1.0, mean_nnz)) * 4.0);
  return ((uint64_t)mixed << 60) | ((uint64_t)bucket << 56) | (nz << 40) |
         (uint64_t)bits_for((uint64_t)d);
}

// Times each candidate width on a sample of the bucket (device time of
// prepare + tiles) and returns the fastest.
cuapss_status tune_bucket(cuapss_ctx* ctx, const BatchIn& in, const Bucket& full, Counters& cnt,
                          int* best_p) {
  cudaStream_t st = ctx->stream;
  Bucket smp;
  int64_t rows = 0;
  for (int q : full.inst) {
    smp.inst.push_back(q);
    rows += in.inst_ptr[q + 1] - in.inst_ptr[q];
    if (rows >= kTuneRows) break;
  }
  uint64_t* ckey = nullptr;
  float* csim = nullptr;
  const int64_t ccap = 1 << 20;
  ST_TRY(ctx->ws.get("tune:key", (size_t)ccap, &ckey));
  ST_TRY(ctx->ws.get("tune:sim", (size_t)ccap, &csim));
  double best = 1e300;
  *best_p = 0;
  for (int p : width_candidates(in.mixed, in.x.d)) {
    CU_TRY(cudaStreamSynchronize(st));
    const auto t0 = std::chrono::steady_clock::now();
    ST_TRY(prepare_bucket(ctx, in, smp, p, "T"));
    smp.ta.unit_counter = cnt.unit;
    smp.ta.cand_count = cnt.cand;
    smp.ta.err = cnt.err;
    smp.ta.cand_key = ckey;
    smp.ta.cand_sim = csim;
    smp.ta.cand_cap = ccap;
    CU_TRY(cudaMemsetAsync(cnt.unit, 0, sizeof(int), st));
    CU_TRY(cudaMemsetAsync(cnt.cand, 0, sizeof(unsigned long long), st));
    CU_TRY(cudaMemsetAsync(cnt.err, 0, sizeof(int), st));
    ST_TRY(launch_bucket(smp, in.mixed, st, false));
    int herr = 0;
    CU_TRY(cudaMemcpyAsync(&herr, cnt.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CU_TRY(cudaStreamSynchronize(st));
    if (herr & kErrTimeout) return CUAPSS_ETIMEOUT;
    if (herr) return CUAPSS_ECUDA;
    const double sec =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (sec < best) {
      best = sec;
      *best_p = smp.p;
    }
  }
  return CUAPSS_OK;
}

float elapsed_ms(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  return ms;
}

// Captures the tile launches of all buckets (with their counter resets) and
// launches them as one graph.
cuapss_status launch_graph(cuapss_ctx* ctx, std::vector<Bucket>& bk, bool mixed,
                           const Counters& cnt) {
  cudaStream_t st = ctx->stream;
  cudaGraph_t g = nullptr;
  CU_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  cuapss_status s = CUAPSS_OK;
  if (cudaMemsetAsync(cnt.unit, 0, sizeof(int) * kNumBuckets, st) != cudaSuccess ||
      cudaMemsetAsync(cnt.cand, 0, sizeof(unsigned long long) * kNumBuckets, st) != cudaSuccess ||
      cudaMemsetAsync(cnt.err, 0, sizeof(int), st) != cudaSuccess)
    s = CUAPSS_ECUDA;
  bool after_tiles = false;
  for (auto& b : bk) {
    if (s == CUAPSS_OK) s = launch_bucket(b, mixed, st, after_tiles);
    after_tiles = after_tiles || b.ntiles > 0;
  }
  const cudaError_t e = cudaStreamEndCapture(st, &g);
  if (s != CUAPSS_OK) {
    if (g) cudaGraphDestroy(g);
    return s;
  }
  CU_TRY(e);
  bool updated = false;
  if (ctx->batch_exec) {
    cudaGraphExecUpdateResultInfo info;
    if (cudaGraphExecUpdate(ctx->batch_exec, g, &info) == cudaSuccess) {
      updated = true;
    } else {
      cudaGetLastError();
      cudaGraphExecDestroy(ctx->batch_exec);
      ctx->batch_exec = nullptr;
    }
  }
  if (ctx->batch_graph) cudaGraphDestroy(ctx->batch_graph);
  ctx->batch_graph = g;
  if (!updated) CU_TRY(cudaGraphInstantiate(&ctx->batch_exec, g, 0));
  CU_TRY(cudaGraphLaunch(ctx->batch_exec, st));
  return CUAPSS_OK;
}

}  // namespace

cuapss_status batch_device(cuapss_ctx* ctx, const DevCsr& x, int k, const int64_t* inst_ptr,
                           const float* tq, cuapss_pairs* out, cuapss_stats* stats,
                           int32_t* bucket_p) {
  if (k < 1 || !inst_ptr || !tq || !out || out->capacity < 0) return CUAPSS_EINVAL;
  if (out->capacity > 0 && (!out->i || !out->j || !out->sim)) return CUAPSS_EINVAL;
  if (inst_ptr[0] != 0 || inst_ptr[k] != x.n) return CUAPSS_EINVAL;
  for (int q = 0; q < k; ++q) {
    if (inst_ptr[q + 1] < inst_ptr[q]) return CUAPSS_EINVAL;
    if (!(tq[q] > 0.0f) || !std::isfinite(tq[q])) return CUAPSS_EINVAL;
  }
  cudaStream_t st = ctx->stream;
  Workspace& ws = ctx->ws;
  const int64_t d = x.d;
  const bool mixed = ctx->opts.precision == CUAPSS_PREC_MIXED;
  const int64_t launches0 = g_launches.load();
  cudaEventRecord(ctx->ev[0], st);
  StageRange nvtx("cuapss_batch_run:prepare");
  // ---- validate + posting counts + frequency remap over all instances
  int32_t* counts = nullptr;
  int32_t* perm = nullptr;
  ST_TRY(ws.get("counts", (size_t)d, &counts));
  ST_TRY(ws.get("perm", (size_t)d, &perm));
  CU_TRY(cudaMemsetAsync(counts, 0, sizeof(int32_t) * d, st));
  double nrm = 1.0;
  ST_TRY(validate_csr(x.rp, x.col, x.val, x.n, d, x.nnz, ctx->opts.norm_tol, ctx->opts.validate,
                      counts, &nrm, ws, "A", st));
  if (nrm * nrm >= 1.9) return CUAPSS_EINVAL;  // fixed-point tail needs ~unit norms
  ST_TRY(feature_perm(counts, d, x.n, ctx->opts.remap, perm, ws, st));
  BatchIn in;
  in.x = x;
  in.k = k;
  in.inst_ptr = inst_ptr;
  in.t = tq;
  in.perm = perm;
  in.nrm = nrm;
  in.mixed = mixed;
  // ---- buckets
  std::vector<Bucket> all(kNumBuckets);
  std::vector<int64_t> bucket_nnz(kNumBuckets, 0), bucket_rows(kNumBuckets, 0);
  for (int q = 0; q < k; ++q) {
    const int64_t n = inst_ptr[q + 1] - inst_ptr[q];
    if (n < 2) continue;  // no pairs
    const int b = bucket_of(n);
    all[b].inst.push_back(q);
    bucket_rows[b] += n;
  }
  Counters cnt;
  ST_TRY(ws.get("batch:unit", kNumBuckets, &cnt.unit));
  ST_TRY(ws.get("batch:cand", kNumBuckets, &cnt.cand));
  ST_TRY(ws.get("batch:err", 1, &cnt.err));
  // mean row nnz per bucket, from the row pointers at instance boundaries
  {
    int64_t* d_iptr = nullptr;
    int64_t* d_at = nullptr;
    ST_TRY(ws.get("batch:iptr", (size_t)k + 1, &d_iptr));
    ST_TRY(ws.get("batch:rpat", (size_t)k + 1, &d_at));
    CU_TRY(cudaMemcpyAsync(d_iptr, inst_ptr, sizeof(int64_t) * (k + 1), cudaMemcpyHostToDevice,
                           st));
    k_gather_i64<<<grid_for(k + 1, kThreads), kThreads, 0, st>>>(x.rp, d_iptr, k + 1, d_at);
    LAUNCH_CHECK();
    std::vector<int64_t> rp_at((size_t)k + 1);
    CU_TRY(cudaMemcpyAsync(rp_at.data(), d_at, sizeof(int64_t) * (k + 1), cudaMemcpyDeviceToHost,
                           st));
    CU_TRY(cudaStreamSynchronize(st));
    for (int b = 0; b < kNumBuckets; ++b)
      for (int q : all[b].inst) bucket_nnz[b] += rp_at[q + 1] - rp_at[q];
  }
  ST_TRY(tiles_init(mixed));  // kernel attributes are set outside the capture
  std::vector<Bucket> bk;
  int32_t used_p[kNumBuckets] = {0, 0, 0};
  for (int b = 0; b < kNumBuckets; ++b) {
    if (all[b].inst.empty()) continue;
    int p = ctx->opts.head_width;
    if (p <= 0) {
      const uint64_t key = tune_key(mixed, b, (double)bucket_nnz[b] / bucket_rows[b], d);
      auto it = ctx->tuned_p.find(key);
      if (it != ctx->tuned_p.end()) {
        p = it->second;
      } else {
        ST_TRY(tune_bucket(ctx, in, all[b], cnt, &p));
        ctx->tuned_p[key] = p;
      }
    }
    const int pq = mixed ? 64 : 32;
    p = (int)std::min<int64_t>(((int64_t)p + pq - 1) / pq * pq, ceil_div(d, pq) * pq);
    if (mixed && p < 64) p = 64;
    ST_TRY(prepare_bucket(ctx, in, all[b], p, "B" + std::to_string(b)));
    used_p[b] = all[b].p;
    bk.push_back(std::move(all[b]));
  }
  if (bucket_p)
    for (int b = 0; b < kNumBuckets; ++b) bucket_p[b] = used_p[b];
  cudaEventRecord(ctx->ev[1], st);
  nvtx.next("cuapss_batch_run:tiles");
  // ---- tiles: all buckets in one graph launch; candidate regions per bucket
  int64_t ntiles = 0, nslots = 0;
  for (auto& b : bk) {
    ntiles += b.ntiles;
    nslots += b.nslots;
  }
  if (ctx->cand_cap == 0) ctx->cand_cap = std::max<int64_t>(1 << 20, 8 * nslots);
  uint64_t* ckey = nullptr;
  float* csim = nullptr;
  std::vector<unsigned long long> hc(kNumBuckets, 0);
  for (int attempt = 0; attempt < 3; ++attempt) {
    // region of each bucket proportional to its rows, at least 64k
    int64_t need = 0;
    std::vector<int64_t> cap(bk.size());
    for (size_t i = 0; i < bk.size(); ++i) {
      const int64_t share = (int64_t)((double)ctx->cand_cap * bk[i].nslots / std::max<int64_t>(1, nslots));
      cap[i] = std::max<int64_t>(share, 1 << 16);
      if (attempt > 0) cap[i] = std::max<int64_t>(cap[i], (int64_t)hc[i] + (int64_t)hc[i] / 4);
      need += cap[i];
    }
    ST_TRY(ws.get("cand:key", (size_t)std::max<int64_t>(need, 1), &ckey));
    ST_TRY(ws.get("cand:sim", (size_t)std::max<int64_t>(need, 1), &csim));
    int64_t off = 0;
    for (size_t i = 0; i < bk.size(); ++i) {
      Bucket& b = bk[i];
      b.cand_off = off;
      b.cand_cap = cap[i];
      off += cap[i];
      b.ta.unit_counter = cnt.unit + i;
      b.ta.cand_count = cnt.cand + i;
      b.ta.err = cnt.err;
      b.ta.cand_key = ckey + b.cand_off;
      b.ta.cand_sim = csim + b.cand_off;
      b.ta.cand_cap = b.cand_cap;
    }
    ST_TRY(launch_graph(ctx, bk, mixed, cnt));
    int herr = 0;
    CU_TRY(cudaMemcpyAsync(hc.data(), cnt.cand, sizeof(unsigned long long) * kNumBuckets,
                           cudaMemcpyDeviceToHost, st));
    CU_TRY(cudaMemcpyAsync(&herr, cnt.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CU_TRY(cudaStreamSynchronize(st));
    if (herr & kErrTimeout) return CUAPSS_ETIMEOUT;
    if (herr) return CUAPSS_ECUDA;
    bool over = false;
    for (size_t i = 0; i < bk.size(); ++i) over |= (int64_t)hc[i] > bk[i].cand_cap;
    if (!over) break;
    int64_t want = 0;
    for (size_t i = 0; i < bk.size(); ++i) want += (int64_t)hc[i];
    ctx->cand_cap = std::max<int64_t>(ctx->cand_cap, want + want / 4);
    if (attempt == 2) return CUAPSS_ENOMEM;
  }
  int64_t ncand = 0;
  for (size_t i = 0; i < bk.size(); ++i) ncand += (int64_t)hc[i];
  cudaEventRecord(ctx->ev[2], st);
  nvtx.next("cuapss_batch_run:finalize");
  // ---- finalize per bucket into one list, then one sort
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
  const int rbits = std::max(1, bits_for((uint64_t)x.n));
  for (size_t i = 0; i < bk.size(); ++i) {
    const Bucket& b = bk[i];
    FinalizeArgs fa{};
    fa.cand_key = b.ta.cand_key;
    fa.cand_sim = b.ta.cand_sim;
    fa.ncand = (int64_t)hc[i];
    fa.rowpermI = fa.rowpermJ = b.S.rowperm;
    fa.nnzI = fa.nnzJ = b.S.nnz_row;
    fa.hnormI = fa.hnormJ = b.S.hnorm;
    fa.rpI = fa.rpJ = b.rp;
    fa.colI = fa.colJ = b.col;
    fa.valI = fa.valJ = b.val;
    fa.t = 1.0f;
    fa.t_row = b.t_row;
    fa.slot_row = b.slot_row;
    fa.eps_c1 = b.ta.eps_c1;
    fa.eps_c0 = b.ta.eps_c0;
    fa.eps_head = b.ta.eps_head;
    fa.self = 1;
    fa.rbits = rbits;
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
  ST_TRY(radix_sort_pairs(okey, oidx, npairs, 2 * rbits, ws, "out", st));
  out->count = npairs;
  cuapss_status result = CUAPSS_OK;
  if (npairs > out->capacity) {
    result = CUAPSS_EOVERFLOW;
  } else if (npairs > 0) {
    if (out->on_device) {
      ST_TRY(launch_split_pairs(okey, oidx, osim, npairs, rbits, out->i, out->j, out->sim, st));
    } else {
      int32_t *di = nullptr, *dj = nullptr;
      float* ds = nullptr;
      ST_TRY(ws.get("out:i", (size_t)npairs, &di));
      ST_TRY(ws.get("out:j", (size_t)npairs, &dj));
      ST_TRY(ws.get("out:s", (size_t)npairs, &ds));
      ST_TRY(launch_split_pairs(okey, oidx, osim, npairs, rbits, di, dj, ds, st));
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
    int64_t most = -1;
    for (auto& b : bk) {
      stats->tail_entries += b.S.ntail;
      stats->tail_products += b.S.tail_products;
      if (b.ntiles > most) {
        most = b.ntiles;
        stats->head_width = b.p;
      }
    }
    stats->ms_preprocess = elapsed_ms(ctx->ev[0], ctx->ev[1]);
    stats->ms_tiles = elapsed_ms(ctx->ev[1], ctx->ev[2]);
    stats->ms_finalize = elapsed_ms(ctx->ev[2], ctx->ev[3]);
    stats->ms_total = elapsed_ms(ctx->ev[0], ctx->ev[3]);
    stats->launches = g_launches.load() - launches0;
  }
  return result;
}

}  // namespace cuapss

using namespace cuapss;

extern "C" cuapss_status cuapss_batch_run(cuapss_ctx* c, const cuapss_csr* x, int32_t k,
                                          const int64_t* inst_ptr, const float* t,
                                          cuapss_pairs* out, cuapss_stats* stats,
                                          int32_t* bucket_p) {
  if (!c) return CUAPSS_EINVAL;
  CU_TRY(cudaSetDevice(c->device));
  DevCsr a;
  ST_TRY(stage_csr(c, x, "X", &a));
  return batch_device(c, a, k, inst_ptr, t, out, stats, bucket_p);
}
