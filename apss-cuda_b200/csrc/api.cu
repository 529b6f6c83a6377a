// C ABI of CuAPSS (include/cuapss.h) and the host orchestration of a join.
//
// The reference's orchestrator, similarity_join_device (fengyilin118/
// APSS-CUDA similarity_search.cu:934-3014), copies 8 fixed partitions to the
// device, builds per-partition indexes, then runs 28 cross-partition joins
// and 8 self-joins, each through a dense n_A x n_B (or n(n-1)/2) float
// accumulator in global memory with a blocking cudaThreadSynchronize after
// every launch, and prints pair counts. Here one call handles a matrix of
// any size: prepare (validate, remap, order, head block, inverted lists),
// one persistent tile launch over the upper triangle of 128 x 128 pair
// tiles with no n^2 buffer, then the exact finalize and a sorted pair list.
#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "ctx.cuh"
#include "index.cuh"
#include "prep.cuh"
#include "prims.cuh"
#include "tiles.cuh"

namespace cuapss {

std::atomic<int64_t> g_launches{0};

namespace {
thread_local char g_last_error[512] = {0};
}

void record_cuda_error(cudaError_t e, const char* what, const char* file, int line) {
  snprintf(g_last_error, sizeof(g_last_error), "%s: %s (%s:%d)", what, cudaGetErrorString(e),
           file, line);
}

const char* last_error_message() { return g_last_error; }

// Per-tile cost model of the mixed-precision tile kernel, whose tensor-core
// side and sparse-tail side mostly overlap, so the slower one sets the pace:
//   head  head_chunk_ns per 64 head features (operand stream and MMAs of a
//         128 x 128 tile),
//   tail  tail_posting_ns per probed tail posting of the J block (one probe
//         of the staged I postings); a block holds 128 x (probed tail
//         non-zeros per row),
//   cost  max(head, tail) + overlap_loss x min(head, tail).
// Fitted to tile-kernel times on the n = d = 1M workload's shape: with
// every tail feature probed at 200,000 rows for p = 768 .. 2048, and with
// the rare features paired explicitly at 200,000 and 1,000,000 rows for
// p = 640 .. 1152 and C = 128 .. 2048 (their postings leave the probed
// tail; the probes left are the costlier hits of the frequent tail
// features). The head width p minimises the cost over multiples of 64; the
// tail non-zeros at each p come from the posting counts in frequency order.
// Explicit rare-feature pairs of one self-join: 8-byte records, offsets of
// 32 bits; the records take at most 40% of the free device memory.
constexpr int64_t kMaxExplicitPairs = 4000000000;
constexpr double kExplicitPairBytes = 8.0, kExplicitMemShare = 0.4;
// Cost of one explicit pair in SM-nanoseconds, against the per-tile cost
// below (SM-nanoseconds of one 128 x 128 tile): its addition in the tile
// kernel (about 4) and its share of the build's count and placement passes
// (about 3.5), measured on the n = d = 1M workload's shape.
constexpr double kExplicitPairSmNs = 7.5;
// The tile kernel that adds explicit records holds them in registers and so
// loads J postings two at a time instead of three: 7% slower per tile at
// equal work (n = 800k, d = 50k: 1,017 against 945 ms with few records).
constexpr double kExplicitKernelFactor = 1.07;
// Self-joins of fewer rows skip the rare-feature planning: its statistics
// kernel and host round trip cost about as much as the pairs could save
// (measured on 4,096 instances of 64..20,000 rows called one by one, and on
// one 20,000-row join: 2.24 -> 2.45 ms).
constexpr int64_t kRareMinRows = 32768;

struct TileCostModel {
  double head_chunk_ns, tail_posting_ns, overlap_loss;
};
constexpr TileCostModel kProbedTail{388.0, 1.6, 0.06};
constexpr TileCostModel kRarePaired{340.0, 1.84, 0.3};
constexpr int kMaxModelHead = 8192;
constexpr double kUnitCostCap = 512.0;  // unit cost cap (tile weights, 1 + tail / mean)

namespace {

// Tail postings still probed at head width p (ranks >= p), without the
// paired rare features (ranks >= rare_rank) when rare_postings > 0.
int64_t probed_postings(int64_t p, int64_t nnz, const std::vector<int64_t>& prefix,
                        int64_t rare_rank, int64_t rare_postings) {
  const int64_t top = (int64_t)prefix.size() - 1;
  int64_t probed = nnz - prefix[(size_t)std::min(p, top)];
  if (rare_postings > 0) probed = p < rare_rank ? std::max<int64_t>(0, probed - rare_postings) : 0;
  return probed;
}

// Modelled SM-nanoseconds of one tile at head width p. The FP32 head runs
// on CUDA cores beside nothing: only its tail side depends on the split.
double tile_ns(int precision, int64_t p, int64_t n, int64_t probed, bool paired) {
  const TileCostModel& m = paired ? kRarePaired : kProbedTail;
  const double tail = m.tail_posting_ns * kBlockRows * ((double)probed / (double)n);
  if (precision != CUAPSS_PREC_MIXED) return tail;
  const double head = m.head_chunk_ns * (double)(p / 64);
  return std::max(head, tail) + m.overlap_loss * std::min(head, tail);
}

// The model's head width and its tile cost.
int best_head_width(int64_t n, int64_t nnz, const std::vector<int64_t>& prefix, int64_t rare_rank,
                    int64_t rare_postings, double* cost) {
  double best = 1e300;
  int best_p = 64;
  const int64_t top = (int64_t)prefix.size() - 1;  // ranks with known counts
  for (int64_t p = 64; p <= std::min<int64_t>(top, kMaxModelHead); p += 64) {
    const int64_t probed = probed_postings(p, nnz, prefix, rare_rank, rare_postings);
    const double c = tile_ns(CUAPSS_PREC_MIXED, p, n, probed, rare_postings > 0);
    if (c < best - 1e-9) {
      best = c;
      best_p = (int)p;
    }
  }
  *cost = best;
  return best_p;
}

}  // namespace

int choose_head_width(int precision, int64_t n, int64_t d, int64_t nnz,
                      const std::vector<int64_t>& prefix, int64_t rare_rank,
                      int64_t rare_postings) {
  const int64_t cap = ((d + 31) / 32) * 32;
  // the FP32 head runs on CUDA cores and pays per feature per pair: its
  // measured optimum on the lognormal/Zipf workloads is a narrow head
  if (precision != CUAPSS_PREC_MIXED) return (int)std::min<int64_t>(64, cap);
  if (n <= 0 || prefix.size() < 2) return (int)std::min<int64_t>(1024, ((d + 63) / 64) * 64);
  double cost = 0.0;
  return best_head_width(n, nnz, prefix, rare_rank, rare_postings, &cost);
}

bool head_bound_plan(int64_t p, int64_t n, int64_t nnz, const std::vector<int64_t>& prefix,
                     const RareCandidate& rare) {
  if (n <= 0 || prefix.size() < 2) return false;
  const bool paired = rare.max_count > 0;
  const TileCostModel& m = paired ? kRarePaired : kProbedTail;
  const int64_t probed =
      probed_postings(p, nnz, prefix, paired ? rare.rank : 0, paired ? rare.postings : 0);
  const double head = m.head_chunk_ns * (double)(p / 64);
  const double tail = m.tail_posting_ns * kBlockRows * ((double)probed / (double)n);
  return head >= 2.0 * tail;
}

TilePlan plan_tiles(int precision, int64_t n, int64_t d, int64_t nnz,
                    const std::vector<int64_t>& prefix,
                    const std::vector<RareCandidate>& cands, int64_t max_pairs, int fixed_p,
                    bool forced) {
  TilePlan plan;
  plan.p = fixed_p > 0 ? fixed_p : choose_head_width(precision, n, d, nnz, prefix);
  if (cands.empty() || n <= 0 || prefix.size() < 2) return plan;
  const double nbk = std::ceil((double)n / kBlockRows);
  const double tiles = nbk * (nbk + 1.0) / 2.0;
  auto cost_at = [&](const RareCandidate* c, int* p_out) {
    const int64_t rank = c ? c->rank : 0, posts = c ? c->postings : 0;
    double per_tile = 0.0;
    int p = fixed_p;
    if (precision == CUAPSS_PREC_MIXED && fixed_p <= 0) {
      p = best_head_width(n, nnz, prefix, rank, posts, &per_tile);
    } else {
      if (p <= 0) p = plan.p;
      per_tile = tile_ns(precision, p, n, probed_postings(p, nnz, prefix, rank, posts), c != nullptr);
    }
    *p_out = p;
    if (c) per_tile *= kExplicitKernelFactor;
    return tiles * per_tile + (c ? (double)c->pairs * kExplicitPairSmNs : 0.0);
  };
  int p0 = plan.p;
  double best = cost_at(nullptr, &p0);
  plan.p = p0;
  for (const RareCandidate& c : cands) {
    if (c.pairs > max_pairs || c.pairs >= (int64_t)UINT32_MAX - 1) continue;
    int pc = 0;
    const double cost = cost_at(&c, &pc);
    if (cost < best || forced) {
      best = cost;
      plan.p = pc;
      plan.rare = c;
    }
  }
  return plan;
}

namespace {

// Candidates of rare_feature_candidates from host counts (same thresholds).
void host_rare_candidates(const int32_t* counts, int64_t d, std::vector<RareCandidate>* out) {
  out->clear();
  for (int C = kMaxRareCount; C >= 16; C >>= 1) {
    RareCandidate c;
    c.max_count = C;
    for (int64_t f = 0; f < d; ++f) {
      const int64_t k = counts[f];
      if (k > C) {
        ++c.rank;
      } else {
        c.pairs += k * (k - 1) / 2;
        c.postings += k;
      }
    }
    if (c.postings > 0) out->push_back(c);
  }
}

}  // namespace

extern "C" cuapss_status cuapss_plan_self_join(int32_t precision, int64_t n, int64_t d,
                                               const int32_t* counts, int64_t max_pairs,
                                               int32_t* head_width, int32_t* rare_max_count,
                                               int64_t* explicit_pairs) {
  if (n < 0 || d < 1 || d > INT32_MAX || !counts || !head_width) return CUAPSS_EINVAL;
  if (precision != CUAPSS_PREC_FP32 && precision != CUAPSS_PREC_MIXED) return CUAPSS_EINVAL;
  for (int64_t f = 0; f < d; ++f)
    if (counts[f] < 0 || counts[f] > n) return CUAPSS_EINVAL;
  // the posting counts of the most frequent features, as rank_count_prefix
  std::vector<int32_t> sorted(counts, counts + d);
  const int64_t top = std::min<int64_t>(d, kMaxModelHead);
  std::partial_sort(sorted.begin(), sorted.begin() + top, sorted.end(), std::greater<int32_t>());
  std::vector<int64_t> prefix((size_t)top + 1, 0);
  for (int64_t k = 0; k < top; ++k) prefix[(size_t)k + 1] = prefix[(size_t)k] + sorted[(size_t)k];
  int64_t nnz = 0;
  for (int64_t f = 0; f < d; ++f) nnz += counts[f];
  std::vector<RareCandidate> rare;
  if (n >= kRareMinRows) host_rare_candidates(counts, d, &rare);
  const int64_t bound = max_pairs > 0 ? std::min(max_pairs, kMaxExplicitPairs) : kMaxExplicitPairs;
  const TilePlan plan = plan_tiles(precision, n, d, nnz, prefix, rare, bound, 0);
  const bool mixed = precision == CUAPSS_PREC_MIXED;
  const int pq = mixed ? 64 : 32;  // as the self-join rounds it
  int p = (int)std::min<int64_t>(((int64_t)plan.p + pq - 1) / pq * pq, ((d + pq - 1) / pq) * pq);
  if (mixed && p < 64) p = 64;
  *head_width = p;
  if (rare_max_count) *rare_max_count = plan.rare.max_count;
  if (explicit_pairs) *explicit_pairs = plan.rare.max_count > 0 ? plan.rare.pairs : 0;
  return CUAPSS_OK;
}

cuapss_status stage_csr(cuapss_ctx* ctx, const cuapss_csr* x, const std::string& tag,
                        DevCsr* out) {
  if (!x || x->n < 0 || x->d < 1 || x->nnz < 0 || x->d > INT32_MAX || x->n >= INT32_MAX)
    return CUAPSS_EINVAL;
  if (!x->rowptr || (x->nnz > 0 && (!x->col || !x->val))) return CUAPSS_EINVAL;
  out->n = x->n;
  out->d = x->d;
  out->nnz = x->nnz;
  if (x->on_device) {
    out->rp = x->rowptr;
    out->col = x->col;
    out->val = x->val;
    return CUAPSS_OK;
  }
  int64_t* rp = nullptr;
  int32_t* col = nullptr;
  float* val = nullptr;
  ST_TRY(ctx->ws.get(tag + ":in_rp", (size_t)x->n + 1, &rp));
  ST_TRY(ctx->ws.get(tag + ":in_col", (size_t)std::max<int64_t>(x->nnz, 1), &col));
  ST_TRY(ctx->ws.get(tag + ":in_val", (size_t)std::max<int64_t>(x->nnz, 1), &val));
  cudaStream_t st = ctx->stream;
  CU_TRY(cudaMemcpyAsync(rp, x->rowptr, sizeof(int64_t) * (x->n + 1), cudaMemcpyHostToDevice, st));
  if (x->nnz > 0) {
    CU_TRY(cudaMemcpyAsync(col, x->col, sizeof(int32_t) * x->nnz, cudaMemcpyHostToDevice, st));
    CU_TRY(cudaMemcpyAsync(val, x->val, sizeof(float) * x->nnz, cudaMemcpyHostToDevice, st));
  }
  out->rp = rp;
  out->col = col;
  out->val = val;
  return CUAPSS_OK;
}

namespace {

float elapsed(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  return ms;
}

}  // namespace

cuapss_status join_device(cuapss_ctx* ctx, const DevCsr& a, const DevCsr* b, float t,
                          cuapss_pairs* out, cuapss_stats* stats, int shard, int nshards) {
  if (nshards < 1 || shard < 0 || shard >= nshards) return CUAPSS_EINVAL;
  const bool self = (b == nullptr);
  const DevCsr& bb = self ? a : *b;
  if (!self && a.d != bb.d) return CUAPSS_EINVAL;
  if (!(t > 0.0f) || !std::isfinite(t)) return CUAPSS_EINVAL;
  if (!out || out->capacity < 0) return CUAPSS_EINVAL;
  if (out->capacity > 0 && (!out->i || !out->j || !out->sim)) return CUAPSS_EINVAL;
  cudaStream_t st = ctx->stream;
  Workspace& ws = ctx->ws;
  const int64_t d = a.d;
  const int64_t launches0 = g_launches.load();
  cudaEventRecord(ctx->ev[0], st);
  StageRange nvtx("cuapss_run:prepare");
  // ---- validate + posting counts + frequency remap ----
  int32_t* counts = nullptr;
  int32_t* perm = nullptr;
  ST_TRY(ws.get("counts", (size_t)d, &counts));
  ST_TRY(ws.get("perm", (size_t)d, &perm));
  CU_TRY(cudaMemsetAsync(counts, 0, sizeof(int32_t) * d, st));
  double nrm_a = 1.0, nrm_b = 1.0;
  const int check = ctx->opts.validate;
  ST_TRY(validate_csr(a.rp, a.col, a.val, a.n, d, a.nnz, ctx->opts.norm_tol, check, counts, &nrm_a,
                      ws, "A", st));
  if (!self)
    ST_TRY(validate_csr(bb.rp, bb.col, bb.val, bb.n, d, bb.nnz, ctx->opts.norm_tol, check, counts,
                        &nrm_b, ws, "B", st));
  else
    nrm_b = nrm_a;
  ST_TRY(feature_perm(counts, d, a.n + (self ? 0 : bb.n), ctx->opts.remap, perm, ws, st));
  const int precision = ctx->opts.precision;
  // Tail features that occur in at most a few rows are paired explicitly
  // (self-joins; a shard builds the pairs of its own tile rows): probing
  // their postings in every tile is
  // almost all misses. They are the highest ranks only under the frequency
  // remap. The threshold and the head width are chosen together: the head
  // is sized against the tail that is still probed, each threshold's pairs
  // cost their build and their additions.
  std::vector<RareCandidate> rare;
  const int forced_rare = ctx->opts.rare_max_count;
  // below kRareMinRows rows the pairs cannot pay for the planning's extra
  // host round trips (unless forced)
  if (self && ctx->opts.remap &&
      (forced_rare > 0 || (forced_rare == 0 && a.n >= kRareMinRows))) {
    ST_TRY(rare_feature_candidates(counts, d, ws, st, &rare));
    if (forced_rare > 0) {
      std::vector<RareCandidate> keep;
      for (const RareCandidate& c : rare)
        if (c.max_count == forced_rare) keep.push_back(c);
      rare.swap(keep);
    }
  }
  const int64_t n_all = a.n + (self ? 0 : bb.n), nnz_all = a.nnz + (self ? 0 : bb.nnz);
  std::vector<int64_t> prefix;
  if (precision == CUAPSS_PREC_MIXED || !rare.empty())
    ST_TRY(rank_count_prefix(counts, d, ctx->opts.remap, kMaxModelHead, ws, st, &prefix));
  int64_t max_pairs = 0;
  if (!rare.empty()) {
    size_t free_b = 0, total_b = 0;
    CU_TRY(cudaMemGetInfo(&free_b, &total_b));
    max_pairs = std::min<int64_t>(
        kMaxExplicitPairs, (int64_t)((double)free_b * kExplicitMemShare / kExplicitPairBytes));
  }
  if (forced_rare > 0 && !rare.empty() && rare[0].pairs > max_pairs) return CUAPSS_ENOMEM;
  const TilePlan plan = plan_tiles(precision, n_all, d, nnz_all, prefix, rare, max_pairs,
                                   ctx->opts.head_width, forced_rare > 0);
  int p = plan.p;
  const bool mixed = precision == CUAPSS_PREC_MIXED;
  const int pq = mixed ? 64 : 32;  // head width granularity of the tile kernels
  p = (int)std::min<int64_t>(((int64_t)p + pq - 1) / pq * pq, ((d + pq - 1) / pq) * pq);
  if (mixed && p < 64) p = 64;
  PrepOptions po;
  po.p = p;
  // Rows are dealt into 128-row blocks by their tail non-zeros, so every
  // block's tail is near the mean: the tail's shared-memory staging fits
  // every block (no chunked staging, the kernel variant with more operand
  // stages) and the tiles' tail work is even. The finalize maps rows back.
  // (a sharded run keeps the caller's order: shard s owns the caller-row
  // blocks b with b % nshards == s, which cuapss_shard_blocks lists)
  po.balance_rows = nshards == 1 ? 1 : 0;
  po.want_head32 = mixed ? 0 : 1;
  po.want_head16 = mixed ? 1 : 0;
  if (plan.rare.max_count > 0) {
    // the head keeps its p ranks in any case
    po.rare_from = std::max<int64_t>(plan.rare.rank, p);
    po.rare_max_count = plan.rare.max_count;
    po.rare_shard = shard;
    po.rare_nshards = nshards;
  }
  const bool head_bound = mixed && head_bound_plan(p, n_all, nnz_all, prefix, plan.rare);
  Side SA, SB;
  SA.rp0 = a.rp;
  SA.col0 = a.col;
  SA.val0 = a.val;
  SA.n = a.n;
  SA.d = d;
  SA.nnz = a.nnz;
  SA.nrm_max = nrm_a;
  ST_TRY(build_side(SA, po, perm, ws, "A", st));
  Side* SJ = &SA;
  if (!self) {
    SB.rp0 = bb.rp;
    SB.col0 = bb.col;
    SB.val0 = bb.val;
    SB.n = bb.n;
    SB.d = d;
    SB.nnz = bb.nnz;
    SB.nrm_max = nrm_b;
    ST_TRY(build_side(SB, po, perm, ws, "B", st));
    SJ = &SB;
  }
  cudaEventRecord(ctx->ev[1], st);
  nvtx.next("cuapss_run:tiles");
  // ---- pair tiles ----
  const double nrm2 = nrm_a * nrm_b;
  TileArgs ta{};
  ta.headI32 = SA.head32;
  ta.nI = SA.n;
  ta.nbI = SA.nb;
  ta.blkmaxI = SA.blk_maxnnz;
  ta.hnormI = SA.hnorm;
  ta.bptrI = SA.bptr;
  ta.bilI_key = SA.bil_key;
  ta.bilI_len = SA.bil_len;
  ta.max_tailI = SA.max_block_tail;
  ta.bilI_u = SA.bil_u;
  ta.headJ32 = SJ->head32;
  ta.nJ = SJ->n;
  ta.nbJ = SJ->nb;
  ta.blkmaxJ = SJ->blk_maxnnz;
  ta.hnormJ = SJ->hnorm;
  ta.hptrJ = SJ->hptr;
  ta.bilJ_rec = SJ->bil_rec;
  if (self && SA.n_explicit > 0) {
    ta.ex_off = SA.ex_off;
    ta.ex_rec = SA.ex_rec;
  }
  ta.p = SA.p;
  ta.self = self ? 1 : 0;
  ta.t = t;
  if (nrm2 >= 1.9) return CUAPSS_EINVAL;  // fixed-point tail needs ~unit norms
  if (d - SA.p > (int64_t)(1u << 20) - 2) return CUAPSS_EINVAL;  // 20-bit tail feature keys
  set_tile_margins(ta, nrm2, mixed);
  // ---- units: I block x J range; an I block's J range is cut into chunks
  // of about equal cost, heavier blocks get shorter ranges. CTAs take units
  // from a counter as they get to them.
  const int grid_max = ctx->sms;
  std::vector<int4> units;
  {
    const double avg = std::max(1.0, (double)SA.ntail / std::max(1, SA.nb));
    auto weight = [&](int I) {
      return 1.0 + (double)(SA.h_bptr[I + 1] - SA.h_bptr[I]) / avg;
    };
    // a shard takes the I blocks with I mod nshards == shard
    double total = 0.0;
    for (int I = shard; I < SA.nb; I += nshards) total += weight(I) * (SJ->nb - (self ? I : 0));
    // about 64 units per CTA: the CTAs take them dynamically, so the last
    // ones to finish wait at most a short unit. A unit costs at most about
    // kUnitCostCap (about 256 tiles of mean weight), so that the J windows
    // of the units running at one time stay within L2: the J operands of a
    // 3,200-tile unit (n = 1M, 64 units per CTA) span 0.8 GB, and the tile
    // kernel then read 4.1 TB from DRAM per launch.
    const double target = std::max(1.0, std::min(total / (grid_max * 64.0), kUnitCostCap));
    for (int I = shard; I < SA.nb; I += nshards) {
      const int jb = self ? I : 0, je = SJ->nb;
      const int chunk = (int)std::max(1.0, std::floor(target / weight(I)));
      for (int j0 = jb; j0 < je; j0 += chunk)
        units.push_back(make_int4(I, j0, std::min(je, j0 + chunk), 0));
    }
  }
  order_units_for_l2(units);
  const int grid = std::max(1, std::min((int)units.size(), grid_max));
  int4* d_units = nullptr;
  ST_TRY(ws.get("tiles:units", std::max<size_t>(units.size(), 1), &d_units));
  if (!units.empty())
    CU_TRY(cudaMemcpyAsync(d_units, units.data(), sizeof(int4) * units.size(),
                           cudaMemcpyHostToDevice, st));
  ta.units = d_units;
  ta.nunits = (int)units.size();
  int64_t ncand = 0;
  int* unit_counter = nullptr;
  int* err = nullptr;
  unsigned long long* ccount = nullptr;
  ST_TRY(ws.get("tiles:unit", 1, &unit_counter));
  ST_TRY(ws.get("tiles:err", 1, &err));
  ST_TRY(ws.get("tiles:ccount", 1, &ccount));
  ta.unit_counter = unit_counter;
  ta.err = err;
  ta.cand_count = ccount;
  if (ctx->cand_cap == 0) ctx->cand_cap = std::max<int64_t>(1 << 20, 8 * (a.n + bb.n));
  int64_t ntiles = 0;
  for (const int4& u : units) ntiles += u.z - u.y;
  for (int attempt = 0; attempt < 3; ++attempt) {
    ST_TRY(ws.get("cand:key", (size_t)ctx->cand_cap, &ta.cand_key));
    ST_TRY(ws.get("cand:sim", (size_t)ctx->cand_cap, &ta.cand_sim));
    ta.cand_cap = ctx->cand_cap;
    CU_TRY(cudaMemsetAsync(unit_counter, 0, sizeof(int), st));
    CU_TRY(cudaMemsetAsync(err, 0, sizeof(int), st));
    CU_TRY(cudaMemsetAsync(ccount, 0, sizeof(unsigned long long), st));
    if (ntiles > 0) {
      if (mixed)
        ST_TRY(launch_tiles_mma(ta, SA.head16, SJ->head16, SA.p, grid, st, false, head_bound));
      else ST_TRY(launch_tiles_fp32(ta, grid, st));
    }
    unsigned long long hc = 0;
    int herr = 0;
    CU_TRY(cudaMemcpyAsync(&hc, ccount, sizeof(hc), cudaMemcpyDeviceToHost, st));
    CU_TRY(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CU_TRY(cudaStreamSynchronize(st));
    if (herr & kErrTimeout) return CUAPSS_ETIMEOUT;
    if (herr) return CUAPSS_ECUDA;
    ncand = (int64_t)hc;
    if (ncand <= ctx->cand_cap) break;
    ctx->cand_cap = ncand + ncand / 4;
    if (attempt == 2) return CUAPSS_ENOMEM;
  }
  cudaEventRecord(ctx->ev[2], st);
  nvtx.next("cuapss_run:finalize");
  // ---- finalize: exact decision, reported similarity, sorted output ----
  uint64_t* okey = nullptr;
  uint32_t* oidx = nullptr;
  float* osim = nullptr;
  unsigned long long* ocount = nullptr;
  unsigned long long* nresc = nullptr;
  const int64_t ocap = std::max<int64_t>(ncand, 1);
  ST_TRY(ws.get("out:key", (size_t)ocap, &okey));
  ST_TRY(ws.get("out:idx", (size_t)ocap, &oidx));
  ST_TRY(ws.get("out:sim", (size_t)ocap, &osim));
  ST_TRY(ws.get("out:count", 2, &ocount));
  nresc = ocount + 1;
  CU_TRY(cudaMemsetAsync(ocount, 0, 2 * sizeof(unsigned long long), st));
  const int rbitsJ = std::max(1, bits_for((uint64_t)SJ->n));
  const int rbitsI = std::max(1, bits_for((uint64_t)SA.n));
  FinalizeArgs fa{};
  fa.cand_key = ta.cand_key;
  fa.cand_sim = ta.cand_sim;
  fa.ncand = ncand;
  fa.rowpermI = SA.rowperm;
  fa.rowpermJ = SJ->rowperm;
  fa.nnzI = SA.nnz_row;
  fa.nnzJ = SJ->nnz_row;
  fa.hnormI = SA.hnorm;
  fa.hnormJ = SJ->hnorm;
  fa.rpI = a.rp;
  fa.colI = a.col;
  fa.valI = a.val;
  fa.rpJ = bb.rp;
  fa.colJ = bb.col;
  fa.valJ = bb.val;
  fa.t = t;
  fa.eps_c1 = ta.eps_c1;
  fa.eps_c0 = ta.eps_c0;
  fa.eps_head = ta.eps_head;
  fa.self = self ? 1 : 0;
  fa.rbits = rbitsJ;
  fa.out_key = okey;
  fa.out_idx = oidx;
  fa.out_sim = osim;
  fa.out_count = ocount;
  fa.out_cap = ocap;
  fa.n_rescored = nresc;
  ST_TRY(launch_finalize(fa, st));
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
    stats->head_width = SA.p;
    stats->tail_entries = SA.ntail + (self ? 0 : SJ->ntail);
    stats->tail_products = SA.tail_products;
    int32_t kmax = 0;
    if (SA.nb > 0)
      cudaMemcpy(&kmax, SA.blk_maxnnz, sizeof(int32_t), cudaMemcpyDeviceToHost);
    stats->max_band = ta.eps_c1 * kmax + ta.eps_c0;
    stats->ms_preprocess = elapsed(ctx->ev[0], ctx->ev[1]);
    stats->ms_index = 0.0;
    stats->ms_tiles = elapsed(ctx->ev[1], ctx->ev[2]);
    stats->ms_finalize = elapsed(ctx->ev[2], ctx->ev[3]);
    stats->ms_total = elapsed(ctx->ev[0], ctx->ev[3]);
    stats->launches = g_launches.load() - launches0;
    stats->explicit_pairs = SA.n_explicit;
    stats->rare_max_count = po.rare_max_count;
  }
  return result;
}

}  // namespace cuapss

using namespace cuapss;

extern "C" {

void cuapss_default_opts(cuapss_opts* o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->device = 0;
  o->stream = nullptr;
  o->precision = CUAPSS_PREC_FP32;
  o->head_width = 0;
  o->remap = 1;
  o->validate = 1;
  o->norm_tol = 1e-4f;
  o->verbose = 0;
  o->rare_max_count = 0;
}

const char* cuapss_status_string(cuapss_status s) {
  switch (s) {
    case CUAPSS_OK: return "ok";
    case CUAPSS_EINVAL: return "invalid argument";
    case CUAPSS_ENOMEM: return "out of memory";
    case CUAPSS_EOVERFLOW: return "output capacity too small";
    case CUAPSS_ETIMEOUT: return "bounded wait timed out";
    case CUAPSS_ECUDA: return "CUDA error";
    case CUAPSS_EBUSY: return "admission refused";
  }
  return "unknown status";
}

int cuapss_abi_version(void) { return CUAPSS_ABI_VERSION; }

cuapss_status cuapss_create(cuapss_ctx** out, const cuapss_opts* opts) {
  if (!out) return CUAPSS_EINVAL;
  *out = nullptr;
  cuapss_opts o;
  if (opts) o = *opts;
  else cuapss_default_opts(&o);
  if (o.precision != CUAPSS_PREC_FP32 && o.precision != CUAPSS_PREC_MIXED) return CUAPSS_EINVAL;
  if (o.head_width < 0 || !(o.norm_tol >= 0.0f)) return CUAPSS_EINVAL;
  if (o.rare_max_count < -1 || o.rare_max_count > kMaxRareCount ||
      (o.rare_max_count > 0 && (o.rare_max_count < 16 ||
                                (o.rare_max_count & (o.rare_max_count - 1)) != 0)))
    return CUAPSS_EINVAL;
  int ndev = 0;
  CU_TRY(cudaGetDeviceCount(&ndev));
  if (o.device < 0 || o.device >= ndev) return CUAPSS_EINVAL;
  CU_TRY(cudaSetDevice(o.device));
  cuapss_ctx* c = new cuapss_ctx();
  c->device = o.device;
  c->opts = o;
  cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, o.device);
  if (o.stream) {
    c->stream = static_cast<cudaStream_t>(o.stream);
  } else {
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete c;
      return CUAPSS_ECUDA;
    }
    c->own_stream = true;
  }
  for (auto& e : c->ev) cudaEventCreate(&e);
  *out = c;
  return CUAPSS_OK;
}

cuapss_status cuapss_destroy(cuapss_ctx* c) {
  if (!c) return CUAPSS_OK;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  if (c->batch_exec) cudaGraphExecDestroy(c->batch_exec);
  if (c->batch_graph) cudaGraphDestroy(c->batch_graph);
  c->ws.release();
  for (auto& e : c->ev)
    if (e) cudaEventDestroy(e);
  if (c->own_stream) cudaStreamDestroy(c->stream);
  delete c;
  return CUAPSS_OK;
}

cuapss_status cuapss_run(cuapss_ctx* c, const cuapss_csr* x, float t, cuapss_pairs* out,
                         cuapss_stats* stats) {
  if (!c) return CUAPSS_EINVAL;
  CU_TRY(cudaSetDevice(c->device));
  DevCsr a;
  ST_TRY(stage_csr(c, x, "X", &a));
  return join_device(c, a, nullptr, t, out, stats);
}

cuapss_status cuapss_run_shard(cuapss_ctx* c, const cuapss_csr* x, float t, int32_t shard,
                               int32_t nshards, cuapss_pairs* out, cuapss_stats* stats) {
  if (!c) return CUAPSS_EINVAL;
  CU_TRY(cudaSetDevice(c->device));
  DevCsr a;
  ST_TRY(stage_csr(c, x, "X", &a));
  return join_device(c, a, nullptr, t, out, stats, shard, nshards);
}

int32_t cuapss_shard_blocks(int64_t n, int32_t shard, int32_t nshards, int32_t* blocks,
                            int64_t capacity) {
  if (n < 0 || nshards < 1 || shard < 0 || shard >= nshards) return -1;
  const int64_t nb = (n + kBlockRows - 1) / kBlockRows;
  int64_t k = 0;
  for (int64_t b = shard; b < nb; b += nshards, ++k)
    if (blocks && k < capacity) blocks[k] = (int32_t)b;
  return (int32_t)k;
}

cuapss_status cuapss_join(cuapss_ctx* c, const cuapss_csr* a, const cuapss_csr* b, float t,
                          cuapss_pairs* out, cuapss_stats* stats) {
  if (!c) return CUAPSS_EINVAL;
  CU_TRY(cudaSetDevice(c->device));
  DevCsr da, db;
  ST_TRY(stage_csr(c, a, "XA", &da));
  ST_TRY(stage_csr(c, b, "XB", &db));
  if (da.d != db.d) return CUAPSS_EINVAL;
  return join_device(c, da, &db, t, out, stats);
}

cuapss_status cuapss_build_index(cuapss_ctx* c, const cuapss_csr* x, int32_t p, int32_t* dim_ptr,
                                 int32_t* idx_row, float* idx_val, int64_t capacity,
                                 int64_t* tail_nnz) {
  if (!c || !dim_ptr || !tail_nnz || p < 0) return CUAPSS_EINVAL;
  CU_TRY(cudaSetDevice(c->device));
  DevCsr a;
  ST_TRY(stage_csr(c, x, "IX", &a));
  if (a.nnz >= INT32_MAX) return CUAPSS_EINVAL;
  cudaStream_t st = c->stream;
  ST_TRY(validate_csr(a.rp, a.col, a.val, a.n, a.d, a.nnz, 0.f, 0, nullptr, nullptr, c->ws, "IX",
                      st));
  int32_t* dp = nullptr;
  ST_TRY(c->ws.get("ri:dimptr", (size_t)a.d + 1, &dp));
  int32_t* rows = nullptr;
  float* vals = nullptr;
  int64_t T = 0;
  ST_TRY(build_ref_index(a.rp, a.col, a.val, a.n, a.d, p, dp, &rows, &vals, &T, c->ws, st));
  *tail_nnz = T;
  if (T > capacity) {
    CU_TRY(cudaStreamSynchronize(st));
    return CUAPSS_EOVERFLOW;
  }
  if (T > 0 && (!idx_row || !idx_val)) return CUAPSS_EINVAL;
  const cudaMemcpyKind kind = x->on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  CU_TRY(cudaMemcpyAsync(dim_ptr, dp, sizeof(int32_t) * (a.d + 1), kind, st));
  if (T > 0) {
    CU_TRY(cudaMemcpyAsync(idx_row, rows, sizeof(int32_t) * T, kind, st));
    CU_TRY(cudaMemcpyAsync(idx_val, vals, sizeof(float) * T, kind, st));
  }
  CU_TRY(cudaStreamSynchronize(st));
  return CUAPSS_OK;
}

cuapss_status cuapss_feature_remap(cuapss_ctx* c, const cuapss_csr* x, int32_t* perm,
                                   int32_t* counts) {
  if (!c || !perm || !counts) return CUAPSS_EINVAL;
  CU_TRY(cudaSetDevice(c->device));
  DevCsr a;
  ST_TRY(stage_csr(c, x, "RX", &a));
  cudaStream_t st = c->stream;
  int32_t* dc = nullptr;
  int32_t* dp = nullptr;
  ST_TRY(c->ws.get("rm:counts", (size_t)a.d, &dc));
  ST_TRY(c->ws.get("rm:perm", (size_t)a.d, &dp));
  CU_TRY(cudaMemsetAsync(dc, 0, sizeof(int32_t) * a.d, st));
  ST_TRY(validate_csr(a.rp, a.col, a.val, a.n, a.d, a.nnz, 0.f, 0, dc, nullptr, c->ws, "RX", st));
  ST_TRY(feature_perm(dc, a.d, a.n, 1, dp, c->ws, st));
  const cudaMemcpyKind kind = x->on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  CU_TRY(cudaMemcpyAsync(perm, dp, sizeof(int32_t) * a.d, kind, st));
  CU_TRY(cudaMemcpyAsync(counts, dc, sizeof(int32_t) * a.d, kind, st));
  CU_TRY(cudaStreamSynchronize(st));
  return CUAPSS_OK;
}

}  // extern "C"
