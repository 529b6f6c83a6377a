// Request server over a resident index (cuapss_server_*): continuous
// batching of query requests with per-query thresholds, ordered appends,
// admission by the working memory of the batches in flight.
//
// Lanes. Each lane is a host thread with its own context (own CUDA stream,
// own grow-only working memory). A free lane takes, under the queue lock, a
// batch of queued query items, concatenates their rows into one batch CSR
// with one threshold per row, runs it with index_query_rows and hands each
// item its slice of the sorted output (rows of one item are contiguous in
// the batch). Lanes run concurrently, so their batches overlap on the GPU;
// requests that arrive while batches run are picked up by the next lane that
// frees up.
//
// Slices. A query request of more than max_batch_rows rows is queued as
// slices of at most max_batch_rows consecutive rows, so one large request
// never holds a lane for longer than one batch, its slices run on several
// lanes at once, and small requests get on the GPU between them. The
// request is finished when its last slice is; its pairs are the slices'
// pairs in slice order (sorted by query row, then index row).
//
// Order. Among the query items queued ahead of the first queued append, a
// lane fills its batch in the order of submit time + kRowMs per row (the
// item's service cost expressed as age): small requests overtake large ones
// until those have waited kRowMs per row longer, which bounds how long a
// large item can be passed over.
//
// Admission. The working memory of a batch is estimated from its rows,
// non-zeros and the head width, plus its expected candidates (a running
// mean of candidates per query row, 24 bytes each for keys, values and
// output). A batch is admitted while the estimates of all batches in flight
// stay within hbm_budget; a lone batch is always admitted.
//
// Streams. Each lane's context runs on a stream of the device's lowest
// (default) priority; appends run on one separate context whose stream has
// the highest priority: the queries queued behind an append wait for it, so
// the block scheduler starts an append's CTAs ahead of pending query CTAs.
// (The other way round, appends starved behind the lanes' persistent tile
// kernels: p99 of the mixed workload 560 ms against 240 ms.) An append only
// builds its rows' segment; the segment merges it calls for run on a thread
// of their own with a third context at the lanes' priority, so no lane and
// no queued query waits for a merge.
//
// Appends are taken in submission order by one lane at a time, when they
// are the oldest queued item; queries queued behind an append wait until
// some lane has taken it. A request is matched against the index rows that
// existed when the first of its batches started (for a sliced request, the
// fewest rows any of its slices saw; pairs with rows appended later are
// dropped), reported in cuapss_request_info.index_rows.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "cuapss.h"
#include "serve.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request;
using ReqPtr = std::shared_ptr<Request>;

// The results of one slice of a sliced query request.
struct Part {
  std::vector<int32_t> oi, oj;
  std::vector<float> os;
  int64_t index_rows = 0;
};

struct Request {
  uint64_t id = 0;
  bool append = false;
  int64_t n = 0, d = 0;
  std::vector<int64_t> rp;
  std::vector<int32_t> col;
  std::vector<float> val;
  std::vector<float> t;
  Clock::time_point submit, start, done;
  bool finished = false;
  bool started = false;
  cuapss_status status = CUAPSS_OK;
  std::vector<int32_t> oi, oj;
  std::vector<float> os;
  int64_t batch_id = -1, batch_rows = 0, index_rows = 0;
  // a slice: the request it belongs to, its number and its first row there
  ReqPtr parent;
  int slice = 0;
  int64_t row_off = 0;
  // a sliced request: its slices' results and how many are still running
  std::vector<Part> parts;
  int slices_left = 0;
};

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace

struct cuapss_server {
  cuapss_index* idx = nullptr;
  int device = 0;
  cuapss_server_opts opts{};
  int head_width = 0;
  std::vector<cuapss_ctx*> lanes;
  cuapss_ctx* append_ctx = nullptr;      // appends, high-priority stream
  cuapss_ctx* merge_ctx = nullptr;       // segment merges, the lanes' priority
  std::thread merger;                    // runs the merges the appends call for
  std::vector<cudaStream_t> streams;     // created here, destroyed after the contexts
  std::vector<std::thread> threads;
  std::mutex mu;
  std::condition_variable cv_work, cv_done, cv_merge;
  bool merge_due = false;
  std::deque<ReqPtr> queue;
  std::unordered_map<uint64_t, ReqPtr> reqs;
  uint64_t next_id = 1;
  int64_t next_batch = 0;
  bool stop = false;
  int64_t inflight_bytes = 0;
  double cand_per_row = 64.0;  // running mean of candidates per query row
};

namespace {

// Age, in ms, that one query row of an item is worth when batches are
// filled (see "Order" above).
constexpr double kRowMs = 0.02;

int64_t estimate_bytes(const cuapss_server* s, int64_t rows, int64_t nnz) {
  const double cand = s->cand_per_row * (double)rows;
  return (int64_t)((double)rows * (2.0 * s->head_width + 256.0) + (double)nnz * 64.0 +
                   cand * 24.0) + (1 << 20);
}

// Records the outcome of a finished query item (under the server lock): a
// whole request is finished; a slice fills its part of the request, which
// is finished with its last slice.
void finish_item(Request& r, cuapss_status st, std::vector<int32_t>&& oi, std::vector<int32_t>&& oj,
                 std::vector<float>&& os, int64_t batch_id, int64_t rows, int64_t rows_seen,
                 Clock::time_point now) {
  r.rp.clear();
  r.col.clear();
  r.val.clear();
  if (!r.parent) {
    r.status = st;
    r.oi = std::move(oi);
    r.oj = std::move(oj);
    r.os = std::move(os);
    r.batch_id = batch_id;
    r.batch_rows = rows;
    r.index_rows = rows_seen;
    r.done = now;
    r.finished = true;
    return;
  }
  Request& p = *r.parent;
  Part& part = p.parts[(size_t)r.slice];
  if (st == CUAPSS_OK) {
    for (auto& v : oi) v += (int32_t)r.row_off;
    part.oi = std::move(oi);
    part.oj = std::move(oj);
    part.os = std::move(os);
  } else if (p.status == CUAPSS_OK) {
    p.status = st;
  }
  part.index_rows = rows_seen;
  p.batch_id = std::max(p.batch_id, batch_id);
  p.batch_rows = std::max(p.batch_rows, rows);
  if (--p.slices_left > 0) return;
  // the last slice: one index view for the request, pairs in slice order
  int64_t view = INT64_MAX;
  for (const Part& q : p.parts) view = std::min(view, q.index_rows);
  p.index_rows = view;
  if (p.status == CUAPSS_OK) {
    size_t m = 0;
    for (const Part& q : p.parts) m += q.oi.size();
    p.oi.reserve(m);
    p.oj.reserve(m);
    p.os.reserve(m);
    for (Part& q : p.parts) {
      for (size_t k = 0; k < q.oi.size(); ++k) {
        if (q.oj[k] >= view) continue;  // a row appended after the request's view
        p.oi.push_back(q.oi[k]);
        p.oj.push_back(q.oj[k]);
        p.os.push_back(q.os[k]);
      }
      q = Part();
    }
  }
  p.parts.clear();
  p.done = now;
  p.finished = true;
}

void run_append(cuapss_server* s, cuapss_ctx* ctx, const ReqPtr& r) {
  cuapss_csr x{r->n, r->d, (int64_t)r->col.size(), r->rp.data(), r->col.data(), r->val.data(), 0};
  // the new rows' segment only: its merges run on the merge thread, so the
  // lane (and the queries queued behind the append) wait for no merge
  const cuapss_status st = cuapss::index_append_segment(ctx, s->idx, &x);
  int64_t rows = 0;
  cuapss_index_info(s->idx, &rows, nullptr, nullptr, nullptr);
  std::lock_guard<std::mutex> lk(s->mu);
  s->merge_due = true;
  s->cv_merge.notify_one();
  r->status = st;
  r->index_rows = rows;
  r->done = Clock::now();
  r->finished = true;
  // the data is no longer needed
  r->rp.clear();
  r->col.clear();
  r->val.clear();
}

// The merge thread: after each append, the merges of the index's trailing
// segments that the size policy calls for, one at a time, on its own
// context. A merge that fails leaves the segments as they were (the index
// stays valid, with more segments).
void merge_loop(cuapss_server* s) {
  std::unique_lock<std::mutex> lk(s->mu);
  while (true) {
    s->cv_merge.wait(lk, [s] { return s->merge_due || s->stop; });
    if (s->stop) break;
    s->merge_due = false;
    lk.unlock();
    for (bool merged = true; merged;)
      if (cuapss::index_merge_step(s->merge_ctx, s->idx, &merged) != CUAPSS_OK) break;
    lk.lock();
  }
}

void run_batch(cuapss_server* s, cuapss_ctx* ctx, std::vector<ReqPtr>& batch, int64_t batch_id,
               int64_t est) {
  // concatenate the requests' rows
  int64_t rows = 0, nnz = 0;
  for (auto& r : batch) {
    rows += r->n;
    nnz += (int64_t)r->col.size();
  }
  std::vector<int64_t> rp((size_t)rows + 1, 0);
  std::vector<int32_t> col((size_t)std::max<int64_t>(nnz, 1));
  std::vector<float> val((size_t)std::max<int64_t>(nnz, 1));
  std::vector<float> t((size_t)std::max<int64_t>(rows, 1));
  std::vector<int64_t> first((size_t)batch.size() + 1, 0);
  {
    int64_t ro = 0, eo = 0;
    for (size_t k = 0; k < batch.size(); ++k) {
      const Request& r = *batch[k];
      first[k] = ro;
      for (int64_t i = 0; i < r.n; ++i) rp[ro + i + 1] = eo + r.rp[i + 1];
      std::copy(r.col.begin(), r.col.end(), col.begin() + eo);
      std::copy(r.val.begin(), r.val.end(), val.begin() + eo);
      std::copy(r.t.begin(), r.t.end(), t.begin() + ro);
      ro += r.n;
      eo += (int64_t)r.col.size();
    }
    first[batch.size()] = ro;
  }
  cuapss_csr q{rows, batch[0]->d, nnz, rp.data(), col.data(), val.data(), 0};
  int64_t cap = std::max<int64_t>(1 << 16, rows * 16);
  std::vector<int32_t> oi, oj;
  std::vector<float> os;
  cuapss_status st = CUAPSS_OK;
  cuapss_stats stats{};
  int64_t rows_seen = 0;
  for (int attempt = 0; attempt < 3; ++attempt) {
    oi.resize((size_t)cap);
    oj.resize((size_t)cap);
    os.resize((size_t)cap);
    cuapss_pairs out{oi.data(), oj.data(), os.data(), cap, 0, 0};
    st = cuapss::index_query_rows(ctx, s->idx, &q, t.data(), &out, &stats, &rows_seen);
    if (st == CUAPSS_EOVERFLOW) {
      cap = out.count;
      continue;
    }
    if (st == CUAPSS_OK) {
      oi.resize((size_t)out.count);
      oj.resize((size_t)out.count);
      os.resize((size_t)out.count);
    }
    break;
  }
  // split by item: pairs are sorted by batch row
  std::vector<size_t> cut(batch.size() + 1, oi.size());
  if (st == CUAPSS_OK) {
    for (size_t k = 0; k <= batch.size(); ++k)
      cut[k] = (size_t)(std::lower_bound(oi.begin(), oi.end(), (int32_t)first[k]) - oi.begin());
  }
  std::vector<std::vector<int32_t>> pi(batch.size()), pj(batch.size());
  std::vector<std::vector<float>> ps(batch.size());
  if (st == CUAPSS_OK) {
    for (size_t k = 0; k < batch.size(); ++k) {
      const size_t a = cut[k], b = cut[k + 1];
      pi[k].resize(b - a);
      for (size_t m = a; m < b; ++m) pi[k][m - a] = oi[m] - (int32_t)first[k];
      pj[k].assign(oj.begin() + a, oj.begin() + b);
      ps[k].assign(os.begin() + a, os.begin() + b);
    }
  }
  const Clock::time_point now = Clock::now();
  std::lock_guard<std::mutex> lk(s->mu);
  for (size_t k = 0; k < batch.size(); ++k)
    finish_item(*batch[k], st, std::move(pi[k]), std::move(pj[k]), std::move(ps[k]), batch_id,
                rows, rows_seen, now);
  if (st == CUAPSS_OK && rows > 0) {
    const double per = (double)stats.candidates / (double)rows;
    s->cand_per_row = 0.8 * s->cand_per_row + 0.2 * per;
  }
  s->inflight_bytes -= est;
}

void lane_loop(cuapss_server* s, int lane) {
  cuapss_ctx* ctx = s->lanes[lane];
  for (;;) {
    std::vector<ReqPtr> batch;
    ReqPtr app;
    int64_t est = 0, bid = 0;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      for (;;) {
        if (!s->queue.empty()) {
          if (s->queue.front()->append) {
            app = s->queue.front();
            s->queue.pop_front();
            app->start = Clock::now();
            break;
          }
          // query items ahead of the first append, cheapest (age + rows) first
          std::vector<size_t> cand;
          for (size_t k = 0; k < s->queue.size() && cand.size() < 1024; ++k) {
            if (s->queue[k]->append) break;
            cand.push_back(k);
          }
          auto key = [&](size_t k) {
            const Request& r = *s->queue[k];
            return std::chrono::duration<double, std::milli>(r.submit.time_since_epoch()).count() +
                   kRowMs * (double)r.n;
          };
          std::stable_sort(cand.begin(), cand.end(),
                           [&](size_t a, size_t b) { return key(a) < key(b); });
          int64_t rows = 0, nnz = 0;
          std::vector<size_t> take;
          for (size_t k : cand) {
            const Request& r = *s->queue[k];
            const int64_t nr = rows + r.n, nz = nnz + (int64_t)r.col.size();
            if (!take.empty() && nr > s->opts.max_batch_rows) continue;
            const int64_t e = estimate_bytes(s, nr, nz);
            if (s->inflight_bytes + e > s->opts.hbm_budget && (!take.empty() || s->inflight_bytes > 0))
              continue;
            rows = nr;
            nnz = nz;
            est = e;
            take.push_back(k);
          }
          if (!take.empty()) {
            const Clock::time_point now = Clock::now();
            std::sort(take.begin(), take.end());
            for (size_t k : take) {
              ReqPtr r = s->queue[k];
              r->start = now;
              Request& owner = r->parent ? *r->parent : *r;
              if (!owner.started) {
                owner.started = true;
                owner.start = now;
              }
              batch.push_back(r);
            }
            for (size_t m = take.size(); m-- > 0;)
              s->queue.erase(s->queue.begin() + (std::ptrdiff_t)take[m]);
            s->inflight_bytes += est;
            bid = s->next_batch++;
            break;
          }
        } else if (s->stop) {
          return;
        }
        s->cv_work.wait(lk);
      }
    }
    if (app) run_append(s, s->append_ctx, app);
    else run_batch(s, ctx, batch, bid, est);
    s->cv_done.notify_all();
    s->cv_work.notify_all();
  }
}

cuapss_status copy_request(const cuapss_csr* x, Request* r) {
  if (!x || x->on_device || x->n < 0 || x->nnz < 0 || !x->rowptr) return CUAPSS_EINVAL;
  if (x->nnz > 0 && (!x->col || !x->val)) return CUAPSS_EINVAL;
  if (x->rowptr[0] != 0 || x->rowptr[x->n] != x->nnz) return CUAPSS_EINVAL;
  r->n = x->n;
  r->d = x->d;
  r->rp.assign(x->rowptr, x->rowptr + x->n + 1);
  r->col.assign(x->col, x->col + x->nnz);
  r->val.assign(x->val, x->val + x->nnz);
  return CUAPSS_OK;
}

uint64_t enqueue(cuapss_server* s, ReqPtr r) {
  std::lock_guard<std::mutex> lk(s->mu);
  r->id = s->next_id++;
  r->submit = Clock::now();
  s->reqs[r->id] = r;
  const int64_t cap = s->opts.max_batch_rows;
  if (r->append || r->n <= cap) {
    s->queue.push_back(r);
  } else {
    // slices of at most max_batch_rows rows
    const int ns = (int)((r->n + cap - 1) / cap);
    r->parts.resize((size_t)ns);
    r->slices_left = ns;
    for (int k = 0; k < ns; ++k) {
      auto sl = std::make_shared<Request>();
      const int64_t lo = (int64_t)k * cap, hi = std::min(r->n, lo + cap);
      sl->parent = r;
      sl->slice = k;
      sl->row_off = lo;
      sl->n = hi - lo;
      sl->d = r->d;
      sl->submit = r->submit;
      const int64_t e0 = r->rp[(size_t)lo], e1 = r->rp[(size_t)hi];
      sl->rp.resize((size_t)(hi - lo) + 1);
      for (int64_t i = lo; i <= hi; ++i) sl->rp[(size_t)(i - lo)] = r->rp[(size_t)i] - e0;
      sl->col.assign(r->col.begin() + e0, r->col.begin() + e1);
      sl->val.assign(r->val.begin() + e0, r->val.begin() + e1);
      sl->t.assign(r->t.begin() + lo, r->t.begin() + hi);
      s->queue.push_back(sl);
    }
    r->rp.clear();
    r->col.clear();
    r->val.clear();
    r->t.clear();
  }
  s->cv_work.notify_all();
  return r->id;
}

}  // namespace

extern "C" {

void cuapss_server_default_opts(cuapss_server_opts* o) {
  if (!o) return;
  o->lanes = 3;
  o->max_batch_rows = 1024;
  o->hbm_budget = (int64_t)16 << 30;
}

cuapss_status cuapss_server_create(cuapss_server** out, cuapss_index* idx, int device,
                                   const cuapss_server_opts* o) {
  if (!out || !idx) return CUAPSS_EINVAL;
  *out = nullptr;
  cuapss_server_opts opts;
  cuapss_server_default_opts(&opts);
  if (o) opts = *o;
  if (opts.lanes < 1 || opts.lanes > 16 || opts.max_batch_rows < 1 || opts.hbm_budget < 1)
    return CUAPSS_EINVAL;
  auto s = std::make_unique<cuapss_server>();
  s->idx = idx;
  s->device = device;
  s->opts = opts;
  int32_t p = 0;
  cuapss_status st = cuapss_index_info(idx, nullptr, nullptr, &p, nullptr);
  if (st != CUAPSS_OK) return st;
  s->head_width = p;
  auto undo = [&s]() {
    for (auto* x : s->lanes) cuapss_destroy(x);
    if (s->append_ctx) cuapss_destroy(s->append_ctx);
    if (s->merge_ctx) cuapss_destroy(s->merge_ctx);
    for (auto q : s->streams) cudaStreamDestroy(q);
  };
  int least = 0, greatest = 0;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess)
    return CUAPSS_ECUDA;
  // the lanes, then the append context, then the merge context
  for (int l = 0; l <= opts.lanes + 1; ++l) {
    const bool append = l == opts.lanes, merge = l == opts.lanes + 1;
    cudaStream_t q = nullptr;
    if (cudaStreamCreateWithPriority(&q, cudaStreamNonBlocking, append ? greatest : least) !=
        cudaSuccess) {
      undo();
      return CUAPSS_ECUDA;
    }
    s->streams.push_back(q);
    cuapss_opts co;
    cuapss_default_opts(&co);
    co.device = device;
    co.stream = q;
    cuapss_ctx* c = nullptr;
    st = cuapss_create(&c, &co);
    if (st != CUAPSS_OK) {
      undo();
      return st;
    }
    if (append) s->append_ctx = c;
    else if (merge) s->merge_ctx = c;
    else s->lanes.push_back(c);
  }
  for (int l = 0; l < opts.lanes; ++l) s->threads.emplace_back(lane_loop, s.get(), l);
  s->merger = std::thread(merge_loop, s.get());
  *out = s.release();
  return CUAPSS_OK;
}

cuapss_status cuapss_server_submit_query(cuapss_server* s, const cuapss_csr* q, const float* t,
                                         uint64_t* ticket) {
  if (!s || !ticket) return CUAPSS_EINVAL;
  auto r = std::make_shared<Request>();
  const cuapss_status st = copy_request(q, r.get());
  if (st != CUAPSS_OK) return st;
  if (q->n > 0 && !t) return CUAPSS_EINVAL;
  for (int64_t i = 0; i < q->n; ++i)
    if (!(t[i] > 0.0f) || !(t[i] < 1e30f)) return CUAPSS_EINVAL;
  r->t.assign(t, t + q->n);
  *ticket = enqueue(s, r);
  return CUAPSS_OK;
}

cuapss_status cuapss_server_submit_append(cuapss_server* s, const cuapss_csr* x,
                                          uint64_t* ticket) {
  if (!s || !ticket) return CUAPSS_EINVAL;
  auto r = std::make_shared<Request>();
  r->append = true;
  const cuapss_status st = copy_request(x, r.get());
  if (st != CUAPSS_OK) return st;
  *ticket = enqueue(s, r);
  return CUAPSS_OK;
}

cuapss_status cuapss_server_wait(cuapss_server* s, uint64_t ticket, int32_t timeout_ms,
                                 cuapss_pairs* out, cuapss_request_info* info) {
  if (!s) return CUAPSS_EINVAL;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return CUAPSS_EINVAL;
  ReqPtr r = it->second;
  auto ready = [&] { return r->finished; };
  if (timeout_ms < 0) {
    s->cv_done.wait(lk, ready);
  } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
    return CUAPSS_ETIMEOUT;
  }
  if (info) {
    info->status = r->status;
    info->pairs = (int64_t)r->oi.size();
    info->queue_ms = ms_between(r->submit, r->start);
    info->latency_ms = ms_between(r->submit, r->done);
    info->batch_id = r->batch_id;
    info->batch_rows = r->batch_rows;
    info->index_rows = r->index_rows;
  }
  if (r->status != CUAPSS_OK) {
    s->reqs.erase(it);
    return r->status;
  }
  if (out) {
    const int64_t m = (int64_t)r->oi.size();
    out->count = m;
    if (m > out->capacity) return CUAPSS_EOVERFLOW;
    if (m > 0 && (!out->i || !out->j || !out->sim || out->on_device)) return CUAPSS_EINVAL;
    std::memcpy(out->i, r->oi.data(), sizeof(int32_t) * m);
    std::memcpy(out->j, r->oj.data(), sizeof(int32_t) * m);
    std::memcpy(out->sim, r->os.data(), sizeof(float) * m);
  }
  s->reqs.erase(it);
  return CUAPSS_OK;
}

cuapss_status cuapss_server_destroy(cuapss_server* s) {
  if (!s) return CUAPSS_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  s->cv_merge.notify_all();
  for (auto& th : s->threads) th.join();
  if (s->merger.joinable()) s->merger.join();
  for (auto* c : s->lanes) cuapss_destroy(c);
  if (s->append_ctx) cuapss_destroy(s->append_ctx);
  if (s->merge_ctx) cuapss_destroy(s->merge_ctx);
  for (auto q : s->streams) cudaStreamDestroy(q);
  delete s;
  return CUAPSS_OK;
}

}  // extern "C"
