/*
 * oracle.c -- CPU restatement of the reference APSS, test infrastructure
 * only (see oracle.h for the reference file:line each function follows).
 * Parity is pinned by tests/golden: the reference's own CPU search
 * (InvertedIndex_search, main.cu:104-141, compiled from its source into
 * oracle/_ref/ by oracle/Makefile) counted pairs on the committed fixture,
 * and this file must reproduce those counts.
 */
#include "oracle.h"

#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int64_t* ptr;  /* [d+1] */
  int32_t* row;  /* [nnz] ascending within a feature */
  float* val;
} csc_t;

static int build_csc(int64_t n, int64_t d, const int64_t* rp, const int32_t* col,
                     const float* val, csc_t* c) {
  const int64_t nnz = rp[n];
  c->ptr = (int64_t*)calloc((size_t)d + 1, sizeof(int64_t));
  c->row = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nnz > 0 ? nnz : 1));
  c->val = (float*)malloc(sizeof(float) * (size_t)(nnz > 0 ? nnz : 1));
  if (!c->ptr || !c->row || !c->val) return -1;
  for (int64_t e = 0; e < nnz; ++e) {
    if (col[e] < 0 || col[e] >= d) return -1;
    c->ptr[col[e] + 1]++;
  }
  for (int64_t f = 0; f < d; ++f) c->ptr[f + 1] += c->ptr[f];
  int64_t* cur = (int64_t*)malloc(sizeof(int64_t) * (size_t)(d > 0 ? d : 1));
  if (!cur) return -1;
  memcpy(cur, c->ptr, sizeof(int64_t) * (size_t)d);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t e = rp[i]; e < rp[i + 1]; ++e) {
      const int64_t k = cur[col[e]]++;
      c->row[k] = (int32_t)i;
      c->val[k] = val[e];
    }
  free(cur);
  return 0;
}

static void free_csc(csc_t* c) {
  free(c->ptr);
  free(c->row);
  free(c->val);
}

/* first position in [lo, hi) with row[pos] > key */
static int64_t upper_bound_i32(const int32_t* a, int64_t lo, int64_t hi, int32_t key) {
  while (lo < hi) {
    const int64_t mid = lo + (hi - lo) / 2;
    if (a[mid] <= key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

typedef struct {
  int32_t* i;
  int32_t* j;
  double* s;
  int64_t n, cap;
} plist_t;

static void plist_push(plist_t* p, int32_t i, int32_t j, double s) {
  if (p->n == p->cap) {
    p->cap = p->cap ? 2 * p->cap : 256;
    p->i = (int32_t*)realloc(p->i, sizeof(int32_t) * (size_t)p->cap);
    p->j = (int32_t*)realloc(p->j, sizeof(int32_t) * (size_t)p->cap);
    p->s = (double*)realloc(p->s, sizeof(double) * (size_t)p->cap);
  }
  p->i[p->n] = i;
  p->j[p->n] = j;
  p->s[p->n] = s;
  p->n++;
}

static int cmp_i32(const void* a, const void* b) {
  const int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
  return (x > y) - (x < y);
}

static int valid_csr(int64_t n, int64_t d, const int64_t* rp, const int32_t* col) {
  if (n < 0 || d < 0 || !rp || rp[0] != 0) return 0;
  for (int64_t i = 0; i < n; ++i) {
    if (rp[i + 1] < rp[i]) return 0;
    for (int64_t e = rp[i]; e < rp[i + 1]; ++e) {
      if (col[e] < 0 || col[e] >= d) return 0;
      if (e > rp[i] && col[e] <= col[e - 1]) return 0;
    }
  }
  return 1;
}

/* Concatenate per-chunk lists in chunk order into the caller's arrays. */
static int64_t gather_chunks(plist_t* chunks, int64_t nch, int64_t cap,
                             int32_t* oi, int32_t* oj, double* os) {
  int64_t total = 0;
  for (int64_t c = 0; c < nch; ++c) {
    for (int64_t k = 0; k < chunks[c].n; ++k, ++total)
      if (total < cap) {
        oi[total] = chunks[c].i[k];
        oj[total] = chunks[c].j[k];
        if (os) os[total] = chunks[c].s[k];
      }
    free(chunks[c].i);
    free(chunks[c].j);
    free(chunks[c].s);
  }
  free(chunks);
  return total;
}

/* Core: rows [r0, r1) of A against the inverted index of B. self=1: only
 * j > i. Accumulation for one pair runs over A's row features ascending. */
static int64_t join_core(int64_t na, const int64_t* arp, const int32_t* acol,
                         const float* aval, int64_t nb, const csc_t* bi, int self,
                         double t, int64_t cap, int32_t* oi, int32_t* oj, double* os) {
  const int64_t CH = 64;
  const int64_t nch = (na + CH - 1) / CH;
  plist_t* chunks = (plist_t*)calloc((size_t)(nch > 0 ? nch : 1), sizeof(plist_t));
#pragma omp parallel
  {
    double* acc = (double*)malloc(sizeof(double) * (size_t)(nb > 0 ? nb : 1));
    unsigned char* seen = (unsigned char*)calloc((size_t)(nb > 0 ? nb : 1), 1);
    int32_t* touched = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nb > 0 ? nb : 1));
#pragma omp for schedule(dynamic, 1)
    for (int64_t c = 0; c < nch; ++c) {
      plist_t* out = &chunks[c];
      const int64_t hi = (c + 1) * CH < na ? (c + 1) * CH : na;
      for (int64_t i = c * CH; i < hi; ++i) {
        int64_t nt = 0;
        for (int64_t e = arp[i]; e < arp[i + 1]; ++e) {
          const int32_t f = acol[e];
          const double x = (double)aval[e];
          int64_t k = bi->ptr[f];
          const int64_t kend = bi->ptr[f + 1];
          if (self) k = upper_bound_i32(bi->row, k, kend, (int32_t)i);
          for (; k < kend; ++k) {
            const int32_t j = bi->row[k];
            if (!seen[j]) {
              seen[j] = 1;
              acc[j] = 0.0;
              touched[nt++] = j;
            }
            acc[j] += x * (double)bi->val[k];
          }
        }
        qsort(touched, (size_t)nt, sizeof(int32_t), cmp_i32);
        for (int64_t q = 0; q < nt; ++q) {
          const int32_t j = touched[q];
          if (acc[j] >= t) plist_push(out, (int32_t)i, j, acc[j]);
          seen[j] = 0;
        }
      }
    }
    free(acc);
    free(seen);
    free(touched);
  }
  return gather_chunks(chunks, nch, cap, oi, oj, os);
}

int64_t oracle_apss_fp64(int64_t n, int64_t d, const int64_t* rowptr,
                         const int32_t* col, const float* val, double t,
                         int64_t cap, int32_t* oi, int32_t* oj, double* os) {
  if (!valid_csr(n, d, rowptr, col)) return -1;
  csc_t c;
  if (build_csc(n, d, rowptr, col, val, &c)) return -1;
  const int64_t r = join_core(n, rowptr, col, val, n, &c, 1, t, cap, oi, oj, os);
  free_csc(&c);
  return r;
}

int64_t oracle_join_fp64(int64_t na, const int64_t* arp, const int32_t* acol,
                         const float* aval, int64_t nb, const int64_t* brp,
                         const int32_t* bcol, const float* bval, int64_t d,
                         double t, int64_t cap, int32_t* oi, int32_t* oj,
                         double* os) {
  if (!valid_csr(na, d, arp, acol) || !valid_csr(nb, d, brp, bcol)) return -1;
  csc_t c;
  if (build_csc(nb, d, brp, bcol, bval, &c)) return -1;
  const int64_t r = join_core(na, arp, acol, aval, nb, &c, 0, t, cap, oi, oj, os);
  free_csc(&c);
  return r;
}

void oracle_pair_sims(const int64_t* rowptr, const int32_t* col,
                      const float* val, int64_t m, const int32_t* pi,
                      const int32_t* pj, double* out) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t q = 0; q < m; ++q) {
    int64_t a = rowptr[pi[q]], ae = rowptr[pi[q] + 1];
    int64_t b = rowptr[pj[q]], be = rowptr[pj[q] + 1];
    double s = 0.0;
    while (a < ae && b < be) {
      if (col[a] < col[b]) ++a;
      else if (col[a] > col[b]) ++b;
      else {
        s += (double)val[a] * (double)val[b];
        ++a;
        ++b;
      }
    }
    out[q] = s;
  }
}

static int cmp_pair(const void* a, const void* b) {
  const int64_t x = *(const int64_t*)a, y = *(const int64_t*)b;
  return (x > y) - (x < y);
}

int64_t oracle_rows_fp64(int64_t n, int64_t d, const int64_t* rowptr,
                         const int32_t* col, const float* val, double t,
                         int64_t m, const int32_t* rows, int64_t cap,
                         int32_t* oi, int32_t* oj, double* os) {
  if (!valid_csr(n, d, rowptr, col)) return -1;
  csc_t c;
  if (build_csc(n, d, rowptr, col, val, &c)) return -1;
  plist_t* per = (plist_t*)calloc((size_t)(m > 0 ? m : 1), sizeof(plist_t));
#pragma omp parallel
  {
    double* acc = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    unsigned char* seen = (unsigned char*)calloc((size_t)(n > 0 ? n : 1), 1);
    int32_t* touched = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
#pragma omp for schedule(dynamic, 1)
    for (int64_t q = 0; q < m; ++q) {
      const int32_t i = rows[q];
      int64_t nt = 0;
      for (int64_t e = rowptr[i]; e < rowptr[i + 1]; ++e) {
        const double x = (double)val[e];
        for (int64_t k = c.ptr[col[e]]; k < c.ptr[col[e] + 1]; ++k) {
          const int32_t j = c.row[k];
          if (j == i) continue;
          if (!seen[j]) {
            seen[j] = 1;
            acc[j] = 0.0;
            touched[nt++] = j;
          }
          acc[j] += x * (double)c.val[k];
        }
      }
      for (int64_t k = 0; k < nt; ++k) {
        const int32_t j = touched[k];
        if (acc[j] >= t)
          plist_push(&per[q], i < j ? i : j, i < j ? j : i, acc[j]);
        seen[j] = 0;
      }
    }
    free(acc);
    free(seen);
    free(touched);
  }
  int64_t tot = 0;
  for (int64_t q = 0; q < m; ++q) tot += per[q].n;
  /* key = (i << 32 | j), value index; sort then dedupe */
  int64_t* keys = (int64_t*)malloc(sizeof(int64_t) * 2 * (size_t)(tot > 0 ? tot : 1));
  double* sims = (double*)malloc(sizeof(double) * (size_t)(tot > 0 ? tot : 1));
  int64_t w = 0;
  for (int64_t q = 0; q < m; ++q) {
    for (int64_t k = 0; k < per[q].n; ++k, ++w) {
      keys[2 * w] = ((int64_t)per[q].i[k] << 32) | (uint32_t)per[q].j[k];
      keys[2 * w + 1] = w;
      sims[w] = per[q].s[k];
    }
    free(per[q].i);
    free(per[q].j);
    free(per[q].s);
  }
  free(per);
  qsort(keys, (size_t)tot, 2 * sizeof(int64_t), cmp_pair);
  int64_t out = 0;
  for (int64_t k = 0; k < tot; ++k) {
    if (k > 0 && keys[2 * k] == keys[2 * (k - 1)]) continue;
    if (out < cap) {
      oi[out] = (int32_t)(keys[2 * k] >> 32);
      oj[out] = (int32_t)(keys[2 * k] & 0xffffffff);
      if (os) os[out] = sims[keys[2 * k + 1]];
    }
    ++out;
  }
  free(keys);
  free(sims);
  free_csc(&c);
  return out;
}

int64_t oracle_index_ref(int64_t n, int64_t d, const int64_t* rowptr,
                         const int32_t* col, const float* val, int32_t p,
                         int32_t* dim_ptr, int32_t* idx_row, float* idx_val) {
  if (!valid_csr(n, d, rowptr, col)) return -1;
  /* generate_index_ptr4: per-feature count of entries with id >= p */
  int64_t* cnt = (int64_t*)calloc((size_t)d + 1, sizeof(int64_t));
  for (int64_t e = 0; e < rowptr[n]; ++e)
    if (col[e] >= p) cnt[col[e]]++;
  /* host exclusive scan (similarity_search.cu:1168-1186) */
  int64_t acc = 0;
  for (int64_t f = 0; f < d; ++f) {
    dim_ptr[f] = (int32_t)acc;
    acc += cnt[f];
  }
  dim_ptr[d] = (int32_t)acc;
  /* construct_Index2 with a serial cursor: rows arrive in ascending order */
  for (int64_t f = 0; f < d; ++f) cnt[f] = dim_ptr[f];
  for (int64_t i = 0; i < n; ++i)
    for (int64_t e = rowptr[i]; e < rowptr[i + 1]; ++e)
      if (col[e] >= p) {
        const int64_t k = cnt[col[e]]++;
        idx_row[k] = (int32_t)i;
        idx_val[k] = val[e];
      }
  free(cnt);
  return acc;
}

static const int32_t* g_cnt_for_sort;
static int cmp_feat(const void* a, const void* b) {
  const int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
  if (g_cnt_for_sort[x] != g_cnt_for_sort[y])
    return g_cnt_for_sort[x] > g_cnt_for_sort[y] ? -1 : 1;
  return (x > y) - (x < y);
}

void oracle_feature_remap(int64_t n, int64_t d, const int64_t* rowptr,
                          const int32_t* col, int32_t* perm, int32_t* counts) {
  memset(counts, 0, sizeof(int32_t) * (size_t)d);
  for (int64_t e = 0; e < rowptr[n]; ++e) counts[col[e]]++;
  int32_t* order = (int32_t*)malloc(sizeof(int32_t) * (size_t)(d > 0 ? d : 1));
  for (int64_t f = 0; f < d; ++f) order[f] = (int32_t)f;
  g_cnt_for_sort = counts;
  qsort(order, (size_t)d, sizeof(int32_t), cmp_feat);
  for (int64_t r = 0; r < d; ++r) perm[order[r]] = (int32_t)r;
  free(order);
}

int oracle_max_threads(void) { return omp_get_max_threads(); }

/* ---------------- OpenMP FP32 hybrid baseline ---------------- */

typedef struct {
  int32_t c;
  float v;
} ent_t;

static int cmp_ent(const void* a, const void* b) {
  const int32_t x = ((const ent_t*)a)->c, y = ((const ent_t*)b)->c;
  return (x > y) - (x < y);
}

struct cpu_hybrid {
  int64_t n;
  int32_t p;
  const int64_t* rowptr;
  ent_t* ent;    /* remapped entries, each row sorted by rank */
  int64_t* hend; /* end of each row's head (rank < p) prefix */
  float* hn;     /* FP32 head norms */
  int64_t* tptr; /* tail inverted lists, rows ascending */
  int32_t* trow;
  float* tval;
};

cpu_hybrid_t* cpu_hybrid_prepare(int64_t n, int64_t d, const int64_t* rowptr,
                                 const int32_t* col, const float* val,
                                 int32_t p, int threads, double* sec_prep) {
  if (!valid_csr(n, d, rowptr, col) || p < 0) return NULL;
  if (threads > 0) omp_set_num_threads(threads);
  const double w0 = omp_get_wtime();
  const int64_t nnz = rowptr[n];
  cpu_hybrid_t* h = (cpu_hybrid_t*)calloc(1, sizeof(cpu_hybrid_t));
  h->n = n;
  h->p = p;
  h->rowptr = rowptr;
  /* frequency remap and per-row re-sort: head = rank < p is a row prefix */
  int32_t* perm = (int32_t*)malloc(sizeof(int32_t) * (size_t)(d > 0 ? d : 1));
  int32_t* cnt = (int32_t*)malloc(sizeof(int32_t) * (size_t)(d > 0 ? d : 1));
  oracle_feature_remap(n, d, rowptr, col, perm, cnt);
  ent_t* ent = (ent_t*)malloc(sizeof(ent_t) * (size_t)(nnz > 0 ? nnz : 1));
  int64_t* hend = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
  float* hn = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < n; ++i) {
    double ss = 0.0;
    int64_t hh = rowptr[i];
    for (int64_t e = rowptr[i]; e < rowptr[i + 1]; ++e) {
      ent[e].c = perm[col[e]];
      ent[e].v = val[e];
    }
    qsort(ent + rowptr[i], (size_t)(rowptr[i + 1] - rowptr[i]), sizeof(ent_t), cmp_ent);
    for (int64_t e = rowptr[i]; e < rowptr[i + 1] && ent[e].c < p; ++e, ++hh)
      ss += (double)ent[e].v * ent[e].v;
    hend[i] = hh;
    hn[i] = (float)sqrt(ss);
  }
  /* tail inverted lists (rows ascending) */
  int64_t* tptr = (int64_t*)calloc((size_t)d + 1, sizeof(int64_t));
  for (int64_t i = 0; i < n; ++i)
    for (int64_t e = hend[i]; e < rowptr[i + 1]; ++e) tptr[ent[e].c + 1]++;
  for (int64_t f = 0; f < d; ++f) tptr[f + 1] += tptr[f];
  const int64_t ntail = tptr[d];
  int32_t* trow = (int32_t*)malloc(sizeof(int32_t) * (size_t)(ntail > 0 ? ntail : 1));
  float* tval = (float*)malloc(sizeof(float) * (size_t)(ntail > 0 ? ntail : 1));
  int64_t* cur = (int64_t*)malloc(sizeof(int64_t) * (size_t)(d > 0 ? d : 1));
  memcpy(cur, tptr, sizeof(int64_t) * (size_t)d);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t e = hend[i]; e < rowptr[i + 1]; ++e) {
      const int64_t k = cur[ent[e].c]++;
      trow[k] = (int32_t)i;
      tval[k] = ent[e].v;
    }
  free(cur);
  free(perm);
  free(cnt);
  h->ent = ent;
  h->hend = hend;
  h->hn = hn;
  h->tptr = tptr;
  h->trow = trow;
  h->tval = tval;
  if (sec_prep) *sec_prep = omp_get_wtime() - w0;
  return h;
}

int64_t cpu_hybrid_query(const cpu_hybrid_t* h, float t, int64_t m,
                         const int64_t* qrows, int64_t q0, int threads,
                         double* sec_query) {
  if (!h) return -1;
  if (threads > 0) omp_set_num_threads(threads);
  const double w0 = omp_get_wtime();
  const int64_t n = h->n;
  const int32_t p = h->p;
  const int64_t* rowptr = h->rowptr;
  const ent_t* ent = h->ent;
  const int64_t* hend = h->hend;
  const float* hn = h->hn;
  const int64_t* tptr = h->tptr;
  const int32_t* trow = h->trow;
  const float* tval = h->tval;
  int64_t found = 0;
#pragma omp parallel reduction(+ : found)
  {
    float* acc = (float*)calloc((size_t)(n > 0 ? n : 1), sizeof(float));
    float* q = (float*)calloc((size_t)(p > 0 ? p : 1), sizeof(float));
#pragma omp for schedule(dynamic, 1)
    for (int64_t k = 0; k < m; ++k) {
      const int64_t i = qrows ? qrows[k] : q0 + k;
      if (i < 0 || i >= n) continue;
      /* tail: feature-parallel accumulation through inverted lists */
      for (int64_t e = hend[i]; e < rowptr[i + 1]; ++e) {
        const int32_t f = ent[e].c;
        const float x = ent[e].v;
        for (int64_t r = upper_bound_i32(trow, tptr[f], tptr[f + 1], (int32_t)i);
             r < tptr[f + 1]; ++r)
          acc[trow[r]] += x * tval[r];
      }
      for (int64_t e = rowptr[i]; e < hend[i]; ++e) q[ent[e].c] = ent[e].v;
      const float hi = hn[i];
      for (int64_t j = i + 1; j < n; ++j) {
        const float a = acc[j];
        acc[j] = 0.0f;
        if (a + hi * hn[j] < t) continue; /* Cauchy-Schwarz prune */
        float s = a;
        for (int64_t e = rowptr[j]; e < hend[j]; ++e) s += q[ent[e].c] * ent[e].v;
        if (s >= t) ++found;
      }
      for (int64_t e = rowptr[i]; e < hend[i]; ++e) q[ent[e].c] = 0.0f;
    }
    free(acc);
    free(q);
  }
  if (sec_query) *sec_query = omp_get_wtime() - w0;
  return found;
}

void cpu_hybrid_free(cpu_hybrid_t* h) {
  if (!h) return;
  free(h->ent);
  free(h->hend);
  free(h->hn);
  free(h->tptr);
  free(h->trow);
  free(h->tval);
  free(h);
}

int64_t cpu_hybrid_apss(int64_t n, int64_t d, const int64_t* rowptr,
                        const int32_t* col, const float* val, float t,
                        int32_t p, int64_t q0, int64_t q1, int threads,
                        double* sec_prep, double* sec_query) {
  cpu_hybrid_t* h = cpu_hybrid_prepare(n, d, rowptr, col, val, p, threads, sec_prep);
  if (!h) return -1;
  if (q1 > n) q1 = n;
  if (q0 < 0) q0 = 0;
  const int64_t found =
      cpu_hybrid_query(h, t, q1 > q0 ? q1 - q0 : 0, NULL, q0, threads, sec_query);
  cpu_hybrid_free(h);
  return found;
}
