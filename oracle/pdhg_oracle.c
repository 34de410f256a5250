/* pdhg_oracle.c — TEST ORACLE: C restatement of the reference r²HPDHG path.
 * See pdhg_oracle.h for scope, the reference files it follows, and how it is pinned.
 * Single-threaded; every sum is taken in the reference's order; compiled with
 * -ffp-contract=off so a*b+c rounds twice, as in the reference's x86-64 build. */
#include "pdhg_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

enum { ST_OPTIMAL, ST_INFEASIBLE, ST_UNBOUNDED, ST_ITERLIMIT, ST_TIMELIMIT, ST_NUMERICAL, ST_NOTSOLVED };

static const double kFirstOrderFast = 1e-4;      /* tolerances.h:9 */
static const double kFirstOrderInfeasible = 1e-8; /* tolerances.h:14 */
static const double kMixedPrecisionSwitch = 1e-6; /* tolerances.h:23 */
static const double kVerifyPrimal = 1e-6, kVerifyDual = 1e-6, kVerifyGap = 1e-6; /* tolerances.h:34-36 */

static void* xmalloc(size_t n) {
  void* p = malloc(n ? n : 1);
  if (!p) {
    fprintf(stderr, "pdhg_oracle: out of memory\n");
    abort();
  }
  return p;
}
static double* dvec(size_t n, double v) {
  double* p = (double*)xmalloc(n * sizeof(double));
  for (size_t i = 0; i < n; ++i) p[i] = v;
  return p;
}
static double dmaxd(double a, double b) { return (a < b) ? b : a; } /* std::max */
static double dmind(double a, double b) { return (b < a) ? b : a; } /* std::min */

/* ------------------------------------------------------------------ CSR (csr.h:19-43) */
typedef struct {
  int rows, cols;
  int64_t* rp;
  int* col;
  double* val;
} csr;

static int64_t csr_nnz(const csr* a) { return a->rp[a->rows]; }
static void csr_free(csr* a) {
  free(a->rp);
  free(a->col);
  free(a->val);
  memset(a, 0, sizeof *a);
}
static csr csr_copy(const csr* a) {
  csr t = *a;
  int64_t nz = csr_nnz(a);
  t.rp = (int64_t*)xmalloc((size_t)(a->rows + 1) * sizeof(int64_t));
  memcpy(t.rp, a->rp, (size_t)(a->rows + 1) * sizeof(int64_t));
  t.col = (int*)xmalloc((size_t)nz * sizeof(int));
  memcpy(t.col, a->col, (size_t)nz * sizeof(int));
  t.val = (double*)xmalloc((size_t)nz * sizeof(double));
  memcpy(t.val, a->val, (size_t)nz * sizeof(double));
  return t;
}
/* transpose (csr.cpp:19-36): rows visited in order, so columns of t come out sorted */
static csr csr_transpose(const csr* a) {
  csr t;
  t.rows = a->cols;
  t.cols = a->rows;
  int64_t nz = csr_nnz(a);
  t.rp = (int64_t*)calloc((size_t)t.rows + 1, sizeof(int64_t));
  for (int64_t k = 0; k < nz; ++k) ++t.rp[a->col[k] + 1];
  for (int i = 0; i < t.rows; ++i) t.rp[i + 1] += t.rp[i];
  t.col = (int*)xmalloc((size_t)nz * sizeof(int));
  t.val = (double*)xmalloc((size_t)nz * sizeof(double));
  int64_t* next = (int64_t*)xmalloc((size_t)(t.rows + 1) * sizeof(int64_t));
  memcpy(next, t.rp, (size_t)t.rows * sizeof(int64_t));
  for (int i = 0; i < a->rows; ++i)
    for (int64_t k = a->rp[i]; k < a->rp[i + 1]; ++k) {
      int64_t p = next[a->col[k]]++;
      t.col[p] = i;
      t.val[p] = a->val[k];
    }
  free(next);
  return t;
}
/* CSR of Aᵀ straight from the model's CSC arrays (csr.cpp:8-16) */
static csr csr_transpose_from_model(const orc_model* M) {
  csr r;
  r.rows = M->n;
  r.cols = M->m;
  int nz = M->col_start[M->n];
  r.rp = (int64_t*)xmalloc((size_t)(M->n + 1) * sizeof(int64_t));
  for (int j = 0; j <= M->n; ++j) r.rp[j] = M->col_start[j];
  r.col = (int*)xmalloc((size_t)nz * sizeof(int));
  memcpy(r.col, M->row_index, (size_t)nz * sizeof(int));
  r.val = (double*)xmalloc((size_t)nz * sizeof(double));
  memcpy(r.val, M->value, (size_t)nz * sizeof(double));
  return r;
}
/* out = a·x, double accumulation, row-sequential (csr.h:30-43) */
static void csr_mul_dd(const csr* a, const double* x, double* out) {
  for (int i = 0; i < a->rows; ++i) {
    double s = 0;
    for (int64_t k = a->rp[i]; k < a->rp[i + 1]; ++k) s += a->val[k] * x[a->col[k]];
    out[i] = s;
  }
}

/* ------------------------------------------------------------------ scaling (scaling.cpp) */
struct orc_scaled {
  int m, n, sense;
  csr A, At, A_orig, At_orig;
  double *c, *col_lower, *col_upper, *row_lower, *row_upper, *row_scale, *col_scale;
  double bound_scale, obj_scale, log10_range;
  int geometric_mean_applied;
  const orc_model* M;
};

static void scale_apply(csr* A, const double* r, const double* c) { /* scaling.cpp:12-15 */
  for (int i = 0; i < A->rows; ++i)
    for (int64_t k = A->rp[i]; k < A->rp[i + 1]; ++k) A->val[k] *= r[i] * c[A->col[k]];
}
static void scale_norms(const csr* A, int inf_norm, double* rn, double* cn) { /* scaling.cpp:18-32 */
  for (int i = 0; i < A->rows; ++i) rn[i] = 0.0;
  for (int j = 0; j < A->cols; ++j) cn[j] = 0.0;
  for (int i = 0; i < A->rows; ++i)
    for (int64_t k = A->rp[i]; k < A->rp[i + 1]; ++k) {
      double a = fabs(A->val[k]);
      if (inf_norm) {
        rn[i] = dmaxd(rn[i], a);
        cn[A->col[k]] = dmaxd(cn[A->col[k]], a);
      } else {
        rn[i] += a;
        cn[A->col[k]] += a;
      }
    }
}
static double safe_inv_sqrt(double v) { return v > 0.0 && isfinite(v) ? 1.0 / sqrt(v) : 1.0; }
static double clampf_gm(double v) { return dmind(dmaxd(v, 1e-20), 1e20); }

orc_scaled* orc_scale(const orc_model* M, const orc_scaling_options* opt) { /* scaling.cpp:37-142 */
  orc_scaled* sp = (orc_scaled*)calloc(1, sizeof(orc_scaled));
  const int m = M->m, n = M->n;
  sp->m = m;
  sp->n = n;
  sp->sense = M->sense;
  sp->M = M;
  sp->At_orig = csr_transpose_from_model(M);
  sp->A_orig = csr_transpose(&sp->At_orig);
  sp->A = csr_copy(&sp->A_orig);
  sp->row_scale = dvec((size_t)m, 1.0);
  sp->col_scale = dvec((size_t)n, 1.0);
  double* rn = dvec((size_t)m, 0.0);
  double* cn = dvec((size_t)n, 0.0);
  double* rf = dvec((size_t)m, 0.0);
  double* cf = dvec((size_t)n, 0.0);
  double log10_range = 0.0;
  {
    double amin = INFINITY, amax = 0.0;
    int64_t nz = csr_nnz(&sp->A_orig);
    for (int64_t k = 0; k < nz; ++k) {
      double v = sp->A_orig.val[k];
      if (v != 0.0) amin = dmind(amin, fabs(v)), amax = dmaxd(amax, fabs(v));
    }
    if (amax > 0) log10_range = log10(amax / amin);
  }
  sp->log10_range = log10_range;
  sp->geometric_mean_applied =
      opt->geometric_mean_iterations > 0 && log10_range >= opt->geometric_mean_min_log10_range;
  if (sp->geometric_mean_applied) {
    const csr* A0 = &sp->A_orig;
    double* r = dvec((size_t)m, 1.0);
    double* c = dvec((size_t)n, 1.0);
    double* lo = dvec((size_t)(m > n ? m : n), 0.0);
    double* hi = dvec((size_t)(m > n ? m : n), 0.0);
    for (int it = 0; it < opt->geometric_mean_iterations; ++it) {
      for (int i = 0; i < m; ++i) lo[i] = INFINITY, hi[i] = 0.0;
      for (int i = 0; i < m; ++i)
        for (int64_t k = A0->rp[i]; k < A0->rp[i + 1]; ++k) {
          double v = fabs(A0->val[k]) * c[A0->col[k]];
          if (v > 0 && isfinite(v)) lo[i] = dmind(lo[i], v), hi[i] = dmaxd(hi[i], v);
        }
      for (int i = 0; i < m; ++i)
        if (hi[i] > 0) r[i] = clampf_gm(1.0 / (sqrt(lo[i]) * sqrt(hi[i])));
      for (int j = 0; j < n; ++j) lo[j] = INFINITY, hi[j] = 0.0;
      for (int i = 0; i < m; ++i)
        for (int64_t k = A0->rp[i]; k < A0->rp[i + 1]; ++k) {
          int j = A0->col[k];
          double v = fabs(A0->val[k]) * r[i];
          if (v > 0 && isfinite(v)) lo[j] = dmind(lo[j], v), hi[j] = dmaxd(hi[j], v);
        }
      for (int j = 0; j < n; ++j)
        if (hi[j] > 0) c[j] = clampf_gm(1.0 / (sqrt(lo[j]) * sqrt(hi[j])));
    }
    scale_apply(&sp->A, r, c);
    memcpy(sp->row_scale, r, (size_t)m * sizeof(double));
    memcpy(sp->col_scale, c, (size_t)n * sizeof(double));
    free(r);
    free(c);
    free(lo);
    free(hi);
  }
  for (int it = 0; it < opt->ruiz_iterations; ++it) {
    scale_norms(&sp->A, 1, rn, cn);
    for (int i = 0; i < m; ++i) rf[i] = safe_inv_sqrt(rn[i]);
    for (int j = 0; j < n; ++j) cf[j] = safe_inv_sqrt(cn[j]);
    scale_apply(&sp->A, rf, cf);
    for (int i = 0; i < m; ++i) sp->row_scale[i] *= rf[i];
    for (int j = 0; j < n; ++j) sp->col_scale[j] *= cf[j];
  }
  if (opt->pock_chambolle) {
    scale_norms(&sp->A, 0, rn, cn);
    for (int i = 0; i < m; ++i) rf[i] = safe_inv_sqrt(rn[i]);
    for (int j = 0; j < n; ++j) cf[j] = safe_inv_sqrt(cn[j]);
    scale_apply(&sp->A, rf, cf);
    for (int i = 0; i < m; ++i) sp->row_scale[i] *= rf[i];
    for (int j = 0; j < n; ++j) sp->col_scale[j] *= cf[j];
  }
  sp->c = dvec((size_t)n, 0.0);
  sp->col_lower = dvec((size_t)n, 0.0);
  sp->col_upper = dvec((size_t)n, 0.0);
  for (int j = 0; j < n; ++j) {
    sp->c[j] = sp->col_scale[j] * (double)M->sense * M->c[j];
    sp->col_lower[j] = M->col_lower[j] / sp->col_scale[j];
    sp->col_upper[j] = M->col_upper[j] / sp->col_scale[j];
  }
  sp->row_lower = dvec((size_t)m, 0.0);
  sp->row_upper = dvec((size_t)m, 0.0);
  for (int i = 0; i < m; ++i) {
    sp->row_lower[i] = sp->row_scale[i] * M->row_lower[i];
    sp->row_upper[i] = sp->row_scale[i] * M->row_upper[i];
  }
  sp->bound_scale = 1.0;
  sp->obj_scale = 1.0;
  if (opt->bound_objective_rescaling) {
    double b2 = 0.0, c2 = 0.0;
    for (int i = 0; i < m; ++i) {
      double lo = isfinite(sp->row_lower[i]) ? fabs(sp->row_lower[i]) : 0.0;
      double up = isfinite(sp->row_upper[i]) ? fabs(sp->row_upper[i]) : 0.0;
      double b = dmaxd(lo, up);
      b2 += b * b;
    }
    for (int j = 0; j < n; ++j) c2 += sp->c[j] * sp->c[j];
    sp->bound_scale = 1.0 / (sqrt(b2) + 1.0);
    sp->obj_scale = 1.0 / (sqrt(c2) + 1.0);
    for (int i = 0; i < m; ++i) sp->row_lower[i] *= sp->bound_scale;
    for (int i = 0; i < m; ++i) sp->row_upper[i] *= sp->bound_scale;
    for (int j = 0; j < n; ++j) sp->col_lower[j] *= sp->bound_scale;
    for (int j = 0; j < n; ++j) sp->col_upper[j] *= sp->bound_scale;
    for (int j = 0; j < n; ++j) sp->c[j] *= sp->obj_scale;
  }
  sp->At = csr_transpose(&sp->A);
  free(rn);
  free(cn);
  free(rf);
  free(cf);
  return sp;
}

void orc_scaled_free(orc_scaled* sp) {
  if (!sp) return;
  csr_free(&sp->A);
  csr_free(&sp->At);
  csr_free(&sp->A_orig);
  csr_free(&sp->At_orig);
  free(sp->c);
  free(sp->col_lower);
  free(sp->col_upper);
  free(sp->row_lower);
  free(sp->row_upper);
  free(sp->row_scale);
  free(sp->col_scale);
  free(sp);
}

long long orc_scaled_get(const orc_scaled* sp, int which, double* dst) {
  const double* src = NULL;
  long long len = 0;
  switch (which) {
    case 0: src = sp->A.val, len = csr_nnz(&sp->A); break;
    case 1: src = sp->At.val, len = csr_nnz(&sp->At); break;
    case 2: src = sp->c, len = sp->n; break;
    case 3: src = sp->col_lower, len = sp->n; break;
    case 4: src = sp->col_upper, len = sp->n; break;
    case 5: src = sp->row_lower, len = sp->m; break;
    case 6: src = sp->row_upper, len = sp->m; break;
    case 7: src = sp->row_scale, len = sp->m; break;
    case 8: src = sp->col_scale, len = sp->n; break;
    default: return -1;
  }
  if (dst) memcpy(dst, src, (size_t)len * sizeof(double));
  return len;
}

void orc_scaled_scalars(const orc_scaled* sp, double* out) {
  out[0] = sp->bound_scale;
  out[1] = sp->obj_scale;
  out[2] = sp->log10_range;
  out[3] = sp->geometric_mean_applied ? 1.0 : 0.0;
}

static void unscale_primal(const orc_scaled* sp, const double* xs, double* x) { /* scaling.cpp:144-150 */
  for (int j = 0; j < sp->n; ++j)
    x[j] = dmind(dmaxd(sp->col_scale[j] * xs[j] / sp->bound_scale, sp->M->col_lower[j]), sp->M->col_upper[j]);
}
static void unscale_dual(const orc_scaled* sp, const double* ys, double* y) { /* scaling.cpp:152-155 */
  for (int i = 0; i < sp->m; ++i) y[i] = sp->row_scale[i] * ys[i] / sp->obj_scale;
}

/* ------------------------------------------------------------------ ‖A‖₂ (csr.cpp:54-132) */
static double tridiag_max_eig(const double* a, const double* b, int k) {
  double lo = 1e300, hi = -1e300;
  for (int i = 0; i < k; ++i) {
    double r = (i > 0 ? fabs(b[i - 1]) : 0.0) + (i + 1 < k ? fabs(b[i]) : 0.0);
    lo = dmind(lo, a[i] - r);
    hi = dmaxd(hi, a[i] + r);
  }
  for (int it = 0; it < 200 && hi - lo > 1e-15 * dmaxd(1.0, fabs(hi)); ++it) {
    double mid = 0.5 * (lo + hi);
    int c = 0;
    double d = 1.0;
    for (int i = 0; i < k; ++i) {
      double bb = i > 0 ? b[i - 1] * b[i - 1] : 0.0;
      d = (a[i] - mid) - (i > 0 ? bb / d : 0.0);
      if (d == 0.0) d = -1e-300;
      if (d < 0) ++c;
    }
    if (c == k) hi = mid;
    else lo = mid;
  }
  return hi;
}

static double estimate_norm2(const csr* a, const csr* at) {
  const int n = a->cols;
  if (n == 0 || csr_nnz(a) == 0) return 0.0;
  const int K = 400; /* min(max(400, 20), 400) */
  const double rel_tol = 1e-12;
  double* v = dvec((size_t)n, 0.0);
  double* vprev = dvec((size_t)n, 0.0);
  double* w = dvec((size_t)n, 0.0);
  double* t = dvec((size_t)a->rows, 0.0);
  double* alpha = dvec(K, 0.0);
  double* beta = dvec(K, 0.0);
  int na = 0, nb = 0;
  uint64_t state = 0x9E3779B97F4A7C15ULL;
  double nv = 0;
  for (int j = 0; j < n; ++j) { /* xorshift64* -> uniform(-1, 1) */
    state ^= state >> 12, state ^= state << 25, state ^= state >> 27;
    v[j] = (double)((state * 0x2545F4914F6CDD1DULL) >> 11) / 9007199254740992.0 * 2.0 - 1.0;
    nv += v[j] * v[j];
  }
  nv = sqrt(nv);
  for (int j = 0; j < n; ++j) v[j] /= nv;
  double theta = 0, theta_old = -1;
  int stagnant = 0;
  for (int k = 0; k < K; ++k) {
    csr_mul_dd(a, v, t);
    csr_mul_dd(at, t, w);
    double al = 0;
    for (int j = 0; j < n; ++j) al += w[j] * v[j];
    double bprev = nb == 0 ? 0.0 : beta[nb - 1];
    double bn = 0;
    for (int j = 0; j < n; ++j) {
      w[j] -= al * v[j] + bprev * vprev[j];
      bn += w[j] * w[j];
    }
    bn = sqrt(bn);
    alpha[na++] = al;
    theta = tridiag_max_eig(alpha, beta, na);
    if (bn <= 1e-14 * dmaxd(1.0, theta)) break;
    beta[nb++] = bn;
    if (theta - theta_old <= rel_tol * theta) {
      if (++stagnant >= 5 && k >= 20) break;
    } else {
      stagnant = 0;
    }
    theta_old = theta;
    for (int j = 0; j < n; ++j) {
      vprev[j] = v[j];
      v[j] = w[j] / bn;
    }
  }
  free(v);
  free(vprev);
  free(w);
  free(t);
  free(alpha);
  free(beta);
  return sqrt(dmaxd(theta, 0.0)) * (1.0 + 1e-4);
}

double orc_norm2(const orc_scaled* sp) { return estimate_norm2(&sp->A, &sp->At); }

/* ------------------------------------------------------------------ backend (cpu_backend.cpp) */
typedef struct {
  size_t len;
  double* d;
  float* f;
} ovec;

struct orc_backend {
  const orc_scaled* sp;
  int mixed;
  /* float copies of the scaled problem (Store<float>) */
  float *Af, *Atf, *cf, *lf, *uf, *rlf, *ruf;
  ovec* vecs;
  int nvec, cap;
};

orc_backend* orc_backend_new(const orc_scaled* sp) {
  orc_backend* b = (orc_backend*)calloc(1, sizeof(orc_backend));
  b->sp = sp;
  int64_t nzA = csr_nnz(&sp->A), nzT = csr_nnz(&sp->At);
  b->Af = (float*)xmalloc((size_t)nzA * sizeof(float));
  for (int64_t k = 0; k < nzA; ++k) b->Af[k] = (float)sp->A.val[k];
  b->Atf = (float*)xmalloc((size_t)nzT * sizeof(float));
  for (int64_t k = 0; k < nzT; ++k) b->Atf[k] = (float)sp->At.val[k];
  const double* src[5] = {sp->c, sp->col_lower, sp->col_upper, sp->row_lower, sp->row_upper};
  float** dst[5] = {&b->cf, &b->lf, &b->uf, &b->rlf, &b->ruf};
  for (int q = 0; q < 5; ++q) {
    size_t len = q < 3 ? (size_t)sp->n : (size_t)sp->m;
    *dst[q] = (float*)xmalloc(len * sizeof(float));
    for (size_t i = 0; i < len; ++i) (*dst[q])[i] = (float)src[q][i];
  }
  return b;
}

void orc_backend_free(orc_backend* b) {
  if (!b) return;
  for (int v = 0; v < b->nvec; ++v) free(b->vecs[v].d), free(b->vecs[v].f);
  free(b->vecs);
  free(b->Af);
  free(b->Atf);
  free(b->cf);
  free(b->lf);
  free(b->uf);
  free(b->rlf);
  free(b->ruf);
  free(b);
}

void orc_backend_set_precision(orc_backend* b, int mixed) {
  if (mixed == b->mixed) return;
  for (int v = 0; v < b->nvec; ++v) {
    ovec* V = &b->vecs[v];
    if (mixed)
      for (size_t i = 0; i < V->len; ++i) V->f[i] = (float)V->d[i];
    else
      for (size_t i = 0; i < V->len; ++i) V->d[i] = (double)V->f[i];
  }
  b->mixed = mixed;
}

int orc_backend_create(orc_backend* b, int dual) {
  if (b->nvec == b->cap) {
    b->cap = b->cap ? 2 * b->cap : 16;
    b->vecs = (ovec*)realloc(b->vecs, (size_t)b->cap * sizeof(ovec));
  }
  ovec* V = &b->vecs[b->nvec];
  V->len = dual ? (size_t)b->sp->m : (size_t)b->sp->n;
  V->d = (double*)calloc(V->len ? V->len : 1, sizeof(double));
  V->f = (float*)calloc(V->len ? V->len : 1, sizeof(float));
  return b->nvec++;
}

void orc_backend_upload(orc_backend* b, int v, const double* src) {
  ovec* V = &b->vecs[v];
  if (b->mixed)
    for (size_t i = 0; i < V->len; ++i) V->f[i] = (float)src[i];
  else
    memcpy(V->d, src, V->len * sizeof(double));
}
void orc_backend_download(orc_backend* b, int v, double* dst) {
  ovec* V = &b->vecs[v];
  if (b->mixed)
    for (size_t i = 0; i < V->len; ++i) dst[i] = (double)V->f[i];
  else
    memcpy(dst, V->d, V->len * sizeof(double));
}
void orc_backend_fill(orc_backend* b, int v, double a) {
  ovec* V = &b->vecs[v];
  if (b->mixed) {
    float t = (float)a;
    for (size_t i = 0; i < V->len; ++i) V->f[i] = t;
  } else {
    for (size_t i = 0; i < V->len; ++i) V->d[i] = a;
  }
}
void orc_backend_copy(orc_backend* b, int dst, int src) {
  if (b->mixed)
    memcpy(b->vecs[dst].f, b->vecs[src].f, b->vecs[src].len * sizeof(float));
  else
    memcpy(b->vecs[dst].d, b->vecs[src].d, b->vecs[src].len * sizeof(double));
}
void orc_backend_axpby(orc_backend* b, double a, int x, double bb, int y) {
  size_t n = b->vecs[y].len;
  if (b->mixed) {
    const float ta = (float)a, tb = (float)bb;
    float *Y = b->vecs[y].f, *X = b->vecs[x].f;
    for (size_t i = 0; i < n; ++i) Y[i] = ta * X[i] + tb * Y[i];
  } else {
    double *Y = b->vecs[y].d, *X = b->vecs[x].d;
    for (size_t i = 0; i < n; ++i) Y[i] = a * X[i] + bb * Y[i];
  }
}
static void spmv_any(const csr* M, const float* valf, int mixed, const ovec* X, ovec* O) {
  for (int i = 0; i < M->rows; ++i) {
    double s = 0;
    if (mixed) {
      for (int64_t k = M->rp[i]; k < M->rp[i + 1]; ++k) s += (double)valf[k] * (double)X->f[M->col[k]];
      O->f[i] = (float)s;
    } else {
      for (int64_t k = M->rp[i]; k < M->rp[i + 1]; ++k) s += M->val[k] * X->d[M->col[k]];
      O->d[i] = s;
    }
  }
}
void orc_backend_spmv(orc_backend* b, int x, int out) {
  spmv_any(&b->sp->A, b->Af, b->mixed, &b->vecs[x], &b->vecs[out]);
}
void orc_backend_spmv_t(orc_backend* b, int y, int out) {
  spmv_any(&b->sp->At, b->Atf, b->mixed, &b->vecs[y], &b->vecs[out]);
}

/* parallel_sum with kReduceChunks = 64 fixed chunks (parallel.h:169-188) */
enum { kReduceChunks = 64 };
static double chunk_sum(int64_t n, const ovec* A, const ovec* B, int mixed, int diff) {
  double part[kReduceChunks] = {0};
  const int chunks = (int)(n < kReduceChunks ? (n < 1 ? 1 : n) : kReduceChunks);
  for (int c = 0; c < chunks; ++c) {
    const int64_t lo = n * c / chunks, hi = n * (c + 1) / chunks;
    double s = 0;
    for (int64_t i = lo; i < hi; ++i) {
      double a = mixed ? (double)A->f[i] : A->d[i];
      double bb = mixed ? (double)B->f[i] : B->d[i];
      if (diff) {
        double d = a - bb;
        s += d * d;
      } else {
        s += a * bb;
      }
    }
    part[c] = s;
  }
  double s = 0;
  for (int c = 0; c < chunks; ++c) s += part[c];
  return s;
}
double orc_backend_dot(orc_backend* b, int x, int y) {
  return chunk_sum((int64_t)b->vecs[x].len, &b->vecs[x], &b->vecs[y], b->mixed, 0);
}
double orc_backend_norm2(orc_backend* b, int x) { return sqrt(orc_backend_dot(b, x, x)); }
double orc_backend_diff_norm2(orc_backend* b, int x, int y) {
  return sqrt(chunk_sum((int64_t)b->vecs[x].len, &b->vecs[x], &b->vecs[y], b->mixed, 1));
}

#define OCLAMP(v, lo, hi) ((v) < (lo) ? (lo) : ((v) > (hi) ? (hi) : (v))) /* cpu_backend.cpp:17-20 */

void orc_backend_primal_step(orc_backend* b, int x, int aty, double tau, int xh) {
  const orc_scaled* sp = b->sp;
  size_t n = (size_t)sp->n;
  if (b->mixed) {
    const float t = (float)tau;
    const float *X = b->vecs[x].f, *G = b->vecs[aty].f;
    float* H = b->vecs[xh].f;
    for (size_t j = 0; j < n; ++j) {
      float v = X[j] - t * (b->cf[j] - G[j]);
      H[j] = OCLAMP(v, b->lf[j], b->uf[j]);
    }
  } else {
    const double *X = b->vecs[x].d, *G = b->vecs[aty].d;
    double* H = b->vecs[xh].d;
    for (size_t j = 0; j < n; ++j) {
      double v = X[j] - tau * (sp->c[j] - G[j]);
      H[j] = OCLAMP(v, sp->col_lower[j], sp->col_upper[j]);
    }
  }
}
void orc_backend_dual_step(orc_backend* b, int y, int ax, double sigma, int yh) {
  const orc_scaled* sp = b->sp;
  size_t m = (size_t)sp->m;
  if (b->mixed) {
    const float s = (float)sigma;
    const float *Y = b->vecs[y].f, *AX = b->vecs[ax].f;
    float* H = b->vecs[yh].f;
    for (size_t i = 0; i < m; ++i) {
      float v = AX[i] - Y[i] / s;
      float cl = OCLAMP(v, b->rlf[i], b->ruf[i]);
      H[i] = Y[i] - s * AX[i] + s * cl;
    }
  } else {
    const double *Y = b->vecs[y].d, *AX = b->vecs[ax].d;
    double* H = b->vecs[yh].d;
    for (size_t i = 0; i < m; ++i) {
      double v = AX[i] - Y[i] / sigma;
      double cl = OCLAMP(v, sp->row_lower[i], sp->row_upper[i]);
      H[i] = Y[i] - sigma * AX[i] + sigma * cl;
    }
  }
}
void orc_backend_r2h_primal(orc_backend* b, int x, int x0, int aty, double tau, double w, double rho, int xh,
                            int xb) {
  const orc_scaled* sp = b->sp;
  size_t n = (size_t)sp->n;
  if (b->mixed) {
    const float t = (float)tau, tw = (float)w, a = (float)(2 * rho), bb = (float)(1 - 2 * rho);
    float *X = b->vecs[x].f, *H = b->vecs[xh].f, *B = b->vecs[xb].f;
    const float *X0 = b->vecs[x0].f, *G = b->vecs[aty].f;
    for (size_t j = 0; j < n; ++j) {
      float v = X[j] - t * (b->cf[j] - G[j]);
      const float h = OCLAMP(v, b->lf[j], b->uf[j]);
      H[j] = h;
      B[j] = 2 * h - X[j];
      X[j] = tw * (a * h + bb * X[j]) + (1 - tw) * X0[j];
    }
  } else {
    const double t = tau, tw = w, a = 2 * rho, bb = 1 - 2 * rho;
    double *X = b->vecs[x].d, *H = b->vecs[xh].d, *B = b->vecs[xb].d;
    const double *X0 = b->vecs[x0].d, *G = b->vecs[aty].d;
    for (size_t j = 0; j < n; ++j) {
      double v = X[j] - t * (sp->c[j] - G[j]);
      const double h = OCLAMP(v, sp->col_lower[j], sp->col_upper[j]);
      H[j] = h;
      B[j] = 2 * h - X[j];
      X[j] = tw * (a * h + bb * X[j]) + (1 - tw) * X0[j];
    }
  }
}
void orc_backend_r2h_dual(orc_backend* b, int y, int y0, int ax, double sigma, double w, double rho, int yh,
                          int yb) {
  const orc_scaled* sp = b->sp;
  size_t m = (size_t)sp->m;
  if (b->mixed) {
    const float s = (float)sigma, tw = (float)w, a = (float)(2 * rho), bb = (float)(1 - 2 * rho);
    float *Y = b->vecs[y].f, *H = b->vecs[yh].f, *B = yb >= 0 ? b->vecs[yb].f : NULL;
    const float *Y0 = b->vecs[y0].f, *AX = b->vecs[ax].f;
    for (size_t i = 0; i < m; ++i) {
      float v = AX[i] - Y[i] / s;
      float cl = OCLAMP(v, b->rlf[i], b->ruf[i]);
      const float h = Y[i] - s * AX[i] + s * cl;
      H[i] = h;
      if (B) B[i] = 2 * h - Y[i];
      Y[i] = tw * (a * h + bb * Y[i]) + (1 - tw) * Y0[i];
    }
  } else {
    const double s = sigma, tw = w, a = 2 * rho, bb = 1 - 2 * rho;
    double *Y = b->vecs[y].d, *H = b->vecs[yh].d, *B = yb >= 0 ? b->vecs[yb].d : NULL;
    const double *Y0 = b->vecs[y0].d, *AX = b->vecs[ax].d;
    for (size_t i = 0; i < m; ++i) {
      double v = AX[i] - Y[i] / s;
      double cl = OCLAMP(v, sp->row_lower[i], sp->row_upper[i]);
      const double h = Y[i] - s * AX[i] + s * cl;
      H[i] = h;
      if (B) B[i] = 2 * h - Y[i];
      Y[i] = tw * (a * h + bb * Y[i]) + (1 - tw) * Y0[i];
    }
  }
}

/* ------------------------------------------------------------------ KKT (cpu_backend.cpp:226-284) */
typedef struct {
  double primal_residual, dual_residual, primal_obj, dual_obj, b_norm, c_norm, primal_max_rel, dual_max_rel;
  double obj_shift;
} kkt_stats;

static double rel_primal(const kkt_stats* k) { return k->primal_residual / (1.0 + k->b_norm); }
static double rel_dual(const kkt_stats* k) { return k->dual_residual / (1.0 + k->c_norm); }
static double rel_gap(const kkt_stats* k) {
  return fabs(k->primal_obj - k->dual_obj) /
         (1.0 + fabs(k->primal_obj + k->obj_shift) + fabs(k->dual_obj + k->obj_shift));
}
static double rel_kkt(const kkt_stats* k) { /* std::max({p, d, g}) */
  double r = rel_primal(k), d = rel_dual(k), g = rel_gap(k);
  double mx = r;
  if (mx < d) mx = d;
  if (mx < g) mx = g;
  return mx;
}
static int kkt_converged(const kkt_stats* k, double eps) { /* termination.h:52-56 */
  if (rel_kkt(k) > eps) return 0;
  if (eps >= kVerifyPrimal) return 1;
  return k->primal_max_rel <= kVerifyPrimal && k->dual_max_rel <= kVerifyDual && rel_gap(k) <= kVerifyGap;
}
static int kkt_finite(const kkt_stats* k) {
  return isfinite(k->primal_residual) && isfinite(k->dual_residual) && isfinite(k->primal_obj) &&
         isfinite(k->dual_obj);
}
static double elem_viol(double v, double lo, double up) {
  if (v < lo) return (lo - v) / (1.0 + fabs(lo));
  if (v > up) return (v - up) / (1.0 + fabs(up));
  return 0.0;
}

static kkt_stats kkt_on_original(const orc_scaled* sp, const double* x, const double* y) {
  const orc_model* M = sp->M;
  const double sense = M->sense;
  const int m = sp->m, n = sp->n;
  kkt_stats k;
  memset(&k, 0, sizeof k);
  double* ax = dvec((size_t)m, 0.0);
  double* aty = dvec((size_t)n, 0.0);
  csr_mul_dd(&sp->A_orig, x, ax);
  csr_mul_dd(&sp->At_orig, y, aty);
  double rp2 = 0, rd2 = 0, b2 = 0, c2 = 0, p = 0, d = 0, cinf = 0, pmax = 0, dmax = 0;
  for (int i = 0; i < m; ++i) {
    const double lo = M->row_lower[i], up = M->row_upper[i];
    const double viol = ax[i] < lo ? lo - ax[i] : (ax[i] > up ? ax[i] - up : 0.0);
    rp2 += viol * viol;
    pmax = dmaxd(pmax, elem_viol(ax[i], lo, up));
    const double bl = isfinite(lo) ? fabs(lo) : 0.0, bu = isfinite(up) ? fabs(up) : 0.0;
    b2 += dmaxd(bl, bu) * dmaxd(bl, bu);
    if (y[i] > 0) {
      if (isfinite(lo)) d += y[i] * lo;
      else rd2 += y[i] * y[i], dmax = dmaxd(dmax, y[i]);
    } else if (y[i] < 0) {
      if (isfinite(up)) d += y[i] * up;
      else rd2 += y[i] * y[i], dmax = dmaxd(dmax, -y[i]);
    }
  }
  for (int j = 0; j < n; ++j) {
    const double cj = sense * M->c[j];
    c2 += cj * cj;
    cinf = dmaxd(cinf, fabs(cj));
    p += cj * x[j];
    pmax = dmaxd(pmax, elem_viol(x[j], M->col_lower[j], M->col_upper[j]));
    const double lam = cj - aty[j];
    const double lo = M->col_lower[j], up = M->col_upper[j];
    double z;
    if (isfinite(lo) && isfinite(up)) z = lam;
    else if (isfinite(lo)) z = dmaxd(lam, 0.0);
    else if (isfinite(up)) z = dmind(lam, 0.0);
    else z = 0.0;
    rd2 += (lam - z) * (lam - z);
    dmax = dmaxd(dmax, fabs(lam - z));
    if (z > 0) d += z * lo;
    else if (z < 0) d += z * up;
  }
  k.primal_residual = sqrt(rp2);
  k.dual_residual = sqrt(rd2);
  k.primal_obj = p;
  k.dual_obj = d;
  k.b_norm = sqrt(b2);
  k.c_norm = sqrt(c2);
  k.primal_max_rel = pmax;
  k.dual_max_rel = dmax / (1.0 + cinf);
  free(ax);
  free(aty);
  return k;
}

static kkt_stats backend_kkt(orc_backend* b, int xs, int ys) {
  const orc_scaled* sp = b->sp;
  double* xsd = dvec((size_t)sp->n, 0.0);
  double* ysd = dvec((size_t)sp->m, 0.0);
  double* x = dvec((size_t)sp->n, 0.0);
  double* y = dvec((size_t)sp->m, 0.0);
  orc_backend_download(b, xs, xsd);
  orc_backend_download(b, ys, ysd);
  unscale_primal(sp, xsd, x);
  unscale_dual(sp, ysd, y);
  kkt_stats k = kkt_on_original(sp, x, y);
  free(xsd);
  free(ysd);
  free(x);
  free(y);
  return k;
}

void orc_backend_kkt(orc_backend* b, int xs, int ys, double* out) {
  kkt_stats k = backend_kkt(b, xs, ys);
  out[0] = k.primal_residual;
  out[1] = k.dual_residual;
  out[2] = k.primal_obj;
  out[3] = k.dual_obj;
  out[4] = k.b_norm;
  out[5] = k.c_norm;
  out[6] = k.primal_max_rel;
  out[7] = k.dual_max_rel;
}

/* ------------------------------------------------------------------ ray test (engine.cpp:82-184) */
typedef struct {
  int primal_infeasible, dual_infeasible;
  double dual_ray_objective, dual_ray_violation, primal_ray_objective, primal_ray_violation;
} ray_result;

static ray_result ray_test(const orc_scaled* sp, const double* dxs, const double* dys, double* r_out,
                           double* d_out) {
  const orc_model* M = sp->M;
  const int m = sp->m, n = sp->n;
  ray_result t;
  memset(&t, 0, sizeof t);
  double* r = dvec((size_t)m, 0.0);
  double* g = dvec((size_t)n, 0.0);
  double rmax = 0;
  for (int i = 0; i < m; ++i) {
    double v = sp->row_scale[i] * dys[i] / sp->obj_scale;
    if (!isfinite(M->row_lower[i])) v = dmind(v, 0.0);
    if (!isfinite(M->row_upper[i])) v = dmaxd(v, 0.0);
    r[i] = v;
    rmax = dmaxd(rmax, fabs(v));
  }
  if (rmax > 0) {
    csr_mul_dd(&sp->At_orig, r, g);
    double* gabs = dvec((size_t)n, 0.0);
    for (int j = 0; j < n; ++j)
      for (int k = M->col_start[j]; k < M->col_start[j + 1]; ++k) gabs[j] += fabs(M->value[k] * r[M->row_index[k]]);
    double obj = 0, viol = 0, mag = 0;
    for (int i = 0; i < m; ++i) {
      const double term = r[i] > 0 ? M->row_lower[i] * r[i] : (r[i] < 0 ? M->row_upper[i] * r[i] : 0.0);
      obj += term;
      mag += fabs(term);
    }
    for (int j = 0; j < n; ++j) {
      const double lam = -g[j], lo = M->col_lower[j], up = M->col_upper[j];
      if (lam > 0) {
        if (isfinite(lo)) obj += lo * lam, mag += gabs[j] * fabs(lo);
        else viol = dmaxd(viol, lam);
      } else if (lam < 0) {
        if (isfinite(up)) obj += up * lam, mag += gabs[j] * fabs(up);
        else viol = dmaxd(viol, -lam);
      }
    }
    const double scale = dmaxd(rmax, viol);
    t.dual_ray_objective = obj / scale;
    t.dual_ray_violation = viol / scale;
    t.primal_infeasible = t.dual_ray_objective > 0 && obj > kFirstOrderInfeasible * mag &&
                          t.dual_ray_violation <= kFirstOrderInfeasible * t.dual_ray_objective;
    if (r_out) memcpy(r_out, r, (size_t)m * sizeof(double));
    free(gabs);
  }
  double* d = dvec((size_t)n, 0.0);
  double* ad = dvec((size_t)m, 0.0);
  double dmax = 0;
  for (int j = 0; j < n; ++j) {
    double v = sp->col_scale[j] * dxs[j] / sp->bound_scale;
    if (isfinite(M->col_lower[j])) v = dmaxd(v, 0.0);
    if (isfinite(M->col_upper[j])) v = dmind(v, 0.0);
    d[j] = v;
    dmax = dmaxd(dmax, fabs(v));
  }
  if (dmax > 0) {
    csr_mul_dd(&sp->A_orig, d, ad);
    double cd = 0, viol = 0, cmag = 0;
    for (int j = 0; j < n; ++j) cd += (double)M->sense * M->c[j] * d[j], cmag += fabs(M->c[j] * d[j]);
    for (int i = 0; i < m; ++i) {
      if (isfinite(M->row_lower[i])) viol = dmaxd(viol, -ad[i]);
      if (isfinite(M->row_upper[i])) viol = dmaxd(viol, ad[i]);
    }
    const double scale = dmaxd(dmax, viol);
    t.primal_ray_objective = cd / scale;
    t.primal_ray_violation = viol / scale;
    t.dual_infeasible = t.primal_ray_objective < 0 && -cd > kFirstOrderInfeasible * cmag &&
                        t.primal_ray_violation <= kFirstOrderInfeasible * -t.primal_ray_objective;
    if (d_out) memcpy(d_out, d, (size_t)n * sizeof(double));
  }
  free(r);
  free(g);
  free(d);
  free(ad);
  return t;
}

/* ------------------------------------------------------------------ engine (r2hpdhg.cpp) */
void orc_default_options(orc_options* o) {
  memset(o, 0, sizeof *o);
  o->tolerance = 1e-8;
  o->iteration_limit = 100000000LL;
  o->check_every = 64;
  o->mixed = 0;
  o->scaling.ruiz_iterations = 10;
  o->scaling.pock_chambolle = 1;
  o->scaling.bound_objective_rescaling = 1;
  o->scaling.geometric_mean_iterations = 12;
  o->scaling.geometric_mean_min_log10_range = 4.5;
  o->reflection = 1.0;
  o->restart_sufficient = 0.2;
  o->restart_necessary = 0.5;
  o->restart_artificial = 0.36;
  o->pid_kp = 0.99;
  o->pid_ki = 0.01;
  o->pid_kd = 0.0;
  o->pid_integral_decay = 0.3;
  o->pid_max_log_step = 2.302585092994046;
}

typedef struct {
  const orc_model* M;
  const orc_options* o;
  orc_scaled* sp;
  orc_backend* b;
  double eta;
  long long fast_it;
  double primal_weight;
  double *dual_ray, *primal_ray; /* certificate of the last verdict */
} ctx_t;

static int record(ctx_t* c, const kkt_stats* k, long long it) { /* engine.cpp:224-235 */
  if (c->fast_it < 0 && rel_kkt(k) <= kFirstOrderFast) c->fast_it = it;
  return kkt_converged(k, c->o->tolerance);
}

static int check_infeasibility(ctx_t* c, int dx, int dy, const kkt_stats* current, char* why, size_t whylen) {
  const orc_scaled* sp = c->sp;
  double* dxs = dvec((size_t)sp->n, 0.0);
  double* dys = dvec((size_t)sp->m, 0.0);
  orc_backend_download(c->b, dx, dxs);
  orc_backend_download(c->b, dy, dys);
  double* r = dvec((size_t)sp->m, 0.0);
  double* d = dvec((size_t)sp->n, 0.0);
  ray_result t = ray_test(sp, dxs, dys, r, d);
  int st = ST_NOTSOLVED;
  if (t.primal_infeasible) {
    memcpy(c->dual_ray, r, (size_t)sp->m * sizeof(double));
    snprintf(why, whylen, "primal infeasible: dual ray certificate (objective %f, violation %f)",
             t.dual_ray_objective, t.dual_ray_violation);
    st = ST_INFEASIBLE;
  } else if (t.dual_infeasible) {
    const int feasible = rel_primal(current) <= kVerifyPrimal && current->primal_max_rel <= kVerifyPrimal;
    memcpy(c->primal_ray, d, (size_t)sp->n * sizeof(double));
    snprintf(why, whylen, "unbounded: primal ray certificate (c'd %f, violation %f)%s", t.primal_ray_objective,
             t.primal_ray_violation,
             feasible ? " at a primal-feasible iterate" : "; iterate not primal-feasible yet");
    st = ST_UNBOUNDED;
  }
  free(dxs);
  free(dys);
  free(r);
  free(d);
  return st;
}

static int finish(ctx_t* c, int status, int xs, int ys, long long it, const char* msg, orc_result* res, double* x,
                  double* y, double* z, double* dual_ray, double* primal_ray) { /* engine.cpp:268-307 */
  const orc_scaled* sp = c->sp;
  const orc_model* M = c->M;
  const int m = sp->m, n = sp->n;
  double* xsd = dvec((size_t)n, 0.0);
  double* ysd = dvec((size_t)m, 0.0);
  double* xo = dvec((size_t)n, 0.0);
  double* ymin = dvec((size_t)m, 0.0);
  orc_backend_download(c->b, xs, xsd);
  orc_backend_download(c->b, ys, ysd);
  unscale_primal(sp, xsd, xo);
  unscale_dual(sp, ysd, ymin);
  kkt_stats k = kkt_on_original(sp, xo, ymin);
  if (!kkt_finite(&k)) status = ST_NUMERICAL;
  if (status == ST_OPTIMAL && !kkt_converged(&k, c->o->tolerance)) status = ST_NUMERICAL;
  const double sense = M->sense;
  double* yo = dvec((size_t)m, 0.0);
  for (int i = 0; i < m; ++i) yo[i] = sense * ymin[i];
  if (z) {
    for (int j = 0; j < n; ++j) {
      double zz = M->c[j];
      for (int p = M->col_start[j]; p < M->col_start[j + 1]; ++p) zz -= M->value[p] * yo[M->row_index[p]];
      z[j] = zz;
    }
  }
  double obj = M->offset;
  for (int j = 0; j < n; ++j) obj += M->c[j] * xo[j];
  res->status = status;
  res->iterations = it;
  res->objective = obj;
  res->dual_objective = sense * k.dual_obj + M->offset;
  res->primal_residual = rel_primal(&k);
  res->dual_residual = rel_dual(&k);
  res->gap = rel_gap(&k);
  res->iterations_to_fast = c->fast_it;
  res->primal_weight = c->primal_weight;
  res->eta = c->eta;
  snprintf(res->message, sizeof res->message, "%s", msg);
  if (status == ST_INFEASIBLE || status == ST_UNBOUNDED) res->objective = res->dual_objective = NAN;
  if (x) memcpy(x, xo, (size_t)n * sizeof(double));
  if (y) memcpy(y, yo, (size_t)m * sizeof(double));
  if (dual_ray && status == ST_INFEASIBLE) memcpy(dual_ray, c->dual_ray, (size_t)m * sizeof(double));
  if (primal_ray && status == ST_UNBOUNDED) memcpy(primal_ray, c->primal_ray, (size_t)n * sizeof(double));
  free(xsd);
  free(ysd);
  free(xo);
  free(ymin);
  free(yo);
  return status;
}

static double initial_primal_weight(const ctx_t* c) { /* engine.cpp:207-218 */
  if (c->o->warm_primal_weight > 0) return c->o->warm_primal_weight;
  if (c->o->scaling.bound_objective_rescaling) return 1.0;
  const orc_scaled* sp = c->sp;
  double c2 = 0, b2 = 0;
  for (int j = 0; j < sp->n; ++j) c2 += sp->c[j] * sp->c[j];
  for (int i = 0; i < sp->m; ++i) {
    const double lo = isfinite(sp->row_lower[i]) ? fabs(sp->row_lower[i]) : 0.0;
    const double up = isfinite(sp->row_upper[i]) ? fabs(sp->row_upper[i]) : 0.0;
    b2 += dmaxd(lo, up) * dmaxd(lo, up);
  }
  return (sqrt(c2) + 1.0) / (sqrt(b2) + 1.0);
}

typedef struct {
  int mixed;
  double target, best;
  int checks_since_best;
  long long switched_at;
} policy_t;

static int policy_on_check(policy_t* p, orc_backend* b, double rk, long long it) { /* engine.cpp:61-79 */
  if (!p->mixed || !b->mixed) return 0;
  if (rk < 0.9 * p->best) {
    p->best = rk;
    p->checks_since_best = 0;
  } else {
    ++p->checks_since_best;
  }
  const int reached = rk <= kMixedPrecisionSwitch && p->target < kMixedPrecisionSwitch;
  const int stalled = p->checks_since_best >= 10;
  if (reached || stalled) {
    orc_backend_set_precision(b, 0);
    p->switched_at = it;
    return 1;
  }
  return 0;
}

static int apply_warm_start(ctx_t* c, int x, int y, policy_t* pol) { /* engine.cpp:237-266 */
  const orc_options* o = c->o;
  if (!o->warm_x && !o->warm_y) return 0;
  const orc_scaled* sp = c->sp;
  const orc_model* M = c->M;
  double* xo = dvec((size_t)sp->n, 0.0);
  double* yo = dvec((size_t)sp->m, 0.0);
  if (o->warm_x) {
    for (int j = 0; j < sp->n; ++j) xo[j] = dmind(dmaxd(o->warm_x[j], M->col_lower[j]), M->col_upper[j]);
  } else {
    double* xs = dvec((size_t)sp->n, 0.0);
    orc_backend_download(c->b, x, xs);
    unscale_primal(sp, xs, xo);
    free(xs);
  }
  if (o->warm_y) {
    for (int i = 0; i < sp->m; ++i) {
      double v = (double)M->sense * o->warm_y[i];
      if (!isfinite(M->row_lower[i])) v = dmind(v, 0.0);
      if (!isfinite(M->row_upper[i])) v = dmaxd(v, 0.0);
      yo[i] = v;
    }
  }
  kkt_stats kw = kkt_on_original(sp, xo, yo);
  const double wr = rel_kkt(&kw);
  if (pol->mixed && c->b->mixed && wr <= kMixedPrecisionSwitch && pol->target < kMixedPrecisionSwitch) {
    orc_backend_set_precision(c->b, 0);
    pol->switched_at = 0;
  }
  double* xs = dvec((size_t)sp->n, 0.0);
  double* ys = dvec((size_t)sp->m, 0.0);
  for (int j = 0; j < sp->n; ++j) xs[j] = sp->bound_scale * xo[j] / sp->col_scale[j];
  for (int i = 0; i < sp->m; ++i) ys[i] = sp->obj_scale * yo[i] / sp->row_scale[i];
  orc_backend_upload(c->b, x, xs);
  orc_backend_upload(c->b, y, ys);
  free(xo);
  free(yo);
  free(xs);
  free(ys);
  return 1;
}

int orc_solve_r2hpdhg(const orc_model* M, const orc_options* o, orc_result* res, double* xout, double* yout,
                      double* zout, double* dual_ray, double* primal_ray) {
  memset(res, 0, sizeof *res);
  ctx_t c;
  memset(&c, 0, sizeof c);
  c.M = M;
  c.o = o;
  c.fast_it = -1;
  c.primal_weight = NAN;
  c.sp = orc_scale(M, &o->scaling);
  c.b = orc_backend_new(c.sp);
  const double norm = orc_norm2(c.sp);
  c.eta = norm > 0 ? 0.998 / norm : 1.0;
  c.dual_ray = dvec((size_t)M->m, 0.0);
  c.primal_ray = dvec((size_t)M->n, 0.0);
  orc_backend* b = c.b;
  policy_t pol = {o->mixed, o->tolerance, 1e300, 0, -1};
  orc_backend_set_precision(b, o->mixed);
  const double eta = c.eta, rho = o->reflection;
  double omega = initial_primal_weight(&c);
  res->initial_primal_weight = omega;

  int x = orc_backend_create(b, 0), x0 = orc_backend_create(b, 0), xh = orc_backend_create(b, 0);
  int xb = orc_backend_create(b, 0), aty = orc_backend_create(b, 0), dx = orc_backend_create(b, 0);
  int y = orc_backend_create(b, 1), y0 = orc_backend_create(b, 1), yh = orc_backend_create(b, 1);
  int yb = orc_backend_create(b, 1), ax = orc_backend_create(b, 1), dy = orc_backend_create(b, 1);

  orc_backend_fill(b, dx, 0.0);
  orc_backend_fill(b, aty, 0.0);
  orc_backend_primal_step(b, dx, aty, 0.0, x);
  orc_backend_fill(b, y, 0.0);
  const int warm = apply_warm_start(&c, x, y, &pol);
  c.primal_weight = omega;
  char msg[256];
  snprintf(msg, sizeof msg, "%s", warm ? "warm start" : "");
  int status;
  if (warm) {
    kkt_stats kw = backend_kkt(b, x, y);
    if (kkt_finite(&kw) && record(&c, &kw, 0)) {
      status = finish(&c, ST_OPTIMAL, x, y, 0, "warm start already optimal", res, xout, yout, zout, dual_ray,
                      primal_ray);
      goto done;
    }
  }
  orc_backend_copy(b, x0, x);
  orc_backend_copy(b, y0, y);
  orc_backend_copy(b, xh, x);
  orc_backend_copy(b, yh, y);

  double pid_integral = 0.0, pid_last = 0.0, best_omega = omega, best_balance = 1e300;
  const int K = o->check_every;
  long long it = 0, inner = 0;
  double r0 = -1.0, r_last = INFINITY;

#define FIXED_POINT_RESIDUAL(out)                                                   \
  do {                                                                              \
    orc_backend_copy(b, dx, xb);                                                    \
    orc_backend_axpby(b, -1.0, xh, 1.0, dx);                                        \
    orc_backend_copy(b, dy, yb);                                                    \
    orc_backend_axpby(b, -1.0, yh, 1.0, dy);                                        \
    orc_backend_spmv(b, dx, ax);                                                    \
    const double px_ = orc_backend_dot(b, dx, dx), py_ = orc_backend_dot(b, dy, dy); \
    const double cross_ = orc_backend_dot(b, dy, ax);                               \
    const double r2_ = omega * px_ + py_ / omega + 2.0 * eta * cross_;              \
    (out) = sqrt(dmaxd(r2_, 0.0));                                                  \
  } while (0)

  for (;;) {
    const double tau = eta / omega, sigma = eta * omega;
    for (int s = 0; s < K; ++s) {
      const double w = (double)(inner + 1) / (double)(inner + 2);
      const int need_residual = (s == K - 1) || inner == 0;
      orc_backend_spmv_t(b, y, aty);
      orc_backend_r2h_primal(b, x, x0, aty, tau, w, rho, xh, xb);
      orc_backend_spmv(b, xb, ax);
      orc_backend_r2h_dual(b, y, y0, ax, sigma, w, rho, yh, need_residual ? yb : -1);
      if (inner == 0) FIXED_POINT_RESIDUAL(r0);
      ++inner;
      ++it;
    }
    double r;
    FIXED_POINT_RESIDUAL(r);
    ++res->checks;
    kkt_stats k = backend_kkt(b, xh, yh);
    if (!kkt_finite(&k) || !isfinite(r)) {
      status = finish(&c, ST_NUMERICAL, xh, yh, it, "non-finite iterate", res, xout, yout, zout, dual_ray,
                      primal_ray);
      goto done;
    }
    if (record(&c, &k, it)) {
      status = finish(&c, ST_OPTIMAL, xh, yh, it, msg, res, xout, yout, zout, dual_ray, primal_ray);
      goto done;
    }
    if (it >= o->iteration_limit) {
      status = finish(&c, ST_ITERLIMIT, xh, yh, it, msg, res, xout, yout, zout, dual_ray, primal_ray);
      goto done;
    }
    if (it >= 4LL * K) {
      char why[256] = "";
      int st = check_infeasibility(&c, dx, dy, &k, why, sizeof why);
      if (st == ST_NOTSOLVED && inner >= K && (it / K) % 4 == 0) {
        orc_backend_copy(b, dx, xh);
        orc_backend_axpby(b, -1.0, x0, 1.0, dx);
        orc_backend_copy(b, dy, yh);
        orc_backend_axpby(b, -1.0, y0, 1.0, dy);
        st = check_infeasibility(&c, dx, dy, &k, why, sizeof why);
        if (st != ST_NOTSOLVED) strncat(why, " (drift since the restart anchor)", sizeof why - strlen(why) - 1);
      }
      if (st != ST_NOTSOLVED) {
        status = finish(&c, st, xh, yh, it, why, res, xout, yout, zout, dual_ray, primal_ray);
        goto done;
      }
    }
    const int promoted = policy_on_check(&pol, b, rel_kkt(&k), it);
    if (promoted) {
      char add[96];
      snprintf(add, sizeof add, "%sfp32 -> fp64 at iteration %lld", msg[0] ? "; " : "", it);
      strncat(msg, add, sizeof msg - strlen(msg) - 1);
    }
    const int ratios_ok = r0 > 0 && isfinite(r0) && r > 0;
    const int restart = promoted ||
                        (ratios_ok && (r <= o->restart_sufficient * r0 ||
                                       (r <= o->restart_necessary * r0 && r > r_last))) ||
                        (double)inner >= o->restart_artificial * (double)it;
    r_last = r;
    if (!restart) continue;

    const double dxn = orc_backend_diff_norm2(b, xh, x0), dyn = orc_backend_diff_norm2(b, yh, y0);
    const int both_pos = rel_dual(&k) > 0 && rel_primal(&k) > 0;
    const double ratio = both_pos ? rel_dual(&k) / rel_primal(&k) : 1.0;
    if (dxn > 1e-16 && dyn > 1e-16 && dxn < 1e12 && dyn < 1e12 && ratio > 1e-8 && ratio < 1e8) {
      const double e = log(dyn) - log(dxn) - log(omega);
      pid_integral = o->pid_integral_decay * pid_integral + e;
      const double step = o->pid_kp * e + o->pid_ki * pid_integral + o->pid_kd * (e - pid_last);
      const double cl = step < -o->pid_max_log_step ? -o->pid_max_log_step
                                                     : (o->pid_max_log_step < step ? o->pid_max_log_step : step);
      omega *= exp(cl);
      pid_last = e;
    } else {
      omega = best_omega;
      pid_integral = pid_last = 0.0;
    }
    const double balance = fabs(log10(ratio));
    if (both_pos && balance < best_balance) {
      best_balance = balance;
      best_omega = omega;
    }
    c.primal_weight = omega;
    ++res->restarts;
    orc_backend_copy(b, x, xh);
    orc_backend_copy(b, x0, xh);
    orc_backend_copy(b, y, yh);
    orc_backend_copy(b, y0, yh);
    inner = 0;
    r_last = INFINITY;
  }
#undef FIXED_POINT_RESIDUAL
done:
  res->switch_iteration = pol.switched_at;
  orc_backend_free(c.b);
  orc_scaled_free(c.sp);
  free(c.dual_ray);
  free(c.primal_ray);
  return status;
}
