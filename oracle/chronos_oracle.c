/* CPU oracle of the solve path in C (FP64, OpenMP).  See chronos_oracle.h.
 * ORACLE TEST INFRASTRUCTURE only; never linked into the product. */
#include "chronos_oracle.h"

#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

static int g_threads = 0;

void oracle_set_threads(int nthreads) { g_threads = nthreads; }

static int nthr(void) { return g_threads > 0 ? g_threads : omp_get_max_threads(); }

void oracle_spmv(const ocsr *A, const double *x, double *y) {
#pragma omp parallel for schedule(static) num_threads(nthr())
  for (int i = 0; i < A->nrows; ++i) {
    double s = 0.0;
    for (int64_t k = A->rp[i]; k < A->rp[i + 1]; ++k) s += A->v[k] * x[A->ci[k]];
    y[i] = s;
  }
}

static double dot(int n, const double *a, const double *b) {
  double s = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : s) num_threads(nthr())
  for (int i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

/* r = b - A x */
static void resid(const ocsr *A, const double *x, const double *b, double *r) {
#pragma omp parallel for schedule(static) num_threads(nthr())
  for (int i = 0; i < A->nrows; ++i) {
    double s = 0.0;
    for (int64_t k = A->rp[i]; k < A->rp[i + 1]; ++k) s += A->v[k] * x[A->ci[k]];
    r[i] = b[i] - s;
  }
}

/* y = y + alpha * (A x) */
static void spmv_add(const ocsr *A, double alpha, const double *x, double *y) {
#pragma omp parallel for schedule(static) num_threads(nthr())
  for (int i = 0; i < A->nrows; ++i) {
    double s = 0.0;
    for (int64_t k = A->rp[i]; k < A->rp[i + 1]; ++k) s += A->v[k] * x[A->ci[k]];
    y[i] += alpha * s;
  }
}

/* x (+)= omega * G'(G r) with a scratch t */
static void smooth(const olevel *L, const double *r, double *t, double *x, int accumulate) {
  oracle_spmv(&L->G, r, t);
  if (accumulate) {
    spmv_add(&L->Gt, L->omega, t, x);
  } else {
    oracle_spmv(&L->Gt, t, x);
#pragma omp parallel for schedule(static) num_threads(nthr())
    for (int i = 0; i < L->n; ++i) x[i] *= L->omega;
  }
}

static void vcycle_rec(int lvl, int nlev, const olevel *lv, const double *b, double *x) {
  const olevel *L = &lv[lvl];
  const int n = L->n;
  if (lvl == nlev - 1) {
    /* x = L' \ (L \ b) */
    memcpy(x, b, sizeof(double) * n);
    for (int j = 0; j < n; ++j) {
      const double *col = L->L + (size_t)j * n;
      x[j] /= col[j];
      const double xj = x[j];
      for (int i = j + 1; i < n; ++i) x[i] -= col[i] * xj;
    }
    for (int j = n - 1; j >= 0; --j) {
      const double *col = L->L + (size_t)j * n;
      double s = x[j];
      for (int i = j + 1; i < n; ++i) s -= col[i] * x[i];
      x[j] = s / col[j];
    }
    return;
  }
  double *r = (double *)malloc(sizeof(double) * n);
  double *t = (double *)malloc(sizeof(double) * n);
  const int nc = L->P.ncols;
  double *rc = (double *)malloc(sizeof(double) * nc);
  double *hc = (double *)malloc(sizeof(double) * nc);
  smooth(L, b, t, x, 0);                         /* x = Minv1(b) */
  for (int k = 1; k < L->nupre; ++k) {
    resid(&L->A, x, b, r);
    smooth(L, r, t, x, 1);
  }
  resid(&L->A, x, b, r);                          /* r = b - A*x */
  oracle_spmv(&L->Pt, r, rc);                     /* r = P'*r */
  vcycle_rec(lvl + 1, nlev, lv, rc, hc);
  spmv_add(&L->P, 1.0, hc, x);                    /* x = x + P*hc */
  for (int k = 0; k < L->nupost; ++k) {
    resid(&L->A, x, b, r);
    smooth(L, r, t, x, 1);
  }
  free(r);
  free(t);
  free(rc);
  free(hc);
}

void oracle_vcycle(int nlev, const olevel *lv, const double *b, double *x) {
  vcycle_rec(0, nlev, lv, b, x);
}

int oracle_pcg_cj(int nlev, const olevel *lv, const ocsr *A, const double *b, double *x,
                  int itmax, double tol, int *iters, double *resvec) {
  const int n = A->nrows;
  int iter = 0, flag = 0;
  const double bnorm = sqrt(dot(n, b, b));
  if (bnorm == 0.0) {
    memset(x, 0, sizeof(double) * n);
    *iters = 0;
    if (resvec) resvec[0] = 0.0;
    return 0;
  }
  double *res = (double *)malloc(sizeof(double) * n);
  double *pres = (double *)malloc(sizeof(double) * n);
  double *p = (double *)calloc(n, sizeof(double));
  double *axp = (double *)calloc(n, sizeof(double));
  resid(A, x, b, res);
  double resiter = sqrt(dot(n, res, res)) / bnorm;
  if (resvec) resvec[0] = resiter;
  int exit_test = itmax <= 0;
  double ptap = 0.0;
  while (!exit_test) {
    iter += 1;
    oracle_vcycle(nlev, lv, res, pres);
    if (iter == 1) {
      memcpy(p, pres, sizeof(double) * n);
    } else {
      const double beta = -dot(n, pres, axp) / ptap;
#pragma omp parallel for schedule(static) num_threads(nthr())
      for (int i = 0; i < n; ++i) p[i] = pres[i] + beta * p[i];
    }
    oracle_spmv(A, p, axp);
    ptap = dot(n, p, axp);
    const double alpha = dot(n, p, res) / ptap;
#pragma omp parallel for schedule(static) num_threads(nthr())
    for (int i = 0; i < n; ++i) {
      x[i] += alpha * p[i];
      res[i] -= alpha * axp[i];
    }
    resiter = sqrt(dot(n, res, res)) / bnorm;
    if (resvec) resvec[iter] = resiter;
    exit_test = resiter < tol || iter == itmax;
  }
  if (resiter > tol) flag = 1;
  free(res);
  free(pres);
  free(p);
  free(axp);
  *iters = iter;
  return flag;
}

int oracle_pmis(int n, const int64_t *S_rp, const int *S_ci, const double *rnd, int *fc) {
  /* column view of S (diagonal removed): S is symmetric on this path, but the
   * sweep uses S(:,inod) for marking and S + S' for the neighbourhood, so
   * build both explicitly */
  int64_t *cp = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t));
  for (int i = 0; i < n; ++i)
    for (int64_t k = S_rp[i]; k < S_rp[i + 1]; ++k)
      if (S_ci[k] != i) cp[S_ci[k] + 1]++;
  for (int j = 0; j < n; ++j) cp[j + 1] += cp[j];
  int *cr = (int *)malloc(sizeof(int) * (cp[n] > 0 ? cp[n] : 1));
  int64_t *pos = (int64_t *)malloc(sizeof(int64_t) * (n > 0 ? n : 1));
  for (int j = 0; j < n; ++j) pos[j] = cp[j];
  for (int i = 0; i < n; ++i)
    for (int64_t k = S_rp[i]; k < S_rp[i + 1]; ++k)
      if (S_ci[k] != i) cr[pos[S_ci[k]]++] = i;
  double *w = (double *)malloc(sizeof(double) * n);
  double *wf = (double *)malloc(sizeof(double) * n);
  for (int j = 0; j < n; ++j) w[j] = (double)(cp[j + 1] - cp[j]) + rnd[j];
  for (int j = 0; j < n; ++j) {
    if (fc[j] == -2) fc[j] = -1;
    wf[j] = fc[j] == -1 ? -1.0 : w[j];
  }
  int *list = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
  int64_t len = 0;
  for (int j = 0; j < n; ++j)
    if (fc[j] == 0) list[len++] = j;
  int64_t ind = 0;
  while (len > 0) {
    const int inod = list[ind];
    if (fc[inod] != 0) {
      list[ind] = list[len - 1];
      --len;
    } else {
      int coarse = 1;
      const double wi = w[inod];
      /* neighbours in S + S': row inod of S and column inod of S */
      for (int64_t k = S_rp[inod]; k < S_rp[inod + 1] && coarse; ++k)
        if (S_ci[k] != inod && wf[S_ci[k]] > wi) coarse = 0;
      for (int64_t k = cp[inod]; k < cp[inod + 1] && coarse; ++k)
        if (wf[cr[k]] > wi) coarse = 0;
      if (!coarse) {
        ++ind;
      } else {
        for (int64_t k = cp[inod]; k < cp[inod + 1]; ++k) {
          fc[cr[k]] = -1;
          wf[cr[k]] = -1.0;
        }
        fc[inod] = 1;
        wf[inod] = -1.0;
        list[ind] = list[len - 1];
        --len;
      }
    }
    if (ind > len - 1) ind = 0;
  }
  int nc = 0, nf = 0;
  for (int j = 0; j < n; ++j) {
    if (fc[j] > 0) fc[j] = ++nc;
    else fc[j] = -(++nf);
  }
  free(cp);
  free(cr);
  free(pos);
  free(w);
  free(wf);
  free(list);
  return nc;
}
