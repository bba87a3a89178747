/*
 * CPU restatement of the reference's FP64 PCG + geometric-multigrid solve path.
 *
 * TEST INFRASTRUCTURE ONLY: this file is the oracle of the parity tests and the "port" CPU
 * baseline.  The product never links, loads or calls it.
 *
 * Every routine restates the reference's generic (CPU) code path in the same operation order,
 * without FP contraction (built with -ffp-contract=off), so that its results are bitwise equal to
 * the reference build of the same inputs:
 *   oc_csr_apply        kernel/lafem/arch/apply_generic.hpp:25-69      (Apply::csr_generic)
 *   oc_axpy             kernel/lafem/arch/axpy_generic.hpp:25-49       (Axpy::value_generic)
 *   oc_dot              kernel/lafem/arch/dot_product_generic.hpp:21-41
 *   oc_norm2            kernel/lafem/arch/norm_generic.hpp:24-33
 *   oc_filter_*         kernel/lafem/arch/unit_filter_generic.hpp:22-37
 *   inverse diagonal    kernel/solver/jacobi_precond.hpp:136-143 + sparse_matrix_csr.hpp:2277-2291
 *                       + component_invert_generic.hpp:21-40
 *   richardson_apply    kernel/solver/richardson.hpp:160-228 with the stopping logic of
 *                       kernel/solver/iterative.hpp:492-507,748-879 (min_iter = max_iter = steps)
 *   oc_mg_vcycle        kernel/solver/multigrid.hpp:1270-1350 (apply, V-cycle),
 *                       :1526-1587 (_apply_coarse), :1713-1838 (_apply_rest),
 *                       :1845-2000 (_apply_prol, fixed coarse-grid correction omega = 1)
 *   oc_pcg_solve        kernel/solver/pcg.hpp:159-286 (correct + _apply_intern) with the stopping
 *                       logic of kernel/solver/iterative.hpp (defaults: tol_abs = 1/eps^2,
 *                       div_rel = 1/eps, div_abs = 1/eps^2, no stagnation check)
 *   sor_generic         kernel/solver/sor_precond.hpp:179-224 (SORPrecondWithBackend<generic, CSR>)
 *   ssor_generic        kernel/solver/ssor_precond.hpp (SSORPrecondWithBackend<generic, CSR>: forward
 *                       and backward insertion, scaling by omega (2 - omega))
 *   sor_coloured,       the coloured sweeps of the reference's CUDA backend (kernel/solver/sor_precond.cu:
 *   ssor_coloured       26-41 and :294-315, kernel/solver/ssor_precond.cu:25-60 and :182-230): y = 0,
 *                       then colour by colour, colours by ascending row count; the colouring itself
 *                       (greedy_colours below, first fit in row order) replaces cusparseDcsrcolor
 * The coarse-grid solve is an exact inverse of the matrix restricted to the free DOFs, formed by
 * Gauss-Jordan elimination with partial pivoting and applied in ascending column order (the same
 * coarse solver the reference-side driver oracle/feat_ref_driver.cpp plugs into the reference).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OC_EPS 2.220446049250313080847e-16

typedef struct
{
  uint64_t rows, cols;
  const uint64_t* row_ptr;
  const uint64_t* col_ind;
  const double* val;
} oc_csr;

/* r = a * op(A) * x + b * y; |b| < eps means y is ignored (apply_generic.hpp:25-69) */
void oc_csr_apply(double* r, double a, const double* x, double b, const double* y, const oc_csr* A,
  int transposed)
{
  const uint64_t nout = transposed ? A->cols : A->rows;
  if(fabs(b) < OC_EPS)
    memset(r, 0, sizeof(double) * nout);
  else if(r != y)
    memcpy(r, y, sizeof(double) * nout);
  if(transposed)
  {
    const double ba = b / a;
    for(uint64_t c = 0; c < A->cols; ++c)
      r[c] = ba * r[c];
    for(uint64_t row = 0; row < A->rows; ++row)
      for(uint64_t i = A->row_ptr[row]; i < A->row_ptr[row + 1]; ++i)
        r[A->col_ind[i]] += A->val[i] * x[row];
    for(uint64_t c = 0; c < A->cols; ++c)
      r[c] = a * r[c];
  }
  else
  {
    for(uint64_t row = 0; row < A->rows; ++row)
    {
      double sum = 0.0;
      const uint64_t end = A->row_ptr[row + 1];
      for(uint64_t i = A->row_ptr[row]; i < end; ++i)
        sum += A->val[i] * x[A->col_ind[i]];
      r[row] = (sum * a) + (b * r[row]);
    }
  }
}

/* r = a * x + y (axpy_generic.hpp:25-49; every alias branch rounds as fl(fl(a*x) + y)) */
void oc_axpy(double* r, double a, const double* x, const double* y, uint64_t n)
{
  if(r == y)
    for(uint64_t i = 0; i < n; ++i)
      r[i] += a * x[i];
  else if(r == x)
    for(uint64_t i = 0; i < n; ++i)
    {
      r[i] *= a;
      r[i] += y[i];
    }
  else
    for(uint64_t i = 0; i < n; ++i)
      r[i] = (a * x[i]) + y[i];
}

double oc_dot(const double* x, const double* y, uint64_t n)
{
  double r = 0.0;
  for(uint64_t i = 0; i < n; ++i)
    r += x[i] * y[i];
  return r;
}

double oc_norm2(const double* x, uint64_t n)
{
  double r = 0.0;
  for(uint64_t i = 0; i < n; ++i)
    r += x[i] * x[i];
  return sqrt(r);
}

void oc_filter_rhs(double* v, const double* vals, const uint64_t* idx, uint64_t ue)
{
  for(uint64_t i = 0; i < ue; ++i)
    v[idx[i]] = vals[i];
}

void oc_filter_def(double* v, const uint64_t* idx, uint64_t ue)
{
  for(uint64_t i = 0; i < ue; ++i)
    v[idx[i]] = 0.0;
}

/* inv_diag_i = omega / a_ii, 0 diagonal when the row has no diagonal entry */
void oc_inv_diag(double* d, const oc_csr* A, double omega)
{
  for(uint64_t row = 0; row < A->rows; ++row)
  {
    double a = 0.0;
    for(uint64_t i = A->row_ptr[row]; i < A->row_ptr[row + 1]; ++i)
      if(A->col_ind[i] == row)
      {
        a = A->val[i];
        break;
      }
    d[row] = omega / a;
  }
}

typedef struct
{
  oc_csr A, P, R;        /* P: this level <- next coarser level; R: next coarser <- this */
  const uint64_t* fidx;  /* Dirichlet DOFs */
  const double* fval;
  uint64_t nf;
} oc_level_in;

typedef struct
{
  oc_level_in in;
  uint64_t n;
  double *rhs, *sol, *def, *cor, *tmp;
  double *inv_diag, *sm_def, *sm_cor;
} oc_level;

typedef struct
{
  int nlevels;
  oc_level* lv;
  double omega;
  int steps;
  uint64_t nfree;
  uint64_t* free_dofs;
  double* cinv;
  /* PCG vectors on the finest level */
  double *r, *p, *t;
  int smoother;          /* 0 Jacobi, 1 SOR, 2 SSOR: the Richardson smoother's preconditioner */
  double sor_omega;      /* SOR / SSOR damping */
  int coloured;          /* 1: the reference's coloured (CUDA) sweeps with greedy_colours */
  uint32_t** corder;     /* per level: rows colour by colour; cofs: colour offsets */
  uint32_t** cofs;
  int* ncol;
  int cycle;             /* 0 V, 1 F, 2 W (MultiGridCycle) */
  int cgc;               /* 0 fixed, 1 energy minimisation, 2 defect minimisation (MultiGridAdaptCGC) */
} oc_mg;

static int coarse_factor(oc_mg* mg)
{
  oc_level* c = &mg->lv[mg->nlevels - 1];
  const uint64_t n = c->n;
  char* dir = (char*)calloc(n, 1);
  for(uint64_t k = 0; k < c->in.nf; ++k)
    dir[c->in.fidx[k]] = 1;
  uint64_t m = 0;
  for(uint64_t i = 0; i < n; ++i)
    m += dir[i] ? 0 : 1;
  mg->nfree = m;
  mg->free_dofs = (uint64_t*)malloc(sizeof(uint64_t) * (m ? m : 1));
  uint64_t* pos = (uint64_t*)malloc(sizeof(uint64_t) * n);
  m = 0;
  for(uint64_t i = 0; i < n; ++i)
  {
    pos[i] = UINT64_MAX;
    if(!dir[i])
    {
      pos[i] = m;
      mg->free_dofs[m++] = i;
    }
  }
  double* a = (double*)calloc(m * m + 1, sizeof(double));
  double* inv = (double*)calloc(m * m + 1, sizeof(double));
  for(uint64_t i = 0; i < m; ++i)
  {
    const uint64_t r = mg->free_dofs[i];
    for(uint64_t k = c->in.A.row_ptr[r]; k < c->in.A.row_ptr[r + 1]; ++k)
    {
      const uint64_t cc = c->in.A.col_ind[k];
      if(pos[cc] != UINT64_MAX)
        a[i * m + pos[cc]] = c->in.A.val[k];
    }
    inv[i * m + i] = 1.0;
  }
  for(uint64_t col = 0; col < m; ++col)
  {
    uint64_t p = col;
    for(uint64_t r = col + 1; r < m; ++r)
      if(fabs(a[r * m + col]) > fabs(a[p * m + col]))
        p = r;
    if(p != col)
      for(uint64_t j = 0; j < m; ++j)
      {
        double t = a[p * m + j];
        a[p * m + j] = a[col * m + j];
        a[col * m + j] = t;
        t = inv[p * m + j];
        inv[p * m + j] = inv[col * m + j];
        inv[col * m + j] = t;
      }
    const double d = a[col * m + col];
    for(uint64_t j = 0; j < m; ++j)
    {
      a[col * m + j] /= d;
      inv[col * m + j] /= d;
    }
    for(uint64_t r = 0; r < m; ++r)
    {
      if(r == col)
        continue;
      const double f = a[r * m + col];
      if(f == 0.0)
        continue;
      for(uint64_t j = 0; j < m; ++j)
      {
        a[r * m + j] -= f * a[col * m + j];
        inv[r * m + j] -= f * inv[col * m + j];
      }
    }
  }
  mg->cinv = inv;
  free(a);
  free(pos);
  free(dir);
  return 0;
}

oc_mg* oc_mg_create(int nlevels, const oc_level_in* levels, double omega, int steps)
{
  oc_mg* mg = (oc_mg*)calloc(1, sizeof(oc_mg));
  mg->nlevels = nlevels;
  mg->omega = omega;
  mg->steps = steps;
  mg->lv = (oc_level*)calloc((size_t)nlevels, sizeof(oc_level));
  for(int l = 0; l < nlevels; ++l)
  {
    oc_level* v = &mg->lv[l];
    v->in = levels[l];
    v->n = levels[l].A.rows;
    v->rhs = (double*)calloc(v->n, sizeof(double));
    v->sol = (double*)calloc(v->n, sizeof(double));
    v->def = (double*)calloc(v->n, sizeof(double));
    v->cor = (double*)calloc(v->n, sizeof(double));
    v->tmp = (double*)calloc(v->n, sizeof(double));
    v->inv_diag = (double*)calloc(v->n, sizeof(double));
    v->sm_def = (double*)calloc(v->n, sizeof(double));
    v->sm_cor = (double*)calloc(v->n, sizeof(double));
    oc_inv_diag(v->inv_diag, &v->in.A, omega);
  }
  coarse_factor(mg);
  const uint64_t n = mg->lv[0].n;
  mg->r = (double*)calloc(n, sizeof(double));
  mg->p = (double*)calloc(n, sizeof(double));
  mg->t = (double*)calloc(n, sizeof(double));
  return mg;
}

void oc_mg_destroy(oc_mg* mg)
{
  if(!mg)
    return;
  for(int l = 0; l < mg->nlevels; ++l)
  {
    oc_level* v = &mg->lv[l];
    free(v->rhs); free(v->sol); free(v->def); free(v->cor); free(v->tmp);
    free(v->inv_diag); free(v->sm_def); free(v->sm_cor);
  }
  if(mg->corder)
    for(int l = 0; l < mg->nlevels; ++l)
    {
      free(mg->corder[l]);
      free(mg->cofs[l]);
    }
  free(mg->corder); free(mg->cofs); free(mg->ncol);
  free(mg->lv);
  free(mg->free_dofs);
  free(mg->cinv);
  free(mg->r); free(mg->p); free(mg->t);
  free(mg);
}

/* SORPrecond (generic): out = copy(in), forward insertion out_i = w (in_i - sum_{j<i} a_ij out_j) / a_ii
 * over the row's entries left of the diagonal in stored order */
static void sor_generic(const oc_csr* A, double* out, const double* in, double w)
{
  const uint64_t n = A->rows;
  memcpy(out, in, sizeof(double) * n);
  for(uint64_t i = 0; i < n; ++i)
  {
    uint64_t col;
    double d = 0.0;
    for(col = A->row_ptr[i]; A->col_ind[col] < i; ++col)
      d += A->val[col] * out[A->col_ind[col]];
    out[i] = w * (in[i] - d) / A->val[col];
  }
}

/* SSORPrecond (generic): forward insertion out_i = (in_i - w d) / a_ii, backward insertion
 * out_i -= w d / a_ii with d over the entries right of the diagonal from the row's end, then
 * out *= w (2 - w) */
static void ssor_generic(const oc_csr* A, double* out, const double* in, double w)
{
  const uint64_t n = A->rows;
  memcpy(out, in, sizeof(double) * n);
  for(uint64_t i = 0; i < n; ++i)
  {
    uint64_t col;
    double d = 0.0;
    for(col = A->row_ptr[i]; A->col_ind[col] < i; ++col)
      d += A->val[col] * out[A->col_ind[col]];
    out[i] = (in[i] - w * d) / A->val[col];
  }
  for(uint64_t i = n; i > 0;)
  {
    --i;
    uint64_t col;
    double d = 0.0;
    for(col = A->row_ptr[i + 1] - 1; A->col_ind[col] > i; --col)
      d += A->val[col] * out[A->col_ind[col]];
    out[i] -= w * d / A->val[col];
  }
  const double sc = w * (2.0 - w);
  for(uint64_t i = 0; i < n; ++i)
    out[i] = out[i] * sc;
}

/* the coloured sweeps: out = 0, then colour by colour (rows of one colour are not coupled) */
static void sor_coloured(const oc_csr* A, double* out, const double* in, double w, const uint32_t* order,
  const uint32_t* cofs, int ncol, int ssor)
{
  memset(out, 0, sizeof(double) * A->rows);
  for(int c = 0; c < ncol; ++c)
    for(uint32_t k = cofs[c]; k < cofs[c + 1]; ++k)
    {
      const uint64_t row = order[k];
      uint64_t col;
      double d = 0.0;
      for(col = A->row_ptr[row]; A->col_ind[col] < row; ++col)
        d += A->val[col] * out[A->col_ind[col]];
      out[row] = ssor ? (in[row] - w * d) / A->val[col] : w * (in[row] - d) / A->val[col];
    }
  if(!ssor)
    return;
  for(int c = 0; c < ncol; ++c)
    for(uint32_t k = cofs[c]; k < cofs[c + 1]; ++k)
    {
      const uint64_t row = order[k];
      uint64_t col;
      double d = 0.0;
      for(col = A->row_ptr[row + 1] - 1; A->col_ind[col] > row; --col)
        d += A->val[col] * out[A->col_ind[col]];
      out[row] -= w * d / A->val[col];
    }
  const double sc = w * (2.0 - w);
  for(uint64_t i = 0; i < A->rows; ++i)
    out[i] = out[i] * sc;
}

/* Greedy colouring of the symmetric pattern of A: rows in ascending order take the smallest colour
 * no already coloured neighbour (a_ij or a_ji stored, j != i) has; colours are then ordered by
 * ascending row count (ties: colour number) and each colour lists its rows in ascending order. */
static int greedy_colours(const oc_csr* A, uint32_t** order_out, uint32_t** cofs_out)
{
  const uint64_t n = A->rows;
  /* transpose pattern */
  uint64_t* tp = (uint64_t*)calloc(n + 1, sizeof(uint64_t));
  const uint64_t nnz = A->row_ptr[n];
  uint64_t* tc = (uint64_t*)malloc(sizeof(uint64_t) * (nnz ? nnz : 1));
  for(uint64_t k = 0; k < nnz; ++k)
    ++tp[A->col_ind[k] + 1];
  for(uint64_t i = 0; i < n; ++i)
    tp[i + 1] += tp[i];
  uint64_t* fill = (uint64_t*)malloc(sizeof(uint64_t) * (n ? n : 1));
  memcpy(fill, tp, sizeof(uint64_t) * n);
  for(uint64_t i = 0; i < n; ++i)
    for(uint64_t k = A->row_ptr[i]; k < A->row_ptr[i + 1]; ++k)
      tc[fill[A->col_ind[k]]++] = i;
  int* colour = (int*)malloc(sizeof(int) * (n ? n : 1));
  int* mark = (int*)malloc(sizeof(int) * (n + 1));
  for(uint64_t i = 0; i <= n; ++i)
    mark[i] = -1;
  int ncol = 0;
  for(uint64_t i = 0; i < n; ++i)
  {
    for(uint64_t k = A->row_ptr[i]; k < A->row_ptr[i + 1]; ++k)
      if(A->col_ind[k] < i)
        mark[colour[A->col_ind[k]]] = (int)i;
    for(uint64_t k = tp[i]; k < tp[i + 1]; ++k)
      if(tc[k] < i)
        mark[colour[tc[k]]] = (int)i;
    int c = 0;
    while(mark[c] == (int)i)
      ++c;
    colour[i] = c;
    if(c + 1 > ncol)
      ncol = c + 1;
  }
  uint64_t* cnt = (uint64_t*)calloc((size_t)ncol, sizeof(uint64_t));
  for(uint64_t i = 0; i < n; ++i)
    ++cnt[colour[i]];
  int* rank = (int*)malloc(sizeof(int) * (size_t)ncol);   /* colours by ascending (count, number) */
  for(int c = 0; c < ncol; ++c)
    rank[c] = c;
  for(int a = 1; a < ncol; ++a)
  {
    const int v = rank[a];
    int b = a - 1;
    while(b >= 0 && (cnt[rank[b]] > cnt[v] || (cnt[rank[b]] == cnt[v] && rank[b] > v)))
    {
      rank[b + 1] = rank[b];
      --b;
    }
    rank[b + 1] = v;
  }
  uint32_t* order = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  uint32_t* cofs = (uint32_t*)malloc(sizeof(uint32_t) * ((size_t)ncol + 1));
  uint32_t pos = 0;
  for(int r = 0; r < ncol; ++r)
  {
    cofs[r] = pos;
    for(uint64_t i = 0; i < n; ++i)
      if(colour[i] == rank[r])
        order[pos++] = (uint32_t)i;
  }
  cofs[ncol] = pos;
  free(tp); free(tc); free(fill); free(colour); free(mark); free(cnt); free(rank);
  *order_out = order;
  *cofs_out = cofs;
  return ncol;
}

/* the smoother's preconditioner: cor = M(def), filtered (JacobiPrecond / SORPrecond / SSORPrecond) */
static void precond_apply(const oc_mg* mg, const oc_level* v, int l, double* cor, const double* def)
{
  const uint64_t n = v->n;
  if(mg->smoother == 0)
  {
    for(uint64_t i = 0; i < n; ++i)
      cor[i] = v->inv_diag[i] * def[i];
  }
  else if(mg->coloured)
    sor_coloured(&v->in.A, cor, def, mg->sor_omega, mg->corder[l], mg->cofs[l], mg->ncol[l], mg->smoother == 2);
  else if(mg->smoother == 1)
    sor_generic(&v->in.A, cor, def, mg->sor_omega);
  else
    ssor_generic(&v->in.A, cor, def, mg->sor_omega);
  oc_filter_def(cor, v->in.fidx, v->in.nf);
}

/* Richardson(omega = 1) with the smoother's preconditioner, min_iter = max_iter = steps:
 * out = smoother(in), out starts at zero (richardson.hpp:160-228). */
static void richardson_apply(const oc_mg* mg, const oc_level* v, double* out, const double* in)
{
  const uint64_t n = v->n;
  memcpy(v->sm_def, in, sizeof(double) * n);
  memset(out, 0, sizeof(double) * n);
  const double def_init = oc_norm2(v->sm_def, n);
  if(!isfinite(def_init))
    return;                                   /* Status::aborted */
  if(def_init <= OC_EPS * OC_EPS)
    return;                                   /* Status::success */
  for(int it = 1;; ++it)
  {
    /* JacobiPrecond / SORPrecond / SSORPrecond::apply, filter_cor */
    precond_apply(mg, v, (int)(v - mg->lv), v->sm_cor, v->sm_def);
    oc_axpy(out, 1.0, v->sm_cor, out, n);
    oc_csr_apply(v->sm_def, -1.0, out, 1.0, in, &v->in.A, 0);
    oc_filter_def(v->sm_def, v->in.fidx, v->in.nf);
    /* _set_new_defect without a norm (min_iter == max_iter): the stored defect stays def_init */
    if(def_init > 1.0 / (OC_EPS * OC_EPS) || def_init > (1.0 / OC_EPS) * def_init)
      return;                                 /* Status::diverged */
    if(it < mg->steps)
      continue;
    return;                                   /* converged test is false; Status::max_iter */
  }
}

static void coarse_apply(const oc_mg* mg, double* x, const double* b)
{
  const oc_level* c = &mg->lv[mg->nlevels - 1];
  memset(x, 0, sizeof(double) * c->n);
  const uint64_t m = mg->nfree;
  for(uint64_t i = 0; i < m; ++i)
  {
    double s = 0.0;
    for(uint64_t j = 0; j < m; ++j)
      s += mg->cinv[i * m + j] * b[mg->free_dofs[j]];
    x[mg->free_dofs[i]] = s;
  }
}

/* MultiGrid::_apply_rest(cur_lvl, cur_smooth) (multigrid.hpp:1713-1840): pre-smoothing and defect on
 * every level but cur_lvl when cur_smooth is false, then restriction to the next coarser level */
static void apply_rest(oc_mg* mg, int cur, int smooth)
{
  const int last = mg->nlevels - 1;
  for(int i = cur; i < last; ++i)
  {
    oc_level* f = &mg->lv[i];
    oc_level* c = &mg->lv[i + 1];
    if(smooth || i > cur)
    {
      richardson_apply(mg, f, f->sol, f->rhs);
      oc_csr_apply(f->def, -1.0, f->sol, 1.0, f->rhs, &f->in.A, 0);
    }
    oc_filter_def(f->def, f->in.fidx, f->in.nf);
    oc_csr_apply(c->rhs, 1.0, f->def, 0.0, c->rhs, &f->in.R, 0);
    oc_filter_def(c->rhs, c->in.fidx, c->in.nf);
  }
}

/* MultiGrid::_apply_prol(cur_lvl, cur_smooth) (multigrid.hpp:1845-1990): prolongation, the (adaptive)
 * coarse-grid correction, post-smoothing on every level but cur_lvl when cur_smooth is false */
static void apply_prol(oc_mg* mg, int cur, int smooth)
{
  const int last = mg->nlevels - 1;
  for(int i = last - 1; i >= cur; --i)
  {
    oc_level* f = &mg->lv[i];
    oc_level* c = &mg->lv[i + 1];
    const uint64_t n = f->n;
    oc_csr_apply(f->cor, 1.0, c->sol, 0.0, f->cor, &f->in.P, 0);
    oc_filter_def(f->cor, f->in.fidx, f->in.nf);
    double w = 1.0;
    if(mg->cgc)
    {
      oc_csr_apply(f->tmp, 1.0, f->cor, 0.0, f->tmp, &f->in.A, 0);
      oc_filter_def(f->tmp, f->in.fidx, f->in.nf);
      if(mg->cgc == 1)
        w = oc_dot(f->def, f->cor, n) / oc_dot(f->tmp, f->cor, n);
      else
        w = oc_dot(f->def, f->tmp, n) / oc_dot(f->tmp, f->tmp, n);
    }
    oc_axpy(f->sol, w, f->cor, f->sol, n);
    if(smooth || i > cur)
    {
      if(mg->cgc)
        oc_axpy(f->def, -w, f->tmp, f->def, n);
      else
      {
        oc_csr_apply(f->def, -1.0, f->sol, 1.0, f->rhs, &f->in.A, 0);
        oc_filter_def(f->def, f->in.fidx, f->in.nf);
      }
      richardson_apply(mg, f, f->cor, f->def);
      oc_axpy(f->sol, 1.0, f->cor, f->sol, n);
    }
  }
}

/* MultiGrid::_apply_smooth_peak + _apply_smooth_def (multigrid.hpp:1591-1700) with the peak smoother */
static void smooth_peak(oc_mg* mg, int l)
{
  oc_level* f = &mg->lv[l];
  oc_csr_apply(f->def, -1.0, f->sol, 1.0, f->rhs, &f->in.A, 0);
  oc_filter_def(f->def, f->in.fidx, f->in.nf);
  richardson_apply(mg, f, f->cor, f->def);
  oc_filter_def(f->cor, f->in.fidx, f->in.nf);
  oc_axpy(f->sol, 1.0, f->cor, f->sol, f->n);
  oc_csr_apply(f->def, -1.0, f->sol, 1.0, f->rhs, &f->in.A, 0);
  oc_filter_def(f->def, f->in.fidx, f->in.nf);
}

static void apply_coarse(oc_mg* mg)
{
  coarse_apply(mg, mg->lv[mg->nlevels - 1].sol, mg->lv[mg->nlevels - 1].rhs);
}

/* cor = MG(def): MultiGrid::_apply_cycle_v / _f / _w (multigrid.hpp:1335-1440) */
int oc_mg_vcycle(oc_mg* mg, double* cor, const double* def)
{
  const int last = mg->nlevels - 1;
  memcpy(mg->lv[0].rhs, def, sizeof(double) * mg->lv[0].n);
  apply_rest(mg, 0, 1);
  if(mg->cycle == 1)
  {
    for(int pk = last - 1; pk > 0; --pk)
    {
      apply_coarse(mg);
      apply_prol(mg, pk, 0);
      smooth_peak(mg, pk);
      apply_rest(mg, pk, 0);
    }
  }
  else if(mg->cycle == 2)
  {
    apply_coarse(mg);
    int counters[64];
    for(int i = 0; i <= last; ++i)
      counters[i] = 0;
    const long num_cgs = 1L << last;
    for(long cgs = 1; cgs < num_cgs; ++cgs)
    {
      int pk = last;
      while(pk > 0)
        if(counters[--pk] == 0)
          break;
      for(int i = last - 1; i > pk; --i)
        counters[i] = 0;
      ++counters[pk];
      apply_prol(mg, pk, 0);
      smooth_peak(mg, pk);
      apply_rest(mg, pk, 0);
      apply_coarse(mg);
    }
  }
  if(mg->cycle != 2)
    apply_coarse(mg);
  apply_prol(mg, 0, 1);
  memcpy(cor, mg->lv[0].sol, sizeof(double) * mg->lv[0].n);
  return 0;
}

/* the smoother's preconditioner: kind 0 Jacobi (the default), 1 SOR, 2 SSOR with damping omega;
 * coloured != 0: the reference's coloured sweeps with greedy_colours (on every level but the coarsest) */
int oc_mg_set_smoother(oc_mg* mg, int kind, double omega, int coloured)
{
  if(kind < 0 || kind > 2)
    return 1;
  mg->smoother = kind;
  mg->sor_omega = omega;
  mg->coloured = kind != 0 && coloured;
  if(mg->coloured && !mg->corder)
  {
    mg->corder = (uint32_t**)calloc((size_t)mg->nlevels, sizeof(uint32_t*));
    mg->cofs = (uint32_t**)calloc((size_t)mg->nlevels, sizeof(uint32_t*));
    mg->ncol = (int*)calloc((size_t)mg->nlevels, sizeof(int));
    for(int l = 0; l < mg->nlevels; ++l)
      mg->ncol[l] = greedy_colours(&mg->lv[l].in.A, &mg->corder[l], &mg->cofs[l]);
  }
  return 0;
}

/* the colouring of level l (greedy_colours): ncol colours, order[n] rows, cofs[ncol + 1] offsets;
 * returns the colour count, or -1 without a coloured smoother */
int oc_mg_colours(const oc_mg* mg, int l, uint32_t* order, uint32_t* cofs)
{
  if(!mg->corder || l < 0 || l >= mg->nlevels)
    return -1;
  if(order)
    memcpy(order, mg->corder[l], sizeof(uint32_t) * mg->lv[l].n);
  if(cofs)
    memcpy(cofs, mg->cofs[l], sizeof(uint32_t) * ((size_t)mg->ncol[l] + 1));
  return mg->ncol[l];
}

/* MultiGrid::set_cycle / set_adapt_cgc */
int oc_mg_set_cycle(oc_mg* mg, int cycle, int cgc)
{
  if(cycle < 0 || cycle > 2 || cgc < 0 || cgc > 2 || mg->nlevels > 62)
    return 1;
  mg->cycle = cycle;
  mg->cgc = cgc;
  return 0;
}

enum { OC_PROGRESS = 0, OC_SUCCESS = 1, OC_ABORTED = 2, OC_DIVERGED = 3, OC_MAX_ITER = 4 };

/* PCG::correct(sol, rhs) preconditioned by one V-cycle (pcg.hpp:159-286).  sol holds the initial
 * guess on entry.  defects[0..iters] receives the defect norms (defects[0] = initial). */
int oc_pcg_solve(oc_mg* mg, double* sol, const double* rhs, double tol_rel, int max_iter,
  double* defects, int* iters_out)
{
  const oc_level* top = &mg->lv[0];
  const uint64_t n = top->n;
  const oc_csr* A = &top->in.A;
  double *r = mg->r, *p = mg->p, *t = mg->t;
  const double tol_abs = 1.0 / (OC_EPS * OC_EPS), div_abs = 1.0 / (OC_EPS * OC_EPS);
  const double div_rel = 1.0 / OC_EPS;

  oc_csr_apply(r, -1.0, sol, 1.0, rhs, A, 0);
  oc_filter_def(r, top->in.fidx, top->in.nf);
  const double def_init = oc_norm2(r, n);
  double def_cur = def_init;
  int it = 0;
  if(defects)
    defects[0] = def_init;
  *iters_out = 0;
  if(!isfinite(def_init))
    return OC_ABORTED;
  if(def_init <= OC_EPS * OC_EPS)
    return OC_SUCCESS;
  oc_mg_vcycle(mg, p, r);
  double gamma = oc_dot(r, p, n);
  for(;;)
  {
    oc_csr_apply(t, 1.0, p, 0.0, t, A, 0);
    oc_filter_def(t, top->in.fidx, top->in.nf);
    const double alpha = gamma / oc_dot(t, p, n);
    oc_axpy(sol, alpha, p, sol, n);
    oc_axpy(r, -alpha, t, r, n);
    ++it;
    def_cur = oc_norm2(r, n);
    if(defects)
      defects[it] = def_cur;
    *iters_out = it;
    if(!isfinite(def_cur))
      return OC_ABORTED;
    if(def_cur > div_abs || def_cur > div_rel * def_init)
      return OC_DIVERGED;
    if(def_cur <= tol_abs && (def_cur <= tol_rel * def_init || def_cur <= 0.0))
      return OC_SUCCESS;
    if(it >= max_iter)
      return OC_MAX_ITER;
    oc_mg_vcycle(mg, t, r);
    const double gamma2 = gamma;
    gamma = oc_dot(r, t, n);
    const double beta = gamma / gamma2;
    oc_axpy(p, beta, p, t, n);
  }
}

/* Plain PCG with a Jacobi preconditioner (or none when omega == 0), on one matrix, for the
 * reference's known-answer iteration counts (kernel/solver/basic_solver-test.cpp:98-140). */
int oc_pcg_jacobi(const oc_csr* A, const uint64_t* fidx, uint64_t nf, double omega, double* sol,
  const double* rhs, double tol_rel, int max_iter, int* iters_out)
{
  const uint64_t n = A->rows;
  double* r = (double*)calloc(n, sizeof(double));
  double* p = (double*)calloc(n, sizeof(double));
  double* t = (double*)calloc(n, sizeof(double));
  double* d = (double*)calloc(n, sizeof(double));
  if(omega > 0.0)
    oc_inv_diag(d, A, omega);
  int status = OC_PROGRESS;
  const double tol_abs = 1.0 / (OC_EPS * OC_EPS);
  oc_csr_apply(r, -1.0, sol, 1.0, rhs, A, 0);
  oc_filter_def(r, fidx, nf);
  const double def_init = oc_norm2(r, n);
  int it = 0;
#define OC_PRECOND(z, v)                                            \
  do {                                                              \
    if(omega > 0.0) for(uint64_t i_ = 0; i_ < n; ++i_) z[i_] = d[i_] * v[i_]; \
    else memcpy(z, v, sizeof(double) * n);                          \
    oc_filter_def(z, fidx, nf);                                     \
  } while(0)
  if(!isfinite(def_init))
    status = OC_ABORTED;
  else if(def_init <= OC_EPS * OC_EPS)
    status = OC_SUCCESS;
  else
  {
    OC_PRECOND(p, r);
    double gamma = oc_dot(r, p, n);
    for(;;)
    {
      oc_csr_apply(t, 1.0, p, 0.0, t, A, 0);
      oc_filter_def(t, fidx, nf);
      const double alpha = gamma / oc_dot(t, p, n);
      oc_axpy(sol, alpha, p, sol, n);
      oc_axpy(r, -alpha, t, r, n);
      ++it;
      const double def_cur = oc_norm2(r, n);
      if(!isfinite(def_cur)) { status = OC_ABORTED; break; }
      if(def_cur <= tol_abs && def_cur <= tol_rel * def_init) { status = OC_SUCCESS; break; }
      if(it >= max_iter) { status = OC_MAX_ITER; break; }
      OC_PRECOND(t, r);
      const double gamma2 = gamma;
      gamma = oc_dot(r, t, n);
      oc_axpy(p, gamma / gamma2, p, t, n);
    }
  }
#undef OC_PRECOND
  *iters_out = it;
  free(r); free(p); free(t); free(d);
  return status;
}
