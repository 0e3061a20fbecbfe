/*
 * or_linsys.c -- oracle (test infrastructure only): influence-coefficient
 * rows and the block LU solve of the reference.
 *
 *   src/linsys/mod_linsys.f90    initialize_linsys :109-267,
 *                                assemble_linsys :279-344,
 *                                solve_linsys :352-482
 *   src/aeroel/mod_surfpan.f90   build_row_surfpan :378-439,
 *                                build_row_static_surfpan :448-481,
 *                                add_wake_surfpan :489-535,
 *                                compute_pot_surfpan :579-601,
 *                                compute_psi_surfpan :610-629
 *   src/aeroel/mod_vortlatt.f90  build_row_vortlatt :143-192,
 *                                build_row_static_vortlatt :201-237,
 *                                add_wake_vortlatt :280-322,
 *                                compute_pot_vortlatt :331-355,
 *                                compute_psi_vortlatt :365-391
 *
 * The dense kernels are plain restatements of LAPACK/BLAS dgetrf (partial
 * pivoting, first maximum wins, like idamax), dgetrs, dlaswp, dtrsm and
 * dgemm; the tests pin them against the LAPACK that scipy links.
 *
 * One deliberate difference: build_row_static_vortlatt zeroes the column
 * b_static(:,ie) inside an OpenMP loop over rows (mod_vortlatt.f90:216),
 * which races with other rows when static surface panels and vortex-lattice
 * rows are mixed; the oracle leaves b_static as initialised (all zero) and
 * writes rows only.  For all-vortex-lattice or all-surface-panel static sets
 * the two agree.
 */
#include "or_internal.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define A_(i, j) A[(size_t)(j) * (size_t)lda + (size_t)(i)]

int or_dgetrf(int m, int n, double *A, int lda, int *ipiv) {
  int info = 0, mn = m < n ? m : n;
  for (int j = 0; j < mn; ++j) {
    int p = j;
    double amax = fabs(A_(j, j));
    for (int i = j + 1; i < m; ++i)
      if (fabs(A_(i, j)) > amax) {
        amax = fabs(A_(i, j));
        p = i;
      }
    ipiv[j] = p + 1;
    if (A_(p, j) != 0.0) {
      if (p != j)
        for (int c = 0; c < n; ++c) {
          double t = A_(j, c);
          A_(j, c) = A_(p, c);
          A_(p, c) = t;
        }
      double r = 1.0 / A_(j, j);
      for (int i = j + 1; i < m; ++i) A_(i, j) *= r;
    } else if (info == 0) {
      info = j + 1;
    }
#pragma omp parallel for schedule(static) if ((size_t)(m - j) * (n - j) > 65536)
    for (int c = j + 1; c < n; ++c) {
      double t = A_(j, c);
      if (t != 0.0)
        for (int i = j + 1; i < m; ++i) A_(i, c) -= A_(i, j) * t;
    }
  }
  return info;
}

void or_dlaswp(int n, double *A, int lda, int k1, int k2, const int *ipiv) {
  for (int i = k1 - 1; i < k2; ++i) {
    int ip = ipiv[i] - 1;
    if (ip != i)
      for (int c = 0; c < n; ++c) {
        double t = A_(i, c);
        A_(i, c) = A_(ip, c);
        A_(ip, c) = t;
      }
  }
}

/* B := inv(L) B, L unit lower (m x m), B m x n */
void or_dtrsm_llnu(int m, int n, const double *A, int lda, double *B, int ldb) {
#pragma omp parallel for schedule(static)
  for (int c = 0; c < n; ++c)
    for (int k = 0; k < m; ++k) {
      double t = B[(size_t)c * ldb + k];
      if (t != 0.0)
        for (int i = k + 1; i < m; ++i) B[(size_t)c * ldb + i] -= t * A_(i, k);
    }
}

/* B := B inv(U), U upper non-unit (n x n), B m x n */
void or_dtrsm_runn(int m, int n, const double *A, int lda, double *B, int ldb) {
  for (int j = 0; j < n; ++j) {
    for (int k = 0; k < j; ++k) {
      double t = A_(k, j);
      if (t != 0.0)
        for (int i = 0; i < m; ++i) B[(size_t)j * ldb + i] -= t * B[(size_t)k * ldb + i];
    }
    double r = 1.0 / A_(j, j);
    for (int i = 0; i < m; ++i) B[(size_t)j * ldb + i] *= r;
  }
}

/* C -= A B */
void or_dgemm_nn_minus(int m, int n, int k, const double *A, int lda,
                       const double *B, int ldb, double *C, int ldc) {
#pragma omp parallel for schedule(static)
  for (int j = 0; j < n; ++j)
    for (int l = 0; l < k; ++l) {
      double t = B[(size_t)j * ldb + l];
      if (t != 0.0)
        for (int i = 0; i < m; ++i) C[(size_t)j * ldc + i] -= t * A_(i, l);
    }
}

void or_dgetrs(int n, int nrhs, const double *A, int lda, const int *ipiv,
               double *B, int ldb) {
  or_dlaswp(nrhs, B, ldb, 1, n, ipiv);
  for (int c = 0; c < nrhs; ++c) {
    double *b = B + (size_t)c * ldb;
    for (int k = 0; k < n; ++k)
      if (b[k] != 0.0)
        for (int i = k + 1; i < n; ++i) b[i] -= b[k] * A_(i, k);
    for (int k = n - 1; k >= 0; --k) {
      if (b[k] != 0.0) {
        b[k] /= A_(k, k);
        double t = b[k];
        for (int i = 0; i < k; ++i) b[i] -= t * A_(i, k);
      }
    }
  }
}

/* ---------------------------------------------------------------- rows */
typedef struct {
  const dust_fmm_params *prm;
  or_pan_t *el; /* implicit elements */
  int nwake, n_impl;
  or_pan_t *wk;
  const int *impl;
} rowctx;

/* compute_pot_{surfpan,vortlatt}(A, b, pos, i, j) */
static void compute_pot(const rowctx *c, int j, const double *pos, int i_row,
                        double *A, double *b) {
  const or_pan_t *p = &c->el[j];
  double dou = (i_row != j) ? or_pot_dou(c->prm, p, pos) : -2.0 * OR_PI;
  *A = -dou;
  *b = (p->kind == DUST_ELEM_SURFPAN) ? or_pot_sou(p, dou, pos) : 0.0;
}
/* compute_psi_{surfpan,vortlatt}(A, b, pos, nor, i, j) */
static void compute_psi(const rowctx *c, int j, const double *pos,
                        const double *nor, int i_row, double *A, double *b) {
  const or_pan_t *p = &c->el[j];
  double vd[3];
  or_vel_dou(c->prm, p, pos, vd);
  *A = vd[0] * nor[0] + vd[1] * nor[1] + vd[2] * nor[2];
  if (p->kind == DUST_ELEM_SURFPAN) {
    double vs[3];
    or_vel_sou(c->prm, p, pos, vs);
    *b = -vs[0] * nor[0] + -vs[1] * nor[1] + -vs[2] * nor[2];
  } else {
    *b = (i_row == j) ? 4.0 * OR_PI : 0.0;
  }
}

static double nor_rel(const or_pan_t *p) { return p->sig; }
static double nor_static(const or_pan_t *p, const double *u_inf, const double *uvort) {
  /* nor . (-wind - uvort) */
  return p->nor[0] * (-u_inf[0] - uvort[0]) + p->nor[1] * (-u_inf[1] - uvort[1]) +
         p->nor[2] * (-u_inf[2] - uvort[2]);
}

static void build_row_static(const rowctx *c, double *A, int lda, double *bst,
                             int nst, int ie, int ista, int iend) {
  const or_pan_t *r = &c->el[ie];
  for (int j = ista; j <= iend; ++j) {
    double b1;
    if (r->kind == DUST_ELEM_SURFPAN)
      compute_pot(c, j, r->cen, ie, &A_(ie, j), &b1);
    else
      compute_psi(c, j, r->cen, r->nor, ie, &A_(ie, j), &b1);
    bst[(size_t)j * nst + ie] = b1;
  }
}

/* Row ie of A (element (ie, j) at A[j * lda + ie - roff]) and b[ie - roff]:
 * roff = 0 for the full system, roff = ie with lda = 1 for a single row. */
static void build_row(const rowctx *c, double *A, int lda, const double *bst,
                      int nst, const double *uvort, double *b, int ie, int ista,
                      int iend, int roff) {
  const or_pan_t *r = &c->el[ie];
  const double *u = c->prm->u_inf;
  b[ie - roff] = 0.0;
  for (int j = 0; j < ista; ++j)
    b[ie - roff] = b[ie - roff] + bst[(size_t)j * nst + ie] * nor_static(&c->el[j], u, uvort + 3 * j);
  for (int j = ista; j <= iend; ++j) {
    double b1;
    if (r->kind == DUST_ELEM_SURFPAN) {
      compute_pot(c, j, r->cen, ie, &A[(size_t)j * lda + (size_t)(ie - roff)], &b1);
      b[ie - roff] = b[ie - roff] + b1 * nor_rel(&c->el[j]);
    } else {
      compute_psi(c, j, r->cen, r->nor, ie, &A[(size_t)j * lda + (size_t)(ie - roff)], &b1);
      if (ie == j) {
        /* nor_ie . (ub_ie - wind - uvort_j) with j == ie */
        b[ie - roff] = b[ie - roff] + b1 * nor_rel(&c->el[ie]);
      } else {
        b[ie - roff] = b[ie - roff] + b1 * nor_rel(&c->el[j]);
      }
    }
  }
}

static void add_wake(const rowctx *c, double *A, int lda, double *b, int ie,
                     int ista, int iend, int roff) {
  const or_pan_t *r = &c->el[ie];
  for (int j = 0; j < c->n_impl; ++j) {
    int i1 = c->impl[2 * j] - 1, i2 = c->impl[2 * j + 1] - 1;
    if (r->kind == DUST_ELEM_SURFPAN) {
      if (i1 >= ista && i1 <= iend && i2 >= ista && i2 <= iend) {
        double a = -or_pot_dou(c->prm, &c->wk[j], r->cen);
        A[(size_t)i1 * lda + (size_t)(ie - roff)] = A[(size_t)i1 * lda + (size_t)(ie - roff)] + a;
        A[(size_t)i2 * lda + (size_t)(ie - roff)] = A[(size_t)i2 * lda + (size_t)(ie - roff)] - a;
      }
    } else {
      if (i1 >= ista && i1 <= iend) {
        double vd[3];
        or_vel_dou(c->prm, &c->wk[j], r->cen, vd);
        double a = vd[0] * r->nor[0] + vd[1] * r->nor[1] + vd[2] * r->nor[2];
        A[(size_t)i1 * lda + (size_t)(ie - roff)] = A[(size_t)i1 * lda + (size_t)(ie - roff)] + a;
        if (i2 >= 0) A[(size_t)i2 * lda + (size_t)(ie - roff)] = A[(size_t)i2 * lda + (size_t)(ie - roff)] - a;
      }
    }
  }
  for (int j = c->n_impl; j < c->nwake; ++j) {
    double a;
    if (r->kind == DUST_ELEM_SURFPAN) {
      a = -or_pot_dou(c->prm, &c->wk[j], r->cen);
    } else {
      double vd[3];
      or_vel_dou(c->prm, &c->wk[j], r->cen, vd);
      a = vd[0] * r->nor[0] + vd[1] * r->nor[1] + vd[2] * r->nor[2];
    }
    b[ie - roff] = b[ie - roff] - a * c->wk[j].mag;
  }
}

static void ctx_load(rowctx *c, const dust_fmm_params *prm, int rank,
                     const dust_panels *el, const dust_wake_rows *wk) {
  c->prm = prm;
  c->el = (or_pan_t *)malloc(sizeof(or_pan_t) * rank);
  for (int j = 0; j < rank; ++j) or_pan_build(el, j, prm->u_inf, &c->el[j]);
  c->nwake = wk ? wk->pan.n : 0;
  c->n_impl = wk ? wk->n_impl : 0;
  c->impl = wk ? wk->impl_ind : NULL;
  c->wk = (or_pan_t *)malloc(sizeof(or_pan_t) * (c->nwake + 1));
  for (int j = 0; j < c->nwake; ++j) or_pan_build(&wk->pan, j, prm->u_inf, &c->wk[j]);
}
static void ctx_free(rowctx *c) {
  free(c->el);
  free(c->wk);
}

/* initialize_linsys without the LU (mod_linsys.f90:109-229): the static
 * rows (columns 0..nst-1) and the static wake into A (rank x rank,
 * column-major), bst (nst x nst) and b. */
void or_linsys_init(const dust_fmm_params *prm, int rank, int nst,
                    const dust_panels *elems, const dust_wake_rows *wake, double *A,
                    double *bst, double *b) {
  int lda = rank;
  rowctx c;
  ctx_load(&c, prm, rank, elems, wake);
#pragma omp parallel for schedule(dynamic)
  for (int ie = 0; ie < nst; ++ie) build_row_static(&c, A, lda, bst, nst, ie, 0, nst - 1);
#pragma omp parallel for schedule(dynamic)
  for (int ie = 0; ie < nst; ++ie) add_wake(&c, A, lda, b, ie, 0, nst - 1, 0);
  ctx_free(&c);
}

/* assemble_linsys with uvort given (mod_linsys.f90:279-344): moving columns
 * of the static rows, all columns of the moving rows, the right-hand side
 * and the wake terms; the static block of A (its LU) is not touched. */
void or_linsys_step(const dust_fmm_params *prm, int rank, int nst,
                    const dust_panels *elems, const dust_wake_rows *wake, double *A,
                    const double *bst, double *b) {
  int n = rank, lda = rank;
  rowctx c;
  ctx_load(&c, prm, rank, elems, wake);
  double *uv = (double *)calloc(3 * (size_t)n, sizeof(double));
  if (elems->uvort) memcpy(uv, elems->uvort, sizeof(double) * 3 * n);
#pragma omp parallel for schedule(dynamic)
  for (int ie = 0; ie < n; ++ie) {
    if (ie < nst)
      build_row(&c, A, lda, bst, nst, uv, b, ie, nst, n - 1, 0);
    else
      build_row(&c, A, lda, bst, nst, uv, b, ie, 0, n - 1, 0);
  }
#pragma omp parallel for schedule(dynamic)
  for (int ie = 0; ie < n; ++ie) {
    if (ie < nst)
      add_wake(&c, A, lda, b, ie, nst, n - 1, 0);
    else
      add_wake(&c, A, lda, b, ie, 0, n - 1, 0);
  }
  free(uv);
  ctx_free(&c);
}

int or_linsys_run(const dust_fmm_params *prm, int rank, int nstatic,
                  const dust_panels *elems_init, const dust_panels *elems_step,
                  const dust_wake_rows *wake_init, const dust_wake_rows *wake_step,
                  double *A_out, double *b_out, double *res) {
  int n = rank, nst = nstatic, nmv = rank - nstatic, lda = rank;
  double *A = (double *)calloc((size_t)n * n, sizeof(double));
  double *b = (double *)calloc(n, sizeof(double));
  double *bst = (double *)calloc((size_t)(nst > 0 ? nst : 1) * (nst > 0 ? nst : 1),
                                 sizeof(double));
  int *P = (int *)calloc(n, sizeof(int));
  int info = 0;
  or_linsys_init(prm, rank, nst, elems_init, wake_init, A, bst, b);
  if (nst > 0) {
    info = or_dgetrf(nst, nst, A, lda, P);
    if (info) goto done;
  }
  or_linsys_step(prm, rank, nst, elems_step, wake_step, A, bst, b);
  if (A_out) memcpy(A_out, A, sizeof(double) * (size_t)n * n);
  if (b_out) memcpy(b_out, b, sizeof(double) * n);
  /* solve_linsys */
  if (nst > 0 && nmv > 0) {
    double *Asd = (double *)malloc(sizeof(double) * (size_t)nst * nmv);
    double *Ads = (double *)malloc(sizeof(double) * (size_t)nmv * nst);
    for (int j = 0; j < nmv; ++j)
      for (int i = 0; i < nst; ++i) Asd[(size_t)j * nst + i] = A_(i, nst + j);
    for (int j = 0; j < nst; ++j)
      for (int i = 0; i < nmv; ++i) Ads[(size_t)j * nmv + i] = A_(nst + i, j);
    or_dlaswp(nmv, Asd, nst, 1, nst, P);
    or_dtrsm_llnu(nst, nmv, A, lda, Asd, nst);
    or_dtrsm_runn(nmv, nst, A, lda, Ads, nmv);
    or_dgemm_nn_minus(nmv, nmv, nst, Ads, nmv, Asd, nst, &A_(nst, nst), lda);
    for (int j = 0; j < nmv; ++j)
      for (int i = 0; i < nst; ++i) A_(i, nst + j) = Asd[(size_t)j * nst + i];
    for (int j = 0; j < nst; ++j)
      for (int i = 0; i < nmv; ++i) A_(nst + i, j) = Ads[(size_t)j * nmv + i];
    free(Asd);
    free(Ads);
  }
  if (nmv > 0) {
    info = or_dgetrf(nmv, nmv, &A_(nst, nst), lda, P + nst);
    if (info) goto done;
  }
  if (nst > 0 && nmv > 0) {
    /* dlaswp on A(nst+1:rank, 1:nst) */
    for (int i = 0; i < nmv; ++i) {
      int ip = P[nst + i] - 1;
      if (ip != i)
        for (int cc = 0; cc < nst; ++cc) {
          double t = A_(nst + i, cc);
          A_(nst + i, cc) = A_(nst + ip, cc);
          A_(nst + ip, cc) = t;
        }
    }
  }
  for (int i = nst; i < n; ++i) P[i] += nst;
  memcpy(res, b, sizeof(double) * n);
  or_dgetrs(n, 1, A, lda, P, res, n);
done:
  free(A);
  free(b);
  free(bst);
  free(P);
  return info ? DUST_ERR_SINGULAR : DUST_OK;
}

/* Selected rows of the system as assemble_linsys builds them when every
 * element is moving (nstatic = 0: build_row over all columns, then
 * add_wake; mod_linsys.f90:279-344): row r of the output is element
 * rows[r]; A_rows is nrows x rank row-major, b_rows nrows. */
int or_linsys_rows(const dust_fmm_params *prm, int rank, const dust_panels *elems,
                   const dust_wake_rows *wake, int nrows, const int *rows,
                   double *A_rows, double *b_rows) {
  rowctx c;
  ctx_load(&c, prm, rank, elems, wake);
  double *uv = (double *)calloc(3 * (size_t)rank, sizeof(double));
  if (elems->uvort) memcpy(uv, elems->uvort, sizeof(double) * 3 * rank);
  int bad = 0;
#pragma omp parallel for schedule(dynamic)
  for (int r = 0; r < nrows; ++r) {
    int ie = rows[r];
    if (ie < 0 || ie >= rank) {
      bad = 1;
      continue;
    }
    double *Ar = A_rows + (size_t)r * rank;
    double *br = b_rows + r;
    for (int j = 0; j < rank; ++j) Ar[j] = 0.0;
    *br = 0.0;
    build_row(&c, Ar, 1, NULL, 1, uv, br, ie, 0, rank - 1, ie);
    add_wake(&c, Ar, 1, br, ie, 0, rank - 1, ie);
  }
  free(uv);
  ctx_free(&c);
  return bad ? 6 : 0;
}
