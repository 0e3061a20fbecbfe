/*
 * or_pressure.c -- oracle (test infrastructure only): the pressure integral
 * equation of one time step.
 *
 *   src/linsys/mod_linsys.f90            A_pres from the surface-panel block
 *                                        of A before the wake correction
 *                                        (:184-187 at initialize_linsys,
 *                                        :318-323 at assemble_linsys); LU of
 *                                        its static block (:250-257)
 *   src/linsys/mod_pressure_equation.f90 initialize_pressure_sys :44-79
 *                                        (b_static_pres), assemble_pressure_sys
 *                                        :139-235 (rotational terms of the
 *                                        particles, end vortices and wake
 *                                        panels), solve_pressure_sys :243-387
 *   src/aeroel/mod_surfpan.f90           build_row_surfpan :396-437 (the
 *                                        Bernoulli source terms of b_pres)
 *
 * The Bernoulli source of each surface panel (press_normvel_der,
 * mod_pressure_equation.f90:395-455, which needs the surface velocities of
 * the loads computation) is an input.  Elements are ordered static first;
 * the surface panels keep that order (idSurfPan).  The block LU uses the
 * dense restatements of or_linsys.c.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "or_internal.h"

/* compute_pot of element j at the centre of surface panel i (global
 * indices): a = -dou (the diagonal -(-2 pi)), b1 = source potential */
static void pot_pair(const dust_fmm_params *prm, const or_pan_t *el, int i, int j, double *a,
                     double *b1) {
  const or_pan_t *p = &el[j];
  const double *pos = el[i].cen;
  double dou = (i != j) ? or_pot_dou(prm, p, pos) : -2.0 * OR_PI;
  *a = -dou;
  *b1 = (p->kind == DUST_ELEM_SURFPAN) ? or_pot_sou(p, dou, pos) : 0.0;
}

static void cross3(const double *a, const double *b, double *r) {
  r[0] = a[1] * b[2] - a[2] * b[1];
  r[1] = a[2] * b[0] - a[0] * b[2];
  r[2] = a[0] * b[1] - a[1] * b[0];
}
static double norm3(const double *v) { return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }

int or_pressure_run(const dust_fmm_params *prm, int rank, int nstatic,
                    const dust_panels *elems_init, const dust_panels *elems_step,
                    const double *bern, int n, const double *cen, const double *dir,
                    const double *mag, const double *r_vortex, const double *vel,
                    const dust_panels *wake, const double *wake_vv, const dust_lines *end_vort,
                    const double *end_vv, double *A_out, double *b_out, double *res) {
  or_pan_t *e0 = (or_pan_t *)malloc(sizeof(or_pan_t) * (size_t)rank);
  or_pan_t *e1 = (or_pan_t *)malloc(sizeof(or_pan_t) * (size_t)rank);
  for (int j = 0; j < rank; ++j) {
    or_pan_build(elems_init, j, prm->u_inf, &e0[j]);
    or_pan_build(elems_step, j, prm->u_inf, &e1[j]);
  }
  /* idSurfPan / idSurfPanG2L */
  int *id = (int *)malloc(sizeof(int) * (size_t)(rank + 1));
  int *g2l = (int *)malloc(sizeof(int) * (size_t)(rank + 1));
  int nsp = 0, nsst = 0;
  for (int j = 0; j < rank; ++j) {
    g2l[j] = -1;
    if (e1[j].kind == DUST_ELEM_SURFPAN) {
      g2l[j] = nsp;
      id[nsp++] = j;
      if (j < nstatic) ++nsst;
    }
  }
  const int nsmv = nsp - nsst;
  double *A = (double *)calloc((size_t)(nsp > 0 ? nsp : 1) * (nsp > 0 ? nsp : 1), sizeof(double));
  double *bsp = (double *)calloc((size_t)(nsst > 0 ? nsst : 1) * (nsst > 0 ? nsst : 1),
                                 sizeof(double));
  double *b = (double *)calloc((size_t)(nsp > 0 ? nsp : 1), sizeof(double));
  int *P = (int *)calloc((size_t)(nsp > 0 ? nsp : 1), sizeof(int));
  int info = 0;
#define AP(i, j) A[(size_t)(j) * nsp + (i)]
  /* initialize_linsys: static rows x static columns (A and b_static) */
#pragma omp parallel for schedule(dynamic)
  for (int i = 0; i < nsst; ++i)
    for (int j = 0; j < nsst; ++j) {
      double a, b1;
      pot_pair(prm, e0, id[i], id[j], &a, &b1);
      AP(i, j) = a;
      bsp[(size_t)j * nsst + i] = b1;
    }
  if (nsst > 0) {
    info = or_dgetrf(nsst, nsst, A, nsp, P);
    if (info) goto done;
  }
  /* assemble_linsys: static rows x moving columns, moving rows x all */
#pragma omp parallel for schedule(dynamic)
  for (int i = 0; i < nsp; ++i) {
    const int gi = id[i];
    const int static_row = gi < nstatic;
    for (int j = static_row ? nsst : 0; j < nsp; ++j) {
      double a, b1;
      pot_pair(prm, e1, gi, id[j], &a, &b1);
      AP(i, j) = a;
    }
    /* build_row_surfpan: Bernoulli source terms (:396-437) */
    double s = 0.0;
    if (bern) {
      if (static_row)
        for (int j = 0; j < nsst; ++j) s = s + bsp[(size_t)j * nsst + i] * bern[j];
      for (int j = static_row ? nstatic : 0; j < rank; ++j) {
        if (e1[j].kind != DUST_ELEM_SURFPAN) continue;
        double a, b1;
        pot_pair(prm, e1, gi, j, &a, &b1);
        s = s + b1 * bern[g2l[j]];
      }
    }
    b[i] = s;
  }
  /* assemble_pressure_sys: rotational terms (:170-226) */
  {
    or_pan_t *wk = NULL;
    or_line_t *ln = NULL;
    int nw = wake ? wake->n : 0, nl = end_vort ? end_vort->n : 0;
    wk = (or_pan_t *)malloc(sizeof(or_pan_t) * (size_t)(nw + 1));
    ln = (or_line_t *)malloc(sizeof(or_line_t) * (size_t)(nl + 1));
    for (int j = 0; j < nw; ++j) or_pan_build(wake, j, prm->u_inf, &wk[j]);
    for (int j = 0; j < nl; ++j) or_line_build(end_vort, j, &ln[j]);
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < nsp; ++i) {
      const double *ec = e1[id[i]].cen;
      double s = b[i];
      for (int q = 0; q < n; ++q) { /* (c.1) particles */
        double d[3], w[3];
        for (int k = 0; k < 3; ++k) d[k] = cen[3 * (size_t)q + k] - ec[k];
        cross3(dir + 3 * (size_t)q, vel + 3 * (size_t)q, w);
        const double dw = d[0] * w[0] + d[1] * w[1] + d[2] * w[2];
        const double rr = sqrt((d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) +
                               r_vortex[q] * r_vortex[q]);
        s = s + dw * mag[q] / (rr * rr * rr);
      }
      for (int j = 0; j < nl; ++j) { /* (c.2) end vortices */
        double d1[3], d2[3], c1[3], c2[3];
        const double *v1 = end_vv + 6 * (size_t)j, *v2 = v1 + 3;
        for (int k = 0; k < 3; ++k) {
          d1[k] = ln[j].ver[0][k] - ec[k];
          d2[k] = ln[j].ver[1][k] - ec[k];
        }
        cross3(d1, v1, c1);
        cross3(d2, v2, c2);
        const double n1 = norm3(d1), n2 = norm3(d2);
        const double n13 = n1 * n1 * n1, n23 = n2 * n2 * n2;
        double t = 0.0;
        for (int k = 0; k < 3; ++k) t += ln[j].edge_vec[k] * (c1[k] / n13 + c2[k] / n23);
        s = s - 0.5 * ln[j].mag * t;
      }
      for (int j = 0; j < nw; ++j) { /* (c.3) wake panels */
        const or_pan_t *p = &wk[j];
        for (int e = 0; e < p->nv; ++e) {
          const int en = (e + 1) % p->nv;
          double d1[3], d2[3], c1[3], c2[3];
          const double *v1 = wake_vv + 12 * (size_t)j + 3 * e, *v2 = wake_vv + 12 * (size_t)j + 3 * en;
          for (int k = 0; k < 3; ++k) {
            d1[k] = p->ver[e][k] - ec[k];
            d2[k] = p->ver[en][k] - ec[k];
          }
          cross3(d1, v1, c1);
          cross3(d2, v2, c2);
          const double n1 = norm3(d1), n2 = norm3(d2);
          const double n13 = n1 * n1 * n1, n23 = n2 * n2 * n2;
          double t = 0.0;
          for (int k = 0; k < 3; ++k) t += p->edge_vec[e][k] * (c1[k] / n13 + c2[k] / n23);
          s = s - 0.5 * p->mag * t;
        }
      }
      b[i] = s;
    }
    free(wk);
    free(ln);
  }
  if (A_out) memcpy(A_out, A, sizeof(double) * (size_t)nsp * nsp);
  if (b_out) memcpy(b_out, b, sizeof(double) * (size_t)nsp);
  /* solve_pressure_sys (:243-387): the solve_linsys sequence on A_pres */
  if (nsst > 0 && nsmv > 0) {
    double *Asd = (double *)malloc(sizeof(double) * (size_t)nsst * nsmv);
    double *Ads = (double *)malloc(sizeof(double) * (size_t)nsmv * nsst);
    for (int j = 0; j < nsmv; ++j)
      for (int i = 0; i < nsst; ++i) Asd[(size_t)j * nsst + i] = AP(i, nsst + j);
    for (int j = 0; j < nsst; ++j)
      for (int i = 0; i < nsmv; ++i) Ads[(size_t)j * nsmv + i] = AP(nsst + i, j);
    or_dlaswp(nsmv, Asd, nsst, 1, nsst, P);
    or_dtrsm_llnu(nsst, nsmv, A, nsp, Asd, nsst);
    or_dtrsm_runn(nsmv, nsst, A, nsp, Ads, nsmv);
    or_dgemm_nn_minus(nsmv, nsmv, nsst, Ads, nsmv, Asd, nsst, &AP(nsst, nsst), nsp);
    for (int j = 0; j < nsmv; ++j)
      for (int i = 0; i < nsst; ++i) AP(i, nsst + j) = Asd[(size_t)j * nsst + i];
    for (int j = 0; j < nsst; ++j)
      for (int i = 0; i < nsmv; ++i) AP(nsst + i, j) = Ads[(size_t)j * nsmv + i];
    free(Asd);
    free(Ads);
  }
  if (nsmv > 0) {
    info = or_dgetrf(nsmv, nsmv, &AP(nsst, nsst), nsp, P + nsst);
    if (info) goto done;
  }
  if (nsst > 0 && nsmv > 0) {
    for (int i = 0; i < nsmv; ++i) {
      int ip = P[nsst + i] - 1;
      if (ip != i)
        for (int c = 0; c < nsst; ++c) {
          double t = AP(nsst + i, c);
          AP(nsst + i, c) = AP(nsst + ip, c);
          AP(nsst + ip, c) = t;
        }
    }
  }
  for (int i = nsst; i < nsp; ++i) P[i] += nsst;
  memcpy(res, b, sizeof(double) * (size_t)nsp);
  if (nsp > 0) or_dgetrs(nsp, 1, A, nsp, P, res, nsp);
#undef AP
done:
  free(e0);
  free(e1);
  free(id);
  free(g2l);
  free(A);
  free(bsp);
  free(b);
  free(P);
  return info ? DUST_ERR_SINGULAR : DUST_OK;
}

/* The particles' rotational term of assemble_pressure_sys alone
 * (mod_pressure_equation.f90:170-186) at n_pts points: out[i] = sum over
 * the n particles of dist . (dir x vel) mag / (|dist|^2 + r_v^2)^(3/2),
 * dist = x_p - pts_i (the CPU baseline's sampled pressure assembly). */
int or_pressure_particles(int n_pts, const double *pts, int n, const double *cen,
                          const double *dir, const double *mag, const double *r_vortex,
                          const double *vel, double *out) {
#pragma omp parallel for schedule(dynamic, 4)
  for (int i = 0; i < n_pts; ++i) {
    const double *ec = pts + 3 * (size_t)i;
    double s = 0.0;
    for (int q = 0; q < n; ++q) {
      double d[3], w[3];
      for (int k = 0; k < 3; ++k) d[k] = cen[3 * (size_t)q + k] - ec[k];
      cross3(dir + 3 * (size_t)q, vel + 3 * (size_t)q, w);
      const double dw = d[0] * w[0] + d[1] * w[1] + d[2] * w[2];
      const double rr =
          sqrt((d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) + r_vortex[q] * r_vortex[q]);
      s = s + dw * mag[q] / (rr * rr * rr);
    }
    out[i] = s;
  }
  return DUST_OK;
}
