/*
 * or_elements.c -- oracle (test infrastructure only): panel, line and
 * particle influence kernels of the reference.
 *
 *   src/aeroel/mod_doublet.f90   potential_calc_doublet :113-168,
 *                                velocity_calc_doublet :178-248
 *   src/aeroel/mod_surfpan.f90   potential_calc_sou_surfpan :173-258,
 *                                velocity_calc_sou_surfpan :268-357,
 *                                compute_vel_surfpan :641-658,
 *                                calc_geo_data_surfpan :888-951,
 *                                get_vort_vel_surfpan :962-977
 *   src/aeroel/mod_vortlatt.f90  compute_vel_vortlatt :403-415,
 *                                calc_geo_data_vortlatt :601-669
 *   src/aeroel/mod_vortline.f90  compute_vel_vortline :126-170,
 *                                calc_geo_data_vortline :240-256
 */
#include "or_internal.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static inline void cross3(const double *a, const double *b, double *r) {
  r[0] = a[1] * b[2] - a[2] * b[1];
  r[1] = a[2] * b[0] - a[0] * b[2];
  r[2] = a[0] * b[1] - a[1] * b[0];
}
static inline double dot3(const double *a, const double *b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
static inline double norm3(const double *v) { return sqrt(dot3(v, v)); }

/* next_qua / next_tri (src/general/mod_param.f90:94-97), 0-based */
static inline int nxt(int nv, int i) { return (i + 1) % nv; }

void or_pan_build(const dust_panels *pan, int j, const double *u_inf,
                  or_pan_t *p) {
  memset(p, 0, sizeof(*p));
  int nv = pan->n_ver ? pan->n_ver[j] : 4;
  p->nv = nv;
  p->kind = pan->kind ? pan->kind[j] : DUST_ELEM_VORTLATT;
  for (int v = 0; v < 4; ++v)
    for (int d = 0; d < 3; ++d) p->ver[v][d] = pan->ver[12 * (size_t)j + 3 * v + d];
  for (int d = 0; d < 3; ++d) {
    double s = 0.0;
    for (int v = 0; v < nv; ++v) s += p->ver[v][d];
    p->cen[d] = s / (double)nv;
  }
  double nor[3], a[3], b[3];
  if (nv == 4) {
    for (int d = 0; d < 3; ++d) {
      a[d] = p->ver[2][d] - p->ver[0][d];
      b[d] = p->ver[3][d] - p->ver[1][d];
    }
  } else {
    for (int d = 0; d < 3; ++d) {
      a[d] = p->ver[2][d] - p->ver[1][d];
      b[d] = p->ver[0][d] - p->ver[1][d];
    }
  }
  cross3(a, b, nor);
  p->area = 0.5 * norm3(nor);
  if (p->kind == DUST_ELEM_VORTLATT && norm3(nor) < 1e-16) nor[2] = 1e-16;
  double nn = norm3(nor);
  for (int d = 0; d < 3; ++d) p->nor[d] = nor[d] / nn;
  double tanl[3];
  for (int d = 0; d < 3; ++d)
    tanl[d] = 0.5 * (p->ver[nv - 1][d] + p->ver[0][d]) - p->cen[d];
  double tn = norm3(tanl);
  for (int d = 0; d < 3; ++d) p->tang[0][d] = tanl[d] / tn;
  cross3(p->nor, p->tang[0], p->tang[1]);
  p->max_edge = 0.0;
  for (int v = 0; v < nv; ++v) {
    for (int d = 0; d < 3; ++d) p->edge_vec[v][d] = p->ver[nxt(nv, v)][d] - p->ver[v][d];
    p->edge_len[v] = norm3(p->edge_vec[v]);
    if (v == 0 || p->edge_len[v] > p->max_edge) p->max_edge = p->edge_len[v];
  }
  for (int v = 0; v < nv; ++v)
    for (int d = 0; d < 3; ++d) p->edge_uni[v][d] = p->edge_vec[v][d] / p->edge_len[v];
  for (int v = 0; v < nv; ++v) {
    p->cosTi[v] = dot3(p->edge_uni[v], p->tang[0]);
    p->sinTi[v] = dot3(p->edge_uni[v], p->tang[1]);
    double dv[3] = {p->ver[v][0] - p->cen[0], p->ver[v][1] - p->cen[1],
                    p->ver[v][2] - p->cen[2]};
    double pr = dot3(dv, p->nor);
    for (int d = 0; d < 3; ++d) p->verp[v][d] = p->ver[v][d] - p->nor[d] * pr;
  }
  p->mag = pan->mag ? pan->mag[j] : 0.0;
  double rel[3];
  for (int d = 0; d < 3; ++d) {
    double ub = pan->ub ? pan->ub[3 * (size_t)j + d] : 0.0;
    double uv = pan->uvort ? pan->uvort[3 * (size_t)j + d] : 0.0;
    rel[d] = ub - (u_inf ? u_inf[d] : 0.0) - uv;
  }
  p->sig = dot3(p->nor, rel);
}

void or_line_build(const dust_lines *ln, int j, or_line_t *l) {
  for (int v = 0; v < 2; ++v)
    for (int d = 0; d < 3; ++d) l->ver[v][d] = ln->ver[6 * (size_t)j + 3 * v + d];
  for (int d = 0; d < 3; ++d) {
    l->cen[d] = (l->ver[0][d] + l->ver[1][d]) / 2.0;
    l->edge_vec[d] = l->ver[1][d] - l->ver[0][d];
  }
  l->edge_len = norm3(l->edge_vec);
  for (int d = 0; d < 3; ++d) l->edge_uni[d] = l->edge_vec[d] / l->edge_len;
  l->mag = ln->mag ? ln->mag[j] : 0.0;
}

or_elemctx *or_elemctx_build(const dust_elements *el, const double *u_inf) {
  or_elemctx *c = (or_elemctx *)calloc(1, sizeof(or_elemctx));
  if (u_inf) memcpy(c->u_inf, u_inf, sizeof(c->u_inf));
  if (!el) return c;
  c->nbody = el->body.n;
  c->nwake = el->wake.n;
  c->nline = el->end_vort.n;
  c->body = (or_pan_t *)malloc(sizeof(or_pan_t) * (c->nbody + 1));
  c->wake = (or_pan_t *)malloc(sizeof(or_pan_t) * (c->nwake + 1));
  c->line = (or_line_t *)malloc(sizeof(or_line_t) * (c->nline + 1));
  for (int j = 0; j < c->nbody; ++j) or_pan_build(&el->body, j, u_inf, &c->body[j]);
  for (int j = 0; j < c->nwake; ++j) or_pan_build(&el->wake, j, u_inf, &c->wake[j]);
  for (int j = 0; j < c->nline; ++j) or_line_build(&el->end_vort, j, &c->line[j]);
  return c;
}

void or_elemctx_free(or_elemctx *c) {
  if (!c) return;
  free(c->body);
  free(c->wake);
  free(c->line);
  free(c);
}

/* potential_calc_doublet, mod_doublet.f90:113-168 */
double or_pot_dou(const dust_fmm_params *prm, const or_pan_t *p, const double *pos) {
  double r[3] = {pos[0] - p->cen[0], pos[1] - p->cen[1], pos[2] - p->cen[2]};
  double radius = norm3(r);
  double zQ = dot3(r, p->nor);
  double dou;
  if (radius > prm->far_field_ratio_doublet * p->max_edge) {
    dou = zQ * p->area / pow(radius, 3.0);
  } else {
    dou = 0.0;
    int nv = p->nv;
    for (int i1 = 0; i1 < nv; ++i1) {
      int im1 = (i1 + nv - 1) % nv;
      double ei[3] = {-(pos[0] - p->ver[i1][0]), -(pos[1] - p->ver[i1][1]),
                      -(pos[2] - p->ver[i1][2])};
      double en = norm3(ei);
      for (int d = 0; d < 3; ++d) ei[d] = ei[d] / en;
      double ep = dot3(ei, p->edge_vec[i1]), em = dot3(ei, p->edge_vec[im1]);
      double ap1[3], am1[3];
      for (int d = 0; d < 3; ++d) {
        ap1[d] = p->edge_vec[i1][d] - ei[d] * ep;
        am1[d] = -p->edge_vec[im1][d] + ei[d] * em;
      }
      double ap1n = norm3(ap1), am1n = norm3(am1), cr[3];
      cross3(am1, ap1, cr);
      double sinB = dot3(ei, cr) / (ap1n * am1n);
      double cosB = dot3(am1, ap1) / (ap1n * am1n);
      dou += atan2(sinB, cosB);
    }
    double gb = (double)(nv - 2) * OR_PI;
    if (dou < -gb + 1.0e-5)
      dou = dou + gb;
    else if (dou > gb - 1.0e-5)
      dou = dou - gb;
  }
  return dou;
}

/* velocity_calc_doublet, mod_doublet.f90:178-248 */
void or_vel_dou(const dust_fmm_params *prm, const or_pan_t *p, const double *pos,
                double *v) {
  double rv[3] = {pos[0] - p->cen[0], pos[1] - p->cen[1], pos[2] - p->cen[2]};
  double radius = norm3(rv);
  v[0] = v[1] = v[2] = 0.0;
  if (radius > prm->far_field_ratio_doublet * p->max_edge) {
    double rn = dot3(rv, p->nor);
    double rati = 3.0 * p->area * rn / pow(radius, 5.0);
    double phix = rati * dot3(rv, p->tang[0]);
    double phiy = rati * dot3(rv, p->tang[1]);
    double pdou = p->area * (-pow(radius, 2.0) + 3.0 * pow(rn, 2.0)) / pow(radius, 5.0);
    for (int d = 0; d < 3; ++d)
      v[d] = p->tang[0][d] * phix + p->tang[1][d] * phiy + p->nor[d] * pdou;
  } else {
    for (int i1 = 0; i1 < p->nv; ++i1) {
      int ip1 = nxt(p->nv, i1);
      double av[3] = {pos[0] - p->ver[i1][0], pos[1] - p->ver[i1][1],
                      pos[2] - p->ver[i1][2]};
      double ai = dot3(av, p->edge_uni[i1]);
      double R1 = norm3(av);
      double b2[3] = {pos[0] - p->ver[ip1][0], pos[1] - p->ver[ip1][1],
                      pos[2] - p->ver[ip1][2]};
      double R2 = norm3(b2);
      double hv[3];
      for (int d = 0; d < 3; ++d) hv[d] = av[d] - ai * p->edge_uni[i1][d];
      double hi = norm3(hv), cr[3];
      cross3(p->edge_uni[i1], hv, cr);
      double L = p->edge_len[i1];
      if (hi > L * prm->rankine_rad) {
        double f = ((L - ai) / R2 + ai / R1) / pow(hi, 2.0);
        for (int d = 0; d < 3; ++d) v[d] = v[d] + f * cr[d];
      } else if (R1 > L * prm->cutoff_rad && R2 > L * prm->cutoff_rad) {
        double rr = prm->rankine_rad * L;
        double f = ((L - ai) / R2 + ai / R1) / pow(rr, 2.0);
        for (int d = 0; d < 3; ++d) v[d] = v[d] + f * cr[d];
      }
    }
  }
}

/* potential_calc_sou_surfpan, mod_surfpan.f90:173-258 (ff_ratio 10) */
double or_pot_sou(const or_pan_t *p, double dou, const double *pos) {
  double r[3] = {pos[0] - p->cen[0], pos[1] - p->cen[1], pos[2] - p->cen[2]};
  double radius = norm3(r);
  if (radius > 10.0 * p->max_edge) return p->area / radius;
  double zQ = dot3(r, p->nor);
  double Qp[3] = {pos[0] - zQ * p->nor[0], pos[1] - zQ * p->nor[1],
                  pos[2] - zQ * p->nor[2]};
  double sou = 0.0;
  for (int i1 = 0; i1 < p->nv; ++i1) {
    int ip1 = nxt(p->nv, i1);
    double a[3] = {pos[0] - p->verp[i1][0], pos[1] - p->verp[i1][1],
                   pos[2] - p->verp[i1][2]};
    double b[3] = {pos[0] - p->verp[ip1][0], pos[1] - p->verp[ip1][1],
                   pos[2] - p->verp[ip1][2]};
    double R1 = norm3(a), R2 = norm3(b);
    double den = R1 + R2 - p->edge_len[i1];
    if (den < 1e-6) {
      double a2[3] = {pos[0] - p->ver[i1][0], pos[1] - p->ver[i1][1],
                      pos[2] - p->ver[i1][2]};
      double b2[3] = {pos[0] - p->ver[ip1][0], pos[1] - p->ver[ip1][1],
                      pos[2] - p->ver[ip1][2]};
      R1 = norm3(a2);
      R2 = norm3(b2);
      den = R1 + R2 - p->edge_len[i1];
    }
    double souLog = log((R1 + R2 + p->edge_len[i1]) / den);
    double q[3] = {Qp[0] - p->verp[i1][0], Qp[1] - p->verp[i1][1],
                   Qp[2] - p->verp[i1][2]};
    double cr[3];
    cross3(q, p->edge_vec[i1], cr);
    double vi = -dot3(cr, p->nor) / p->edge_len[i1];
    sou = sou + vi * souLog;
  }
  return sou - zQ * dou;
}

/* velocity_calc_sou_surfpan, mod_surfpan.f90:268-357 (ff_ratio 10) */
void or_vel_sou(const dust_fmm_params *prm, const or_pan_t *p, const double *pos,
                double *v) {
  double rv[3] = {pos[0] - p->cen[0], pos[1] - p->cen[1], pos[2] - p->cen[2]};
  double radius = norm3(rv);
  double phix, phiy, pdou;
  if (radius > 10.0 * p->max_edge) {
    double r3 = pow(radius, 3.0);
    phix = -p->area * dot3(rv, p->tang[0]) / r3;
    phiy = -p->area * dot3(rv, p->tang[1]) / r3;
    pdou = -p->area * dot3(rv, p->nor) / r3;
  } else {
    phix = 0.0;
    phiy = 0.0;
    for (int i1 = 0; i1 < p->nv; ++i1) {
      int ip1 = nxt(p->nv, i1);
      double a[3] = {pos[0] - p->verp[i1][0], pos[1] - p->verp[i1][1],
                     pos[2] - p->verp[i1][2]};
      double b[3] = {pos[0] - p->verp[ip1][0], pos[1] - p->verp[ip1][1],
                     pos[2] - p->verp[ip1][2]};
      double R1 = norm3(a), R2 = norm3(b), L = p->edge_len[i1];
      double souLog = (R1 + R2 - L < 1e-12) ? 0.0 : log((R1 + R2 + L) / (R1 + R2 - L));
      phix = phix + p->sinTi[i1] * souLog;
      phiy = phiy - p->cosTi[i1] * souLog;
    }
    pdou = or_pot_dou(prm, p, pos);
    phix = -phix;
    phiy = -phiy;
    pdou = -pdou;
  }
  for (int d = 0; d < 3; ++d)
    v[d] = p->tang[0][d] * phix + p->tang[1][d] * phiy + p->nor[d] * pdou;
}

/* compute_vel_vortline, mod_vortline.f90:126-170 */
void or_vel_line(const dust_fmm_params *prm, const or_line_t *l, const double *pos,
                 double *v) {
  double av[3] = {pos[0] - l->ver[0][0], pos[1] - l->ver[0][1], pos[2] - l->ver[0][2]};
  double ai = dot3(av, l->edge_uni);
  double R1 = norm3(av);
  double b[3] = {pos[0] - l->ver[1][0], pos[1] - l->ver[1][1], pos[2] - l->ver[1][2]};
  double R2 = norm3(b);
  double hv[3];
  for (int d = 0; d < 3; ++d) hv[d] = av[d] - ai * l->edge_uni[d];
  double hi = norm3(hv), cr[3], vd[3] = {0, 0, 0};
  cross3(l->edge_uni, hv, cr);
  double L = l->edge_len;
  if (hi > L * prm->rankine_rad) {
    double f = ((L - ai) / R2 + ai / R1) / pow(hi, 2.0);
    for (int d = 0; d < 3; ++d) vd[d] = f * cr[d];
  } else if (R1 > L * prm->cutoff_rad && R2 > L * prm->cutoff_rad) {
    double rr = prm->rankine_rad * L;
    double f = ((L - ai) / R2 + ai / R1) / pow(rr, 2.0);
    for (int d = 0; d < 3; ++d) vd[d] = f * cr[d];
  }
  for (int d = 0; d < 3; ++d) v[d] = vd[d] * l->mag;
}

/* compute_vel_surfpan :641-658 / compute_vel_vortlatt :403-415 */
void or_vel_pan(const dust_fmm_params *prm, const or_pan_t *p, const double *pos,
                double *v) {
  double vd[3];
  or_vel_dou(prm, p, pos, vd);
  if (p->kind == DUST_ELEM_SURFPAN) {
    double vs[3];
    or_vel_sou(prm, p, pos, vs);
    for (int d = 0; d < 3; ++d) v[d] = vd[d] * p->mag - vs[d] * p->sig;
  } else {
    for (int d = 0; d < 3; ++d) v[d] = vd[d] * p->mag;
  }
}

void or_elements_vel_accum(const dust_fmm_params *prm, const or_elemctx *c,
                           const double *pos, double *vel) {
  double v[3];
  if (c) {
    for (int j = 0; j < c->nbody; ++j) {
      or_vel_pan(prm, &c->body[j], pos, v);
      for (int d = 0; d < 3; ++d) vel[d] = vel[d] + v[d] / (4.0 * OR_PI);
    }
    for (int j = 0; j < c->nwake; ++j) {
      or_vel_pan(prm, &c->wake[j], pos, v);
      for (int d = 0; d < 3; ++d) vel[d] = vel[d] + v[d] / (4.0 * OR_PI);
    }
    for (int j = 0; j < c->nline; ++j) {
      or_vel_line(prm, &c->line[j], pos, v);
      for (int d = 0; d < 3; ++d) vel[d] = vel[d] + v[d] / (4.0 * OR_PI);
    }
  }
  for (int d = 0; d < 3; ++d) vel[d] = vel[d] + prm->u_inf[d];
}

int or_elements_vel(const dust_fmm_params *prm, int n_pts, const double *pts,
                    const dust_elements *elems, double *vel) {
  or_elemctx *c = or_elemctx_build(elems, prm->u_inf);
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < n_pts; ++i) {
    double v[3] = {0, 0, 0};
    or_elements_vel_accum(prm, c, pts + 3 * i, v);
    for (int d = 0; d < 3; ++d) vel[3 * i + d] = v[d];
  }
  or_elemctx_free(c);
  return DUST_OK;
}

/* get_vort_vel over wake%vort_p = particles then end vortices */
int or_points_uvort(const dust_fmm_params *prm, int n_pts, const double *pts,
                    int n, const double *cen, const double *dir,
                    const double *mag, const double *r_vortex,
                    const dust_lines *end_vort, double *uvort) {
  int nl = end_vort ? end_vort->n : 0;
  or_line_t *ls = (or_line_t *)malloc(sizeof(or_line_t) * (nl + 1));
  for (int j = 0; j < nl; ++j) or_line_build(end_vort, j, &ls[j]);
#pragma omp parallel for schedule(dynamic, 4)
  for (int i = 0; i < n_pts; ++i) {
    const double *pos = pts + 3 * i;
    double u[3] = {0, 0, 0};
    for (int q = 0; q < n; ++q) {
      double dist[3] = {pos[0] - cen[3 * q], pos[1] - cen[3 * q + 1],
                        pos[2] - cen[3 * q + 2]};
      double distn = norm3(dist);
      double dn = sqrt(distn * distn + r_vortex[q] * r_vortex[q]);
      double c = -1.0 / (dn * dn * dn), cr[3];
      cross3(dist, dir + 3 * q, cr);
      for (int d = 0; d < 3; ++d) u[d] = u[d] + (c * cr[d] * mag[q]) / (4.0 * OR_PI);
    }
    for (int j = 0; j < nl; ++j) {
      double v[3];
      or_vel_line(prm, &ls[j], pos, v);
      for (int d = 0; d < 3; ++d) u[d] = u[d] + v[d] / (4.0 * OR_PI);
    }
    for (int d = 0; d < 3; ++d) uvort[3 * i + d] = u[d];
  }
  free(ls);
  return DUST_OK;
}

int or_panel_geometry(const dust_panels *pan, double *cen, double *nor,
                      double *area) {
  for (int j = 0; j < pan->n; ++j) {
    or_pan_t p;
    or_pan_build(pan, j, NULL, &p);
    for (int d = 0; d < 3; ++d) {
      if (cen) cen[3 * j + d] = p.cen[d];
      if (nor) nor[3 * j + d] = p.nor[d];
    }
    if (area) area[j] = p.area;
  }
  return DUST_OK;
}

double or_potential_doublet(const dust_fmm_params *prm, const dust_panels *pan,
                            int j, const double *pos) {
  or_pan_t p;
  or_pan_build(pan, j, prm->u_inf, &p);
  return or_pot_dou(prm, &p, pos);
}
void or_velocity_doublet(const dust_fmm_params *prm, const dust_panels *pan, int j,
                         const double *pos, double *v) {
  or_pan_t p;
  or_pan_build(pan, j, prm->u_inf, &p);
  or_vel_dou(prm, &p, pos, v);
}
double or_potential_source(const dust_fmm_params *prm, const dust_panels *pan,
                           int j, double dou, const double *pos) {
  or_pan_t p;
  (void)prm;
  or_pan_build(pan, j, NULL, &p);
  return or_pot_sou(&p, dou, pos);
}
void or_velocity_source(const dust_fmm_params *prm, const dust_panels *pan, int j,
                        const double *pos, double *v) {
  or_pan_t p;
  or_pan_build(pan, j, NULL, &p);
  or_vel_sou(prm, &p, pos, v);
}
