/*
 * or_wake.c -- oracle (test infrastructure): the particle loop of
 * complete_wake, src/aeroel/mod_wake.f90:1309-1355, and its penetration
 * avoidance (avoid_collision, :2350-2534), in plain C (FP64, built with
 * -ffp-contract=off: every product and sum rounded on its own, in the
 * reference's left-to-right order).  norm2 is restated as the square root of
 * the sum of squares.  The panel-wake bookkeeping and the shedding of
 * update_wake / complete_wake are restated in wake_oracle.py.
 */
#include <math.h>
#include <stdlib.h>

#include "or_internal.h"

static double or_norm3(const double *v) { return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }

int or_particles_update(const dust_update_params *u, int n, double *cen, double *dir,
                        const double *mag, const double *vel, double *stretch,
                        const double *rotu, int *free_flag, int *n_freed) {
  if (!u || n < 0 || !n_freed || u->ndt_update_wake == 0) return DUST_ERR_BAD_ARG;
  const double nd = (double)u->ndt_update_wake;
  int freed = 0;
  for (int ip = 0; ip < n; ++ip) {
    if (free_flag[ip]) continue; /* :1320 */
    double *c = cen + 3 * (size_t)ip, *d = dir + 3 * (size_t)ip, *s = stretch + 3 * (size_t)ip;
    const double *v = vel + 3 * (size_t)ip;
    double p[3];
    for (int k = 0; k < 3; ++k) p[k] = c[k] + v[k] * u->dt * nd; /* :1321-1322 */
    int in = 1;
    for (int k = 0; k < 3; ++k) in = in && p[k] >= u->box_min[k];
    for (int k = 0; k < 3; ++k) in = in && p[k] <= u->box_max[k]; /* :1324-1325 */
    if (!in) {
      free_flag[ip] = 1; /* :1347-1351 */
      ++freed;
      continue;
    }
    for (int k = 0; k < 3; ++k) c[k] = p[k]; /* :1326 */
    if (!(u->vortstretch || u->diffusion)) continue; /* :1328 */
    const double m = mag[ip];
    if (u->divergence_filtering) { /* :1331-1334 */
      const double *r = rotu + 3 * (size_t)ip;
      const double nr = or_norm3(r), kf = u->filt_eta / nd;
      for (int k = 0; k < 3; ++k) s[k] = s[k] - kf * (d[k] * m - r[k] * m / nr);
    }
    double a[3]; /* :1337-1345 */
    for (int k = 0; k < 3; ++k) a[k] = d[k] * m + s[k] * u->dt * nd;
    const double an = or_norm3(a);
    if (an != 0.0)
      for (int k = 0; k < 3; ++k) d[k] = a[k] / an;
  }
  *n_freed = freed;
  return DUST_OK;
}

/* avoid_collision, src/aeroel/mod_wake.f90:2350-2534: the velocity of one
 * particle corrected against every element of elems_tot in order.  Both
 * branches keep the reference's expressions: the surface-panel branch uses
 * the signed normal distance, the vortex-ring branch norm2(dist * n) (a
 * componentwise product) and doubles the layer thickness at every ring that
 * passes its approach test (:2470). */
static void or_avoid_collision(const dust_pa_params *pa, const dust_update_params *u,
                               const or_pan_t *el, const double *ub, int nel,
                               const double *cen, double r_vortex, const double *vel_in,
                               double *vel_out) {
  const double nd = (double)u->ndt_update_wake;
  const double rad_mult = pa->check_radius, elrad_mult = pa->element_radius;
  double blthick = r_vortex; /* :2377 */
  const double r2d2 = sqrt(2.0) / 2.0;
  double vel[3] = {vel_in[0], vel_in[1], vel_in[2]};
  for (int ie = 0; ie < nel; ++ie) {
    const or_pan_t *e = &el[ie];
    const double *eub = ub ? ub + 3 * (size_t)ie : NULL;
    double dist1[3], n[3], relvel[3];
    for (int k = 0; k < 3; ++k) dist1[k] = cen[k] - e->cen[k];
    double elrad = e->edge_len[0];
    for (int v = 1; v < e->nv; ++v)
      if (e->edge_len[v] > elrad) elrad = e->edge_len[v];
    elrad = elrad * r2d2;
    const double check_radius = u->dt * pa->u_ref * rad_mult + elrad;
    const double distn = or_norm3(dist1);
    if (!(distn < check_radius)) continue;
    for (int k = 0; k < 3; ++k) {
      relvel[k] = vel[k] - (eub ? eub[k] : 0.0);
      n[k] = e->nor[k];
    }
    double dist1_nor, normvel, dt_part, dist2_nor, pos2[3], dist2[3];
    normvel = relvel[0] * n[0] + relvel[1] * n[1] + relvel[2] * n[2];
    if (e->kind == DUST_ELEM_SURFPAN) { /* :2389-2446 */
      dist1_nor = dist1[0] * n[0] + dist1[1] * n[1] + dist1[2] * n[2];
      if (dist1_nor < 0.0 || normvel >= 0.0) continue;
      double t = dist1_nor / (-normvel);
      if (!(t > 0.0)) t = 0.0; /* max(t, 0) */
      dt_part = t < u->dt ? t : u->dt;
      for (int k = 0; k < 3; ++k) {
        pos2[k] = cen[k] + relvel[k] * dt_part;
        dist2[k] = pos2[k] - e->cen[k];
      }
      dist2_nor = dist2[0] * n[0] + dist2[1] * n[1] + dist2[2] * n[2];
    } else { /* vortex ring, :2448-2507 */
      double dn[3] = {dist1[0] * n[0], dist1[1] * n[1], dist1[2] * n[2]};
      dist1_nor = or_norm3(dn);
      const double sdn = dist1[0] * n[0] + dist1[1] * n[1] + dist1[2] * n[2];
      if (sdn * normvel >= 0.0) continue;
      double t = fabs(dist1_nor) / fabs(normvel);
      if (!(t > 0.0)) t = 0.0;
      dt_part = t < u->dt ? t : u->dt;
      for (int k = 0; k < 3; ++k) {
        pos2[k] = cen[k] + relvel[k] * dt_part;
        dist2[k] = pos2[k] - e->cen[k];
      }
      double d2n[3] = {dist2[0] * n[0], dist2[1] * n[1], dist2[2] * n[2]};
      dist2_nor = or_norm3(d2n);
      blthick = 2.0 * blthick;
    }
    if (!(dist2_nor <= blthick)) continue;
    double tv[3];
    for (int k = 0; k < 3; ++k) tv[k] = dist2[k] - n[k] * dist2_nor;
    const double dist2_tan = or_norm3(tv);
    if (!(dist2_tan < elrad_mult * elrad)) continue;
    double normvel_corr;
    if (dt_part < u->dt) {
      normvel_corr = -dist1_nor / (u->dt * nd);
    } else {
      const double dampf = dist2_nor / blthick;
      normvel_corr = normvel + (blthick - dist2_nor) / (u->dt * nd) * dampf;
    }
    double newvel[3], tanvel[3];
    for (int k = 0; k < 3; ++k) newvel[k] = vel[k] + (normvel_corr - normvel) * n[k];
    normvel_corr = newvel[0] * n[0] + newvel[1] * n[1] + newvel[2] * n[2];
    const double nv0 = vel[0] * n[0] + vel[1] * n[1] + vel[2] * n[2];
    for (int k = 0; k < 3; ++k) tanvel[k] = vel[k] - nv0 * n[k];
    const double tanvel2 = tanvel[0] * tanvel[0] + tanvel[1] * tanvel[1] + tanvel[2] * tanvel[2];
    const double nveldiff = nv0 * nv0 - normvel_corr * normvel_corr + tanvel2;
    if (tanvel2 > 0.0 && normvel_corr * nv0 >= 0.0 && nveldiff >= 0.0) {
      const double f = sqrt(nveldiff) / sqrt(tanvel2);
      for (int k = 0; k < 3; ++k) tanvel[k] = tanvel[k] * f;
    }
    for (int k = 0; k < 3; ++k) vel[k] = tanvel[k] + normvel_corr * n[k];
  }
  for (int k = 0; k < 3; ++k) vel_out[k] = vel[k];
}

/* complete_wake's particle loop with use_pa (:1309-1355): avoid_collision
 * on every live particle (its velocity written back), then the update of
 * or_particles_update. */
int or_particles_update_pa(const dust_update_params *u, const dust_pa_params *pa,
                           const dust_panels *elems, int n, double *cen, double *dir,
                           const double *mag, const double *r_vortex, double *vel,
                           double *stretch, const double *rotu, int *free_flag, int *n_freed) {
  if (!u || !pa || !elems || n < 0 || !n_freed) return DUST_ERR_BAD_ARG;
  const int nel = elems->n;
  or_pan_t *el = (or_pan_t *)malloc(sizeof(or_pan_t) * (size_t)(nel + 1));
  for (int j = 0; j < nel; ++j) or_pan_build(elems, j, NULL, &el[j]);
#pragma omp parallel for schedule(dynamic, 64)
  for (int ip = 0; ip < n; ++ip) {
    if (free_flag[ip]) continue;
    double vo[3];
    or_avoid_collision(pa, u, el, elems->ub, nel, cen + 3 * (size_t)ip, r_vortex[ip],
                       vel + 3 * (size_t)ip, vo);
    for (int k = 0; k < 3; ++k) vel[3 * (size_t)ip + k] = vo[k];
  }
  free(el);
  return or_particles_update(u, n, cen, dir, mag, vel, stretch, rotu, free_flag, n_freed);
}
