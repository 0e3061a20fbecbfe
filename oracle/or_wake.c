/*
 * or_wake.c -- oracle (test infrastructure): the particle loop of
 * complete_wake, src/aeroel/mod_wake.f90:1309-1355, in plain C (FP64,
 * built with -ffp-contract=off: every product and sum rounded on its own, in
 * the reference's left-to-right order).  Penetration avoidance (use_pa,
 * :1313-1318, off by default) is not restated.  norm2 is restated as the
 * square root of the sum of squares.
 */
#include <math.h>

#include "dust_oracle.h"

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
