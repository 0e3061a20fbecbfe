/* or_internal.h -- oracle internals (test infrastructure only). */
#ifndef OR_INTERNAL_H
#define OR_INTERNAL_H

#include "dust_oracle.h"

/* pi = 4*atan(1) (src/general/mod_param.f90:92) */
#define OR_PI 3.14159265358979323846

/* A panel with the derived data of calc_geo_data_surfpan
 * (mod_surfpan.f90:888-951) / calc_geo_data_vortlatt (mod_vortlatt.f90:
 * 601-669). */
typedef struct {
  int nv, kind;
  double ver[4][3], cen[3], nor[3], tang[2][3];
  double edge_vec[4][3], edge_len[4], edge_uni[4][3], area, max_edge;
  double verp[4][3], cosTi[4], sinTi[4];
  double mag;
  double sig; /* nor . (ub - wind - uvort): surface-panel source strength */
} or_pan_t;

typedef struct {
  double ver[2][3], cen[3], edge_vec[3], edge_len, edge_uni[3], mag;
} or_line_t;

typedef struct {
  int nbody, nwake, nline;
  or_pan_t *body, *wake;
  or_line_t *line;
  double u_inf[3];
} or_elemctx;

void or_pan_build(const dust_panels *pan, int j, const double *u_inf,
                  or_pan_t *out);
void or_line_build(const dust_lines *ln, int j, or_line_t *out);
or_elemctx *or_elemctx_build(const dust_elements *el, const double *u_inf);
void or_elemctx_free(or_elemctx *c);

double or_pot_dou(const dust_fmm_params *prm, const or_pan_t *p, const double *pos);
void or_vel_dou(const dust_fmm_params *prm, const or_pan_t *p, const double *pos,
                double *v);
double or_pot_sou(const or_pan_t *p, double dou, const double *pos);
void or_vel_sou(const dust_fmm_params *prm, const or_pan_t *p, const double *pos,
                double *v);
void or_vel_line(const dust_fmm_params *prm, const or_line_t *l, const double *pos,
                 double *v);
/* compute_vel of a body/wake panel (x 4 pi) */
void or_vel_pan(const dust_fmm_params *prm, const or_pan_t *p, const double *pos,
                double *v);

/* vel += sum over elements of compute_vel/(4 pi), then vel += u_inf, in the
 * order of apply_multipole (mod_octree.f90:1350-1373) */
void or_elements_vel_accum(const dust_fmm_params *prm, const or_elemctx *c,
                           const double *pos, double *vel);

#endif
