// elements.cuh -- panel / line influence kernels (device functions).
//
// Device restatement of the reference's influence routines:
//   src/aeroel/mod_doublet.f90   potential_calc_doublet :113-168,
//                                velocity_calc_doublet :178-248
//   src/aeroel/mod_surfpan.f90   potential_calc_sou_surfpan :173-258,
//                                velocity_calc_sou_surfpan :268-357,
//                                calc_geo_data_surfpan :888-951
//   src/aeroel/mod_vortlatt.f90  calc_geo_data_vortlatt :601-669
//   src/aeroel/mod_vortline.f90  compute_vel_vortline :126-170
// The velocity routines return 4*pi times the velocity, as the reference's
// do (the caller divides by 4*pi).
#pragma once

#include "dust_common.cuh"

// Derived geometry of one flat panel, one 8-byte-aligned record per panel
// (AoS: an influence evaluation touches most fields of one panel).
struct PanelGeo {
  double ver[4][3];
  double cen[3], nor[3], tang[2][3];
  double edge_vec[4][3], edge_uni[4][3], edge_len[4];
  double verp[4][3], cosTi[4], sinTi[4];
  double area, max_edge, mag, sig;  // sig = nor.(ub - wind - uvort)
  double sig0;                       // nor.(-wind - uvort) (static RHS columns)
  int nv, kind;
};

struct LineGeo {
  double ver[2][3], edge_uni[3], edge_len, mag;
};

struct RegParams {  // regularisation constants used by the kernels
  double ff_dou;     // far_field_ratio_doublet
  double r_rankine;  // rankine_rad
  double r_cutoff;   // cutoff_rad
};

__host__ __device__ inline double d3dot(const double *a, const double *b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
__host__ __device__ inline void d3cross(const double *a, const double *b, double *r) {
  r[0] = a[1] * b[2] - a[2] * b[1];
  r[1] = a[2] * b[0] - a[0] * b[2];
  r[2] = a[0] * b[1] - a[1] * b[0];
}

// calc_geo_data_surfpan / calc_geo_data_vortlatt from the vertices.
__host__ __device__ inline void panel_build(const double *ver12, int nv, int kind,
                                            double mag, const double *ub,
                                            const double *uvort, const double *u_inf,
                                            PanelGeo &p) {
  p.nv = nv;
  p.kind = kind;
  for (int v = 0; v < 4; ++v)
    for (int d = 0; d < 3; ++d) p.ver[v][d] = ver12[3 * v + d];
  for (int d = 0; d < 3; ++d) {
    double s = 0.0;
    for (int v = 0; v < nv; ++v) s += p.ver[v][d];
    p.cen[d] = s / (double)nv;
  }
  double a[3], b[3], nor[3];
  for (int d = 0; d < 3; ++d) {
    if (nv == 4) {
      a[d] = p.ver[2][d] - p.ver[0][d];
      b[d] = p.ver[3][d] - p.ver[1][d];
    } else {
      a[d] = p.ver[2][d] - p.ver[1][d];
      b[d] = p.ver[0][d] - p.ver[1][d];
    }
  }
  d3cross(a, b, nor);
  double nn = sqrt(d3dot(nor, nor));
  p.area = 0.5 * nn;
  if (kind == DUST_ELEM_VORTLATT && nn < 1e-16) {
    nor[2] = 1e-16;
    nn = sqrt(d3dot(nor, nor));
  }
  for (int d = 0; d < 3; ++d) p.nor[d] = nor[d] / nn;
  double tanl[3];
  for (int d = 0; d < 3; ++d) tanl[d] = 0.5 * (p.ver[nv - 1][d] + p.ver[0][d]) - p.cen[d];
  double tn = sqrt(d3dot(tanl, tanl));
  for (int d = 0; d < 3; ++d) p.tang[0][d] = tanl[d] / tn;
  d3cross(p.nor, p.tang[0], p.tang[1]);
  p.max_edge = 0.0;
  for (int v = 0; v < 4; ++v) {
    if (v < nv) {
      int vn = (v + 1) % nv;
      for (int d = 0; d < 3; ++d) p.edge_vec[v][d] = p.ver[vn][d] - p.ver[v][d];
      p.edge_len[v] = sqrt(d3dot(p.edge_vec[v], p.edge_vec[v]));
      if (v == 0 || p.edge_len[v] > p.max_edge) p.max_edge = p.edge_len[v];
      for (int d = 0; d < 3; ++d) p.edge_uni[v][d] = p.edge_vec[v][d] / p.edge_len[v];
      p.cosTi[v] = d3dot(p.edge_uni[v], p.tang[0]);
      p.sinTi[v] = d3dot(p.edge_uni[v], p.tang[1]);
      double dv[3] = {p.ver[v][0] - p.cen[0], p.ver[v][1] - p.cen[1], p.ver[v][2] - p.cen[2]};
      double pr = d3dot(dv, p.nor);
      for (int d = 0; d < 3; ++d) p.verp[v][d] = p.ver[v][d] - p.nor[d] * pr;
    } else {
      for (int d = 0; d < 3; ++d) p.edge_vec[v][d] = p.edge_uni[v][d] = p.verp[v][d] = 0.0;
      p.edge_len[v] = 1.0;
      p.cosTi[v] = p.sinTi[v] = 0.0;
    }
  }
  p.mag = mag;
  double rel[3], rel0[3];
  for (int d = 0; d < 3; ++d) {
    rel0[d] = -(u_inf ? u_inf[d] : 0.0) - (uvort ? uvort[d] : 0.0);
    rel[d] = (ub ? ub[d] : 0.0) - (u_inf ? u_inf[d] : 0.0) - (uvort ? uvort[d] : 0.0);
  }
  p.sig = d3dot(p.nor, rel);
  p.sig0 = d3dot(p.nor, rel0);
}

__host__ __device__ inline void line_build(const double *ver6, double mag, LineGeo &l) {
  for (int v = 0; v < 2; ++v)
    for (int d = 0; d < 3; ++d) l.ver[v][d] = ver6[3 * v + d];
  double e[3] = {l.ver[1][0] - l.ver[0][0], l.ver[1][1] - l.ver[0][1],
                 l.ver[1][2] - l.ver[0][2]};
  l.edge_len = sqrt(d3dot(e, e));
  for (int d = 0; d < 3; ++d) l.edge_uni[d] = e[d] / l.edge_len;
  l.mag = mag;
}

// potential_calc_doublet: solid angle (per-vertex atan2 + Gauss-Bonnet) or
// far-field dipole.
__device__ inline double pot_dou(const RegParams &rp, const PanelGeo &p, const double *pos) {
  double r[3] = {pos[0] - p.cen[0], pos[1] - p.cen[1], pos[2] - p.cen[2]};
  double radius = sqrt(d3dot(r, r));
  double zQ = d3dot(r, p.nor);
  if (radius > rp.ff_dou * p.max_edge) return zQ * p.area / (radius * radius * radius);
  double dou = 0.0;
  int nv = p.nv;
  for (int i1 = 0; i1 < nv; ++i1) {
    int im1 = (i1 + nv - 1) % nv;
    double ei[3] = {p.ver[i1][0] - pos[0], p.ver[i1][1] - pos[1], p.ver[i1][2] - pos[2]};
    double en = sqrt(d3dot(ei, ei));
    for (int d = 0; d < 3; ++d) ei[d] = ei[d] / en;
    double ep = d3dot(ei, p.edge_vec[i1]), em = d3dot(ei, p.edge_vec[im1]);
    double ap1[3], am1[3];
    for (int d = 0; d < 3; ++d) {
      ap1[d] = p.edge_vec[i1][d] - ei[d] * ep;
      am1[d] = -p.edge_vec[im1][d] + ei[d] * em;
    }
    double ap1n = sqrt(d3dot(ap1, ap1)), am1n = sqrt(d3dot(am1, am1)), cr[3];
    d3cross(am1, ap1, cr);
    double den = ap1n * am1n;
    dou += atan2(d3dot(ei, cr) / den, d3dot(am1, ap1) / den);
  }
  double gb = (double)(nv - 2) * DUST_PI;
  if (dou < -gb + 1.0e-5)
    dou += gb;
  else if (dou > gb - 1.0e-5)
    dou -= gb;
  return dou;
}

// velocity_calc_doublet: vortex ring with Rankine core + cutoff, far field.
__device__ inline void vel_dou(const RegParams &rp, const PanelGeo &p, const double *pos,
                               double *v) {
  double rv[3] = {pos[0] - p.cen[0], pos[1] - p.cen[1], pos[2] - p.cen[2]};
  double r2 = d3dot(rv, rv);
  double radius = sqrt(r2);
  v[0] = v[1] = v[2] = 0.0;
  if (radius > rp.ff_dou * p.max_edge) {
    double rn = d3dot(rv, p.nor);
    double r5 = r2 * r2 * radius;
    double rati = 3.0 * p.area * rn / r5;
    double phix = rati * d3dot(rv, p.tang[0]);
    double phiy = rati * d3dot(rv, p.tang[1]);
    double pdou = p.area * (-r2 + 3.0 * rn * rn) / r5;
    for (int d = 0; d < 3; ++d)
      v[d] = p.tang[0][d] * phix + p.tang[1][d] * phiy + p.nor[d] * pdou;
    return;
  }
  for (int i1 = 0; i1 < p.nv; ++i1) {
    int ip1 = (i1 + 1) % p.nv;
    double av[3] = {pos[0] - p.ver[i1][0], pos[1] - p.ver[i1][1], pos[2] - p.ver[i1][2]};
    double ai = d3dot(av, p.edge_uni[i1]);
    double R1 = sqrt(d3dot(av, av));
    double bv[3] = {pos[0] - p.ver[ip1][0], pos[1] - p.ver[ip1][1], pos[2] - p.ver[ip1][2]};
    double R2 = sqrt(d3dot(bv, bv));
    double hv[3];
    for (int d = 0; d < 3; ++d) hv[d] = av[d] - ai * p.edge_uni[i1][d];
    double hi2 = d3dot(hv, hv);
    double hi = sqrt(hi2), cr[3];
    d3cross(p.edge_uni[i1], hv, cr);
    double L = p.edge_len[i1];
    double f;
    if (hi > L * rp.r_rankine) {
      f = ((L - ai) / R2 + ai / R1) / hi2;
    } else if (R1 > L * rp.r_cutoff && R2 > L * rp.r_cutoff) {
      double rr = rp.r_rankine * L;
      f = ((L - ai) / R2 + ai / R1) / (rr * rr);
    } else {
      continue;
    }
    for (int d = 0; d < 3; ++d) v[d] += f * cr[d];
  }
}

// potential_calc_sou_surfpan (far-field ratio fixed at 10 in the reference).
__device__ inline double pot_sou(const PanelGeo &p, double dou, const double *pos) {
  double r[3] = {pos[0] - p.cen[0], pos[1] - p.cen[1], pos[2] - p.cen[2]};
  double radius = sqrt(d3dot(r, r));
  if (radius > 10.0 * p.max_edge) return p.area / radius;
  double zQ = d3dot(r, p.nor);
  double Qp[3] = {pos[0] - zQ * p.nor[0], pos[1] - zQ * p.nor[1], pos[2] - zQ * p.nor[2]};
  double sou = 0.0;
  for (int i1 = 0; i1 < p.nv; ++i1) {
    int ip1 = (i1 + 1) % p.nv;
    double a[3] = {pos[0] - p.verp[i1][0], pos[1] - p.verp[i1][1], pos[2] - p.verp[i1][2]};
    double b[3] = {pos[0] - p.verp[ip1][0], pos[1] - p.verp[ip1][1],
                   pos[2] - p.verp[ip1][2]};
    double R1 = sqrt(d3dot(a, a)), R2 = sqrt(d3dot(b, b));
    double L = p.edge_len[i1];
    double den = R1 + R2 - L;
    if (den < 1e-6) {
      double a2[3] = {pos[0] - p.ver[i1][0], pos[1] - p.ver[i1][1], pos[2] - p.ver[i1][2]};
      double b2[3] = {pos[0] - p.ver[ip1][0], pos[1] - p.ver[ip1][1],
                      pos[2] - p.ver[ip1][2]};
      R1 = sqrt(d3dot(a2, a2));
      R2 = sqrt(d3dot(b2, b2));
      den = R1 + R2 - L;
    }
    double souLog = log((R1 + R2 + L) / den);
    double q[3] = {Qp[0] - p.verp[i1][0], Qp[1] - p.verp[i1][1], Qp[2] - p.verp[i1][2]};
    double cr[3];
    d3cross(q, p.edge_vec[i1], cr);
    sou += (-d3dot(cr, p.nor) / L) * souLog;
  }
  return sou - zQ * dou;
}

// velocity_calc_sou_surfpan.
__device__ inline void vel_sou(const RegParams &rp, const PanelGeo &p, const double *pos,
                               double *v) {
  double rv[3] = {pos[0] - p.cen[0], pos[1] - p.cen[1], pos[2] - p.cen[2]};
  double radius = sqrt(d3dot(rv, rv));
  double phix, phiy, pdou;
  if (radius > 10.0 * p.max_edge) {
    double r3 = radius * radius * radius;
    phix = -p.area * d3dot(rv, p.tang[0]) / r3;
    phiy = -p.area * d3dot(rv, p.tang[1]) / r3;
    pdou = -p.area * d3dot(rv, p.nor) / r3;
  } else {
    phix = 0.0;
    phiy = 0.0;
    for (int i1 = 0; i1 < p.nv; ++i1) {
      int ip1 = (i1 + 1) % p.nv;
      double a[3] = {pos[0] - p.verp[i1][0], pos[1] - p.verp[i1][1],
                     pos[2] - p.verp[i1][2]};
      double b[3] = {pos[0] - p.verp[ip1][0], pos[1] - p.verp[ip1][1],
                     pos[2] - p.verp[ip1][2]};
      double R1 = sqrt(d3dot(a, a)), R2 = sqrt(d3dot(b, b)), L = p.edge_len[i1];
      double souLog = (R1 + R2 - L < 1e-12) ? 0.0 : log((R1 + R2 + L) / (R1 + R2 - L));
      phix += p.sinTi[i1] * souLog;
      phiy -= p.cosTi[i1] * souLog;
    }
    pdou = pot_dou(rp, p, pos);
    phix = -phix;
    phiy = -phiy;
    pdou = -pdou;
  }
  for (int d = 0; d < 3; ++d)
    v[d] = p.tang[0][d] * phix + p.tang[1][d] * phiy + p.nor[d] * pdou;
}

// compute_vel_vortline (x 4 pi).
__device__ inline void vel_line(const RegParams &rp, const LineGeo &l, const double *pos,
                                double *v) {
  double av[3] = {pos[0] - l.ver[0][0], pos[1] - l.ver[0][1], pos[2] - l.ver[0][2]};
  double ai = d3dot(av, l.edge_uni);
  double R1 = sqrt(d3dot(av, av));
  double bv[3] = {pos[0] - l.ver[1][0], pos[1] - l.ver[1][1], pos[2] - l.ver[1][2]};
  double R2 = sqrt(d3dot(bv, bv));
  double hv[3];
  for (int d = 0; d < 3; ++d) hv[d] = av[d] - ai * l.edge_uni[d];
  double hi2 = d3dot(hv, hv);
  double hi = sqrt(hi2), cr[3];
  d3cross(l.edge_uni, hv, cr);
  double L = l.edge_len, f = 0.0;
  if (hi > L * rp.r_rankine)
    f = ((L - ai) / R2 + ai / R1) / hi2;
  else if (R1 > L * rp.r_cutoff && R2 > L * rp.r_cutoff)
    f = ((L - ai) / R2 + ai / R1) / ((rp.r_rankine * L) * (rp.r_rankine * L));
  for (int d = 0; d < 3; ++d) v[d] = f * cr[d] * l.mag;
}

// compute_vel of a body or wake panel (x 4 pi).
__device__ inline void vel_pan(const RegParams &rp, const PanelGeo &p, const double *pos,
                               double *v) {
  double vd[3];
  vel_dou(rp, p, pos, vd);
  if (p.kind == DUST_ELEM_SURFPAN) {
    double vs[3];
    vel_sou(rp, p, pos, vs);
    for (int d = 0; d < 3; ++d) v[d] = vd[d] * p.mag - vs[d] * p.sig;
  } else {
    for (int d = 0; d < 3; ++d) v[d] = vd[d] * p.mag;
  }
}

// vel_pan for a point inside the panel's far-field radius, with the
// per-vertex quantities shared between the edges: the distances to the
// vertices and to the projected vertices are computed once per vertex (the
// reference's loops recompute each at both of its edges), reciprocal
// distances replace the divisions by them, the solid angle's atan2 takes its
// two arguments unscaled (atan2(y/d, x/d) = atan2(y, x) for d > 0), and the
// Rankine-core test compares squares.  Same branches and formulas as
// vel_pan (vel_dou, vel_sou, pot_dou), equal up to rounding; points beyond
// the far-field radii go to vel_pan.
template <int NV>
__device__ inline void vel_pan_near_t(const RegParams &rp, const PanelGeo &p, const double *pos,
                                      double *v) {
  const double rv[3] = {pos[0] - p.cen[0], pos[1] - p.cen[1], pos[2] - p.cen[2]};
  const double r2 = d3dot(rv, rv);
  const double radius = sqrt(r2);
  const bool sp = p.kind == DUST_ELEM_SURFPAN;
  const bool dou_far = radius > rp.ff_dou * p.max_edge;
  const bool sou_far = radius > 10.0 * p.max_edge;
  if (dou_far && (!sp || sou_far)) {
    vel_pan(rp, p, pos, v);
    return;
  }
  constexpr int nv = NV;
  double dv[NV][3], R[NV], iR[NV];
#pragma unroll
  for (int i = 0; i < nv; ++i) {
    for (int d = 0; d < 3; ++d) dv[i][d] = pos[d] - p.ver[i][d];
    const double q = d3dot(dv[i], dv[i]);
    R[i] = sqrt(q);
    iR[i] = 1.0 / R[i];
  }
  double vd[3] = {0.0, 0.0, 0.0};
  if (dou_far) {
    vel_dou(rp, p, pos, vd);
  } else {
#pragma unroll
    for (int i1 = 0; i1 < nv; ++i1) {
      const int ip1 = i1 + 1 == nv ? 0 : i1 + 1;
      const double *eu = p.edge_uni[i1];
      const double L = p.edge_len[i1];
      const double ai = d3dot(dv[i1], eu);
      double hv[3], cr[3];
      for (int d = 0; d < 3; ++d) hv[d] = dv[i1][d] - ai * eu[d];
      const double hi2 = d3dot(hv, hv);
      d3cross(eu, hv, cr);
      const double rr = rp.r_rankine * L;
      double f;
      if (hi2 > rr * rr) {
        f = ((L - ai) * iR[ip1] + ai * iR[i1]) / hi2;
      } else if (R[i1] > L * rp.r_cutoff && R[ip1] > L * rp.r_cutoff) {
        f = ((L - ai) * iR[ip1] + ai * iR[i1]) / (rr * rr);
      } else {
        continue;
      }
      for (int d = 0; d < 3; ++d) vd[d] += f * cr[d];
    }
  }
  if (!sp) {
    for (int d = 0; d < 3; ++d) v[d] = vd[d] * p.mag;
    return;
  }
  double vs[3];
  if (sou_far) {
    vel_sou(rp, p, pos, vs);
  } else {
    double Rp[NV];
#pragma unroll
    for (int i = 0; i < nv; ++i) {
      const double a[3] = {pos[0] - p.verp[i][0], pos[1] - p.verp[i][1], pos[2] - p.verp[i][2]};
      Rp[i] = sqrt(d3dot(a, a));
    }
    double phix = 0.0, phiy = 0.0;
#pragma unroll
    for (int i1 = 0; i1 < nv; ++i1) {
      const int ip1 = i1 + 1 == nv ? 0 : i1 + 1;
      const double L = p.edge_len[i1], s = Rp[i1] + Rp[ip1];
      const double souLog = (s - L < 1e-12) ? 0.0 : log((s + L) / (s - L));
      phix += p.sinTi[i1] * souLog;
      phiy -= p.cosTi[i1] * souLog;
    }
    double pdou;
    if (dou_far) {
      pdou = d3dot(rv, p.nor) * p.area / (radius * radius * radius);
    } else {
      double dou = 0.0;
#pragma unroll
    for (int i1 = 0; i1 < nv; ++i1) {
        const int im1 = i1 == 0 ? nv - 1 : i1 - 1;
        double ei[3], ap1[3], am1[3], cr[3];
        for (int d = 0; d < 3; ++d) ei[d] = -dv[i1][d] * iR[i1];
        const double ep = d3dot(ei, p.edge_vec[i1]), em = d3dot(ei, p.edge_vec[im1]);
        for (int d = 0; d < 3; ++d) {
          ap1[d] = p.edge_vec[i1][d] - ei[d] * ep;
          am1[d] = -p.edge_vec[im1][d] + ei[d] * em;
        }
        d3cross(am1, ap1, cr);
        dou += atan2(d3dot(ei, cr), d3dot(am1, ap1));
      }
      const double gb = (double)(nv - 2) * DUST_PI;
      if (dou < -gb + 1.0e-5)
        dou += gb;
      else if (dou > gb - 1.0e-5)
        dou -= gb;
      pdou = dou;
    }
    for (int d = 0; d < 3; ++d)
      vs[d] = -(p.tang[0][d] * phix + p.tang[1][d] * phiy + p.nor[d] * pdou);
  }
  for (int d = 0; d < 3; ++d) v[d] = vd[d] * p.mag - vs[d] * p.sig;
}

__device__ inline void vel_pan_near(const RegParams &rp, const PanelGeo &p, const double *pos,
                                    double *v) {
  if (p.nv == 4)
    vel_pan_near_t<4>(rp, p, pos, v);
  else
    vel_pan_near_t<3>(rp, p, pos, v);
}
