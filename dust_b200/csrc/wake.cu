// wake.cu -- the particles' explicit Euler step of complete_wake
// (src/aeroel/mod_wake.f90:1309-1355): move, cull outside the particle box,
// divergence filtering of the stretching term and the update of the
// particle direction, optionally after penetration avoidance (avoid_collision,
// :2350-2534).  One thread per particle; the arithmetic follows the
// reference's expressions operation by operation with explicitly rounded
// intrinsics (no fused multiply-adds), so the result equals a plain FP64
// evaluation of the same expressions, as the CPU oracle writes them.  The
// reference takes vector lengths with Fortran's norm2, which gfortran may
// evaluate as a scaled sum of squares; here (and in the oracle) the length
// is sqrt(x*x + y*y + z*z), which can differ from that in the last unit of
// the result.
#include <algorithm>
#include <cstring>

#include "dust_common.cuh"
#include "fmm_internal.h"

static inline unsigned nblk(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

__device__ __forceinline__ double norm3(double x, double y, double z) {
  return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
}

// the move, culling and direction update of one live particle (:1320-1352)
__device__ __forceinline__ void particle_step(const dust_update_params &u, int i, double *cen,
                                              double *dir, const double *mag,
                                              const double *vel, double *str,
                                              const double *rotu, int *free_flag,
                                              int *n_freed) {
  const double nd = (double)u.ndt_update_wake;
  // pos_p = cen + vel * dt * ndt, kept if inside the box  (:1321-1326)
  double p[3];
  bool in = true;
  for (int c = 0; c < 3; ++c) {
    p[c] = __dadd_rn(cen[3 * (size_t)i + c], __dmul_rn(__dmul_rn(vel[3 * (size_t)i + c], u.dt), nd));
    in = in && p[c] >= u.box_min[c] && p[c] <= u.box_max[c];
  }
  if (!in) {
    // outside the particle box: the slot is freed (:1347-1351)
    free_flag[i] = 1;
    atomicAdd(n_freed, 1);
    return;
  }
  for (int c = 0; c < 3; ++c) cen[3 * (size_t)i + c] = p[c];
  if (!(u.vortstretch || u.diffusion)) return;
  const double m = mag[i];
  double d[3], s[3];
  for (int c = 0; c < 3; ++c) {
    d[c] = dir[3 * (size_t)i + c];
    s[c] = str[3 * (size_t)i + c];
  }
  if (u.divergence_filtering) {
    // stretch -= filt_eta / ndt * (dir mag - rotu mag / |rotu|)  (:1331-1334)
    const double *r = rotu + 3 * (size_t)i;
    const double nr = norm3(r[0], r[1], r[2]);
    const double k = __ddiv_rn(u.filt_eta, nd);
    for (int c = 0; c < 3; ++c) {
      const double in_c = __dsub_rn(__dmul_rn(d[c], m), __ddiv_rn(__dmul_rn(r[c], m), nr));
      s[c] = __dsub_rn(s[c], __dmul_rn(k, in_c));
      str[3 * (size_t)i + c] = s[c];
    }
  }
  // alpha = dir mag + stretch dt ndt; dir = alpha / |alpha|  (:1337-1345)
  double a[3];
  for (int c = 0; c < 3; ++c)
    a[c] = __dadd_rn(__dmul_rn(d[c], m), __dmul_rn(__dmul_rn(s[c], u.dt), nd));
  const double an = norm3(a[0], a[1], a[2]);
  if (an != 0.0)
    for (int c = 0; c < 3; ++c) dir[3 * (size_t)i + c] = __ddiv_rn(a[c], an);
}

__global__ void k_particles_update(dust_update_params u, int n, double *cen, double *dir,
                                   const double *mag, const double *vel, double *str,
                                   const double *rotu, int *free_flag, int *n_freed) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || free_flag[i]) return;
  particle_step(u, i, cen, dir, mag, vel, str, rotu, free_flag, n_freed);
}

// ------------------------------------------------- penetration avoidance
// One element's record for avoid_collision: centre, unit normal and the
// largest edge of calc_geo_data (mod_surfpan.f90:888-951,
// mod_vortlatt.f90:601-669) in the operation order of the CPU oracle's panel
// set-up, the body velocity ub and the kind.
struct PaRec {
  double cen[3], nor[3], ub[3], elrad;
  int kind, pad;
};

__global__ void k_pa_records(int n, const int *n_ver, const int *kind, const double *ver,
                             const double *ub, PaRec *out) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const double *v = ver + 12 * (size_t)j;
  const int nv = n_ver ? n_ver[j] : 4;
  PaRec r;
  r.kind = kind ? kind[j] : DUST_ELEM_VORTLATT;
  r.pad = 0;
  for (int d = 0; d < 3; ++d) {
    double s = 0.0;
    for (int k = 0; k < nv; ++k) s = __dadd_rn(s, v[3 * k + d]);
    r.cen[d] = __ddiv_rn(s, (double)nv);
  }
  double a[3], b[3];
  for (int d = 0; d < 3; ++d) {
    if (nv == 4) {
      a[d] = __dsub_rn(v[6 + d], v[d]);
      b[d] = __dsub_rn(v[9 + d], v[3 + d]);
    } else {
      a[d] = __dsub_rn(v[6 + d], v[3 + d]);
      b[d] = __dsub_rn(v[d], v[3 + d]);
    }
  }
  double nr[3] = {__dsub_rn(__dmul_rn(a[1], b[2]), __dmul_rn(a[2], b[1])),
                  __dsub_rn(__dmul_rn(a[2], b[0]), __dmul_rn(a[0], b[2])),
                  __dsub_rn(__dmul_rn(a[0], b[1]), __dmul_rn(a[1], b[0]))};
  if (r.kind == DUST_ELEM_VORTLATT && norm3(nr[0], nr[1], nr[2]) < 1e-16) nr[2] = 1e-16;
  const double nn = norm3(nr[0], nr[1], nr[2]);
  for (int d = 0; d < 3; ++d) r.nor[d] = __ddiv_rn(nr[d], nn);
  double mx = 0.0;
  for (int k = 0; k < nv; ++k) {
    const int k1 = (k + 1) % nv;
    const double e0 = __dsub_rn(v[3 * k1], v[3 * k]), e1 = __dsub_rn(v[3 * k1 + 1], v[3 * k + 1]),
                 e2 = __dsub_rn(v[3 * k1 + 2], v[3 * k + 2]);
    const double el = norm3(e0, e1, e2);
    if (k == 0 || el > mx) mx = el;
  }
  r.elrad = __dmul_rn(mx, __ddiv_rn(__dsqrt_rn(2.0), 2.0));
  for (int d = 0; d < 3; ++d) r.ub[d] = ub ? ub[3 * (size_t)j + d] : 0.0;
  out[j] = r;
}

#define PA_T 128
#define PA_TILE 64
// avoid_collision (:2350-2534) against every element in order, then the
// Euler step.  Element records are staged through shared memory a tile at a
// time; every thread walks the tile in the same order (broadcast reads).
__global__ void __launch_bounds__(PA_T) k_particles_update_pa(
    dust_update_params u, dust_pa_params pa, int nel, const PaRec *__restrict__ el, int n,
    double *cen, double *dir, const double *mag, const double *rvort, double *vel, double *str,
    const double *rotu, int *free_flag, int *n_freed) {
  __shared__ PaRec s_el[PA_TILE];
  const int i = blockIdx.x * PA_T + threadIdx.x;
  const bool act = i < n && !free_flag[i];
  const double nd = (double)u.ndt_update_wake;
  const double dtnd = __dmul_rn(u.dt, nd);
  double pos1[3] = {0, 0, 0}, v[3] = {0, 0, 0}, blthick = 0.0;
  if (act) {
    for (int c = 0; c < 3; ++c) {
      pos1[c] = cen[3 * (size_t)i + c];
      v[c] = vel[3 * (size_t)i + c];
    }
    blthick = rvort[i];  // :2377
  }
  const double cr0 = __dmul_rn(__dmul_rn(u.dt, pa.u_ref), pa.check_radius);
  for (int t0 = 0; t0 < nel; t0 += PA_TILE) {
    __syncthreads();
    const int m = min(PA_TILE, nel - t0);
    const int words = sizeof(PaRec) / 8;
    for (int w = threadIdx.x; w < m * words; w += PA_T)
      ((double *)s_el)[w] = ((const double *)(el + t0))[w];
    __syncthreads();
    if (!act) continue;
    for (int q = 0; q < m; ++q) {
      const PaRec &e = s_el[q];
      double d1[3];
      for (int c = 0; c < 3; ++c) d1[c] = __dsub_rn(pos1[c], e.cen[c]);
      const double check_radius = __dadd_rn(cr0, e.elrad);
      const double distn = norm3(d1[0], d1[1], d1[2]);
      if (!(distn < check_radius)) continue;
      const double *nn = e.nor;
      double rv[3];
      for (int c = 0; c < 3; ++c) rv[c] = __dsub_rn(v[c], e.ub[c]);
      const double normvel =
          __dadd_rn(__dadd_rn(__dmul_rn(rv[0], nn[0]), __dmul_rn(rv[1], nn[1])), __dmul_rn(rv[2], nn[2]));
      double dist1_nor, dt_part, dist2_nor, d2[3];
      if (e.kind == DUST_ELEM_SURFPAN) {  // :2389-2446
        dist1_nor = __dadd_rn(__dadd_rn(__dmul_rn(d1[0], nn[0]), __dmul_rn(d1[1], nn[1])),
                              __dmul_rn(d1[2], nn[2]));
        if (dist1_nor < 0.0 || normvel >= 0.0) continue;
        double tt = __ddiv_rn(dist1_nor, -normvel);
        if (!(tt > 0.0)) tt = 0.0;
        dt_part = tt < u.dt ? tt : u.dt;
        for (int c = 0; c < 3; ++c)
          d2[c] = __dsub_rn(__dadd_rn(pos1[c], __dmul_rn(rv[c], dt_part)), e.cen[c]);
        dist2_nor = __dadd_rn(__dadd_rn(__dmul_rn(d2[0], nn[0]), __dmul_rn(d2[1], nn[1])),
                              __dmul_rn(d2[2], nn[2]));
      } else {  // vortex ring, :2448-2507
        dist1_nor = norm3(__dmul_rn(d1[0], nn[0]), __dmul_rn(d1[1], nn[1]), __dmul_rn(d1[2], nn[2]));
        const double sdn = __dadd_rn(__dadd_rn(__dmul_rn(d1[0], nn[0]), __dmul_rn(d1[1], nn[1])),
                                     __dmul_rn(d1[2], nn[2]));
        if (__dmul_rn(sdn, normvel) >= 0.0) continue;
        double tt = __ddiv_rn(fabs(dist1_nor), fabs(normvel));
        if (!(tt > 0.0)) tt = 0.0;
        dt_part = tt < u.dt ? tt : u.dt;
        for (int c = 0; c < 3; ++c)
          d2[c] = __dsub_rn(__dadd_rn(pos1[c], __dmul_rn(rv[c], dt_part)), e.cen[c]);
        dist2_nor = norm3(__dmul_rn(d2[0], nn[0]), __dmul_rn(d2[1], nn[1]), __dmul_rn(d2[2], nn[2]));
        blthick = __dmul_rn(2.0, blthick);
      }
      if (!(dist2_nor <= blthick)) continue;
      const double dist2_tan = norm3(__dsub_rn(d2[0], __dmul_rn(nn[0], dist2_nor)),
                                     __dsub_rn(d2[1], __dmul_rn(nn[1], dist2_nor)),
                                     __dsub_rn(d2[2], __dmul_rn(nn[2], dist2_nor)));
      if (!(dist2_tan < __dmul_rn(pa.element_radius, e.elrad))) continue;
      double nvc;
      if (dt_part < u.dt) {
        nvc = __ddiv_rn(-dist1_nor, dtnd);
      } else {
        const double dampf = __ddiv_rn(dist2_nor, blthick);
        nvc = __dadd_rn(normvel, __dmul_rn(__ddiv_rn(__dsub_rn(blthick, dist2_nor), dtnd), dampf));
      }
      double nw[3], tv[3];
      for (int c = 0; c < 3; ++c) nw[c] = __dadd_rn(v[c], __dmul_rn(__dsub_rn(nvc, normvel), nn[c]));
      nvc = __dadd_rn(__dadd_rn(__dmul_rn(nw[0], nn[0]), __dmul_rn(nw[1], nn[1])), __dmul_rn(nw[2], nn[2]));
      const double nv0 =
          __dadd_rn(__dadd_rn(__dmul_rn(v[0], nn[0]), __dmul_rn(v[1], nn[1])), __dmul_rn(v[2], nn[2]));
      for (int c = 0; c < 3; ++c) tv[c] = __dsub_rn(v[c], __dmul_rn(nv0, nn[c]));
      const double tv2 =
          __dadd_rn(__dadd_rn(__dmul_rn(tv[0], tv[0]), __dmul_rn(tv[1], tv[1])), __dmul_rn(tv[2], tv[2]));
      const double nvd = __dadd_rn(__dsub_rn(__dmul_rn(nv0, nv0), __dmul_rn(nvc, nvc)), tv2);
      if (tv2 > 0.0 && __dmul_rn(nvc, nv0) >= 0.0 && nvd >= 0.0) {
        const double f = __ddiv_rn(__dsqrt_rn(nvd), __dsqrt_rn(tv2));
        for (int c = 0; c < 3; ++c) tv[c] = __dmul_rn(tv[c], f);
      }
      for (int c = 0; c < 3; ++c) v[c] = __dadd_rn(tv[c], __dmul_rn(nvc, nn[c]));
    }
  }
  if (!act) return;
  for (int c = 0; c < 3; ++c) vel[3 * (size_t)i + c] = v[c];
  particle_step(u, i, cen, dir, mag, vel, str, rotu, free_flag, n_freed);
}

static int update_args_ok(const dust_update_params *u, int n, const void *cen, const void *dir,
                          const void *mag, const void *vel, const void *str, const void *rotu,
                          const void *free_flag, const void *n_freed) {
  if (!u || n < 0 || !n_freed) return 0;
  if (n > 0 && (!cen || !dir || !mag || !vel || !str || !free_flag)) return 0;
  if (n > 0 && u->divergence_filtering && (u->vortstretch || u->diffusion) && !rotu) return 0;
  if (u->ndt_update_wake == 0) return 0;
  return 1;
}

extern "C" int dust_particles_update_device(const dust_update_params *u, int n, double *cen,
                                            double *dir, const double *mag, const double *vel,
                                            double *stretch, const double *rotu,
                                            int *free_flag, int *n_freed, void *stream) {
  if (!update_args_ok(u, n, cen, dir, mag, vel, stretch, rotu, free_flag, n_freed))
    return DUST_ERR_BAD_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  DUST_CUDA(cudaMemsetAsync(n_freed, 0, sizeof(int), st));
  if (n > 0)
    k_particles_update<<<nblk((size_t)n, 256), 256, 0, st>>>(*u, n, cen, dir, mag, vel, stretch,
                                                              rotu, free_flag, n_freed);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}

static DevBuf g_pa_rec;  // element records of the penetration-avoidance entry point

extern "C" int dust_particles_update_pa_device(const dust_update_params *u,
                                               const dust_pa_params *pa,
                                               const dust_panels *elems, int n, double *cen,
                                               double *dir, const double *mag,
                                               const double *r_vortex, double *vel,
                                               double *stretch, const double *rotu,
                                               int *free_flag, int *n_freed, void *stream) {
  if (!update_args_ok(u, n, cen, dir, mag, vel, stretch, rotu, free_flag, n_freed) || !pa ||
      !elems || elems->n < 0 || (elems->n > 0 && !elems->ver) || (n > 0 && !r_vortex))
    return DUST_ERR_BAD_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const int nel = elems->n;
  DUST_TRY(devbuf_grow(g_pa_rec, sizeof(PaRec) * (size_t)std::max(nel, 1)));
  PaRec *rec = (PaRec *)g_pa_rec.p;
  if (nel > 0)
    k_pa_records<<<nblk((size_t)nel, 128), 128, 0, st>>>(nel, elems->n_ver, elems->kind,
                                                         elems->ver, elems->ub, rec);
  DUST_CUDA(cudaMemsetAsync(n_freed, 0, sizeof(int), st));
  if (n > 0)
    k_particles_update_pa<<<nblk((size_t)n, PA_T), PA_T, 0, st>>>(
        *u, *pa, nel, rec, n, cen, dir, mag, r_vortex, vel, stretch, rotu, free_flag, n_freed);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}

extern "C" int dust_particles_update(const dust_update_params *u, int n, double *cen,
                                     double *dir, const double *mag, const double *vel,
                                     double *stretch, const double *rotu, int *free_flag,
                                     int *n_freed) {
  if (!update_args_ok(u, n, cen, dir, mag, vel, stretch, rotu, free_flag, n_freed))
    return DUST_ERR_BAD_ARG;
  if (n == 0) {
    *n_freed = 0;
    return DUST_OK;
  }
  const bool want_rot = u->divergence_filtering && (u->vortstretch || u->diffusion);
  const size_t v3 = (size_t)n * 3 * sizeof(double), v1 = (size_t)n * sizeof(double);
  // one device block: cen, dir, vel, stretch, rotu (3 n each), mag (n),
  // free flags (n ints), the counter
  const size_t bytes = 5 * v3 + v1 + (size_t)n * sizeof(int) + 256;
  // kept across calls (one host thread), so a step loop allocates nothing
  static DevBuf stage;
  DUST_TRY(devbuf_grow(stage, bytes));
  char *b = (char *)stage.p;
  double *dc = (double *)b, *dd = (double *)(b + v3), *dv = (double *)(b + 2 * v3),
         *ds = (double *)(b + 3 * v3), *dr = (double *)(b + 4 * v3), *dm = (double *)(b + 5 * v3);
  int *df = (int *)(b + 5 * v3 + v1);
  int *dn = (int *)(((uintptr_t)(df + n) + 15) & ~(uintptr_t)15);
  cudaStream_t st = 0;
  int s = DUST_OK;
  if (cudaMemcpyAsync(dc, cen, v3, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(dd, dir, v3, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(dv, vel, v3, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(ds, stretch, v3, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      (want_rot && cudaMemcpyAsync(dr, rotu, v3, cudaMemcpyHostToDevice, st) != cudaSuccess) ||
      cudaMemcpyAsync(dm, mag, v1, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(df, free_flag, (size_t)n * sizeof(int), cudaMemcpyHostToDevice, st) !=
          cudaSuccess)
    s = DUST_ERR_CUDA;
  if (s == DUST_OK)
    s = dust_particles_update_device(u, n, dc, dd, dm, dv, ds, want_rot ? dr : nullptr, df, dn,
                                     st);
  if (s == DUST_OK &&
      (cudaMemcpyAsync(cen, dc, v3, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
       cudaMemcpyAsync(dir, dd, v3, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
       cudaMemcpyAsync(stretch, ds, v3, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
       cudaMemcpyAsync(free_flag, df, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, st) !=
           cudaSuccess ||
       cudaMemcpyAsync(n_freed, dn, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
       cudaStreamSynchronize(st) != cudaSuccess))
    s = DUST_ERR_CUDA;
  if (s == DUST_ERR_CUDA) dust_set_last_error("particle update copies", __FILE__, __LINE__);
  return s;
}
