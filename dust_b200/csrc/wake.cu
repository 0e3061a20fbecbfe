// wake.cu -- the particles' explicit Euler step of complete_wake
// (src/aeroel/mod_wake.f90:1309-1355): move, cull outside the particle box,
// divergence filtering of the stretching term and the update of the
// particle direction.  One thread per particle; the arithmetic follows the
// reference's expressions operation by operation with explicitly rounded
// intrinsics (no fused multiply-adds), so the result equals a plain FP64
// evaluation of the same expressions, as the CPU oracle writes them.  The
// reference takes vector lengths with Fortran's norm2, which gfortran may
// evaluate as a scaled sum of squares; here (and in the oracle) the length
// is sqrt(x*x + y*y + z*z), which can differ from that in the last unit of
// the result.  Penetration avoidance (use_pa, :1312-1317) is not part of
// this step.
#include <cstring>

#include "dust_common.cuh"

static inline unsigned nblk(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

__device__ __forceinline__ double norm3(double x, double y, double z) {
  return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
}

__global__ void k_particles_update(dust_update_params u, int n, double *cen, double *dir,
                                   const double *mag, const double *vel, double *str,
                                   const double *rotu, int *free_flag, int *n_freed) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || free_flag[i]) return;
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
  char *b = nullptr;
  DUST_CUDA(cudaMalloc((void **)&b, bytes));
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
  cudaFree(b);
  return s;
}
