// capi.cu -- extern "C" entry points of the FMM path and library utilities.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "dust_common.cuh"
#include "fmm_internal.h"

static std::mutex g_err_mu;
static std::string g_err;

void dust_set_last_error(const char *msg, const char *file, int line) {
  std::lock_guard<std::mutex> lk(g_err_mu);
  char buf[512];
  snprintf(buf, sizeof(buf), "%s (%s:%d)", msg ? msg : "?", file, line);
  g_err = buf;
}

extern "C" const char *dust_last_error(void) {
  std::lock_guard<std::mutex> lk(g_err_mu);
  return g_err.c_str();
}

extern "C" const char *dust_status_string(int s) {
  switch (s) {
    case DUST_OK: return "ok";
    case DUST_ERR_CUDA: return "CUDA error";
    case DUST_ERR_OUT_OF_BOX: return "particle outside the octree box";
    case DUST_ERR_SINGULAR: return "singular matrix (zero pivot)";
    case DUST_ERR_NOT_CONVERGED: return "iterative solve did not converge";
    case DUST_ERR_TIMEOUT: return "bounded device wait timed out";
    case DUST_ERR_BAD_ARG: return "invalid argument";
    case DUST_ERR_NO_DEVICE: return "no usable CUDA device";
    case DUST_ERR_CAPACITY: return "size above the supported maximum";
    default: return "unknown status";
  }
}

extern "C" int dust_device_ok(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return DUST_ERR_NO_DEVICE;
  cudaDeviceProp p;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return DUST_ERR_NO_DEVICE;
  if (cudaGetDeviceProperties(&p, dev) != cudaSuccess) return DUST_ERR_NO_DEVICE;
  if (p.major != 10) return DUST_ERR_NO_DEVICE;
  return DUST_OK;
}

// Sizes of the ABI structs, for binding checks.
extern "C" int dust_abi_sizes(int64_t *out, int n) {
  int64_t s[] = {(int64_t)sizeof(dust_fmm_params), (int64_t)sizeof(dust_panels),
                 (int64_t)sizeof(dust_lines),      (int64_t)sizeof(dust_elements),
                 (int64_t)sizeof(dust_fmm_stats),  (int64_t)sizeof(dust_solve_report),
                 (int64_t)sizeof(dust_wake_rows),  (int64_t)sizeof(dust_update_params),
                 (int64_t)sizeof(dust_pa_params),  (int64_t)sizeof(dust_wake_params),
                 (int64_t)sizeof(dust_te)};
  int m = (int)(sizeof(s) / sizeof(s[0]));
  for (int i = 0; i < n && i < m; ++i) out[i] = s[i];
  return m;
}

static int64_t n_elem_of(const dust_elements *e) {
  if (!e) return 0;
  return (int64_t)e->body.n + e->wake.n + e->end_vort.n;
}

extern "C" int dust_fmm_apply(dust_octree *o, int n, const double *cen, const double *dir,
                              const double *mag, const double *r_vortex,
                              const dust_elements *elems, double *vel, double *stretch,
                              double *rotu) {
  if (!o || n < 0 || (n > 0 && (!cen || !dir || !mag || !r_vortex || !vel)))
    return DUST_ERR_BAD_ARG;
  cudaStream_t st = o->stream;
  size_t N = (size_t)(n > 0 ? n : 1);
  DUST_TRY(devbuf_grow(o->h_in, N * 8 * 8));
  DUST_TRY(devbuf_grow(o->h_out, N * 9 * 8));
  double *dc = (double *)o->h_in.p, *dd = dc + 3 * N, *dm = dd + 3 * N, *dr = dm + N;
  double *ov = (double *)o->h_out.p, *os = ov + 3 * N, *orr = os + 3 * N;
  if (n > 0) {
    DUST_CUDA(cudaMemcpyAsync(dc, cen, (size_t)n * 24, cudaMemcpyHostToDevice, st));
    DUST_CUDA(cudaMemcpyAsync(dd, dir, (size_t)n * 24, cudaMemcpyHostToDevice, st));
    DUST_CUDA(cudaMemcpyAsync(dm, mag, (size_t)n * 8, cudaMemcpyHostToDevice, st));
    DUST_CUDA(cudaMemcpyAsync(dr, r_vortex, (size_t)n * 8, cudaMemcpyHostToDevice, st));
  }
  ElemDev e;
  DUST_TRY(elem_build_device(elems ? &elems->body : nullptr, elems ? &elems->wake : nullptr,
                             elems ? &elems->end_vort : nullptr, o->prm.u_inf,
                             reg_params(&o->prm), true, o->el_raw, o->el_geo, e, st));
  DUST_TRY(fmm_run_device(o, n, dc, dd, dm, dr, st));
  DUST_TRY(fmm_finish_device(o, n, e, ov, stretch ? os : nullptr, rotu ? orr : nullptr, st));
  if (n > 0) {
    DUST_CUDA(cudaMemcpyAsync(vel, ov, (size_t)n * 24, cudaMemcpyDeviceToHost, st));
    if (stretch)
      DUST_CUDA(cudaMemcpyAsync(stretch, os, (size_t)n * 24, cudaMemcpyDeviceToHost, st));
    if (rotu) DUST_CUDA(cudaMemcpyAsync(rotu, orr, (size_t)n * 24, cudaMemcpyDeviceToHost, st));
  }
  DUST_CUDA(cudaStreamSynchronize(st));
  return fmm_collect_stats(o, n, n_elem_of(elems));
}

extern "C" int dust_fmm_apply_device(dust_octree *o, int n, const double *cen,
                                     const double *dir, const double *mag,
                                     const double *r_vortex, const dust_elements *elems,
                                     double *vel, double *stretch, double *rotu, void *stream,
                                     int sync) {
  if (!o || n < 0 || (n > 0 && (!cen || !dir || !mag || !r_vortex || !vel)))
    return DUST_ERR_BAD_ARG;
  cudaStream_t st = stream ? (cudaStream_t)stream : o->stream;
  ElemDev e;
  DUST_TRY(elem_build_device(elems ? &elems->body : nullptr, elems ? &elems->wake : nullptr,
                             elems ? &elems->end_vort : nullptr, o->prm.u_inf,
                             reg_params(&o->prm), false, o->el_raw, o->el_geo, e, st));
  DUST_TRY(fmm_run_device(o, n, cen, dir, mag, r_vortex, st));
  DUST_TRY(fmm_finish_device(o, n, e, vel, stretch, rotu, st));
  if (sync) DUST_CUDA(cudaStreamSynchronize(st));
  if (o->timing || sync) return fmm_collect_stats(o, n, n_elem_of(elems));
  return DUST_OK;
}

// ------------------------------------------------ the FMM in two halves
// prepare_wake's octree part (sort_particles + calculate_multipole,
// mod_wake.f90:797-800) and apply_multipole_panels (:801), then
// update_wake's apply_multipole (:1115-1118): the particles enter the tree
// once per step and serve both the panels' uvort and the particles' own
// velocities.

extern "C" int dust_fmm_prepare(dust_octree *o, int n, const double *cen, const double *dir,
                                const double *mag, const double *r_vortex, int n_pts,
                                const double *pts) {
  if (!o || n < 0 || n_pts < 0 || (n > 0 && (!cen || !dir || !mag || !r_vortex)) ||
      (n_pts > 0 && !pts))
    return DUST_ERR_BAD_ARG;
  cudaStream_t st = o->stream;
  size_t N = (size_t)(n > 0 ? n : 1);
  DUST_TRY(devbuf_grow(o->h_in, N * 8 * 8));
  DUST_TRY(devbuf_grow(o->h_pts, (size_t)std::max(n_pts, 1) * 24));
  double *dc = (double *)o->h_in.p, *dd = dc + 3 * N, *dm = dd + 3 * N, *dr = dm + N;
  if (n > 0) {
    DUST_CUDA(cudaMemcpyAsync(dc, cen, (size_t)n * 24, cudaMemcpyHostToDevice, st));
    DUST_CUDA(cudaMemcpyAsync(dd, dir, (size_t)n * 24, cudaMemcpyHostToDevice, st));
    DUST_CUDA(cudaMemcpyAsync(dm, mag, (size_t)n * 8, cudaMemcpyHostToDevice, st));
    DUST_CUDA(cudaMemcpyAsync(dr, r_vortex, (size_t)n * 8, cudaMemcpyHostToDevice, st));
  }
  if (n_pts > 0)
    DUST_CUDA(cudaMemcpyAsync(o->h_pts.p, pts, (size_t)n_pts * 24, cudaMemcpyHostToDevice, st));
  o->prepared_n = -1;
  const int s = fmm_prepare_device(o, n, dc, dd, dm, dr, n_pts, (const double *)o->h_pts.p, st);
  if (s != DUST_OK) o->prepared_n = -1;
  return s;
}

extern "C" int dust_fmm_prepare_device(dust_octree *o, int n, const double *cen,
                                       const double *dir, const double *mag,
                                       const double *r_vortex, int n_pts, const double *pts,
                                       void *stream) {
  if (!o || n < 0 || n_pts < 0 || (n > 0 && (!cen || !dir || !mag || !r_vortex)) ||
      (n_pts > 0 && !pts))
    return DUST_ERR_BAD_ARG;
  cudaStream_t st = stream ? (cudaStream_t)stream : o->stream;
  DUST_TRY(devbuf_grow(o->h_pts, (size_t)std::max(n_pts, 1) * 24));
  if (n_pts > 0)
    DUST_CUDA(cudaMemcpyAsync(o->h_pts.p, pts, (size_t)n_pts * 24, cudaMemcpyDeviceToDevice, st));
  o->prepared_n = -1;
  const int s =
      fmm_prepare_device(o, n, cen, dir, mag, r_vortex, n_pts, (const double *)o->h_pts.p, st);
  if (s != DUST_OK) o->prepared_n = -1;
  return s;
}

extern "C" int dust_fmm_points_uvort_device(dust_octree *o, const dust_lines *end_vort,
                                            double *uvort, void *stream) {
  if (!o || o->prepared_n < 0 || (o->prepared_pts > 0 && !uvort)) return DUST_ERR_BAD_ARG;
  if (end_vort && (end_vort->n < 0 || (end_vort->n > 0 && (!end_vort->ver || !end_vort->mag))))
    return DUST_ERR_BAD_ARG;
  cudaStream_t st = stream ? (cudaStream_t)stream : o->stream;
  ElemDev e;
  DUST_TRY(elem_build_device(nullptr, nullptr, end_vort, o->prm.u_inf, reg_params(&o->prm),
                             false, o->el_raw, o->el_geo, e, st));
  return fmm_points_uvort_device(o, e, uvort, st);
}

extern "C" int dust_fmm_points_uvort(dust_octree *o, const dust_lines *end_vort, double *uvort) {
  if (!o || o->prepared_n < 0 || (o->prepared_pts > 0 && !uvort)) return DUST_ERR_BAD_ARG;
  if (end_vort && (end_vort->n < 0 || (end_vort->n > 0 && (!end_vort->ver || !end_vort->mag))))
    return DUST_ERR_BAD_ARG;
  const int n_pts = o->prepared_pts;
  if (n_pts == 0) return DUST_OK;
  cudaStream_t st = o->stream;
  DUST_TRY(devbuf_grow(o->h_out, (size_t)n_pts * 24));
  double *du = (double *)o->h_out.p;
  ElemDev e;
  DUST_TRY(elem_build_device(nullptr, nullptr, end_vort, o->prm.u_inf, reg_params(&o->prm),
                             true, o->el_raw, o->el_geo, e, st));
  DUST_TRY(fmm_points_uvort_device(o, e, du, st));
  DUST_CUDA(cudaMemcpyAsync(uvort, du, (size_t)n_pts * 24, cudaMemcpyDeviceToHost, st));
  DUST_CUDA(cudaStreamSynchronize(st));
  return DUST_OK;
}

extern "C" int dust_fmm_finish_device(dust_octree *o, const dust_elements *elems, double *vel,
                                      double *stretch, double *rotu, void *stream, int sync) {
  if (!o || o->prepared_n < 0 || (o->prepared_n > 0 && !vel)) return DUST_ERR_BAD_ARG;
  const int n = o->prepared_n;
  cudaStream_t st = stream ? (cudaStream_t)stream : o->stream;
  ElemDev e;
  DUST_TRY(elem_build_device(elems ? &elems->body : nullptr, elems ? &elems->wake : nullptr,
                             elems ? &elems->end_vort : nullptr, o->prm.u_inf,
                             reg_params(&o->prm), false, o->el_raw, o->el_geo, e, st));
  DUST_TRY(fmm_near_device(o, st));
  DUST_TRY(fmm_finish_device(o, n, e, vel, stretch, rotu, st));
  if (sync) DUST_CUDA(cudaStreamSynchronize(st));
  if (o->timing || sync) return fmm_collect_stats(o, n, n_elem_of(elems));
  return DUST_OK;
}

extern "C" int dust_fmm_finish(dust_octree *o, const dust_elements *elems, double *vel,
                               double *stretch, double *rotu) {
  if (!o || o->prepared_n < 0 || (o->prepared_n > 0 && !vel)) return DUST_ERR_BAD_ARG;
  const int n = o->prepared_n;
  cudaStream_t st = o->stream;
  size_t N = (size_t)(n > 0 ? n : 1);
  DUST_TRY(devbuf_grow(o->h_out, N * 9 * 8));
  double *ov = (double *)o->h_out.p, *os = ov + 3 * N, *orr = os + 3 * N;
  ElemDev e;
  DUST_TRY(elem_build_device(elems ? &elems->body : nullptr, elems ? &elems->wake : nullptr,
                             elems ? &elems->end_vort : nullptr, o->prm.u_inf,
                             reg_params(&o->prm), true, o->el_raw, o->el_geo, e, st));
  DUST_TRY(fmm_near_device(o, st));
  DUST_TRY(fmm_finish_device(o, n, e, ov, stretch ? os : nullptr, rotu ? orr : nullptr, st));
  if (n > 0) {
    DUST_CUDA(cudaMemcpyAsync(vel, ov, (size_t)n * 24, cudaMemcpyDeviceToHost, st));
    if (stretch)
      DUST_CUDA(cudaMemcpyAsync(stretch, os, (size_t)n * 24, cudaMemcpyDeviceToHost, st));
    if (rotu) DUST_CUDA(cudaMemcpyAsync(rotu, orr, (size_t)n * 24, cudaMemcpyDeviceToHost, st));
  }
  DUST_CUDA(cudaStreamSynchronize(st));
  return fmm_collect_stats(o, n, n_elem_of(elems));
}
