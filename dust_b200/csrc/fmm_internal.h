// fmm_internal.h -- handle layout and internal entry points of the FMM.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "dust_common.cuh"
#include "elements.cuh"

struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
};
void devbuf_free(DevBuf &b);
int devbuf_grow(DevBuf &b, size_t bytes);

// Everything a kernel needs, passed by value.
struct FmmDev {
  TreeGeom G;
  uint32_t n;
  int p, nm, nm1, nD;
  int use_vs, use_df, use_vd;
  double nu_inf;
  double u_inf[3];
  const double *dtab[DUST_MAXLEV + 1];
  int kdlen[DUST_MAXLEV + 1][3];
  const uint16_t *idxsum;
  const uint32_t *cstart, *perm;
  const double *P;  // sorted SoA: x y z ax ay az sigma
  const uint8_t *flags;
  const uint32_t *cidx;
  const uint32_t *act_key;
  const uint8_t *act_lev;
  const uint32_t *leaf_ci;
  uint32_t n_leaves;
  double *A, *B, *Gx;  // multipole a, local b (deg p), local g (deg p+1)
  double *out;         // sorted-order vel(3), stretch(3), rotu(3), SoA
  int64_t *counters;   // [0] M2L pairs, [1] P2P pairs
  double inv_fact[224];
};

struct ElemDev {
  const PanelGeo *body, *wake;
  const LineGeo *lines;
  int nbody, nwake, nline;
  RegParams rp;
};

struct dust_octree {
  dust_fmm_params prm;
  TreeGeom G;
  int p, nm, nm1, nD;
  uint64_t ncell_tot = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t last_stream = nullptr;  // stream of the last evaluation
  cudaEvent_t ev[12];  // phases [0..5], M2L kernel [6, 7], far element kernel [8, 9],
                       // start of the particles' near field [10]
  bool kev_m2l = false, kev_far = false;  // whether [6, 7] / [8, 9] were recorded
  bool timing = false;
  DevBuf dtab[DUST_MAXLEV + 1];
  int kdlen[DUST_MAXLEV + 1][3];
  DevBuf idxsum;
  // per-call buffers (grown on demand, kept across calls)
  DevBuf keys, keys_s, vals, perm, cnt, cstart, part, flags, ind, cidx, lidx;
  DevBuf act_key, act_lev, leaf_ci, mp, outs, cub_tmp, small;
  DevBuf h_in, h_out, h_pts, el_geo, el_raw;  // staging of host-API calls
  DevBuf ffbuf;                        // far-field panel records
  DevBuf elem_work;                    // FP32C element sums: far sums, near-pair list
  size_t near_cap = 0;                 // capacity of the near-pair list
  DevBuf dtabs[DUST_MAXLEV + 1];       // dimensionless scalar M2L tables (FP64)
  DevBuf dtab32[DUST_MAXLEV + 1];      // dimensionless scalar M2L tables (FP32)
  DevBuf jsum;                         // scalar M2L index table [n][slot][lane]
  int m2l_nJ = 0, m2l_SL = 0, m2l_P = 0;  // L indices, 32-lane slots, table stride
  DevBuf m2l_buf;                      // class-sorted M2L target lists
  DevBuf m2l_bat;                      // M2L batch descriptors
  uint32_t *m2l_list = nullptr;
  DevBuf ahat;                         // pre-scaled M2L source coefficients
  DevBuf shift;                        // M2M / L2L term tables of every level
  const void *shift_t[DUST_MAXLEV + 1][3], *shift_o[DUST_MAXLEV + 1][3];
  int shift_n[DUST_MAXLEV + 1][3];
  uint32_t ahat_c0 = 0;
  int m2l_cnt[8 * (DUST_MAXLEV + 1)];
  int64_t n_active = 0, n_leaves = 0;
  int64_t act_off[DUST_MAXLEV + 3];
  int bad_particle = -1;
  int prepared_n = -1;    // particles of the last prepared tree (-1: none)
  int prepared_pts = 0;   // evaluation points sorted into it (kept in h_pts)
  FmmDev dev;
  dust_fmm_stats stats;
};

int fmm_run_device(dust_octree *o, int n, const double *cen, const double *dir,
                   const double *mag, const double *rv, cudaStream_t st);
// the two halves of fmm_run_device: tree, multipoles and locals; then the
// particles' L2P + P2P
int fmm_prepare_device(dust_octree *o, int n, const double *cen, const double *dir,
                       const double *mag, const double *rv, int n_pts, const double *pts,
                       cudaStream_t st);
int fmm_near_device(dust_octree *o, cudaStream_t st);
// particles -> the prepared points through the tree, plus the lines directly
int fmm_points_uvort_device(dust_octree *o, const ElemDev &lines, double *uv, cudaStream_t st);
int fmm_finish_device(dust_octree *o, int n, const ElemDev &e, double *vel, double *str,
                      double *rot, cudaStream_t st);
int fmm_collect_stats(dust_octree *o, int n, int64_t n_elem);

// elements.cu
int elem_build_device(const dust_panels *body, const dust_panels *wake,
                      const dust_lines *lines, const double *u_inf, const RegParams &rp,
                      bool host_arrays, DevBuf &raw, DevBuf &geo, ElemDev &out,
                      cudaStream_t st);
RegParams reg_params(const dust_fmm_params *prm);
// velocity at n device points from the elements of e (x 1/4pi) plus u_inf
int elements_vel_points(const ElemDev &e, int n, const double *pts, const double *u_inf,
                        double *vel, cudaStream_t st);
// the particles' uvort kernels with the end vortices of `lines`
int points_uvort_device(const dust_fmm_params *prm, int n_pts, const double *pts, int n,
                        const double *cen, const double *dir, const double *mag,
                        const double *rv, const ElemDev &lines, double *uv, cudaStream_t st);
// Argument check shared by the uvort entry points: the points and the
// output when there are points, the four particle arrays when there are
// particles, the end vortices' vertices and strengths when there are any.
bool uvort_args_ok(const dust_fmm_params *prm, int n_pts, const double *pts, int n,
                   const double *cen, const double *dir, const double *mag,
                   const double *r_vortex, const dust_lines *end_vort, const double *uvort);

// m2l.cu
int m2l_batch_tables(dust_octree *o);
int m2l_prepare(dust_octree *o, FmmDev &d, cudaStream_t st);
int m2l_all_levels(dust_octree *o, FmmDev &d, cudaStream_t st);
int m2l_scale_sources(dust_octree *o, FmmDev &d, cudaStream_t st);


// direct.cu
int elem_output_device(FmmDev &d, const ElemDev &e, DevBuf &ffbuf, DevBuf &work,
                       size_t &near_cap, int precision, double *vel, double *str, double *rot,
                       cudaStream_t st, cudaEvent_t *kev = nullptr, bool *kev_done = nullptr);
// Morton order of n particles over the octree box (10 bits per axis): the
// permutation in scratch (grown to morton_perm_bytes(n) if needed)
size_t morton_perm_bytes(int n, cudaStream_t st);
int morton_perm(const dust_fmm_params *prm, int n, const double *cen, DevBuf &scratch,
                uint32_t **perm, size_t *used, cudaStream_t st);
int points_uvort_run(const dust_fmm_params *prm, int n_pts, const double *pts, int n,
                     const double *cen, const double *dir, const double *mag, const double *rv,
                     const ElemDev &lines, DevBuf &scratch, double *uv, cudaStream_t st);

// gemv.cu: y = alpha A x + beta y and y = alpha A^T x + beta y (A column-major
// m x k, device arrays), and out[0] = max |v_i|, out[1] = ||v||_2 (device)
template <typename T>
int gemv_n(cudaStream_t st, int m, int k, T alpha, const T *A, int lda, const T *x, T beta, T *y);
template <typename T>
int gemv_t(cudaStream_t st, int m, int k, T alpha, const T *A, int lda, const T *x, T beta, T *y);
int vec_absmax_nrm2(cudaStream_t st, int n, const double *v, double *out_dev);
