// schur_mixed.cu -- mixed-precision solve of the static/moving system.
//
// The reference factors the static block once and, every step, updates the
// moving block by a Schur complement in FP64 (src/linsys/mod_linsys.f90:
// 352-482).  Here the same block structure is used in low precision as a
// preconditioner and FP64 accuracy is recovered by iterative refinement:
//
//   once:      Ainv = A_ss^-1 from the FP64 LU of the static block, kept in FP32
//   per step:  Y = Ainv A_sd                    (tensor-core TF32 GEMM)
//              S = A_dd - A_ds Y                (tensor-core TF32 GEMM)
//              S = P L U                        (FP32 LU, tensor-core updates)
//   refine:    r = b - A x   (FP64, blockwise, unfactored blocks)
//              y_s = Ainv r_s;  x_d = S^-1 (r_d - A_ds y_s);  x_s = y_s - Y x_d
//              x += [x_s; x_d]   until ||r||_inf <= tol ||A||_inf ||x||_inf
#include <cublas_v2.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "dust_common.cuh"
#include "linsys_internal.h"
#include "lu.cuh"

static inline unsigned nblk(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

int gemm_tf32_acc(cudaStream_t st, int m, int n, int k, const float *A, int lda, const float *B,
                  int ldb, float *C, int ldc, float sign);
int gemm_tf32_error(cudaStream_t st);

// dst (rows x cols, ldd) = (float) src (ldS)
__global__ void k_blk_f32(int rows, int cols, const double *src, int lds, float *dst, int ldd) {
  size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t tot = (size_t)rows * cols;
  for (; e < tot; e += (size_t)gridDim.x * blockDim.x) {
    int j = (int)(e / rows), i = (int)(e % rows);
    dst[(size_t)i + (size_t)j * ldd] = (float)src[(size_t)i + (size_t)j * lds];
  }
}
__global__ void k_eye(int n, double *X) {
  size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t tot = (size_t)n * n;
  for (; e < tot; e += (size_t)gridDim.x * blockDim.x) {
    int j = (int)(e / n), i = (int)(e % n);
    X[e] = (i == j) ? 1.0 : 0.0;
  }
}
__global__ void k_vec_f32(int n, const double *a, float *b) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}
__global__ void k_vec_add(int n, const float *d, double *x) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] += (double)d[i];
}
// row sums of |A| for the full matrix: static block from As, the rest from
// A; blockIdx.y takes a chunk of RA_COLS columns, rows are coalesced
#define RA_COLS 256
__global__ void k_rowabs_blocks(int n, int nst, const double *As, const double *A, double *rs) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int j0 = blockIdx.y * RA_COLS, j1 = min(n, j0 + RA_COLS);
  double s = 0.0;
  for (int j = j0; j < j1; ++j) {
    double v = (i < nst && j < nst) ? As[(size_t)i + (size_t)j * nst] : A[(size_t)i + (size_t)j * n];
    s += fabs(v);
  }
  atomicAdd(rs + i, s);
}

int build_static_inverse(dust_linsys *L) {
  const int nst = L->nst, n = L->n;
  size_t nn = (size_t)nst * nst;
  DevBuf X;
  DUST_TRY(devbuf_grow(X, nn * 8));
  double *Xp = (double *)X.p;
  k_eye<<<2048, 256, 0, L->st>>>(nst, Xp);
  // A_ss^-1 = U^-1 L^-1 P from the static LU kept in A(1:nst,1:nst)
  DUST_TRY(lu_getrs<double>(L->cb, L->st, nst, nst, (const double *)L->A.p, n, (const int *)L->piv.p,
                            Xp, nst));
  DUST_TRY(devbuf_grow(L->ainv32, nn * 4));
  k_blk_f32<<<2048, 256, 0, L->st>>>(nst, nst, Xp, nst, (float *)L->ainv32.p, nst);
  DUST_CUDA(cudaStreamSynchronize(L->st));
  devbuf_free(X);
  L->ainv_ready = true;
  return DUST_OK;
}

int linsys_solve_schur_mixed(dust_linsys *L, double *x, double tol, int max_iter,
                             dust_solve_report *rep) {
  const int n = L->n, nst = L->nst, nmv = L->nmv;
  cudaStream_t st = L->st;
  cublasSetStream(L->cb, st);
  cublasSetPointerMode(L->cb, CUBLAS_POINTER_MODE_HOST);
  if (nst > 0 && !L->ainv_ready) DUST_TRY(build_static_inverse(L));
  const double *A = (const double *)L->A.p;
  const double *As = (const double *)L->As.p;
  const float *Ainv = (const float *)L->ainv32.p;
  // work: Y (nst x nmv), S (nmv x nmv), Ads32 (nmv x nst), Asd32 (nst x nmv),
  // vectors
  size_t need = 4 * ((size_t)nst * nmv * 3 + (size_t)nmv * nmv + (size_t)n * 4) + 8 * (size_t)n * 4 +
                (size_t)nmv * 8 + 8192;
  DUST_TRY(devbuf_grow(L->mx, need));
  char *b = (char *)L->mx.p;
  auto take = [&](size_t bytes) {
    char *p = b;
    b += (bytes + 255) / 256 * 256;
    return p;
  };
  float *Y = (float *)take((size_t)nst * nmv * 4);
  float *S = (float *)take((size_t)nmv * nmv * 4);
  float *Ads = (float *)take((size_t)nmv * nst * 4);
  float *Asd = (float *)take((size_t)nst * nmv * 4);
  float *r32 = (float *)take((size_t)n * 4);
  float *d32 = (float *)take((size_t)n * 4);
  float *t32 = (float *)take((size_t)n * 4);
  double *r = (double *)take((size_t)n * 8);
  double *rs = (double *)take((size_t)n * 8);
  int *piv = (int *)take((size_t)nmv * 4 + 64);
  int *info = piv + nmv;
  int *perm = (int *)take((size_t)nmv * 4);
  double *nrm = (double *)take(64);  // max |.| and 2-norms of the residual and x
  const bool use_perm = (size_t)nmv * 4 <= 200 * 1024;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  if (nmv > 0) {
    k_blk_f32<<<2048, 256, 0, st>>>(nst, nmv, A + (size_t)nst * n, n, Asd, nst);
    k_blk_f32<<<2048, 256, 0, st>>>(nmv, nst, A + nst, n, Ads, nmv);
    // S = A_mm - A_ms Ainv A_sm (Y = Ainv A_sm is kept, so S can be rebuilt)
    auto build_s = [&]() -> int {
      k_blk_f32<<<1024, 256, 0, st>>>(nmv, nmv, A + nst + (size_t)nst * n, n, S, nmv);
      if (nst > 0) DUST_TRY(gemm_tf32_acc(st, nmv, nmv, nst, Ads, nmv, Y, nst, S, nmv, -1.0f));
      DUST_CUDA(cudaGetLastError());
      return DUST_OK;
    };
    if (nst > 0) {
      DUST_CUDA(cudaMemsetAsync(Y, 0, (size_t)nst * nmv * 4, st));
      DUST_TRY(gemm_tf32_acc(st, nst, nmv, nst, Ainv, nst, Asd, nst, Y, nst, 1.0f));
    }
    DUST_TRY(build_s());
    DUST_TRY(lu_getrf_auto<float>(L->cb, st, L->lu, nmv, S, nmv, piv, info, 1,
                                  use_perm ? perm : nullptr, 0.0, build_s, &L->last_pivoted));
    DUST_TRY(gemm_tf32_error(st));
    int hinfo = 0;
    DUST_CUDA(cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, st));
    DUST_CUDA(cudaStreamSynchronize(st));
    if (hinfo) return DUST_ERR_SINGULAR;
  }
  cudaEventRecord(e1, st);
  DUST_CUDA(cudaMemsetAsync(rs, 0, (size_t)n * 8, st));
  k_rowabs_blocks<<<dim3(nblk(n, 128), nblk(n, RA_COLS)), 128, 0, st>>>(n, nst, As, A, rs);
  DUST_TRY(vec_absmax_nrm2(st, n, rs, nrm));
  double anorm = 0.0;
  DUST_CUDA(cudaMemcpyAsync(&anorm, nrm, 8, cudaMemcpyDeviceToHost, st));
  DUST_CUDA(cudaMemsetAsync(x, 0, (size_t)n * 8, st));
  DUST_CUDA(cudaMemcpyAsync(r, L->b.p, (size_t)n * 8, cudaMemcpyDeviceToDevice, st));
  double worst = 1e300;
  int it = 0;
  for (it = 0; it <= max_iter; ++it) {
    if (it > 0) {
      // r = b - A x, blockwise with the unfactored static block
      DUST_CUDA(cudaMemcpyAsync(r, L->b.p, (size_t)n * 8, cudaMemcpyDeviceToDevice, st));
      if (nst > 0) DUST_TRY(gemv_n<double>(st, nst, nst, -1.0, As, nst, x, 1.0, r));
      if (nmv > 0) {
        // columns nst.. of all rows, and the static columns of the moving rows
        DUST_TRY(gemv_n<double>(st, n, nmv, -1.0, A + (size_t)nst * n, n, x + nst, 1.0, r));
        if (nst > 0) DUST_TRY(gemv_n<double>(st, nmv, nst, -1.0, A + nst, n, x, 1.0, r + nst));
      }
      DUST_TRY(vec_absmax_nrm2(st, n, r, nrm));
      DUST_TRY(vec_absmax_nrm2(st, n, x, nrm + 2));
      double hh[4];
      DUST_CUDA(cudaMemcpyAsync(hh, nrm, 32, cudaMemcpyDeviceToHost, st));
      DUST_CUDA(cudaStreamSynchronize(st));
      const double hr = hh[0], hx = hh[2];
      double den = anorm * fabs(hx);
      worst = den > 0 ? fabs(hr) / den : fabs(hr);
      if (worst <= tol || it == max_iter) break;
    }
    // d = M^-1 r (FP32)
    k_vec_f32<<<nblk(n, 256), 256, 0, st>>>(n, r, r32);
    if (nst > 0) {
      // y_s = Ainv r_s  (in d32[0:nst])
      DUST_TRY(gemv_n<float>(st, nst, nst, 1.0f, Ainv, nst, r32, 0.0f, d32));
    }
    if (nmv > 0) {
      DUST_CUDA(cudaMemcpyAsync(t32, r32 + nst, (size_t)nmv * 4, cudaMemcpyDeviceToDevice, st));
      if (nst > 0) DUST_TRY(gemv_n<float>(st, nmv, nst, -1.0f, Ads, nmv, d32, 1.0f, t32));
      DUST_TRY(lu_getrs<float>(L->cb, st, nmv, 1, S, nmv, piv, t32, nmv,
                               use_perm ? perm : nullptr));
      DUST_CUDA(cudaMemcpyAsync(d32 + nst, t32, (size_t)nmv * 4, cudaMemcpyDeviceToDevice, st));
      if (nst > 0) DUST_TRY(gemv_n<float>(st, nst, nmv, -1.0f, Y, nst, t32, 1.0f, d32));
    }
    k_vec_add<<<nblk(n, 256), 256, 0, st>>>(n, d32, x);
  }
  DUST_CUDA(cudaGetLastError());
  if (rep) {
    rep->mode_used = DUST_SOLVE_MIXED;
    rep->iterations = it;
    rep->residual = worst;
    cudaEventElapsedTime(&rep->ms_factor, e0, e1);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return worst <= tol ? DUST_OK : DUST_ERR_NOT_CONVERGED;
}
