// solve.cu -- dense solves: the plain FP64 LU path and the mixed-precision
// path (FP32 LU, tensor-core trailing updates, FP64 iterative refinement).
//
// The plain path is LAPACK's dgetrf + dgetrs as the reference calls them
// (src/linsys/mod_linsys.f90:470-474).  The mixed path factors an FP32 copy
// of A and recovers FP64 accuracy by refinement: r = B - A X in FP64 (A kept
// in FP64), d = U^-1 L^-1 P r in FP32, X += d, until
// ||r||_inf <= tol * ||A||_inf ||X||_inf.
#include <cublas_v2.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "dust_common.cuh"
#include "linsys_internal.h"
#include "lu.cuh"

static inline unsigned nblk(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

__global__ void k_to_f32(size_t n, const double *a, float *b) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (; i < n; i += (size_t)gridDim.x * blockDim.x) b[i] = (float)a[i];
}
__global__ void k_add_f32(size_t n, const float *d, double *x) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (; i < n; i += (size_t)gridDim.x * blockDim.x) x[i] += (double)d[i];
}
// row sums |A| (for ||A||_inf), one thread per row, column-major
__global__ void k_rowabs(int n, const double *A, double *rs) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0.0;
  for (int j = 0; j < n; ++j) s += fabs(A[(size_t)i + (size_t)j * n]);
  rs[i] = s;
}
// per column: max |r| and max |x|
__global__ void k_colmax(int n, int nrhs, const double *R, const double *X, double *out) {
  int c = blockIdx.x;
  double mr = 0.0, mx = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    mr = fmax(mr, fabs(R[(size_t)c * n + i]));
    mx = fmax(mx, fabs(X[(size_t)c * n + i]));
  }
  for (int o = 16; o > 0; o >>= 1) {
    mr = fmax(mr, __shfl_down_sync(0xffffffffu, mr, o));
    mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
  }
  __shared__ double sr[32], sx[32];
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    sr[w] = mr;
    sx[w] = mx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < (int)(blockDim.x >> 5); ++q) {
      mr = fmax(mr, sr[q]);
      mx = fmax(mx, sx[q]);
    }
    out[2 * c] = fmax(mr, sr[0]);
    out[2 * c + 1] = fmax(mx, sx[0]);
  }
}

int mixed_solve_device(cublasHandle_t cb, cudaStream_t st, LuWork &lu, DevBuf &w32,
                       DevBuf &wrk, int n, int nrhs, const double *A64, const double *B,
                       double *X, double tol, int max_iter, int use_tc,
                       dust_solve_report *rep) {
  size_t nn = (size_t)n * n, nr = (size_t)n * nrhs;
  DUST_TRY(devbuf_grow(w32, nn * 4 + nr * 4 + (size_t)n * 4 + 256));
  DUST_TRY(devbuf_grow(wrk, nr * 8 + (size_t)n * 8 + (size_t)nrhs * 16 + 64 + 256));
  float *A32 = (float *)w32.p;
  float *D32 = A32 + nn;
  int *ipiv = (int *)(D32 + nr);
  double *R = (double *)wrk.p;
  double *rs = R + nr;
  double *cm = rs + n;
  int *info = (int *)(cm + 2 * nrhs);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  k_to_f32<<<1184, 256, 0, st>>>(nn, A64, A32);
  int piv = 1;
  int s = lu_getrf_auto<float>(cb, st, lu, n, A32, n, ipiv, info, use_tc, nullptr, 0.0,
                               [&]() -> int {
                                 k_to_f32<<<1184, 256, 0, st>>>(nn, A64, A32);
                                 DUST_CUDA(cudaGetLastError());
                                 return DUST_OK;
                               },
                               &piv);
  if (rep) rep->pivoted = piv;
  cudaEventRecord(e1, st);
  if (s != DUST_OK) return s;
  int hinfo = 0;
  DUST_CUDA(cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, st));
  DUST_CUDA(cudaStreamSynchronize(st));
  if (rep) cudaEventElapsedTime(&rep->ms_factor, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (hinfo) return DUST_ERR_SINGULAR;
  k_rowabs<<<nblk(n, 128), 128, 0, st>>>(n, A64, rs);
  int imax = 0;
  double anorm = 0.0;
  cublasSetStream(cb, st);
  cublasSetPointerMode(cb, CUBLAS_POINTER_MODE_HOST);
  if (cublasIdamax(cb, n, rs, 1, &imax) != CUBLAS_STATUS_SUCCESS) return DUST_ERR_CUDA;
  DUST_CUDA(cudaMemcpyAsync(&anorm, rs + imax - 1, 8, cudaMemcpyDeviceToHost, st));
  // X0 = LU \ B (in FP32)
  DUST_CUDA(cudaMemsetAsync(X, 0, nr * 8, st));
  DUST_CUDA(cudaMemcpyAsync(R, B, nr * 8, cudaMemcpyDeviceToDevice, st));
  std::vector<double> hcm(2 * (size_t)nrhs);
  const double one = 1.0, mone = -1.0;
  int it = 0;
  double worst = 0.0;
  for (it = 0; it <= max_iter; ++it) {
    if (it > 0) {
      // R = B - A X (FP64)
      DUST_CUDA(cudaMemcpyAsync(R, B, nr * 8, cudaMemcpyDeviceToDevice, st));
      if (cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_N, n, nrhs, n, &mone, A64, n, X, n, &one, R,
                      n) != CUBLAS_STATUS_SUCCESS)
        return DUST_ERR_CUDA;
      k_colmax<<<nrhs, 256, 0, st>>>(n, nrhs, R, X, cm);
      DUST_CUDA(cudaMemcpyAsync(hcm.data(), cm, 16 * (size_t)nrhs, cudaMemcpyDeviceToHost, st));
      DUST_CUDA(cudaStreamSynchronize(st));
      worst = 0.0;
      for (int c = 0; c < nrhs; ++c) {
        double den = anorm * hcm[2 * c + 1];
        double rel = den > 0 ? hcm[2 * c] / den : hcm[2 * c];
        worst = std::max(worst, rel);
      }
      if (worst <= tol) break;
      if (it == max_iter) break;
    }
    k_to_f32<<<256, 256, 0, st>>>(nr, R, D32);
    if (piv == 0)
      DUST_TRY(lu_getrs_nopiv<float>(st, lu, n, nrhs, A32, n, D32, n));
    else
      DUST_TRY(lu_getrs<float>(cb, st, n, nrhs, A32, n, ipiv, D32, n));
    k_add_f32<<<256, 256, 0, st>>>(nr, D32, X);
  }
  DUST_CUDA(cudaGetLastError());
  if (rep) {
    rep->iterations = it;
    rep->residual = worst;
    rep->mode_used = DUST_SOLVE_MIXED;
  }
  return worst <= tol ? DUST_OK : DUST_ERR_NOT_CONVERGED;
}

// LU64 on device arrays: A copied into the work matrix F unless it already
// is F's storage, F = P L U (lu_getrf), X = U^-1 L^-1 P B (lu_getrs).
static int dense_lu64_device(cublasHandle_t cb, cudaStream_t st, LuWork &lu, DevBuf &F,
                             DevBuf &piv, int n, int nrhs, const double *A, const double *B,
                             double *X, dust_solve_report *r) {
  const size_t nn = (size_t)n * n, nr = (size_t)n * nrhs;
  if (A != F.p) DUST_TRY(devbuf_grow(F, nn * 8));
  DUST_TRY(devbuf_grow(piv, (size_t)n * 4 + 64));
  int *ipiv = (int *)piv.p;
  int *info = ipiv + n;
  cudaEvent_t e0, e1, e2;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventCreate(&e2);
  int s = DUST_OK;
  cudaEventRecord(e0, st);
  if (A != F.p && cudaMemcpyAsync(F.p, A, nn * 8, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    s = DUST_ERR_CUDA;
  int pivd = 1;
  if (s == DUST_OK) {
    // A is F's storage only when the caller factors in place (then it cannot
    // be restored, and the pivoted path runs directly)
    if (A != F.p)
      s = lu_getrf_auto<double>(cb, st, lu, n, (double *)F.p, n, ipiv, info, 0, nullptr, 1e-8,
                                [&]() -> int {
                                  DUST_CUDA(cudaMemcpyAsync(F.p, A, nn * 8,
                                                            cudaMemcpyDeviceToDevice, st));
                                  return DUST_OK;
                                },
                                &pivd);
    else
      s = lu_getrf<double>(cb, st, lu, n, (double *)F.p, n, ipiv, info, 0);
  }
  if (r) r->pivoted = pivd;
  cudaEventRecord(e1, st);
  int hinfo = 0;
  if (s == DUST_OK) {
    cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) s = DUST_ERR_CUDA;
    else if (hinfo) s = DUST_ERR_SINGULAR;
  }
  if (s == DUST_OK) {
    if (X != B && cudaMemcpyAsync(X, B, nr * 8, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
      s = DUST_ERR_CUDA;
    if (s == DUST_OK)
      s = pivd == 0 ? lu_getrs_nopiv<double>(st, lu, n, nrhs, (const double *)F.p, n, X, n)
                    : lu_getrs<double>(cb, st, n, nrhs, (const double *)F.p, n, ipiv, X, n);
    cudaEventRecord(e2, st);
  }
  if (s == DUST_OK && cudaStreamSynchronize(st) == cudaSuccess && r) {
    cudaEventElapsedTime(&r->ms_factor, e0, e1);
    cudaEventElapsedTime(&r->ms_solve, e1, e2);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaEventDestroy(e2);
  if (r) r->mode_used = DUST_SOLVE_LU64;
  return s;
}

// Work areas of the device-array dense solve, kept between calls (grown,
// never shrunk) so that repeated solves of one size allocate nothing after
// the first; one set per process, guarded by a mutex.
namespace {
struct DenseWork {
  std::mutex mu;
  cublasHandle_t cb = nullptr;
  DevBuf F, piv, w32, wrk;
  LuWork lu;
};
DenseWork &dense_work() {
  static DenseWork *w = new DenseWork();  // never destroyed: no teardown at exit
  return *w;
}
}  // namespace

extern "C" int dust_dense_solve_device(int n, int nrhs, const double *A, const double *B,
                                       double *X, int mode, double tol,
                                       dust_solve_report *rep, void *stream) {
  if (n <= 0 || nrhs <= 0 || !A || !B || !X) return DUST_ERR_BAD_ARG;
  if (mode != DUST_SOLVE_LU64 && mode != DUST_SOLVE_MIXED) return DUST_ERR_BAD_ARG;
  if (X == A) return DUST_ERR_BAD_ARG;
  DenseWork &w = dense_work();
  std::lock_guard<std::mutex> g(w.mu);
  if (!w.cb && cublasCreate(&w.cb) != CUBLAS_STATUS_SUCCESS) {
    w.cb = nullptr;
    return DUST_ERR_CUDA;
  }
  cudaStream_t st = (cudaStream_t)stream;
  cublasSetStream(w.cb, st);
  dust_solve_report r;
  memset(&r, 0, sizeof(r));
  int s;
  if (mode == DUST_SOLVE_LU64) {
    s = dense_lu64_device(w.cb, st, w.lu, w.F, w.piv, n, nrhs, A, B, X, &r);
  } else {
    if (X == B) return DUST_ERR_BAD_ARG;
    s = mixed_solve_device(w.cb, st, w.lu, w.w32, w.wrk, n, nrhs, A, B, X,
                           tol > 0 ? tol : 1e-12, 30, 1, &r);
  }
  if (rep) *rep = r;
  return s;
}

extern "C" int dust_dense_solve(int n, int nrhs, const double *A, const double *B, double *X,
                                int mode, double tol, dust_solve_report *rep) {
  if (n <= 0 || nrhs <= 0 || !A || !B || !X) return DUST_ERR_BAD_ARG;
  if (mode != DUST_SOLVE_LU64 && mode != DUST_SOLVE_MIXED) return DUST_ERR_BAD_ARG;
  cudaStream_t st;
  cublasHandle_t cb;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return DUST_ERR_CUDA;
  if (cublasCreate(&cb) != CUBLAS_STATUS_SUCCESS) {
    cudaStreamDestroy(st);
    return DUST_ERR_CUDA;
  }
  cublasSetStream(cb, st);
  DevBuf dA, dB, dX, dF, piv, w32, wrk;
  LuWork lu;
  dust_solve_report r;
  memset(&r, 0, sizeof(r));
  size_t nn = (size_t)n * n, nr = (size_t)n * nrhs;
  int s = DUST_OK;
  if ((s = devbuf_grow(dA, nn * 8)) == DUST_OK && (s = devbuf_grow(dB, nr * 8)) == DUST_OK &&
      (s = devbuf_grow(dX, nr * 8 + 64)) == DUST_OK) {
    cudaMemcpyAsync(dA.p, A, nn * 8, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dB.p, B, nr * 8, cudaMemcpyHostToDevice, st);
    if (mode == DUST_SOLVE_LU64) {
      // factored in a second device copy, so that the unpivoted attempt can
      // be undone
      s = dense_lu64_device(cb, st, lu, dF, piv, n, nrhs, (const double *)dA.p,
                            (const double *)dB.p, (double *)dX.p, &r);
    } else {
      s = mixed_solve_device(cb, st, lu, w32, wrk, n, nrhs, (const double *)dA.p,
                             (const double *)dB.p, (double *)dX.p, tol > 0 ? tol : 1e-12, 30,
                             1, &r);
    }
    if (s == DUST_OK || s == DUST_ERR_NOT_CONVERGED) {
      if (cudaMemcpyAsync(X, dX.p, nr * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
          cudaStreamSynchronize(st) != cudaSuccess)
        s = DUST_ERR_CUDA;
    }
  }
  devbuf_free(dA);
  devbuf_free(dB);
  devbuf_free(dX);
  devbuf_free(dF);
  devbuf_free(piv);
  devbuf_free(w32);
  devbuf_free(wrk);
  devbuf_free(lu.sync);
  devbuf_free(lu.np);
  devbuf_free(lu.np_x);
  cublasDestroy(cb);
  cudaStreamDestroy(st);
  if (rep) *rep = r;
  return s;
}


int linsys_solve_iterative(dust_linsys *L, int mode, double *x_dev, dust_solve_report *rep) {
  int s = DUST_ERR_BAD_ARG;
  if (mode == DUST_SOLVE_MIXED)
    s = linsys_solve_schur_mixed(L, x_dev, 1e-14, 30, rep);
  else if (mode == DUST_SOLVE_GMRES_NN)
    s = linsys_gmres_nn(L, x_dev, rep);
  if (s == DUST_OK) {
    L->factored = true;
    return DUST_OK;
  }
  if (s != DUST_ERR_NOT_CONVERGED && s != DUST_ERR_SINGULAR) return s;
  // plain LU remains the fallback (the step's result is then exact LU)
  if (rep) rep->fell_back = 1;
  DUST_TRY(linsys_solve_lu64(L, x_dev));
  if (rep) rep->mode_used = DUST_SOLVE_LU64;
  return DUST_OK;
}
