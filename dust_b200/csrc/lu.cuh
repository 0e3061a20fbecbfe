// lu.cuh -- dense LU with partial pivoting on the device (column-major).
//
// Blocked right-looking LU as LAPACK dgetrf (partial pivoting, first
// maximum wins like idamax), used by solve_linsys's sequence
// (src/linsys/mod_linsys.f90:352-482).  Panels are factored by one CTA
// (rows in registers), a thread-block cluster or a cooperative grid,
// whichever the panel's height allows (lu.cu); trailing updates are GEMMs.
#pragma once

#include <cublas_v2.h>

#include "dust_common.cuh"
#include "fmm_internal.h"

struct LuWork {
  DevBuf sync;   // barrier counters, error flag, partials, candidate rows
  DevBuf np;     // unpivoted LU: max |l| word, inverse triangles of every
                 // diagonal block (kept for lu_getrs_nopiv)
  DevBuf np_x;   // lu_getrs_nopiv: the intermediate Y = L^-1 B
  int nsm = 0;
};

// Factors the m x n column-major matrix A (lda) in place: ipiv (1-based,
// relative to A's first row) as LAPACK.  *info_dev receives the first zero
// pivot (1-based) or stays 0; the returned status reports launch errors and
// barrier timeouts.  `gemm_update` selects the trailing update:
// 0 = cuBLAS DGEMM/SGEMM (plain), 1 = tcgen05 TF32 (FP32 only).  With
// `perm` (n ints, n <= 51,200) the row permutation is also accumulated
// (perm[i] = original row now at row i), for lu_getrs.
template <typename T>
int lu_getrf(cublasHandle_t cb, cudaStream_t st, LuWork &w, int n, T *A, int lda,
             int *ipiv, int *info_dev, int gemm_update, int *perm = nullptr);

// Row interchanges of rows [k1, k2) (0-based) given ipiv (1-based, absolute
// row numbers relative to A), applied to columns [c0, c1) of A.
template <typename T>
void lu_laswp(cudaStream_t st, T *A, int lda, int c0, int c1, int k1, int k2,
              const int *ipiv);

// Solves A X = B with the factors (nrhs columns, ldb); the row interchanges
// from `perm` (lu_getrf's) in one gather when given, else from ipiv.
template <typename T>
int lu_getrs(cublasHandle_t cb, cudaStream_t st, int n, int nrhs, const T *A, int lda,
             const int *ipiv, T *B, int ldb, const int *perm = nullptr);

// Unpivoted blocked LU of the n x n column-major A (lu_np.cu): L unit lower
// and U upper in place, ipiv (when given) the identity, perm (when given)
// the identity permutation, *lmax the largest |l(i,j)| (infinity after a
// zero diagonal).  The factors are partial pivoting's own when *lmax < 1 (no
// interchange would have been made).  `gemm_update` as for lu_getrf.
template <typename T>
int lu_getrf_nopiv(cublasHandle_t cb, cudaStream_t st, LuWork &w, int n, T *A, int lda,
                   int *ipiv, int gemm_update, int *perm, float *lmax);

// Solves A X = B (X over B, nrhs columns, ldb) with the factors of the last
// lu_getrf_nopiv on this LuWork (same A, n): forward and backward block
// substitution with the kept inverse triangles, one launch per 64-row block.
template <typename T>
int lu_getrs_nopiv(cudaStream_t st, LuWork &w, int n, int nrhs, const T *A, int lda, T *B,
                   int ldb);

// lu_getrf through the unpivoted factorisation when its multipliers certify
// it (max |l| < 1 - margin: partial pivoting would interchange no row), else
// restore() puts the unfactored matrix back into A and lu_getrf factors it
// with pivoting.  *pivoted tells which ran.  A zero diagonal always takes
// the pivoted path (which reports it in info as dgetrf does).
template <typename T, typename Restore>
int lu_getrf_auto(cublasHandle_t cb, cudaStream_t st, LuWork &w, int n, T *A, int lda,
                  int *ipiv, int *info_dev, int gemm_update, int *perm, double margin,
                  Restore restore, int *pivoted) {
  float lmax = INFINITY;
  DUST_TRY(lu_getrf_nopiv<T>(cb, st, w, n, A, lda, ipiv, gemm_update, perm, &lmax));
  if ((double)lmax < 1.0 - margin) {
    DUST_CUDA(cudaMemsetAsync(info_dev, 0, sizeof(int), st));
    if (pivoted) *pivoted = 0;
    return DUST_OK;
  }
  DUST_TRY(restore());
  if (pivoted) *pivoted = 1;
  return lu_getrf<T>(cb, st, w, n, A, lda, ipiv, info_dev, gemm_update, perm);
}
