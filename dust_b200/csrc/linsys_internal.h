// linsys_internal.h -- linear-system handle and internal entry points.
#pragma once

#include <cublas_v2.h>

#include "dust_common.cuh"
#include "elements.cuh"
#include "fmm_internal.h"
#include "gnn_internal.h"
#include "lu.cuh"

struct dust_linsys {
  int n = 0, nst = 0, nmv = 0;
  dust_fmm_params prm;
  RegParams rp;
  cudaStream_t st = nullptr;
  cublasHandle_t cb = nullptr;
  DevBuf A;     // column-major rank x rank, FP64; static block holds its LU
  DevBuf As;    // unfactored static block (nst x nst) for residuals
  DevBuf b, bst, piv, info, geo, raw, impl, work, A32, gm;
  DevBuf ainv32;  // FP32 inverse of the static block (mixed solve)
  DevBuf mx;      // mixed-solve work: Schur complement, coupling blocks, vectors
  DevBuf mvb;     // unfactored moving block (LU64 step), restored if the
                  // unpivoted LU is not certified
  int static_pivoted = 0, last_pivoted = 0;  // which LU ran (lu_getrf_auto)
  DevBuf permv;          // net row permutation of the pivots (lu_getrs)
  bool perm_ok = false;  // permv holds the static-only system's permutation
  bool ainv_ready = false;
  struct dust_precond *pc = nullptr;  // learned preconditioner (GMRES_NN)
  DevBuf kr;                          // GMRES Krylov basis and vectors
  LuWork lu;
  const PanelGeo *el = nullptr, *wk = nullptr;
  int nwake = 0, n_impl = 0;
  bool assembled = false, factored = false, keep_static_copy = true;
};

int linsys_solve_lu64(dust_linsys *L, double *res_dev);
int linsys_solve_iterative(dust_linsys *L, int mode, double *x_dev, dust_solve_report *rep);
// Static/moving Schur solve in FP32/TF32 refined to FP64 (tol on the
// normwise backward error ||b-Ax|| / (||A|| ||x||), max_iter refinements).
int linsys_solve_schur_mixed(dust_linsys *L, double *x, double tol, int max_iter,
                             dust_solve_report *rep);
void linsys_shift_pivots(cudaStream_t st, int *P, int n, int off);

// Mixed-precision dense solve on device arrays: FP32 LU (tensor-core
// trailing updates when use_tc) of A64, FP64 iterative refinement to `tol`.
int mixed_solve_device(cublasHandle_t cb, cudaStream_t st, LuWork &lu, DevBuf &w32,
                       DevBuf &wrk, int n, int nrhs, const double *A64, const double *B,
                       double *X, double tol, int max_iter, int use_tc,
                       dust_solve_report *rep);

// the assembled (unfactored) system as a view, and Y = A X through it
SysView linsys_view(const dust_linsys *L);
int linsys_matmat(const dust_linsys *L, int ncols, const double *X, int ldx, double *Y, int ldy,
                  cudaStream_t st, cublasHandle_t cb);
int linsys_gmres_nn(dust_linsys *L, double *x, dust_solve_report *rep);
// Ainv = A_ss^-1 (FP32) from the static block's FP64 LU, once per handle
int build_static_inverse(dust_linsys *L);
