// linsys.cu -- influence-coefficient (AIC) assembly and the block LU solve.
//
// Replaces src/linsys/mod_linsys.f90 (initialize_linsys :109-267,
// assemble_linsys :279-344, solve_linsys :352-482) and the row builders of
// src/aeroel/mod_surfpan.f90 (:378-535, :579-629) and
// src/aeroel/mod_vortlatt.f90 (:143-391).
//
// Layout: A is the reference's column-major A(rank, rank) in HBM (FP64),
// elements ordered static first then moving.  One thread computes one
// coefficient; a CTA covers 32 rows x 8 columns with the 8 column panels
// staged in shared memory, so the column-major stores of a warp are
// contiguous.  The right-hand-side contributions of a CTA are reduced per
// row in shared memory and added with one atomic per row and CTA.
#include <cublas_v2.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "dust_common.cuh"
#include "elements.cuh"
#include "fmm_internal.h"
#include "linsys_internal.h"
#include "lu.cuh"

static inline unsigned nblk(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

// compute_pot (surface-panel row) / compute_psi (vortex-lattice row) of
// element `col` (index j) at the collocation point of `row` (index ie).
__device__ inline void aic_entry(const RegParams &rp, int rkind, const double *rcen,
                                 const double *rnor, int ie, const PanelGeo &col, int j,
                                 double &a, double &b1) {
  if (rkind == DUST_ELEM_SURFPAN) {
    double dou = (ie != j) ? pot_dou(rp, col, rcen) : -2.0 * DUST_PI;
    a = -dou;
    b1 = (col.kind == DUST_ELEM_SURFPAN) ? pot_sou(col, dou, rcen) : 0.0;
  } else {
    double vd[3];
    vel_dou(rp, col, rcen, vd);
    a = vd[0] * rnor[0] + vd[1] * rnor[1] + vd[2] * rnor[2];
    if (col.kind == DUST_ELEM_SURFPAN) {
      double vs[3];
      vel_sou(rp, col, rcen, vs);
      b1 = -vs[0] * rnor[0] + -vs[1] * rnor[1] + -vs[2] * rnor[2];
    } else {
      b1 = (ie == j) ? 4.0 * DUST_PI : 0.0;
    }
  }
}

#define AIC_RX 32
#define AIC_CY 8

// mode 0: static init rows/cols: A(ie,j) and bst(ie,j) = b1
// mode 1: step: A(ie,j) and b(ie) += b1 * sig(j)
__global__ void __launch_bounds__(AIC_RX *AIC_CY)
    k_aic(const PanelGeo *__restrict__ el, RegParams rp, int r0, int r1, int c0, int c1,
          double *A, int lda, double *bst, int nst, double *b, int mode) {
  __shared__ PanelGeo s_col[AIC_CY];
  __shared__ double s_red[AIC_CY][AIC_RX];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int ie = r0 + blockIdx.x * AIC_RX + tx;
  const int jc0 = c0 + blockIdx.y * AIC_CY;
  const int words = sizeof(PanelGeo) / 8;
  const int tid = ty * AIC_RX + tx;
  for (int w = tid; w < AIC_CY * words; w += AIC_RX * AIC_CY) {
    int q = w / words, ww = w % words;
    int j = jc0 + q;
    if (j < c1) ((double *)&s_col[q])[ww] = ((const double *)(el + j))[ww];
  }
  __syncthreads();
  const int j = jc0 + ty;
  double term = 0.0;
  if (ie < r1 && j < c1) {
    const PanelGeo &rw = el[ie];
    double rcen[3] = {rw.cen[0], rw.cen[1], rw.cen[2]};
    double rnor[3] = {rw.nor[0], rw.nor[1], rw.nor[2]};
    double a, b1;
    aic_entry(rp, rw.kind, rcen, rnor, ie, s_col[ty], j, a, b1);
    A[(size_t)ie + (size_t)j * lda] = a;
    if (mode == 0) {
      bst[(size_t)ie + (size_t)j * nst] = b1;
    } else {
      // surfpan row: b1 * nor_j.(ub_j - wind - uvort_j); vortlatt row: the
      // diagonal uses element ie's normal and ub with uvort of j == ie
      term = b1 * s_col[ty].sig;
    }
  }
  if (mode == 1) {
    s_red[ty][tx] = term;
    __syncthreads();
    if (ty == 0 && ie < r1) {
      double s = 0.0;
      for (int q = 0; q < AIC_CY; ++q) s += s_red[q][tx];
      if (s != 0.0) atomicAdd(b + ie, s);
    }
  }
}

// static columns of static rows: b(ie) += sum_j bst(ie,j) nor_j.(-wind - uvort_j);
// blockIdx.y takes a chunk of RS_COLS columns (partial sums added atomically)
#define RS_COLS 256
__global__ void k_rhs_static(const PanelGeo *el, const double *bst, int nst, double *b) {
  __shared__ double s_sig[RS_COLS];
  const int j0 = blockIdx.y * RS_COLS, j1 = min(nst, j0 + RS_COLS);
  for (int j = j0 + (int)threadIdx.x; j < j1; j += blockDim.x) s_sig[j - j0] = el[j].sig0;
  __syncthreads();
  const int ie = blockIdx.x * blockDim.x + threadIdx.x;
  if (ie >= nst) return;
  double s = 0.0;
  for (int j = j0; j < j1; ++j) s += bst[(size_t)ie + (size_t)j * nst] * s_sig[j - j0];
  atomicAdd(b + ie, s);
}

// add_wake_surfpan (mod_surfpan.f90:489-535) / add_wake_vortlatt
// (mod_vortlatt.f90:280-322) for rows [r0, r1) with column range
// [ista, iend] (0-based, inclusive).  One thread owns one row.
__global__ void k_add_wake(const PanelGeo *el, const PanelGeo *wk, int nwake, int n_impl,
                           const int *impl, RegParams rp, int r0, int r1, int ista, int iend,
                           double *A, int lda, double *b, int do_rhs) {
  int ie = r0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (ie >= r1) return;
  const PanelGeo &rw = el[ie];
  double rcen[3] = {rw.cen[0], rw.cen[1], rw.cen[2]};
  double rnor[3] = {rw.nor[0], rw.nor[1], rw.nor[2]};
  const bool sp = rw.kind == DUST_ELEM_SURFPAN;
  for (int j = 0; j < n_impl; ++j) {
    int i1 = impl[2 * j] - 1, i2 = impl[2 * j + 1] - 1;
    if (sp) {
      if (i1 >= ista && i1 <= iend && i2 >= ista && i2 <= iend) {
        double a = -pot_dou(rp, wk[j], rcen);
        A[(size_t)ie + (size_t)i1 * lda] += a;
        A[(size_t)ie + (size_t)i2 * lda] -= a;
      }
    } else if (i1 >= ista && i1 <= iend) {
      double vd[3];
      vel_dou(rp, wk[j], rcen, vd);
      double a = vd[0] * rnor[0] + vd[1] * rnor[1] + vd[2] * rnor[2];
      A[(size_t)ie + (size_t)i1 * lda] += a;
      if (i2 >= 0) A[(size_t)ie + (size_t)i2 * lda] -= a;
    }
  }
  if (!do_rhs) return;
  double s = 0.0;
  for (int j = n_impl; j < nwake; ++j) {
    double a;
    if (sp) {
      a = -pot_dou(rp, wk[j], rcen);
    } else {
      double vd[3];
      vel_dou(rp, wk[j], rcen, vd);
      a = vd[0] * rnor[0] + vd[1] * rnor[1] + vd[2] * rnor[2];
    }
    s -= a * wk[j].mag;
  }
  b[ie] += s;
}

// ------------------------------------------------------------------- host
static int load_geometry(dust_linsys *L, const dust_panels *elems, const dust_wake_rows *wake,
                         bool host = true) {
  if (!elems || elems->n != L->n) return DUST_ERR_BAD_ARG;
  ElemDev e;
  DUST_TRY(elem_build_device(elems, wake ? &wake->pan : nullptr, nullptr, L->prm.u_inf, L->rp,
                             host, L->raw, L->geo, e, L->st));
  L->el = e.body;
  L->wk = e.wake;
  L->nwake = e.nwake;
  L->n_impl = wake ? wake->n_impl : 0;
  if (L->n_impl > L->nwake || L->n_impl < 0) return DUST_ERR_BAD_ARG;
  if (L->n_impl > 0) {
    DUST_TRY(devbuf_grow(L->impl, (size_t)L->n_impl * 2 * sizeof(int)));
    DUST_CUDA(cudaMemcpyAsync(L->impl.p, wake->impl_ind, (size_t)L->n_impl * 2 * sizeof(int),
                              host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                              L->st));
  }
  return DUST_OK;
}

static void launch_aic(dust_linsys *L, int r0, int r1, int c0, int c1, int mode) {
  if (r1 <= r0 || c1 <= c0) return;
  dim3 blk(AIC_RX, AIC_CY), grd(nblk(r1 - r0, AIC_RX), nblk(c1 - c0, AIC_CY));
  k_aic<<<grd, blk, 0, L->st>>>(L->el, L->rp, r0, r1, c0, c1, (double *)L->A.p, L->n,
                               (double *)L->bst.p, L->nst, (double *)L->b.p, mode);
}

static void launch_wake(dust_linsys *L, int r0, int r1, int ista, int iend, int do_rhs) {
  if (r1 <= r0) return;
  k_add_wake<<<nblk(r1 - r0, 128), 128, 0, L->st>>>(
      L->el, L->wk, L->nwake, L->n_impl, (const int *)L->impl.p, L->rp, r0, r1, ista, iend,
      (double *)L->A.p, L->n, (double *)L->b.p, do_rhs);
}

extern "C" int dust_linsys_create(int rank, int nstatic, const dust_fmm_params *prm,
                                  const dust_panels *elems, const dust_wake_rows *wake,
                                  dust_linsys **out) {
  if (!out || !prm || rank <= 0 || nstatic < 0 || nstatic > rank || !elems ||
      elems->n != rank)
    return DUST_ERR_BAD_ARG;
  *out = nullptr;
  dust_linsys *L = new dust_linsys();
  L->n = rank;
  L->nst = nstatic;
  L->nmv = rank - nstatic;
  L->prm = *prm;
  L->rp = reg_params(prm);
  if (cudaStreamCreateWithFlags(&L->st, cudaStreamNonBlocking) != cudaSuccess ||
      cublasCreate(&L->cb) != CUBLAS_STATUS_SUCCESS) {
    delete L;
    return DUST_ERR_CUDA;
  }
  cublasSetStream(L->cb, L->st);
  int st = DUST_OK;
  size_t n = rank, ns = std::max(nstatic, 1);
  if ((st = devbuf_grow(L->A, n * n * 8)) || (st = devbuf_grow(L->b, n * 8 * 4)) ||
      (st = devbuf_grow(L->bst, ns * ns * 8)) || (st = devbuf_grow(L->piv, n * 4 + 64)) ||
      (st = devbuf_grow(L->info, 64))) {
    dust_linsys_destroy(L);
    return st;
  }
  cudaMemsetAsync(L->A.p, 0, n * n * 8, L->st);
  cudaMemsetAsync(L->b.p, 0, n * 8, L->st);
  cudaMemsetAsync(L->bst.p, 0, ns * ns * 8, L->st);
  st = load_geometry(L, elems, wake);
  if (st == DUST_OK && nstatic > 0) {
    // initialize_linsys: static rows x static columns, static wake, LU once
    launch_aic(L, 0, nstatic, 0, nstatic, 0);
    launch_wake(L, 0, nstatic, 0, nstatic - 1, 0);
    if (cudaGetLastError() != cudaSuccess) st = DUST_ERR_CUDA;
    if (st == DUST_OK && L->keep_static_copy) {
      // unfactored static block for refinement (see dust_linsys_solve)
    }
    if (st == DUST_OK) {
      DevBuf &As = L->As;
      if ((st = devbuf_grow(As, (size_t)nstatic * nstatic * 8)) == DUST_OK) {
        cudaMemcpy2DAsync(As.p, (size_t)nstatic * 8, L->A.p, n * 8, (size_t)nstatic * 8, nstatic,
                          cudaMemcpyDeviceToDevice, L->st);
        st = lu_getrf_auto<double>(
            L->cb, L->st, L->lu, nstatic, (double *)L->A.p, rank, (int *)L->piv.p,
            (int *)L->info.p, 0, nullptr, 1e-8,
            [&]() -> int {
              DUST_CUDA(cudaMemcpy2DAsync(L->A.p, n * 8, As.p, (size_t)nstatic * 8,
                                          (size_t)nstatic * 8, nstatic, cudaMemcpyDeviceToDevice,
                                          L->st));
              return DUST_OK;
            },
            &L->static_pivoted);
        if (st == DUST_OK) {
          int info = 0;
          cudaMemcpy(&info, L->info.p, sizeof(int), cudaMemcpyDeviceToHost);
          if (info) st = DUST_ERR_SINGULAR;
        }
      }
    }
  }
  if (st == DUST_OK && cudaStreamSynchronize(L->st) != cudaSuccess) st = DUST_ERR_CUDA;
  if (st != DUST_OK) {
    dust_linsys_destroy(L);
    return st;
  }
  *out = L;
  return DUST_OK;
}

extern "C" int dust_linsys_destroy(dust_linsys *L) {
  if (!L) return DUST_OK;
  if (L->st) cudaStreamSynchronize(L->st);
  DevBuf *bufs[] = {&L->A,  &L->As, &L->b,    &L->bst,  &L->piv, &L->info, &L->geo,
                    &L->raw, &L->impl, &L->work, &L->lu.sync, &L->lu.np, &L->lu.np_x, &L->A32, &L->gm, &L->ainv32, &L->mx, &L->kr,
                    &L->mvb, &L->permv};
  for (DevBuf *b : bufs) devbuf_free(*b);
  if (L->cb) cublasDestroy(L->cb);
  if (L->st) cudaStreamDestroy(L->st);
  delete L;
  return DUST_OK;
}

static int assemble(dust_linsys *L, const dust_panels *elems, const dust_wake_rows *wake,
                    bool host) {
  if (!L) return DUST_ERR_BAD_ARG;
  DUST_TRY(load_geometry(L, elems, wake, host));
  const int n = L->n, nst = L->nst;
  DUST_CUDA(cudaMemsetAsync(L->b.p, 0, (size_t)n * 8, L->st));
  // build_row: static rows get the moving columns, moving rows all columns
  if (nst > 0) {
    k_rhs_static<<<dim3(nblk(nst, 128), nblk(nst, RS_COLS)), 128, 0, L->st>>>(
        L->el, (const double *)L->bst.p, nst, (double *)L->b.p);
    launch_aic(L, 0, nst, nst, n, 1);
  }
  launch_aic(L, nst, n, 0, n, 1);
  // add_wake: static rows over the moving columns, moving rows over all
  launch_wake(L, 0, nst, nst, n - 1, 1);
  launch_wake(L, nst, n, 0, n - 1, 1);
  DUST_CUDA(cudaGetLastError());
  L->factored = false;
  L->assembled = true;
  return DUST_OK;
}

extern "C" int dust_linsys_assemble(dust_linsys *L, const dust_panels *elems,
                                    const dust_wake_rows *wake) {
  return assemble(L, elems, wake, true);
}
extern "C" int dust_linsys_assemble_device(dust_linsys *L, const dust_panels *elems,
                                           const dust_wake_rows *wake) {
  return assemble(L, elems, wake, false);
}

extern "C" int dust_linsys_get_system(dust_linsys *L, double *A, double *b) {
  if (!L || !L->assembled) return DUST_ERR_BAD_ARG;
  if (L->factored) return DUST_ERR_BAD_ARG;
  if (A)
    DUST_CUDA(cudaMemcpyAsync(A, L->A.p, (size_t)L->n * L->n * 8, cudaMemcpyDeviceToHost, L->st));
  if (b) DUST_CUDA(cudaMemcpyAsync(b, L->b.p, (size_t)L->n * 8, cudaMemcpyDeviceToHost, L->st));
  DUST_CUDA(cudaStreamSynchronize(L->st));
  return DUST_OK;
}

// solve_linsys: Schur update of the moving block + LU + solve (FP64).
int linsys_solve_lu64(dust_linsys *L, double *res_dev) {
  const int n = L->n, nst = L->nst, nmv = L->nmv;
  double *A = (double *)L->A.p;
  int *P = (int *)L->piv.p;
  cublasSetStream(L->cb, L->st);
  const double one = 1.0, mone = -1.0;
  if (nst > 0 && nmv > 0) {
    lu_laswp<double>(L->st, A + 0, n, nst, n, 0, nst, P);
    if (cublasDtrsm(L->cb, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N,
                    CUBLAS_DIAG_UNIT, nst, nmv, &one, A, n, A + (size_t)nst * n,
                    n) != CUBLAS_STATUS_SUCCESS)
      return DUST_ERR_CUDA;
    if (cublasDtrsm(L->cb, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N,
                    CUBLAS_DIAG_NON_UNIT, nmv, nst, &one, A, n, A + nst,
                    n) != CUBLAS_STATUS_SUCCESS)
      return DUST_ERR_CUDA;
    if (cublasDgemm(L->cb, CUBLAS_OP_N, CUBLAS_OP_N, nmv, nmv, nst, &mone, A + nst, n,
                    A + (size_t)nst * n, n, &one, A + nst + (size_t)nst * n,
                    n) != CUBLAS_STATUS_SUCCESS)
      return DUST_ERR_CUDA;
  }
  if (nmv > 0) {
    // the moving block (Schur complement) is kept unfactored in mvb until the
    // certified unpivoted LU has been accepted
    double *Amm = A + nst + (size_t)nst * n;
    DUST_TRY(devbuf_grow(L->mvb, (size_t)nmv * nmv * 8));
    DUST_CUDA(cudaMemcpy2DAsync(L->mvb.p, (size_t)nmv * 8, Amm, n * 8, (size_t)nmv * 8, nmv,
                                cudaMemcpyDeviceToDevice, L->st));
    DUST_TRY(lu_getrf_auto<double>(
        L->cb, L->st, L->lu, nmv, Amm, n, P + nst, (int *)L->info.p, 0, nullptr, 1e-8,
        [&]() -> int {
          DUST_CUDA(cudaMemcpy2DAsync(Amm, n * 8, L->mvb.p, (size_t)nmv * 8, (size_t)nmv * 8,
                                      nmv, cudaMemcpyDeviceToDevice, L->st));
          return DUST_OK;
        },
        &L->last_pivoted));
    int info = 0;
    DUST_CUDA(cudaMemcpy(&info, L->info.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (info) return DUST_ERR_SINGULAR;
    if (nst > 0) {
      // dlaswp on A(nst+1:rank, 1:nst) with the moving pivots, then make
      // them global
      lu_laswp<double>(L->st, A + nst, n, 0, nst, 0, nmv, P + nst);
      linsys_shift_pivots(L->st, P + nst, nmv, nst);
    }
  }
  L->factored = true;
  DUST_CUDA(cudaMemcpyAsync(res_dev, L->b.p, (size_t)n * 8, cudaMemcpyDeviceToDevice, L->st));
  // the pivots' net row permutation, applied as one gather instead of n
  // dependent interchanges; a system without moving rows keeps its pivots,
  // so its permutation is built once
  const int *perm = nullptr;
  if ((size_t)n * 8 <= 200 * 1024) {
    if (nmv > 0 || !L->perm_ok) {
      std::vector<int> piv(n), pm(n);
      DUST_CUDA(cudaMemcpyAsync(piv.data(), P, (size_t)n * 4, cudaMemcpyDeviceToHost, L->st));
      DUST_CUDA(cudaStreamSynchronize(L->st));
      for (int i = 0; i < n; ++i) pm[i] = i;
      for (int i = 0; i < n; ++i) {
        const int q = piv[i] - 1;
        if (q < 0 || q >= n) return DUST_ERR_BAD_ARG;
        std::swap(pm[i], pm[q]);
      }
      DUST_TRY(devbuf_grow(L->permv, (size_t)n * 4));
      DUST_CUDA(cudaMemcpyAsync(L->permv.p, pm.data(), (size_t)n * 4, cudaMemcpyHostToDevice,
                                L->st));
      DUST_CUDA(cudaStreamSynchronize(L->st));
      L->perm_ok = nmv == 0;
    }
    perm = (const int *)L->permv.p;
  }
  DUST_TRY(lu_getrs<double>(L->cb, L->st, n, 1, A, n, P, res_dev, n, perm));
  return DUST_OK;
}

__global__ void k_shift(int *P, int n, int off) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) P[i] += off;
}
void linsys_shift_pivots(cudaStream_t st, int *P, int n, int off) {
  if (n > 0) k_shift<<<nblk(n, 128), 128, 0, st>>>(P, n, off);
}

static int solve(dust_linsys *L, int mode, double *res, dust_solve_report *rep, bool host) {
  if (!L || !res || !L->assembled) return DUST_ERR_BAD_ARG;
  if (L->factored) return DUST_ERR_BAD_ARG;  // assemble before every solve
  DUST_TRY(devbuf_grow(L->work, (size_t)L->n * 8 * 8));
  double *x = (double *)L->work.p;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, L->st);
  int st = DUST_OK;
  dust_solve_report r;
  memset(&r, 0, sizeof(r));
  L->last_pivoted = 0;
  if (mode == DUST_SOLVE_LU64) {
    st = linsys_solve_lu64(L, x);
    r.mode_used = DUST_SOLVE_LU64;
    r.pivoted = L->static_pivoted | L->last_pivoted;
  } else if (mode == DUST_SOLVE_MIXED || mode == DUST_SOLVE_GMRES_NN) {
    st = linsys_solve_iterative(L, mode, x, &r);
    r.pivoted = L->static_pivoted | L->last_pivoted;
  } else {
    st = DUST_ERR_BAD_ARG;
  }
  cudaEventRecord(e1, L->st);
  if (st == DUST_OK) {
    if (cudaMemcpyAsync(res, x, (size_t)L->n * 8,
                        host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                        L->st) != cudaSuccess)
      st = DUST_ERR_CUDA;
    if (cudaStreamSynchronize(L->st) != cudaSuccess) st = DUST_ERR_CUDA;
    cudaEventElapsedTime(&r.ms_solve, e0, e1);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rep) *rep = r;
  return st;
}

extern "C" int dust_linsys_solve(dust_linsys *L, int mode, double *res,
                                 dust_solve_report *rep) {
  return solve(L, mode, res, rep, true);
}
extern "C" int dust_linsys_solve_device(dust_linsys *L, int mode, double *res,
                                        dust_solve_report *rep) {
  return solve(L, mode, res, rep, false);
}
