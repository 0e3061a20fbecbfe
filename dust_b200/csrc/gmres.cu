// gmres.cu -- learned-preconditioned FP64 GMRES for the time-stepping system.
//
// Restarted GMRES(m) with right preconditioning A P u = b, x = P u.  With a
// static block, P is block lower-triangular on the static/moving split:
//   z_s = Ainv v_s,   z_d = [M (0; v_d - A_ds z_s)]_d,
// with Ainv = A_ss^-1 (FP32, built once from the static LU, as the mixed
// solve uses it) and M = (I + O) D^-1 from the graph network of gnn.cu
// evaluated on the current matrix, so the network only has to approximate
// the moving bodies' part; without one, P = M.  The warm start is x0 = P b.  Matrix-vector products use
// the assembled blocks directly (static block from its unfactored copy), so
// nothing is refactored.  Orthogonalisation is classical Gram-Schmidt applied
// twice; the small Hessenberg least-squares problem is solved on the host
// with Givens rotations.  Converged when ||b - A x||_2 <= tol ||b||_2 (true
// residual at every restart); otherwise DUST_ERR_NOT_CONVERGED and the caller
// falls back to the plain LU of solve_linsys (mod_linsys.f90:352-482).
#include <cublas_v2.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "dust_common.cuh"
#include "linsys_internal.h"

static inline unsigned nblk(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

#define GM_RESTART 50
#define GM_MAXIT 400
#define GM_TOL 1e-11

SysView linsys_view(const dust_linsys *L) {
  SysView v;
  v.n = L->n;
  v.nst = L->nst;
  v.As = (const double *)L->As.p;
  v.A = (const double *)L->A.p;
  return v;
}

// Y (n x nc) = A X with the assembled blocks
int linsys_matmat(const dust_linsys *L, int nc, const double *X, int ldx, double *Y, int ldy,
                  cudaStream_t st, cublasHandle_t cb) {
  const int n = L->n, nst = L->nst, nmv = L->nmv;
  const double *A = (const double *)L->A.p, *As = (const double *)L->As.p;
  const double one = 1.0, zero = 0.0;
  cublasSetStream(cb, st);
  cublasSetPointerMode(cb, CUBLAS_POINTER_MODE_HOST);
  auto gemm = [&](int m, int k, const double *Ap, int lda, const double *Xp, double *Yp,
                  const double *beta) {
    return cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_N, m, nc, k, &one, Ap, lda, Xp, ldx, beta, Yp,
                       ldy) == CUBLAS_STATUS_SUCCESS;
  };
  bool ok = true;
  if (nc == 1) {
    // one vector: matrix-vector products (bandwidth bound)
    auto gemv = [&](int m, int k, const double *Ap, int lda, const double *Xp, double *Yp,
                    const double *beta) {
      return gemv_n<double>(st, m, k, 1.0, Ap, lda, Xp, *beta, Yp) == DUST_OK;
    };
    if (nst == 0) {
      ok = gemv(n, n, A, n, X, Y, &zero);
    } else {
      ok = gemv(nst, nst, As, nst, X, Y, &zero);
      if (nmv > 0) {
        ok = ok && gemv(nst, nmv, A + (size_t)nst * n, n, X + nst, Y, &one);
        ok = ok && gemv(nmv, nst, A + nst, n, X, Y + nst, &zero);
        ok = ok && gemv(nmv, nmv, A + nst + (size_t)nst * n, n, X + nst, Y + nst, &one);
      }
    }
    return ok ? DUST_OK : DUST_ERR_CUDA;
  }
  if (nst == 0) {
    ok = gemm(n, n, A, n, X, Y, &zero);
  } else {
    ok = gemm(nst, nst, As, nst, X, Y, &zero);
    if (nmv > 0) {
      ok = ok && gemm(nst, nmv, A + (size_t)nst * n, n, X + nst, Y, &one);
      ok = ok && gemm(nmv, nst, A + nst, n, X, Y + nst, &zero);
      ok = ok && gemm(nmv, nmv, A + nst + (size_t)nst * n, n, X + nst, Y + nst, &one);
    }
  }
  return ok ? DUST_OK : DUST_ERR_CUDA;
}

__global__ void k_pc_pack(int n, int C, const double *dinv, const double *AZ, const double *Z,
                          const double *b, const double *x, float *Y, float *T) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)n * C) return;
  const int i = (int)(e / C), c = (int)(e % C);
  if (c < C - 1) {
    Y[e] = (float)(dinv[i] * AZ[i + (size_t)c * n]);
    T[e] = (float)Z[i + (size_t)c * n];
  } else {
    Y[e] = (float)(dinv[i] * b[i]);
    T[e] = (float)x[i];
  }
}

int pc_pack_sample(int n, int C, const double *dinv, const double *AZ, const double *Z,
                   const double *b, const double *x, float *Y, float *T, cudaStream_t st) {
  k_pc_pack<<<nblk((size_t)n * C, 256), 256, 0, st>>>(n, C, dinv, AZ, Z, b, x, Y, T);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}

__global__ void k_to_f32(int n, const double *a, float *b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}
__global__ void k_to_f64(int n, const float *a, double *b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (double)a[i];
}

// z = P v (see the file comment); tmp: 2 n doubles + 2 nst floats
static int gm_precond(dust_linsys *L, dust_precond *P, const double *v, double *z, char *tmp,
                      cudaStream_t st, cublasHandle_t cb) {
  const int n = L->n, nst = L->nst, nmv = L->nmv;
  if (nst == 0) {
    pc_apply(P, v, z, st);
    return DUST_OK;
  }
  double *t = (double *)tmp, *y = t + n;
  float *v32 = (float *)(y + n), *z32 = v32 + nst;
  k_to_f32<<<nblk(nst, 256), 256, 0, st>>>(nst, v, v32);
  DUST_TRY(gemv_n<float>(st, nst, nst, 1.0f, (const float *)L->ainv32.p, nst, v32, 0.0f, z32));
  k_to_f64<<<nblk(nst, 256), 256, 0, st>>>(nst, z32, z);
  if (nmv == 0) return DUST_OK;
  DUST_CUDA(cudaMemsetAsync(t, 0, (size_t)nst * 8, st));
  DUST_CUDA(cudaMemcpyAsync(t + nst, v + nst, (size_t)nmv * 8, cudaMemcpyDeviceToDevice, st));
  DUST_TRY(gemv_n<double>(st, nmv, nst, -1.0, (const double *)L->A.p + nst, n, z, 1.0, t + nst));
  pc_apply(P, t, y, st);
  DUST_CUDA(cudaMemcpyAsync(z + nst, y + nst, (size_t)nmv * 8, cudaMemcpyDeviceToDevice, st));
  return DUST_OK;
}

__global__ void k_scale(int n, double a, const double *x, double *y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = a * x[i];
}
__global__ void k_sub(int n, const double *b, const double *ax, double *r) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) r[i] = b[i] - ax[i];
}
__global__ void k_add(int n, const double *u, double *x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] += u[i];
}

int linsys_gmres_nn(dust_linsys *L, double *x, dust_solve_report *rep) {
  dust_precond *P = L->pc;
  if (!P || P->n != L->n) return DUST_ERR_NOT_CONVERGED;
  const int n = L->n, m = GM_RESTART;
  cudaStream_t st = L->st;
  cublasHandle_t cb = L->cb;
  cublasSetStream(cb, st);
  // the network runs on its own stream, ordered after the assembly
  cudaEvent_t ev;
  DUST_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  DUST_CUDA(cudaEventRecord(ev, st));
  DUST_CUDA(cudaStreamWaitEvent(P->st, ev, 0));
  int s = pc_infer(P, linsys_view(L));
  if (s == DUST_OK && cudaEventRecord(ev, P->st) != cudaSuccess) s = DUST_ERR_CUDA;
  if (s == DUST_OK && cudaStreamWaitEvent(st, ev, 0) != cudaSuccess) s = DUST_ERR_CUDA;
  cudaEventDestroy(ev);
  if (s != DUST_OK) return s;
  // V (n x (m+1)), z, w, r, u and the projections h (m+1) on the device
  if (L->nst > 0 && !L->ainv_ready) DUST_TRY(build_static_inverse(L));
  // hd: two Gram-Schmidt projections of m+1 and the new norm, read in one copy
  const size_t nhd = 2 * (size_t)(m + 1) + 2;
  DUST_TRY(devbuf_grow(L->kr, (size_t)n * 8 * (m + 1 + 6) + nhd * 8 + (size_t)L->nst * 8 + 512));
  double *V = (double *)L->kr.p, *z = V + (size_t)n * (m + 1), *w = z + n, *r = w + n,
         *u = r + n, *hd = u + n;
  char *ptmp = (char *)(hd + nhd);  // gm_precond scratch
  auto precond = [&](const double *v, double *out) { return gm_precond(L, P, v, out, ptmp, st, cb); };
  const double *b = (const double *)L->b.p;
  cublasSetPointerMode(cb, CUBLAS_POINTER_MODE_HOST);
  auto nrm2 = [&](const double *v, double *out) {  // synchronises the stream
    double h2[2];
    return vec_absmax_nrm2(st, n, v, hd + 2 * (m + 1)) == DUST_OK &&
           cudaMemcpyAsync(h2, hd + 2 * (m + 1), 16, cudaMemcpyDeviceToHost, st) == cudaSuccess &&
           cudaStreamSynchronize(st) == cudaSuccess && ((*out = h2[1]), true);
  };
  auto resid = [&]() -> int {  // r = b - A x
    DUST_TRY(linsys_matmat(L, 1, x, n, w, n, st, cb));
    k_sub<<<nblk(n, 256), 256, 0, st>>>(n, b, w, r);
    return DUST_OK;
  };
  double bnorm = 0.0;
  if (!nrm2(b, &bnorm)) return DUST_ERR_CUDA;
  if (bnorm == 0.0) {
    DUST_CUDA(cudaMemsetAsync(x, 0, (size_t)n * 8, st));
    if (rep) rep->mode_used = DUST_SOLVE_GMRES_NN;
    return DUST_OK;
  }
  DUST_TRY(precond(b, x));  // warm start x0 = P b
  DUST_TRY(resid());
  double beta = 0.0;
  if (!nrm2(r, &beta)) return DUST_ERR_CUDA;
  int it = 0;
  std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), y(m), hh(nhd);
  while (beta > GM_TOL * bnorm && it < GM_MAXIT) {
    k_scale<<<nblk(n, 256), 256, 0, st>>>(n, 1.0 / beta, r, V);
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int k = 0;
    bool done = false;
    while (k < m && it < GM_MAXIT && !done) {
      DUST_TRY(precond(V + (size_t)k * n, z));
      DUST_TRY(linsys_matmat(L, 1, z, n, w, n, st, cb));
      double *hc = &H[(size_t)k * (m + 1)];
      std::fill(hc, hc + m + 1, 0.0);
      // classical Gram-Schmidt, twice; both projections and the norm of the
      // result stay on the device until one copy to the host
      for (int pass = 0; pass < 2; ++pass) {
        double *hp = hd + (size_t)pass * (m + 1);
        DUST_TRY(gemv_t<double>(st, n, k + 1, 1.0, V, n, w, 0.0, hp));
        DUST_TRY(gemv_n<double>(st, n, k + 1, -1.0, V, n, hp, 1.0, w));
      }
      DUST_TRY(vec_absmax_nrm2(st, n, w, hd + 2 * (m + 1)));
      DUST_CUDA(cudaMemcpyAsync(hh.data(), hd, sizeof(double) * nhd, cudaMemcpyDeviceToHost, st));
      DUST_CUDA(cudaStreamSynchronize(st));
      for (int q = 0; q <= k; ++q) hc[q] = hh[q] + hh[(size_t)(m + 1) + q];
      const double hn = hh[2 * (size_t)(m + 1) + 1];
      hc[k + 1] = hn;
      if (hn > 0.0) k_scale<<<nblk(n, 256), 256, 0, st>>>(n, 1.0 / hn, w, V + (size_t)(k + 1) * n);
      // Givens rotations on the new column
      for (int q = 0; q < k; ++q) {
        const double t = cs[q] * hc[q] + sn[q] * hc[q + 1];
        hc[q + 1] = -sn[q] * hc[q] + cs[q] * hc[q + 1];
        hc[q] = t;
      }
      const double den = std::hypot(hc[k], hc[k + 1]);
      cs[k] = den > 0 ? hc[k] / den : 1.0;
      sn[k] = den > 0 ? hc[k + 1] / den : 0.0;
      hc[k] = den;
      hc[k + 1] = 0.0;
      g[k + 1] = -sn[k] * g[k];
      g[k] = cs[k] * g[k];
      ++k;
      ++it;
      if (std::fabs(g[k]) <= GM_TOL * bnorm || hn == 0.0) done = true;
    }
    // y = H(1:k,1:k) \ g(1:k); x += P (V y)
    for (int q = k - 1; q >= 0; --q) {
      double sum = g[q];
      for (int c = q + 1; c < k; ++c) sum -= H[(size_t)c * (m + 1) + q] * y[c];
      const double d = H[(size_t)q * (m + 1) + q];
      y[q] = d != 0.0 ? sum / d : 0.0;
    }
    DUST_CUDA(cudaMemcpyAsync(hd, y.data(), sizeof(double) * k, cudaMemcpyHostToDevice, st));
    DUST_TRY(gemv_n<double>(st, n, k, 1.0, V, n, hd, 0.0, u));
    DUST_TRY(precond(u, z));
    k_add<<<nblk(n, 256), 256, 0, st>>>(n, z, x);
    DUST_TRY(resid());
    if (!nrm2(r, &beta)) return DUST_ERR_CUDA;
  }
  DUST_CUDA(cudaGetLastError());
  if (rep) {
    rep->mode_used = DUST_SOLVE_GMRES_NN;
    rep->iterations = it;
    rep->residual = beta / bnorm;
  }
  return beta <= GM_TOL * bnorm ? DUST_OK : DUST_ERR_NOT_CONVERGED;
}
