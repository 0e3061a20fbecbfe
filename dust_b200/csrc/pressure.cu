// pressure.cu -- the pressure integral equation of the reference, on the GPU.
//
//   src/linsys/mod_linsys.f90            A_pres: the surface-panel block of A
//                                        before the wake correction (:184-187
//                                        at initialize_linsys, :318-323 at
//                                        assemble_linsys); LU of its static
//                                        block once (:250-257)
//   src/linsys/mod_pressure_equation.f90 initialize_pressure_sys :44-79,
//                                        assemble_pressure_sys :139-235,
//                                        solve_pressure_sys :243-387
//   src/aeroel/mod_surfpan.f90           build_row_surfpan :396-437 (the
//                                        Bernoulli source terms of b_pres)
//
// The system is the surface-panel sub-block of the influence matrix
// (surface panels keep the element order, static first).  Its right-hand
// side adds to the Bernoulli source terms (caller-supplied sources times the
// source-potential influence) the rotational terms: every particle
//   dist . (dir x vel) mag / (|dist|^2 + r_v^2)^(3/2),  dist = x_p - centre,
// an O(n_sp x N) direct sum evaluated like the uvort sum (particles staged
// in shared memory, several centres per thread, chunks of particles over
// blockIdx.y added atomically; FP64, or with the system's DUST_PREC_FP32C
// packed FP32 pairs on Morton-sorted, tile-relative coordinates with FP64
// accumulation across tiles), and the edges of the end vortices and
// wake panels with their vertex velocities (one thread per row).  The solve
// is solve_linsys's sequence on A_pres (static LU reused, Schur update and
// LU of the moving block, getrs), through the same code as the main system.
#include <cublas_v2.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "dust_common.cuh"
#include "elements.cuh"
#include "fmm_internal.h"
#include "linsys_internal.h"
#include "lu.cuh"

static inline unsigned nblk(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

struct dust_pressure {
  int n = 0, nsp = 0, nsst = 0, nst = 0;  // elements, surface panels, static ones
  std::vector<int> h_id;
  DevBuf id, g2l, bsp, kinds;
  DevBuf sort;               // Morton-sorted particle copy of the FP32C sum
  DevBuf stage;              // device copies of the host-array entry points' inputs
  dust_linsys *S = nullptr;  // the pressure system as a linear-system object
};

__global__ void k_kinds(int n, const PanelGeo *el, int *kind) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) kind[j] = el[j].kind;
}

// A_pres(i, j) = -dou of surface panel id[j] at the centre of id[i] (the
// diagonal -(-2 pi)); with bsp, the source potential b1 too (static block)
#define PA_RX 32
#define PA_CY 8
__global__ void __launch_bounds__(PA_RX *PA_CY)
    k_pres_aic(const PanelGeo *__restrict__ el, const int *__restrict__ id, RegParams rp, int r0,
               int r1, int c0, int c1, double *A, int lda, double *bsp, int ldb) {
  __shared__ PanelGeo s_col[PA_CY];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i = r0 + blockIdx.x * PA_RX + tx;
  const int jc0 = c0 + blockIdx.y * PA_CY;
  const int words = sizeof(PanelGeo) / 8;
  for (int w = ty * PA_RX + tx; w < PA_CY * words; w += PA_RX * PA_CY) {
    int q = w / words, ww = w % words;
    int j = jc0 + q;
    if (j < c1) ((double *)&s_col[q])[ww] = ((const double *)(el + id[j]))[ww];
  }
  __syncthreads();
  const int j = jc0 + ty;
  if (i >= r1 || j >= c1) return;
  const int gi = id[i], gj = id[j];
  const double *pos = el[gi].cen;
  const double dou = gi != gj ? pot_dou(rp, s_col[ty], pos) : -2.0 * DUST_PI;
  A[(size_t)i + (size_t)j * lda] = -dou;
  if (bsp) bsp[(size_t)i + (size_t)j * ldb] = pot_sou(s_col[ty], dou, pos);
}

// Bernoulli source terms of build_row_surfpan (:396-437), one warp per row:
// static rows: sum_j<nsst bsp(i, j) src(j) + moving surface panels' b1 src;
// moving rows: every surface panel's b1 src.
__global__ void k_pres_bern(const PanelGeo *__restrict__ el, const int *__restrict__ id,
                            const int *__restrict__ g2l, RegParams rp, int nsp, int nsst, int nst,
                            int n, const double *bsp, const double *src, double *b) {
  const int lane = threadIdx.x & 31;
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= nsp) return;
  const int gi = id[i];
  const bool st = gi < nst;
  const double *pos = el[gi].cen;
  double s = 0.0;
  if (st)
    for (int j = lane; j < nsst; j += 32) s += bsp[(size_t)i + (size_t)j * nsst] * src[j];
  for (int gj = (st ? nst : 0) + lane; gj < n; gj += 32) {
    const int lj = g2l[gj];
    if (lj < 0) continue;
    const double dou = gi != gj ? pot_dou(rp, el[gj], pos) : -2.0 * DUST_PI;
    s += pot_sou(el[gj], dou, pos) * src[lj];
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) b[i] = s;
}

__device__ __forceinline__ double rsqrt_p(double x) {
  // FP32 seed, one Householder step in FP64: relative error at the FP64
  // rounding level for a normal FP32-range x > 0
  const double y = (double)rsqrtf((float)x);
  const double e = fma(-x * y, y, 1.0);
  return fma(y * e, fma(0.375, e, 0.5), y);
}

// (c.1) particles (:170-186): a tile of particles (x, w = mag dir x vel,
// r_v^2) in shared memory, PR_PPT centres per thread
#define PR_T 128
#define PR_TILE 128
#define PR_PPT 4
__global__ void __launch_bounds__(PR_T) k_pres_particles(const PanelGeo *__restrict__ el,
                                                         const int *__restrict__ id, int nsp,
                                                         int n, const double *cen,
                                                         const double *dir, const double *mag,
                                                         const double *rv, const double *vel,
                                                         int chunk, double *b) {
  __shared__ double s_q[PR_TILE][8];
  const int t0 = blockIdx.x * PR_T * PR_PPT + threadIdx.x;
  const int q_lo = blockIdx.y * chunk, q_hi = min(n, q_lo + chunk);
  double pos[PR_PPT][3], acc[PR_PPT];
#pragma unroll
  for (int k = 0; k < PR_PPT; ++k) {
    const int t = t0 + k * PR_T;
    for (int c = 0; c < 3; ++c) pos[k][c] = t < nsp ? el[id[t]].cen[c] : 0.0;
    acc[k] = 0.0;
  }
  for (int q0 = q_lo; q0 < q_hi; q0 += PR_TILE) {
    __syncthreads();
    const int m = min(PR_TILE, q_hi - q0);
    if ((int)threadIdx.x < m) {
      const int q = q0 + threadIdx.x;
      const double *d = dir + 3 * (size_t)q, *v = vel + 3 * (size_t)q;
      const double mg = mag[q], r = rv[q];
      double *w = s_q[threadIdx.x];
      w[0] = cen[3 * (size_t)q];
      w[1] = cen[3 * (size_t)q + 1];
      w[2] = cen[3 * (size_t)q + 2];
      w[3] = r * r;
      w[4] = mg * (d[1] * v[2] - d[2] * v[1]);
      w[5] = mg * (d[2] * v[0] - d[0] * v[2]);
      w[6] = mg * (d[0] * v[1] - d[1] * v[0]);
    }
    __syncthreads();
#pragma unroll 2
    for (int u = 0; u < m; ++u) {
      const double2 *w = (const double2 *)s_q[u];
      const double2 X = w[0], Y = w[1], Z = w[2], P = w[3];
      // X = (x, y), Y = (z, r_v^2), Z = (wx, wy), P = (wz, -)
#pragma unroll
      for (int k = 0; k < PR_PPT; ++k) {
        const double dx = X.x - pos[k][0], dy = X.y - pos[k][1], dz = Y.x - pos[k][2];
        const double r2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, Y.y)));
        const double ir = rsqrt_p(r2);
        const double dw = fma(dx, Z.x, fma(dy, Z.y, dz * P.x));
        acc[k] = fma(dw * ir, ir * ir, acc[k]);
      }
    }
  }
#pragma unroll
  for (int k = 0; k < PR_PPT; ++k) {
    const int t = t0 + k * PR_T;
    if (t < nsp) atomicAdd(b + t, acc[k]);
  }
}

// FP32C form of (c.1) on Morton-sorted particles: a tile of 128 consecutive
// sorted particles is spatially compact, so coordinates relative to the
// tile's first particle are rounded to FP32 once per tile; pairs of
// particles are evaluated together in packed FP32 (f32x2), partial sums of a
// tile in FP32 added into FP64.  Sorted block: X (double, 3 n), F (float:
// -w x, -w y, -w z, r_v^2; w = mag dir x vel).
__global__ void k_pres_gather(int n, const uint32_t *perm, const double *cen, const double *dir,
                              const double *mag, const double *rv, const double *vel,
                              double *X, float *F) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const uint32_t q = perm[t];
  const double *d = dir + 3 * (size_t)q, *v = vel + 3 * (size_t)q;
  const double m = mag[q];
  for (int k = 0; k < 3; ++k) X[(size_t)k * n + t] = cen[3 * (size_t)q + k];
  F[t] = (float)(-m * (d[1] * v[2] - d[2] * v[1]));
  F[(size_t)n + t] = (float)(-m * (d[2] * v[0] - d[0] * v[2]));
  F[2 * (size_t)n + t] = (float)(-m * (d[0] * v[1] - d[1] * v[0]));
  F[3 * (size_t)n + t] = (float)(rv[q] * rv[q]);
}

#define PF_T 128
#define PF_TILE 128
#define PF_PPT 4
__global__ void __launch_bounds__(PF_T) k_pres_particles_f32(const PanelGeo *__restrict__ el,
                                                             const int *__restrict__ id, int nsp,
                                                             int n, const double *X,
                                                             const float *F, int chunk,
                                                             double *b) {
  // value k of particle q at [q / 2][2 k + q % 2]: -x, -y, -z (tile-relative),
  // r_v^2, -w (three)
  __shared__ __align__(16) float s_pk[PF_TILE / 2][16];
  __shared__ double s_ref[3];
  int t[PF_PPT];
  double pos[PF_PPT][3], acc[PF_PPT];
#pragma unroll
  for (int k = 0; k < PF_PPT; ++k) {
    t[k] = (blockIdx.x * PF_PPT + k) * PF_T + threadIdx.x;
    for (int c = 0; c < 3; ++c) pos[k][c] = t[k] < nsp ? el[id[t[k]]].cen[c] : 0.0;
    acc[k] = 0.0;
  }
  const int q_lo = blockIdx.y * chunk, q_hi = min(n, q_lo + chunk);
  for (int q0 = q_lo; q0 < q_hi; q0 += PF_TILE) {
    __syncthreads();
    const int q = q0 + threadIdx.x;
    const int m = min(PF_TILE, q_hi - q0);
    if (threadIdx.x < 3) s_ref[threadIdx.x] = X[(size_t)threadIdx.x * n + q0];
    __syncthreads();
    {
      // particles beyond the chunk: far away, no strength
      float val[8] = {-1.0e6f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f, 0.f};
      if ((int)threadIdx.x < m) {
        val[0] = (float)(s_ref[0] - X[q]);
        val[1] = (float)(s_ref[1] - X[(size_t)n + q]);
        val[2] = (float)(s_ref[2] - X[2 * (size_t)n + q]);
        val[3] = F[3 * (size_t)n + q];
        val[4] = F[q];
        val[5] = F[(size_t)n + q];
        val[6] = F[2 * (size_t)n + q];
      }
      for (int k = 0; k < 8; ++k) s_pk[threadIdx.x >> 1][2 * k + (threadIdx.x & 1)] = val[k];
    }
    __syncthreads();
    float px[PF_PPT], py[PF_PPT], pz[PF_PPT];
    float2 V[PF_PPT];
#pragma unroll
    for (int k = 0; k < PF_PPT; ++k) {
      px[k] = (float)(pos[k][0] - s_ref[0]);
      py[k] = (float)(pos[k][1] - s_ref[1]);
      pz[k] = (float)(pos[k][2] - s_ref[2]);
      V[k] = make_float2(0.f, 0.f);
    }
    const int mp = (m + 1) >> 1;
#pragma unroll 2
    for (int u = 0; u < mp; ++u) {
      const float4 P0 = *(const float4 *)&s_pk[u][0], P1 = *(const float4 *)&s_pk[u][4],
                   P2 = *(const float4 *)&s_pk[u][8], P3 = *(const float4 *)&s_pk[u][12];
      const float2 nx = make_float2(P0.x, P0.y), ny = make_float2(P0.z, P0.w),
                   nz = make_float2(P1.x, P1.y), s2 = make_float2(P1.z, P1.w),
                   wx = make_float2(P2.x, P2.y), wy = make_float2(P2.z, P2.w),
                   wz = make_float2(P3.x, P3.y);
#pragma unroll
      for (int k = 0; k < PF_PPT; ++k) {
        // d = centre - x_q; (x_q - centre) . w = d . (-w)
        const float2 dx = __fadd2_rn(make_float2(px[k], px[k]), nx),
                     dy = __fadd2_rn(make_float2(py[k], py[k]), ny),
                     dz = __fadd2_rn(make_float2(pz[k], pz[k]), nz);
        const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, s2)));
        const float2 ir = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
        const float2 c = __fmul2_rn(__fmul2_rn(ir, ir), ir);
        const float2 dw = __ffma2_rn(dx, wx, __ffma2_rn(dy, wy, __fmul2_rn(dz, wz)));
        V[k] = __ffma2_rn(c, dw, V[k]);
      }
    }
#pragma unroll
    for (int k = 0; k < PF_PPT; ++k) acc[k] += (double)(V[k].x + V[k].y);
  }
#pragma unroll
  for (int k = 0; k < PF_PPT; ++k)
    if (t[k] < nsp) atomicAdd(b + t[k], acc[k]);
}

// one edge term: -0.5 mag edge . (d1 x v1 / |d1|^3 + d2 x v2 / |d2|^3)
__device__ __forceinline__ double edge_term(const double *p1, const double *p2,
                                            const double *v1, const double *v2,
                                            const double *c) {
  double d1[3], d2[3];
  for (int k = 0; k < 3; ++k) {
    d1[k] = p1[k] - c[k];
    d2[k] = p2[k] - c[k];
  }
  const double c1[3] = {d1[1] * v1[2] - d1[2] * v1[1], d1[2] * v1[0] - d1[0] * v1[2],
                        d1[0] * v1[1] - d1[1] * v1[0]};
  const double c2[3] = {d2[1] * v2[2] - d2[2] * v2[1], d2[2] * v2[0] - d2[0] * v2[2],
                        d2[0] * v2[1] - d2[1] * v2[0]};
  const double n1 = sqrt(d1[0] * d1[0] + d1[1] * d1[1] + d1[2] * d1[2]);
  const double n2 = sqrt(d2[0] * d2[0] + d2[1] * d2[1] + d2[2] * d2[2]);
  const double n13 = n1 * n1 * n1, n23 = n2 * n2 * n2;
  double t = 0.0;
  for (int k = 0; k < 3; ++k) t += (p2[k] - p1[k]) * (c1[k] / n13 + c2[k] / n23);
  return t;
}

// (c.2) end vortices and (c.3) wake panels (:188-226), one thread per row
__global__ void k_pres_wake(const PanelGeo *__restrict__ el, const int *__restrict__ id, int nsp,
                            int nw, const int *wnv, const double *wver, const double *wmag,
                            const double *wvv, int ne, const double *ever, const double *emag,
                            const double *evv, double *b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nsp) return;
  const double *c = el[id[i]].cen;
  double s = 0.0;
  for (int j = 0; j < ne; ++j) {
    const double *v = ever + 6 * (size_t)j, *u = evv + 6 * (size_t)j;
    s -= 0.5 * emag[j] * edge_term(v, v + 3, u, u + 3, c);
  }
  for (int j = 0; j < nw; ++j) {
    const int nv = wnv ? wnv[j] : 4;
    const double *v = wver + 12 * (size_t)j, *u = wvv + 12 * (size_t)j;
    const double m = wmag ? wmag[j] : 0.0;
    double t = 0.0;
    for (int e = 0; e < nv; ++e) {
      const int en = (e + 1) % nv;
      t += edge_term(v + 3 * e, v + 3 * en, u + 3 * e, u + 3 * en, c);
    }
    s -= 0.5 * m * t;
  }
  if (s != 0.0) atomicAdd(b + i, s);
}

// ------------------------------------------------------------ entry points
static void pressure_free(dust_pressure *p) {
  if (!p) return;
  devbuf_free(p->id);
  devbuf_free(p->g2l);
  devbuf_free(p->bsp);
  devbuf_free(p->kinds);
  devbuf_free(p->sort);
  devbuf_free(p->stage);
  if (p->S) dust_linsys_destroy(p->S);
  delete p;
}

extern "C" int dust_pressure_create(dust_linsys *ls, dust_pressure **out) {
  if (!ls || !out || !ls->el) return DUST_ERR_BAD_ARG;
  *out = nullptr;
  dust_pressure *p = new dust_pressure();
  p->n = ls->n;
  p->nst = ls->nst;
  cudaStream_t st = ls->st;
  int s = devbuf_grow(p->kinds, (size_t)p->n * 4);
  if (s != DUST_OK) {
    pressure_free(p);
    return s;
  }
  k_kinds<<<nblk(p->n, 128), 128, 0, st>>>(p->n, ls->el, (int *)p->kinds.p);
  std::vector<int> kind(p->n), g2l(p->n, -1);
  if (cudaMemcpyAsync(kind.data(), p->kinds.p, (size_t)p->n * 4, cudaMemcpyDeviceToHost, st) !=
          cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess) {
    pressure_free(p);
    return DUST_ERR_CUDA;
  }
  for (int j = 0; j < p->n; ++j)
    if (kind[j] == DUST_ELEM_SURFPAN) {
      g2l[j] = (int)p->h_id.size();
      p->h_id.push_back(j);
      if (j < p->nst) ++p->nsst;
    }
  p->nsp = (int)p->h_id.size();
  const int nsp = p->nsp, nsst = p->nsst;
  if (nsp == 0) {
    *out = p;
    return DUST_OK;
  }
  // the pressure system as a linear-system object: A, b, pivots, LU work
  dust_linsys *S = new dust_linsys();
  p->S = S;
  S->n = nsp;
  S->nst = nsst;
  S->nmv = nsp - nsst;
  S->prm = ls->prm;
  S->rp = ls->rp;
  if (cudaStreamCreateWithFlags(&S->st, cudaStreamNonBlocking) != cudaSuccess ||
      cublasCreate(&S->cb) != CUBLAS_STATUS_SUCCESS) {
    pressure_free(p);
    return DUST_ERR_CUDA;
  }
  cublasSetStream(S->cb, S->st);
  const size_t N = nsp, NS = std::max(nsst, 1);
  if ((s = devbuf_grow(S->A, N * N * 8)) || (s = devbuf_grow(S->b, N * 8 * 4)) ||
      (s = devbuf_grow(S->piv, N * 4 + 64)) || (s = devbuf_grow(S->info, 64)) ||
      (s = devbuf_grow(p->id, N * 4)) || (s = devbuf_grow(p->g2l, (size_t)p->n * 4)) ||
      (s = devbuf_grow(p->bsp, NS * NS * 8)) ||
      (nsst > 0 && (s = devbuf_grow(S->As, (size_t)nsst * nsst * 8)))) {
    pressure_free(p);
    return s;
  }
  // ordered after the linsys' own work
  if (cudaStreamSynchronize(st) != cudaSuccess ||
      cudaMemcpyAsync(p->id.p, p->h_id.data(), N * 4, cudaMemcpyHostToDevice, S->st) !=
          cudaSuccess ||
      cudaMemcpyAsync(p->g2l.p, g2l.data(), (size_t)p->n * 4, cudaMemcpyHostToDevice, S->st) !=
          cudaSuccess ||
      cudaMemsetAsync(S->A.p, 0, N * N * 8, S->st) != cudaSuccess) {
    pressure_free(p);
    return DUST_ERR_CUDA;
  }
  if (nsst > 0) {
    // initialize_linsys / initialize_pressure_sys: static block, b_static_pres,
    // LU of the static block once
    dim3 blk(PA_RX, PA_CY), grd(nblk(nsst, PA_RX), nblk(nsst, PA_CY));
    k_pres_aic<<<grd, blk, 0, S->st>>>(ls->el, (const int *)p->id.p, ls->rp, 0, nsst, 0, nsst,
                                       (double *)S->A.p, nsp, (double *)p->bsp.p, nsst);
    cudaMemcpy2DAsync(S->As.p, (size_t)nsst * 8, S->A.p, N * 8, (size_t)nsst * 8, nsst,
                      cudaMemcpyDeviceToDevice, S->st);
    s = lu_getrf_auto<double>(
        S->cb, S->st, S->lu, nsst, (double *)S->A.p, nsp, (int *)S->piv.p, (int *)S->info.p, 0,
        nullptr, 1e-8,
        [&]() -> int {
          DUST_CUDA(cudaMemcpy2DAsync(S->A.p, N * 8, S->As.p, (size_t)nsst * 8,
                                      (size_t)nsst * 8, nsst, cudaMemcpyDeviceToDevice, S->st));
          return DUST_OK;
        },
        &S->static_pivoted);
    if (s == DUST_OK) {
      int info = 0;
      if (cudaMemcpy(&info, S->info.p, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        s = DUST_ERR_CUDA;
      else if (info)
        s = DUST_ERR_SINGULAR;
    }
  }
  if (s == DUST_OK && cudaStreamSynchronize(S->st) != cudaSuccess) s = DUST_ERR_CUDA;
  if (s != DUST_OK) {
    pressure_free(p);
    return s;
  }
  *out = p;
  return DUST_OK;
}

extern "C" int dust_pressure_destroy(dust_pressure *p) {
  pressure_free(p);
  return DUST_OK;
}

extern "C" int dust_pressure_size(const dust_pressure *p, int *n_sp, int *nstatic_sp) {
  if (!p) return DUST_ERR_BAD_ARG;
  if (n_sp) *n_sp = p->nsp;
  if (nstatic_sp) *nstatic_sp = p->nsst;
  return DUST_OK;
}

// b[i] += term[id[i]]: the particle term evaluated at the element centres
__global__ void k_pres_add_term(int nsp, const int *id, const double *term, double *b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nsp) b[i] += term[id[i]];
}

static int pres_assemble(dust_pressure *p, const dust_linsys *ls, const double *bern, int n,
                         const double *cen, const double *dir, const double *mag,
                         const double *r_vortex, const double *vel, const double *pterm,
                         const dust_panels *wake, const double *wake_vv,
                         const dust_lines *end_vort, const double *end_vv, void *stream);

extern "C" int dust_pressure_assemble_device(dust_pressure *p, const dust_linsys *ls,
                                             const double *bern, int n, const double *cen,
                                             const double *dir, const double *mag,
                                             const double *r_vortex, const double *vel,
                                             const dust_panels *wake, const double *wake_vv,
                                             const dust_lines *end_vort, const double *end_vv,
                                             void *stream) {
  return pres_assemble(p, ls, bern, n, cen, dir, mag, r_vortex, vel, nullptr, wake, wake_vv,
                       end_vort, end_vv, stream);
}

extern "C" int dust_pressure_assemble_terms_device(dust_pressure *p, const dust_linsys *ls,
                                                   const double *bern, const double *pterm,
                                                   const dust_panels *wake,
                                                   const double *wake_vv,
                                                   const dust_lines *end_vort,
                                                   const double *end_vv, void *stream) {
  if (!pterm) return DUST_ERR_BAD_ARG;
  return pres_assemble(p, ls, bern, 0, nullptr, nullptr, nullptr, nullptr, nullptr, pterm, wake,
                       wake_vv, end_vort, end_vv, stream);
}

static int pres_assemble(dust_pressure *p, const dust_linsys *ls, const double *bern, int n,
                         const double *cen, const double *dir, const double *mag,
                         const double *r_vortex, const double *vel, const double *pterm,
                         const dust_panels *wake, const double *wake_vv,
                         const dust_lines *end_vort, const double *end_vv, void *stream) {
  if (!p || !ls || !ls->el || ls->n != p->n || n < 0) return DUST_ERR_BAD_ARG;
  if (n > 0 && (!cen || !dir || !mag || !r_vortex || !vel)) return DUST_ERR_BAD_ARG;
  const int nw = wake ? wake->n : 0, ne = end_vort ? end_vort->n : 0;
  if (nw < 0 || ne < 0 || (nw > 0 && (!wake->ver || !wake_vv)) ||
      (ne > 0 && (!end_vort->ver || !end_vort->mag || !end_vv)))
    return DUST_ERR_BAD_ARG;
  if (p->nsp == 0) return DUST_OK;
  dust_linsys *S = p->S;
  cudaStream_t st = (cudaStream_t)stream;
  // the caller's stream and the linsys' assembly come first
  DUST_CUDA(cudaStreamSynchronize(ls->st));
  const int nsp = p->nsp, nsst = p->nsst;
  const int *id = (const int *)p->id.p;
  double *A = (double *)S->A.p, *b = (double *)S->b.p;
  // assemble_linsys :318-323: static rows x moving columns, moving rows x all
  dim3 blk(PA_RX, PA_CY);
  if (nsst > 0 && nsp > nsst)
    k_pres_aic<<<dim3(nblk(nsst, PA_RX), nblk(nsp - nsst, PA_CY)), blk, 0, st>>>(
        ls->el, id, ls->rp, 0, nsst, nsst, nsp, A, nsp, nullptr, 0);
  if (nsp > nsst)
    k_pres_aic<<<dim3(nblk(nsp - nsst, PA_RX), nblk(nsp, PA_CY)), blk, 0, st>>>(
        ls->el, id, ls->rp, nsst, nsp, 0, nsp, A, nsp, nullptr, 0);
  // b_pres: Bernoulli source terms (or zero), then the rotational terms
  if (bern)
    k_pres_bern<<<nblk((size_t)nsp * 32, 128), 128, 0, st>>>(
        ls->el, id, (const int *)p->g2l.p, ls->rp, nsp, nsst, ls->nst, p->n,
        (const double *)p->bsp.p, bern, b);
  else
    DUST_CUDA(cudaMemsetAsync(b, 0, (size_t)nsp * 8, st));
  if (n > 0 && ls->prm.precision == DUST_PREC_FP32C) {
    uint32_t *perm = nullptr;
    size_t used = morton_perm_bytes(n, st);
    const size_t N = (size_t)n;
    const size_t off_x = used, off_f = off_x + (24 * N + 255) / 256 * 256;
    DUST_TRY(devbuf_grow(p->sort, off_f + 16 * N + 256));
    DUST_TRY(morton_perm(&ls->prm, n, cen, p->sort, &perm, &used, st));
    double *X = (double *)((char *)p->sort.p + off_x);
    float *F = (float *)((char *)p->sort.p + off_f);
    k_pres_gather<<<nblk(n, 256), 256, 0, st>>>(n, perm, cen, dir, mag, r_vortex, vel, X, F);
    const int nbx = (int)nblk(nsp, PF_T * PF_PPT);
    const int target = 148 * 8;
    int ny = std::max(1, std::min((n + PF_TILE - 1) / PF_TILE, (target + nbx - 1) / nbx));
    int chunk = (n + ny - 1) / ny;
    chunk = (chunk + PF_TILE - 1) / PF_TILE * PF_TILE;
    ny = (n + chunk - 1) / chunk;
    k_pres_particles_f32<<<dim3(nbx, ny), PF_T, 0, st>>>(ls->el, id, nsp, n, X, F, chunk, b);
  } else if (n > 0) {
    const int nbx = (int)nblk(nsp, PR_T * PR_PPT);
    const int target = 148 * 8;
    int ny = std::max(1, std::min((n + PR_TILE - 1) / PR_TILE, (target + nbx - 1) / nbx));
    int chunk = (n + ny - 1) / ny;
    chunk = (chunk + PR_TILE - 1) / PR_TILE * PR_TILE;
    ny = (n + chunk - 1) / chunk;
    k_pres_particles<<<dim3(nbx, ny), PR_T, 0, st>>>(ls->el, id, nsp, n, cen, dir, mag,
                                                     r_vortex, vel, chunk, b);
  }
  if (pterm) k_pres_add_term<<<nblk(nsp, 128), 128, 0, st>>>(nsp, id, pterm, b);
  if (nw + ne > 0)
    k_pres_wake<<<nblk(nsp, 128), 128, 0, st>>>(ls->el, id, nsp, nw, wake ? wake->n_ver : nullptr,
                                                wake ? wake->ver : nullptr,
                                                wake ? wake->mag : nullptr, wake_vv, ne,
                                                end_vort ? end_vort->ver : nullptr,
                                                end_vort ? end_vort->mag : nullptr, end_vv, b);
  DUST_CUDA(cudaGetLastError());
  DUST_CUDA(cudaStreamSynchronize(st));
  S->assembled = true;
  S->factored = false;
  return DUST_OK;
}

extern "C" int dust_pressure_solve_device(dust_pressure *p, double *res, void *stream) {
  if (!p || !res) return DUST_ERR_BAD_ARG;
  if (p->nsp == 0) return DUST_OK;
  dust_linsys *S = p->S;
  if (!S->assembled || S->factored) return DUST_ERR_BAD_ARG;  // assemble before every solve
  (void)stream;
  DUST_TRY(linsys_solve_lu64(S, res));
  DUST_CUDA(cudaStreamSynchronize(S->st));
  return DUST_OK;
}

extern "C" int dust_pressure_get_system(dust_pressure *p, double *A, double *b) {
  if (!p) return DUST_ERR_BAD_ARG;
  if (p->nsp == 0) return DUST_OK;
  dust_linsys *S = p->S;
  if (!S->assembled || S->factored) return DUST_ERR_BAD_ARG;
  const size_t N = p->nsp;
  if (A) DUST_CUDA(cudaMemcpy(A, S->A.p, N * N * 8, cudaMemcpyDeviceToHost));
  if (b) DUST_CUDA(cudaMemcpy(b, S->b.p, N * 8, cudaMemcpyDeviceToHost));
  return DUST_OK;
}

// Host-array variants: the inputs are copied to the device (one staging
// buffer kept by the handle), the solution back to the host.  pterm (host,
// rank values) replaces the particle arrays when the particles' term was
// evaluated with uvort (dust_points_uvort_pressure).
static int pres_assemble_host(dust_pressure *p, const dust_linsys *ls, const double *bern, int n,
                              const double *cen, const double *dir, const double *mag,
                              const double *r_vortex, const double *vel, const double *pterm,
                              const dust_panels *wake, const double *wake_vv,
                              const dust_lines *end_vort, const double *end_vv) {
  if (!p || !ls || n < 0) return DUST_ERR_BAD_ARG;
  if (n > 0 && (!cen || !dir || !mag || !r_vortex || !vel)) return DUST_ERR_BAD_ARG;
  const int nw = wake ? wake->n : 0, ne = end_vort ? end_vort->n : 0;
  if (nw < 0 || ne < 0 || (nw > 0 && (!wake->ver || !wake_vv)) ||
      (ne > 0 && (!end_vort->ver || !end_vort->mag || !end_vv)))
    return DUST_ERR_BAD_ARG;
  if (p->nsp == 0) return DUST_OK;
  const size_t N = (size_t)n, R = pterm ? (size_t)ls->n : 0;
  auto al = [](size_t b) { return (b + 255) / 256 * 256; };
  size_t off = 0;
  const size_t o_b = off; off += al((bern ? p->nsp : 0) * 8);
  const size_t o_c = off; off += al(24 * N);
  const size_t o_d = off; off += al(24 * N);
  const size_t o_m = off; off += al(8 * N);
  const size_t o_r = off; off += al(8 * N);
  const size_t o_v = off; off += al(24 * N);
  const size_t o_pt = off; off += al(8 * R);
  const size_t o_wv = off; off += al(96 * (size_t)nw);
  const size_t o_wn = off; off += al(4 * (size_t)nw);
  const size_t o_wm = off; off += al(8 * (size_t)nw);
  const size_t o_wvv = off; off += al(96 * (size_t)nw);
  const size_t o_ev = off; off += al(48 * (size_t)ne);
  const size_t o_em = off; off += al(8 * (size_t)ne);
  const size_t o_evv = off; off += al(48 * (size_t)ne);
  DUST_TRY(devbuf_grow(p->stage, off + 256));
  char *s = (char *)p->stage.p;
  cudaStream_t st = p->S->st;
  auto put = [&](size_t o, const void *src, size_t bytes) -> int {
    if (!src || bytes == 0) return DUST_OK;
    DUST_CUDA(cudaMemcpyAsync(s + o, src, bytes, cudaMemcpyHostToDevice, st));
    return DUST_OK;
  };
  DUST_TRY(put(o_b, bern, (bern ? p->nsp : 0) * 8));
  DUST_TRY(put(o_c, cen, 24 * N));
  DUST_TRY(put(o_d, dir, 24 * N));
  DUST_TRY(put(o_m, mag, 8 * N));
  DUST_TRY(put(o_r, r_vortex, 8 * N));
  DUST_TRY(put(o_v, vel, 24 * N));
  DUST_TRY(put(o_pt, pterm, 8 * R));
  dust_panels dw;
  dust_lines de;
  memset(&dw, 0, sizeof(dw));
  memset(&de, 0, sizeof(de));
  if (nw > 0) {
    DUST_TRY(put(o_wv, wake->ver, 96 * (size_t)nw));
    DUST_TRY(put(o_wn, wake->n_ver, 4 * (size_t)nw));
    DUST_TRY(put(o_wm, wake->mag, 8 * (size_t)nw));
    DUST_TRY(put(o_wvv, wake_vv, 96 * (size_t)nw));
    dw.n = nw;
    dw.ver = (const double *)(s + o_wv);
    dw.n_ver = wake->n_ver ? (const int *)(s + o_wn) : nullptr;
    dw.mag = wake->mag ? (const double *)(s + o_wm) : nullptr;
  }
  if (ne > 0) {
    DUST_TRY(put(o_ev, end_vort->ver, 48 * (size_t)ne));
    DUST_TRY(put(o_em, end_vort->mag, 8 * (size_t)ne));
    DUST_TRY(put(o_evv, end_vv, 48 * (size_t)ne));
    de.n = ne;
    de.ver = (const double *)(s + o_ev);
    de.mag = (const double *)(s + o_em);
  }
  auto D = [&](size_t o, const void *h) { return h ? (const double *)(s + o) : nullptr; };
  return pres_assemble(p, ls, D(o_b, bern), n, D(o_c, cen), D(o_d, dir), D(o_m, mag),
                       D(o_r, r_vortex), D(o_v, vel), D(o_pt, pterm), nw > 0 ? &dw : nullptr,
                       D(o_wvv, nw > 0 ? wake_vv : nullptr), ne > 0 ? &de : nullptr,
                       D(o_evv, ne > 0 ? end_vv : nullptr), st);
}

extern "C" int dust_pressure_assemble(dust_pressure *p, const dust_linsys *ls, const double *bern,
                                      int n, const double *cen, const double *dir,
                                      const double *mag, const double *r_vortex,
                                      const double *vel, const dust_panels *wake,
                                      const double *wake_vv, const dust_lines *end_vort,
                                      const double *end_vv) {
  return pres_assemble_host(p, ls, bern, n, cen, dir, mag, r_vortex, vel, nullptr, wake, wake_vv,
                            end_vort, end_vv);
}

extern "C" int dust_pressure_assemble_terms(dust_pressure *p, const dust_linsys *ls,
                                            const double *bern, const double *pterm,
                                            const dust_panels *wake, const double *wake_vv,
                                            const dust_lines *end_vort, const double *end_vv) {
  if (!pterm) return DUST_ERR_BAD_ARG;
  return pres_assemble_host(p, ls, bern, 0, nullptr, nullptr, nullptr, nullptr, nullptr, pterm,
                            wake, wake_vv, end_vort, end_vv);
}

extern "C" int dust_pressure_solve(dust_pressure *p, double *res) {
  if (!p || !res) return DUST_ERR_BAD_ARG;
  if (p->nsp == 0) return DUST_OK;
  DUST_TRY(devbuf_grow(p->stage, (size_t)p->nsp * 8 + 256));
  double *x = (double *)p->stage.p;
  DUST_TRY(dust_pressure_solve_device(p, x, nullptr));
  DUST_CUDA(cudaMemcpy(res, x, (size_t)p->nsp * 8, cudaMemcpyDeviceToHost));
  return DUST_OK;
}
