// gnn.cu -- learned sparse approximate inverse for the moving-body system.
//
// The influence matrix of a moving-body case changes every step
// (build_row_*, mod_linsys.f90:279-344), so the reference refactors its
// moving part each step (solve_linsys, :352-482).  Here a small graph
// network over the panels' k-nearest-neighbour graph emits, from the current
// matrix, a sparse approximate inverse
//     M = (I + O) D^-1,   D = diag(A),   O sparse on the graph's edges,
// that right-preconditions an FP64 GMRES (gmres.cu); with O = 0 it is the
// Jacobi preconditioner, the method without the network.
//
// Network (all FP32, width H = 64, three message-passing layers):
//   node features x_i (8): 1, log|A_ii| - mean, neighbour coupling sum and
//     means of A_ij / A_ii and A_ji / A_jj, mean neighbour distance over its
//     mean, static/moving flag
//   edge features e_ij (4): A_ij / A_ii, A_ji / A_jj, d_ij / mean_i d, 1
//   h0 = relu(W0 x + b0)
//   h(l) = relu(Ws(l) h(l-1) + Wn(l) m(l) + b(l)),  m_i = sum_j w_ij h_j(l-1)
//     with w_ij = |A_ij| / sum_k |A_ik| over the neighbours (self excluded)
//   o_ij = sum_f u_f h_i,f h_j,f + c . e_ij           (self edge included)
// Training (on the GPU, by the kernels below): for a stored system with
// probe vectors Z (+-1) and its solution x*, the columns Y = D^-1 [A Z, b]
// and targets T = [Z, x*] give the loss L = ||Y + O Y - T||_F^2 / (n C),
// i.e. M A z ~ z and M b ~ x*; gradients are propagated by hand through the
// edge outputs, the layers and the aggregation; Adam updates the weights.
#include <cublas_v2.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "dust_common.cuh"
#include "gnn_internal.h"
#include "linsys_internal.h"

static inline unsigned nblk(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

// ------------------------------------------------------------ parameters
// flat layout: W0[H][FIN] b0[H] {Ws[H][H] Wn[H][H] b[H]} x L, u[H] c[EF]
__host__ __device__ inline int pc_off_w0() { return 0; }
__host__ __device__ inline int pc_off_b0() { return PC_H * PC_FIN; }
__host__ __device__ inline int pc_off_ws(int l) {
  return PC_H * PC_FIN + PC_H + l * (2 * PC_H * PC_H + PC_H);
}
__host__ __device__ inline int pc_off_wn(int l) { return pc_off_ws(l) + PC_H * PC_H; }
__host__ __device__ inline int pc_off_bl(int l) { return pc_off_ws(l) + 2 * PC_H * PC_H; }
__host__ __device__ inline int pc_off_u() { return pc_off_ws(PC_L); }
__host__ __device__ inline int pc_off_c() { return pc_off_u() + PC_H; }

// ------------------------------------------------------------ features
// element (i, j) of the assembled system: the static block from its
// unfactored copy, the rest from A
__device__ __forceinline__ double sys_a(const SysView &s, int i, int j) {
  return (i < s.nst && j < s.nst) ? s.As[(size_t)i + (size_t)j * s.nst]
                                  : s.A[(size_t)i + (size_t)j * s.n];
}

__global__ void k_pc_feat(int n, int K, const int *nbr, const float *dist, SysView sv, float *x,
                          float *ef, float *w, double *dinv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double aii = sys_a(sv, i, i);
  const double di = aii != 0.0 ? 1.0 / aii : 1.0;
  dinv[i] = di;
  double sabs = 0.0, sin_ = 0.0, sout = 0.0, sd = 0.0;
  for (int s = 1; s < K; ++s) {
    const int j = nbr[(size_t)i * K + s];
    sabs += fabs(sys_a(sv, i, j));
    sd += dist[(size_t)i * K + s];
  }
  const double dm = sd > 0 ? sd / (K - 1) : 1.0;
  for (int s = 0; s < K; ++s) {
    const int j = nbr[(size_t)i * K + s];
    const double aij = sys_a(sv, i, j), aji = sys_a(sv, j, i), ajj = sys_a(sv, j, j);
    const double in_ = aij * di, out = ajj != 0.0 ? aji / ajj : 0.0;
    float *e = ef + ((size_t)i * K + s) * PC_EF;
    e[0] = (float)in_;
    e[1] = (float)out;
    e[2] = (float)(dist[(size_t)i * K + s] / dm);
    e[3] = 1.f;
    w[(size_t)i * K + s] = (s == 0 || sabs == 0.0) ? 0.f : (float)(fabs(aij) / sabs);
    if (s > 0) {
      sin_ += in_;
      sout += out;
    }
  }
  float *xi = x + (size_t)i * PC_FIN;
  xi[0] = 1.f;
  xi[1] = (float)log(fabs(aii) + 1e-300);
  xi[2] = (float)(sabs * fabs(di));
  xi[3] = (float)(sin_ / (K - 1));
  xi[4] = (float)(sout / (K - 1));
  xi[5] = (float)dm;
  xi[6] = (float)(i < sv.nst ? 0.0 : 1.0);
  xi[7] = 0.f;
}

// sums of the log-diagonal and distance features over the nodes
__global__ void k_pc_feat_stats(int n, const float *x, float *stats) {
  float a = 0.f, b = 0.f;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    a += x[(size_t)i * PC_FIN + 1];
    b += x[(size_t)i * PC_FIN + 5];
  }
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(stats, a);
    atomicAdd(stats + 1, b);
  }
}
// centre the log-diagonal feature and scale the distance feature by its
// mean, so features are O(1) for any geometry scale
__global__ void k_pc_feat_norm(int n, float *x, const float *stats) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  x[(size_t)i * PC_FIN + 1] -= stats[0] / n;
  x[(size_t)i * PC_FIN + 5] /= fmaxf(stats[1] / n, 1e-30f);
}

// ------------------------------------------------------------ forward
// z0 = W0 x + b0, h0 = relu(z0); thread per (node, feature)
__global__ void k_pc_in(int n, const float *P, const float *x, float *z, float *h) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)n * PC_H) return;
  const int i = (int)(e / PC_H), f = (int)(e % PC_H);
  const float *W = P + pc_off_w0() + f * PC_FIN;
  float s = P[pc_off_b0() + f];
  for (int k = 0; k < PC_FIN; ++k) s = fmaf(W[k], x[(size_t)i * PC_FIN + k], s);
  z[e] = s;
  h[e] = fmaxf(s, 0.f);
}

// m_i = sum_j w_ij h_j
__global__ void k_pc_agg(int n, int K, const int *nbr, const float *w, const float *h, float *m) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)n * PC_H) return;
  const int i = (int)(e / PC_H), f = (int)(e % PC_H);
  float s = 0.f;
  for (int q = 1; q < K; ++q)
    s = fmaf(w[(size_t)i * K + q], h[(size_t)nbr[(size_t)i * K + q] * PC_H + f], s);
  m[e] = s;
}

// z = Ws h + Wn m + b, h' = relu(z); a CTA of 64 threads per node row
__global__ void k_pc_layer(int n, const float *P, int l, const float *h, const float *m, float *z,
                           float *hn) {
  __shared__ float sh[PC_H], sm[PC_H];
  const int i = blockIdx.x, f = threadIdx.x;
  sh[f] = h[(size_t)i * PC_H + f];
  sm[f] = m[(size_t)i * PC_H + f];
  __syncthreads();
  const float *Ws = P + pc_off_ws(l) + f * PC_H, *Wn = P + pc_off_wn(l) + f * PC_H;
  float s = P[pc_off_bl(l) + f];
  for (int k = 0; k < PC_H; ++k) s = fmaf(Ws[k], sh[k], fmaf(Wn[k], sm[k], s));
  z[(size_t)i * PC_H + f] = s;
  hn[(size_t)i * PC_H + f] = fmaxf(s, 0.f);
}

// o_ij = sum_f u_f h_i,f h_j,f + c . e_ij; warp per edge
__global__ void k_pc_out(int n, int K, const float *P, const int *nbr, const float *ef,
                         const float *h, float *o) {
  const size_t wid = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (wid >= (size_t)n * K) return;
  const int i = (int)(wid / K);
  const int j = nbr[wid];
  const float *u = P + pc_off_u();
  float s = 0.f;
  for (int f = lane; f < PC_H; f += 32) s += u[f] * h[(size_t)i * PC_H + f] * h[(size_t)j * PC_H + f];
  for (int q = 16; q > 0; q >>= 1) s += __shfl_xor_sync(0xffffffffu, s, q);
  if (lane == 0) {
    const float *c = P + pc_off_c();
    const float *e = ef + wid * PC_EF;
    o[wid] = s + c[0] * e[0] + c[1] * e[1] + c[2] * e[2] + c[3] * e[3];
  }
}

// ------------------------------------------------------------ loss
// R = Y + O Y - T (n x C); squared norms summed into loss
__global__ void k_pc_resid(int n, int K, int C, const int *nbr, const float *o, const float *Y,
                           const float *T, float *R, float *loss) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  float r2 = 0.f;
  if (e < (size_t)n * C) {
    const int i = (int)(e / C), c = (int)(e % C);
    float s = Y[e] - T[e];
    for (int q = 0; q < K; ++q)
      s = fmaf(o[(size_t)i * K + q], Y[(size_t)nbr[(size_t)i * K + q] * C + c], s);
    R[e] = s;
    r2 = s * s;
  }
  for (int q = 16; q > 0; q >>= 1) r2 += __shfl_xor_sync(0xffffffffu, r2, q);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, r2);
}

// ------------------------------------------------------------ backward
// do_ij = scale * sum_c R_ic Y_jc; dc += do_ij e_ij; du_f += do_ij h_i,f h_j,f;
// dh_i += do_ij u h_j, dh_j += do_ij u h_i (warp per edge)
__global__ void k_pc_out_bwd(int n, int K, int C, float scale, const float *P, const int *nbr,
                             const float *ef, const float *h, const float *R, const float *Y,
                             float *G, float *dh) {
  const size_t wid = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (wid >= (size_t)n * K) return;
  const int i = (int)(wid / K), j = nbr[wid];
  float d = 0.f;
  for (int c = lane; c < C; c += 32) d += R[(size_t)i * C + c] * Y[(size_t)j * C + c];
  for (int q = 16; q > 0; q >>= 1) d += __shfl_xor_sync(0xffffffffu, d, q);
  d *= scale;
  if (lane < PC_EF) atomicAdd(G + pc_off_c() + lane, d * ef[wid * PC_EF + lane]);
  const float *u = P + pc_off_u();
  for (int f = lane; f < PC_H; f += 32) {
    const float hi = h[(size_t)i * PC_H + f], hj = h[(size_t)j * PC_H + f];
    atomicAdd(G + pc_off_u() + f, d * hi * hj);
    atomicAdd(dh + (size_t)i * PC_H + f, d * u[f] * hj);
    atomicAdd(dh + (size_t)j * PC_H + f, d * u[f] * hi);
  }
}

// dz = dh * (z > 0), in place
__global__ void k_pc_relu_bwd(size_t cnt, const float *z, float *d) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < cnt && !(z[e] > 0.f)) d[e] = 0.f;
}

// dh_prev_i = Ws^T dz_i, dm_i = Wn^T dz_i (CTA of 64 per node)
__global__ void k_pc_layer_bwd(int n, const float *P, int l, const float *dz, float *dhp,
                               float *dm) {
  __shared__ float sd[PC_H];
  const int i = blockIdx.x, f = threadIdx.x;
  sd[f] = dz[(size_t)i * PC_H + f];
  __syncthreads();
  const float *Ws = P + pc_off_ws(l), *Wn = P + pc_off_wn(l);
  float a = 0.f, b = 0.f;
  for (int k = 0; k < PC_H; ++k) {
    a = fmaf(Ws[k * PC_H + f], sd[k], a);
    b = fmaf(Wn[k * PC_H + f], sd[k], b);
  }
  dhp[(size_t)i * PC_H + f] = a;
  dm[(size_t)i * PC_H + f] = b;
}

// dh_prev_j += w_ij dm_i (scatter over the edges)
__global__ void k_pc_agg_bwd(int n, int K, const int *nbr, const float *w, const float *dm,
                             float *dhp) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)n * PC_H) return;
  const int i = (int)(e / PC_H), f = (int)(e % PC_H);
  const float g = dm[e];
  if (g == 0.f) return;
  for (int q = 1; q < K; ++q)
    atomicAdd(dhp + (size_t)nbr[(size_t)i * K + q] * PC_H + f, w[(size_t)i * K + q] * g);
}

// G[off + f*cols + k] += sum_i dz_i,f a_i,k and G[boff + f] += sum_i dz_i,f
// (boff < 0: none); CTA per chunk of nodes, partial sums in shared memory
#define PC_WG_CHUNK 64
__global__ void k_pc_wgrad(int n, const float *dz, const float *a, int cols, float *G, int off,
                           int boff) {
  extern __shared__ float sacc[];  // PC_H x cols
  const int tid = threadIdx.x;
  const int i0 = blockIdx.x * PC_WG_CHUNK, i1 = min(n, i0 + PC_WG_CHUNK);
  for (int e = tid; e < PC_H * cols; e += blockDim.x) {
    const int f = e / cols, k = e % cols;
    float s = 0.f;
    for (int i = i0; i < i1; ++i) s = fmaf(dz[(size_t)i * PC_H + f], a[(size_t)i * cols + k], s);
    sacc[e] = s;
  }
  __syncthreads();
  for (int e = tid; e < PC_H * cols; e += blockDim.x) atomicAdd(G + off + e, sacc[e]);
  if (boff >= 0)
    for (int f = tid; f < PC_H; f += blockDim.x) {
      float s = 0.f;
      for (int i = i0; i < i1; ++i) s += dz[(size_t)i * PC_H + f];
      atomicAdd(G + boff + f, s);
    }
}

__global__ void k_pc_adam(int np, float *P, const float *G, float *m, float *v, float lr, float b1,
                          float b2, float c1, float c2) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= np) return;
  const float g = G[e];
  m[e] = b1 * m[e] + (1.f - b1) * g;
  v[e] = b2 * v[e] + (1.f - b2) * g * g;
  P[e] -= lr * (m[e] / c1) / (sqrtf(v[e] / c2) + 1e-8f);
}

// ------------------------------------------------------------ host side
static int pc_forward(dust_precond *p, const float *x, const float *ef, const float *w) {
  const int n = p->n, K = p->K;
  cudaStream_t st = p->st;
  const float *P = (const float *)p->par.p;
  float *z = (float *)p->z.p, *h = (float *)p->h.p, *m = (float *)p->m.p;
  const size_t nh = (size_t)n * PC_H;
  k_pc_in<<<nblk(nh, 256), 256, 0, st>>>(n, P, x, z, h);
  for (int l = 0; l < PC_L; ++l) {
    k_pc_agg<<<nblk(nh, 256), 256, 0, st>>>(n, K, (const int *)p->nbr.p, w, h + l * nh,
                                             m + l * nh);
    k_pc_layer<<<n, PC_H, 0, st>>>(n, P, l, h + l * nh, m + l * nh, z + (l + 1) * nh,
                                   h + (l + 1) * nh);
  }
  k_pc_out<<<nblk((size_t)n * K * 32, 256), 256, 0, st>>>(n, K, P, (const int *)p->nbr.p, ef,
                                                           h + PC_L * nh, (float *)p->o.p);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}

// loss and gradient (into p->grad) for stored sample `si`
static int pc_loss_grad(dust_precond *p, int si, float *loss_host) {
  const int n = p->n, K = p->K, C = PC_C;
  cudaStream_t st = p->st;
  PcSample &S = p->samples[si];
  const float *x = (const float *)S.x.p, *ef = (const float *)S.ef.p, *w = (const float *)S.w.p;
  const float *Y = (const float *)S.Y.p, *T = (const float *)S.T.p;
  DUST_TRY(pc_forward(p, x, ef, w));
  const size_t nh = (size_t)n * PC_H;
  float *R = (float *)p->R.p, *ls = (float *)p->loss.p;
  float *G = (float *)p->grad.p;
  float *z = (float *)p->z.p, *h = (float *)p->h.p, *m = (float *)p->m.p;
  float *dh = (float *)p->dh.p, *dhp = (float *)p->dhp.p, *dm = (float *)p->dm.p;
  const int *nbr = (const int *)p->nbr.p;
  DUST_CUDA(cudaMemsetAsync(ls, 0, sizeof(float), st));
  DUST_CUDA(cudaMemsetAsync(G, 0, sizeof(float) * PC_NPAR, st));
  DUST_CUDA(cudaMemsetAsync(dh, 0, sizeof(float) * nh, st));
  k_pc_resid<<<nblk((size_t)n * C, 256), 256, 0, st>>>(n, K, C, nbr, (const float *)p->o.p, Y, T,
                                                        R, ls);
  const float scale = 2.f / ((float)n * C);
  k_pc_out_bwd<<<nblk((size_t)n * K * 32, 256), 256, 0, st>>>(
      n, K, C, scale, (const float *)p->par.p, nbr, ef, h + PC_L * nh, R, Y, G, dh);
  const unsigned nch = nblk(n, PC_WG_CHUNK);
  for (int l = PC_L - 1; l >= 0; --l) {
    // dh holds dL/dh(l+1): mask by z(l+1)
    k_pc_relu_bwd<<<nblk(nh, 256), 256, 0, st>>>(nh, z + (l + 1) * nh, dh);
    k_pc_wgrad<<<nch, 256, PC_H * PC_H * 4, st>>>(n, dh, h + l * nh, PC_H, G, pc_off_ws(l),
                                                   pc_off_bl(l));
    k_pc_wgrad<<<nch, 256, PC_H * PC_H * 4, st>>>(n, dh, m + l * nh, PC_H, G, pc_off_wn(l), -1);
    k_pc_layer_bwd<<<n, PC_H, 0, st>>>(n, (const float *)p->par.p, l, dh, dhp, dm);
    k_pc_agg_bwd<<<nblk(nh, 256), 256, 0, st>>>(n, K, nbr, w, dm, dhp);
    std::swap(dh, dhp);
  }
  k_pc_relu_bwd<<<nblk(nh, 256), 256, 0, st>>>(nh, z, dh);
  k_pc_wgrad<<<nch, 256, PC_H * PC_FIN * 4, st>>>(n, dh, x, PC_FIN, G, pc_off_w0(), pc_off_b0());
  DUST_CUDA(cudaGetLastError());
  if (loss_host) {
    float l = 0.f;
    DUST_CUDA(cudaMemcpyAsync(&l, ls, sizeof(float), cudaMemcpyDeviceToHost, st));
    DUST_CUDA(cudaStreamSynchronize(st));
    *loss_host = l / ((float)n * C);
  }
  return DUST_OK;
}

static int pc_features(dust_precond *p, const SysView &sv, float *x, float *ef, float *w,
                       double *dinv) {
  cudaStream_t st = p->st;
  k_pc_feat<<<nblk(p->n, 128), 128, 0, st>>>(p->n, p->K, (const int *)p->nbr.p,
                                              (const float *)p->dist.p, sv, x, ef, w, dinv);
  float *stats = (float *)p->loss.p + 4;
  DUST_CUDA(cudaMemsetAsync(stats, 0, 2 * sizeof(float), st));
  k_pc_feat_stats<<<64, 256, 0, st>>>(p->n, x, stats);
  k_pc_feat_norm<<<nblk(p->n, 128), 128, 0, st>>>(p->n, x, stats);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}

// forward pass on the current system: edge outputs in p->o, 1/A_ii in p->dinv
int pc_infer(dust_precond *p, const SysView &sv) {
  DUST_TRY(pc_features(p, sv, (float *)p->ix.p, (float *)p->ief.p, (float *)p->iw.p,
                       (double *)p->dinv.p));
  return pc_forward(p, (const float *)p->ix.p, (const float *)p->ief.p, (const float *)p->iw.p);
}

// y = M v = (I + O) D^-1 v (FP64)
__global__ void k_pc_apply(int n, int K, const int *nbr, const float *o, const double *dinv,
                           const double *v, double *y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = dinv[i] * v[i];
  for (int q = 0; q < K; ++q) {
    const int j = nbr[(size_t)i * K + q];
    s += (double)o[(size_t)i * K + q] * dinv[j] * v[j];
  }
  y[i] = s;
}
void pc_apply(dust_precond *p, const double *v, double *y, cudaStream_t st) {
  k_pc_apply<<<nblk(p->n, 128), 128, 0, st>>>(p->n, p->K, (const int *)p->nbr.p,
                                               (const float *)p->o.p, (const double *)p->dinv.p,
                                               v, y);
}

static int pc_alloc_work(dust_precond *p) {
  const size_t n = p->n, nh = n * PC_H, K = p->K;
  DUST_TRY(devbuf_grow(p->h, (PC_L + 1) * nh * 4));
  DUST_TRY(devbuf_grow(p->z, (PC_L + 1) * nh * 4));
  DUST_TRY(devbuf_grow(p->m, PC_L * nh * 4));
  DUST_TRY(devbuf_grow(p->dh, nh * 4));
  DUST_TRY(devbuf_grow(p->dhp, nh * 4));
  DUST_TRY(devbuf_grow(p->dm, nh * 4));
  DUST_TRY(devbuf_grow(p->o, n * K * 4));
  DUST_TRY(devbuf_grow(p->R, n * PC_C * 4));
  DUST_TRY(devbuf_grow(p->loss, 64));
  DUST_TRY(devbuf_grow(p->ix, n * PC_FIN * 4));
  DUST_TRY(devbuf_grow(p->ief, n * K * PC_EF * 4));
  DUST_TRY(devbuf_grow(p->iw, n * K * 4));
  DUST_TRY(devbuf_grow(p->dinv, n * 8));
  return DUST_OK;
}

// -------------------------------------------------------------- C ABI
extern "C" int dust_precond_create(int n, int k, const double *centres, unsigned long long seed,
                                   dust_precond **out) {
  if (!out || n <= 0 || k < 1 || k + 1 > PC_KMAX || !centres || k >= n) return DUST_ERR_BAD_ARG;
  *out = nullptr;
  dust_precond *p = new dust_precond();
  p->n = n;
  p->K = k + 1;
  // k nearest neighbours of every panel centre (slot 0 = the panel itself)
  std::vector<int> nbr((size_t)n * p->K);
  std::vector<float> dist((size_t)n * p->K);
  std::vector<std::pair<double, int>> cand(n);
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j < n; ++j) {
      double d2 = 0.0;
      for (int c = 0; c < 3; ++c) {
        const double dd = centres[3 * (size_t)i + c] - centres[3 * (size_t)j + c];
        d2 += dd * dd;
      }
      cand[j] = {j == i ? -1.0 : d2, j};
    }
    std::partial_sort(cand.begin(), cand.begin() + p->K, cand.end());
    for (int s = 0; s < p->K; ++s) {
      nbr[(size_t)i * p->K + s] = cand[s].second;
      dist[(size_t)i * p->K + s] = (float)sqrt(std::max(cand[s].first, 0.0));
    }
  }
  int st = DUST_OK;
  if (cudaStreamCreateWithFlags(&p->st, cudaStreamNonBlocking) != cudaSuccess) st = DUST_ERR_CUDA;
  if (st == DUST_OK && cublasCreate(&p->cb) != CUBLAS_STATUS_SUCCESS) st = DUST_ERR_CUDA;
  if (st == DUST_OK) st = devbuf_grow(p->nbr, nbr.size() * 4);
  if (st == DUST_OK) st = devbuf_grow(p->dist, dist.size() * 4);
  if (st == DUST_OK) st = devbuf_grow(p->par, PC_NPAR * 4);
  if (st == DUST_OK) st = devbuf_grow(p->grad, PC_NPAR * 4);
  if (st == DUST_OK) st = devbuf_grow(p->am, PC_NPAR * 4);
  if (st == DUST_OK) st = devbuf_grow(p->av, PC_NPAR * 4);
  if (st == DUST_OK) st = pc_alloc_work(p);
  if (st == DUST_OK) {
    cudaMemcpy(p->nbr.p, nbr.data(), nbr.size() * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(p->dist.p, dist.data(), dist.size() * 4, cudaMemcpyHostToDevice);
    // small random hidden weights, output weights zero: the untrained network
    // is the Jacobi preconditioner
    std::mt19937_64 rng(seed);
    std::normal_distribution<float> nd(0.f, 1.f);
    std::vector<float> w(PC_NPAR, 0.f);
    for (int f = 0; f < PC_H; ++f)
      for (int q = 0; q < PC_FIN; ++q) w[pc_off_w0() + f * PC_FIN + q] = nd(rng) / sqrtf(PC_FIN);
    for (int l = 0; l < PC_L; ++l)
      for (int e = 0; e < PC_H * PC_H; ++e) {
        w[pc_off_ws(l) + e] = nd(rng) / sqrtf(2.f * PC_H);
        w[pc_off_wn(l) + e] = nd(rng) / sqrtf(2.f * PC_H);
      }
    cudaMemcpy(p->par.p, w.data(), PC_NPAR * 4, cudaMemcpyHostToDevice);
    cudaMemset(p->am.p, 0, PC_NPAR * 4);
    cudaMemset(p->av.p, 0, PC_NPAR * 4);
    if (cudaGetLastError() != cudaSuccess) st = DUST_ERR_CUDA;
  }
  if (st != DUST_OK) {
    dust_precond_destroy(p);
    return st;
  }
  *out = p;
  return DUST_OK;
}

extern "C" int dust_precond_destroy(dust_precond *p) {
  if (!p) return DUST_OK;
  if (p->st) cudaStreamSynchronize(p->st);
  for (PcSample &s : p->samples) {
    devbuf_free(s.x);
    devbuf_free(s.ef);
    devbuf_free(s.w);
    devbuf_free(s.Y);
    devbuf_free(s.T);
  }
  DevBuf *bufs[] = {&p->nbr, &p->dist, &p->par, &p->grad, &p->am,   &p->av,  &p->h,
                    &p->z,   &p->m,    &p->dh,  &p->dhp,  &p->dm,   &p->o,   &p->R,
                    &p->loss, &p->ix,  &p->ief, &p->iw,   &p->dinv, &p->tmp};
  for (DevBuf *b : bufs) devbuf_free(*b);
  if (p->cb) cublasDestroy(p->cb);
  if (p->st) cudaStreamDestroy(p->st);
  delete p;
  return DUST_OK;
}

extern "C" int dust_precond_num_params(void) { return PC_NPAR; }

extern "C" int dust_precond_get_params(const dust_precond *p, float *w, int count) {
  if (!p || !w || count != PC_NPAR) return DUST_ERR_BAD_ARG;
  DUST_CUDA(cudaMemcpy(w, p->par.p, PC_NPAR * 4, cudaMemcpyDeviceToHost));
  return DUST_OK;
}

extern "C" int dust_precond_set_params(dust_precond *p, const float *w, int count) {
  if (!p || !w || count != PC_NPAR) return DUST_ERR_BAD_ARG;
  DUST_CUDA(cudaMemcpy(p->par.p, w, PC_NPAR * 4, cudaMemcpyHostToDevice));
  p->adam_t = 0;
  DUST_CUDA(cudaMemset(p->am.p, 0, PC_NPAR * 4));
  DUST_CUDA(cudaMemset(p->av.p, 0, PC_NPAR * 4));
  return DUST_OK;
}

// Stores a training sample from an assembled (not yet solved) system and
// its solution x (device): features, Y = D^-1 [A Z, b] and T = [Z, x].
extern "C" int dust_precond_add_sample(dust_precond *p, dust_linsys *L, const double *x_dev,
                                       unsigned long long seed) {
  if (!p || !L || !x_dev || L->n != p->n || !L->assembled || L->factored) return DUST_ERR_BAD_ARG;
  const int n = p->n, K = p->K, C = PC_C, NZ = PC_C - 1;
  cudaStream_t st = p->st;
  DUST_CUDA(cudaStreamSynchronize(L->st));
  const SysView sv = linsys_view(L);
  PcSample S;
  int s = DUST_OK;
  if (s == DUST_OK) s = devbuf_grow(S.x, (size_t)n * PC_FIN * 4);
  if (s == DUST_OK) s = devbuf_grow(S.ef, (size_t)n * K * PC_EF * 4);
  if (s == DUST_OK) s = devbuf_grow(S.w, (size_t)n * K * 4);
  if (s == DUST_OK) s = devbuf_grow(S.Y, (size_t)n * C * 4);
  if (s == DUST_OK) s = devbuf_grow(S.T, (size_t)n * C * 4);
  // work: dinv, Z and A Z (FP64, column-major n x NZ)
  if (s == DUST_OK) s = devbuf_grow(p->tmp, (size_t)n * 8 * (1 + 2 * NZ) + 256);
  if (s == DUST_OK) {
    double *dinv = (double *)p->tmp.p, *Z = dinv + n, *AZ = Z + (size_t)n * NZ;
    s = pc_features(p, sv, (float *)S.x.p, (float *)S.ef.p, (float *)S.w.p, dinv);
    std::mt19937_64 rng(seed);
    std::vector<double> hz((size_t)n * NZ);
    for (double &v : hz) v = (rng() & 1) ? 1.0 : -1.0;
    if (s == DUST_OK &&
        cudaMemcpyAsync(Z, hz.data(), hz.size() * 8, cudaMemcpyHostToDevice, st) != cudaSuccess)
      s = DUST_ERR_CUDA;
    if (s == DUST_OK) s = linsys_matmat(L, NZ, Z, n, AZ, n, st, p->cb);
    if (s == DUST_OK)
      s = pc_pack_sample(n, C, dinv, AZ, Z, (const double *)L->b.p, x_dev, (float *)S.Y.p,
                         (float *)S.T.p, st);
    if (s == DUST_OK && cudaStreamSynchronize(st) != cudaSuccess) s = DUST_ERR_CUDA;
  }
  if (s != DUST_OK) {
    devbuf_free(S.x);
    devbuf_free(S.ef);
    devbuf_free(S.w);
    devbuf_free(S.Y);
    devbuf_free(S.T);
    return s;
  }
  p->samples.push_back(S);
  return DUST_OK;
}

extern "C" int dust_precond_num_samples(const dust_precond *p) {
  return p ? (int)p->samples.size() : 0;
}

// loss and gradient of sample `si` at the current weights (host copies)
extern "C" int dust_precond_loss_grad(dust_precond *p, int si, float *loss, float *grad,
                                      int count) {
  if (!p || si < 0 || si >= (int)p->samples.size() || !loss) return DUST_ERR_BAD_ARG;
  if (grad && count != PC_NPAR) return DUST_ERR_BAD_ARG;
  DUST_TRY(pc_loss_grad(p, si, loss));
  if (grad) DUST_CUDA(cudaMemcpy(grad, p->grad.p, PC_NPAR * 4, cudaMemcpyDeviceToHost));
  return DUST_OK;
}

// the inputs of a stored sample (host arrays; any pointer may be NULL)
extern "C" int dust_precond_get_sample(const dust_precond *p, int si, float *x, float *ef,
                                       float *w, int *nbr, float *Y, float *T) {
  if (!p || si < 0 || si >= (int)p->samples.size()) return DUST_ERR_BAD_ARG;
  const PcSample &S = p->samples[si];
  const size_t n = p->n, K = p->K;
  if (x) DUST_CUDA(cudaMemcpy(x, S.x.p, n * PC_FIN * 4, cudaMemcpyDeviceToHost));
  if (ef) DUST_CUDA(cudaMemcpy(ef, S.ef.p, n * K * PC_EF * 4, cudaMemcpyDeviceToHost));
  if (w) DUST_CUDA(cudaMemcpy(w, S.w.p, n * K * 4, cudaMemcpyDeviceToHost));
  if (nbr) DUST_CUDA(cudaMemcpy(nbr, p->nbr.p, n * K * 4, cudaMemcpyDeviceToHost));
  if (Y) DUST_CUDA(cudaMemcpy(Y, S.Y.p, n * PC_C * 4, cudaMemcpyDeviceToHost));
  if (T) DUST_CUDA(cudaMemcpy(T, S.T.p, n * PC_C * 4, cudaMemcpyDeviceToHost));
  return DUST_OK;
}

// `iters` Adam steps cycling over the stored samples; mean loss of the last
// pass over the samples in *loss_out
extern "C" int dust_precond_train(dust_precond *p, int iters, float lr, float *loss_out) {
  if (!p || iters < 0 || p->samples.empty()) return DUST_ERR_BAD_ARG;
  const float b1 = 0.9f, b2 = 0.999f;
  const int ns = (int)p->samples.size();
  double acc = 0.0;
  int cnt = 0;
  for (int it = 0; it < iters; ++it) {
    const bool last = it >= iters - ns;
    float l = 0.f;
    DUST_TRY(pc_loss_grad(p, it % ns, last ? &l : nullptr));
    if (last) {
      acc += l;
      ++cnt;
    }
    ++p->adam_t;
    const float c1 = 1.f - powf(b1, (float)p->adam_t), c2 = 1.f - powf(b2, (float)p->adam_t);
    k_pc_adam<<<nblk(PC_NPAR, 256), 256, 0, p->st>>>(PC_NPAR, (float *)p->par.p,
                                                      (const float *)p->grad.p, (float *)p->am.p,
                                                      (float *)p->av.p, lr, b1, b2, c1, c2);
  }
  DUST_CUDA(cudaStreamSynchronize(p->st));
  DUST_CUDA(cudaGetLastError());
  if (loss_out) *loss_out = cnt ? (float)(acc / cnt) : 0.f;
  return DUST_OK;
}

extern "C" int dust_linsys_set_precond(dust_linsys *L, dust_precond *p) {
  if (!L || (p && p->n != L->n)) return DUST_ERR_BAD_ARG;
  L->pc = p;
  return DUST_OK;
}
