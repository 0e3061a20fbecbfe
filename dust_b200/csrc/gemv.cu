// gemv.cu -- matrix-vector products and vector reductions of the iterative
// solves (the refinement sweeps of the mixed-precision solve and the GMRES
// of the learned preconditioner): the dgemv / sgemv / idamax / dnrm2 calls
// of LAPACK-style code, here as own kernels.
//
// y = alpha A x + beta y (A column-major m x k): every element of A is read
// once, so the product is bound by HBM.  A CTA owns GV_ROWS rows and a chunk
// of columns; each thread accumulates GV_RPT rows over the chunk with the
// column entries of x staged in shared memory, and the chunk's partial sums
// are added atomically into y (scaled by beta first).  Chunks are sized so
// that the grid covers every SM several times.
// y = alpha A^T x + beta y: one CTA per column (a contiguous dot product),
// reduced in shared memory.
#include <algorithm>

#include "dust_common.cuh"
#include "fmm_internal.h"

static inline unsigned nblk(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

#define GV_T 256
#define GV_RPT 2
#define GV_ROWS (GV_T * GV_RPT)
#define GV_CHUNK 256

template <typename T>
__global__ void k_scal(int m, T beta, T *y) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) y[i] = beta == (T)0 ? (T)0 : beta * y[i];
}

template <typename T>
__global__ void __launch_bounds__(GV_T) k_gemv_n(int m, int k, T alpha, const T *__restrict__ A,
                                                 int lda, const T *__restrict__ x, int chunk,
                                                 T *y) {
  __shared__ T s_x[GV_CHUNK];
  const int r0 = blockIdx.x * GV_ROWS + threadIdx.x;
  const int c0 = blockIdx.y * chunk, c1 = min(k, c0 + chunk);
  T acc[GV_RPT];
#pragma unroll
  for (int u = 0; u < GV_RPT; ++u) acc[u] = (T)0;
  for (int cb = c0; cb < c1; cb += GV_CHUNK) {
    const int cn = min(GV_CHUNK, c1 - cb);
    __syncthreads();
    for (int c = threadIdx.x; c < cn; c += GV_T) s_x[c] = x[cb + c];
    __syncthreads();
#pragma unroll
    for (int u = 0; u < GV_RPT; ++u) {
      const int r = r0 + u * GV_T;
      if (r >= m) continue;
      const T *a = A + (size_t)cb * lda + r;
      T s0 = 0, s1 = 0, s2 = 0, s3 = 0;
      int c = 0;
      for (; c + 4 <= cn; c += 4) {
        s0 += a[(size_t)c * lda] * s_x[c];
        s1 += a[(size_t)(c + 1) * lda] * s_x[c + 1];
        s2 += a[(size_t)(c + 2) * lda] * s_x[c + 2];
        s3 += a[(size_t)(c + 3) * lda] * s_x[c + 3];
      }
      for (; c < cn; ++c) s0 += a[(size_t)c * lda] * s_x[c];
      acc[u] += (s0 + s1) + (s2 + s3);
    }
  }
#pragma unroll
  for (int u = 0; u < GV_RPT; ++u) {
    const int r = r0 + u * GV_T;
    if (r < m) atomicAdd(y + r, alpha * acc[u]);
  }
}

template <typename T>
__global__ void __launch_bounds__(GV_T) k_gemv_t(int m, int k, T alpha, const T *__restrict__ A,
                                                 int lda, const T *__restrict__ x, T beta, T *y) {
  __shared__ T s_r[GV_T / 32];
  const int c = blockIdx.x;
  const T *a = A + (size_t)c * lda;
  T s = 0;
  for (int r = threadIdx.x; r < m; r += GV_T) s += a[r] * x[r];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) s_r[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    T t = 0;
    for (int w = 0; w < GV_T / 32; ++w) t += s_r[w];
    y[c] = alpha * t + (beta == (T)0 ? (T)0 : beta * y[c]);
  }
}

template <typename T>
int gemv_n(cudaStream_t st, int m, int k, T alpha, const T *A, int lda, const T *x, T beta,
           T *y) {
  if (m <= 0) return DUST_OK;
  if (beta != (T)1) k_scal<T><<<nblk(m, 256), 256, 0, st>>>(m, beta, y);
  if (k <= 0) return DUST_OK;
  const int bx = (int)nblk(m, GV_ROWS);
  // enough CTAs for every SM several times over
  int ny = std::max(1, std::min((k + 63) / 64, (148 * 6 + bx - 1) / bx));
  const int chunk = (k + ny - 1) / ny;
  ny = (k + chunk - 1) / chunk;
  k_gemv_n<T><<<dim3(bx, ny), GV_T, 0, st>>>(m, k, alpha, A, lda, x, chunk, y);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}

template <typename T>
int gemv_t(cudaStream_t st, int m, int k, T alpha, const T *A, int lda, const T *x, T beta,
           T *y) {
  if (k <= 0) return DUST_OK;
  k_gemv_t<T><<<k, GV_T, 0, st>>>(m, k, alpha, A, lda, x, beta, y);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}

// out[0] = max_i |v_i| (one CTA), out[1] = sqrt(sum_i v_i^2)
__global__ void __launch_bounds__(1024) k_absmax_nrm2(int n, const double *v, double *out) {
  __shared__ double s_m[32], s_s[32];
  double mx = 0.0, ss = 0.0;
  for (int i = threadIdx.x; i < n; i += 1024) {
    const double a = fabs(v[i]);
    mx = fmax(mx, a);
    ss += a * a;
  }
  for (int o = 16; o > 0; o >>= 1) {
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    ss += __shfl_xor_sync(0xffffffffu, ss, o);
  }
  if ((threadIdx.x & 31) == 0) {
    s_m[threadIdx.x >> 5] = mx;
    s_s[threadIdx.x >> 5] = ss;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0, s = 0.0;
    for (int w = 0; w < 32; ++w) {
      m = fmax(m, s_m[w]);
      s += s_s[w];
    }
    out[0] = m;
    out[1] = sqrt(s);
  }
}

int vec_absmax_nrm2(cudaStream_t st, int n, const double *v, double *out_dev) {
  k_absmax_nrm2<<<1, 1024, 0, st>>>(n, v, out_dev);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}

template int gemv_n<double>(cudaStream_t, int, int, double, const double *, int, const double *,
                            double, double *);
template int gemv_n<float>(cudaStream_t, int, int, float, const float *, int, const float *,
                           float, float *);
template int gemv_t<double>(cudaStream_t, int, int, double, const double *, int, const double *,
                            double, double *);
