// lu_np.cu -- blocked LU without row interchanges, certified against partial
// pivoting (FP64 and FP32), column-major.
//
// Partial pivoting (LAPACK dgetrf, src/linsys/mod_linsys.f90:230-246,
// :470-474) interchanges rows at column j only when some |a(i,j)|, i > j,
// exceeds the diagonal |a(j,j)| at that point of the elimination.  With no
// interchange the multipliers are l(i,j) = a(i,j) / a(j,j), so the
// factorisation computed without pivoting is partial pivoting's own
// whenever every |l(i,j)| < 1.  The surface-panel influence matrices of this
// solver are of that kind (doublet self-influence 2 pi on the diagonal,
// off-diagonal row sums of about 2 pi on a closed body; dgetrf makes no
// interchange on them).  Without the per-column pivot search the panel
// needs no column-by-column barrier across the matrix and the whole
// factorisation is blocks and GEMMs:
//
//   for each block column k (NP_NB wide):
//     k_np_diag   one CTA: unpivoted LU of the diagonal block in shared
//                 memory, its inverse triangles Linv (unit lower) and Uinv
//                 (upper) by substitution, max |l| of the block;
//     k_np_panel  L21 = A21 Uinv (row tiles) and U12 = Linv A12 (column
//                 tiles), 64 x 64 register-tiled products, max |l| of L21;
//     trailing    A22 -= L21 U12 (tcgen05 TF32 GEMM for FP32, DGEMM for
//                 FP64).
//
// The largest |l| is kept as float bits (monotone for non-negative values)
// with atomicMax.  The caller accepts the factors when it is below
// 1 - margin (a margin well above the rounding of the computed multipliers,
// so partial pivoting on the same values would also have kept every
// diagonal); otherwise, and on a zero diagonal, it restores A and runs the
// pivoted factorisation.  ipiv is the identity.
#include <algorithm>
#include <cstring>

#include "lu.cuh"

#define CUBLAS_CHECK(x)                                                   \
  do {                                                                    \
    if ((x) != CUBLAS_STATUS_SUCCESS) {                                   \
      dust_set_last_error("cuBLAS call failed", __FILE__, __LINE__);      \
      return DUST_ERR_CUDA;                                               \
    }                                                                     \
  } while (0)

#define NP_NB 64
#define NP_T 256
#define NP_LD (NP_NB + 1)

__device__ __forceinline__ void np_note_lmax(unsigned *bits, float v) {
  atomicMax(bits, __float_as_uint(v));
}

// Diagonal block: shared a[i * NP_LD + c] (row-major, padded), then the two
// inverse triangles; the block's LU and max |l| back to global memory.
template <typename T>
__global__ void __launch_bounds__(NP_T) k_np_diag(T *A, int lda, int k, int jb, T *Linv,
                                                  T *Uinv, unsigned *lmax_bits) {
  extern __shared__ __align__(16) unsigned char np_sm[];
  T *a = (T *)np_sm;                   // jb x jb, ld NP_LD
  T *inv = a + NP_NB * NP_LD;          // Uinv | Linv, ld NP_LD (Uinv in columns 0..jb)
  T *linv = inv + NP_NB * NP_LD;
  __shared__ float s_lmax;
  const int tid = threadIdx.x;
  if (tid == 0) s_lmax = 0.f;
  for (int e = tid; e < jb * jb; e += NP_T) {
    const int i = e % jb, c = e / jb;
    a[i * NP_LD + c] = A[(size_t)(k + i) + (size_t)(k + c) * lda];
  }
  __syncthreads();
  float lm = 0.f;
  bool zero = false;
  const int i = tid & (NP_NB - 1), cp = tid / NP_NB;  // row, column phase (0..3)
  for (int j = 0; j < jb; ++j) {
    const T piv = a[j * NP_LD + j];
    if (piv == (T)0) zero = true;
    if (cp == 0 && i > j && i < jb) {
      const T l = a[i * NP_LD + j] / piv;
      a[i * NP_LD + j] = l;
      lm = fmaxf(lm, (float)fabs((double)l));
    }
    __syncthreads();
    if (i > j && i < jb) {
      const T l = a[i * NP_LD + j];
      for (int c = j + 1 + cp; c < jb; c += NP_T / NP_NB) a[i * NP_LD + c] -= l * a[j * NP_LD + c];
    }
    __syncthreads();
  }
  if (zero) lm = INFINITY;
  // max |l| of the block (CTA reduction through one shared word)
  for (int o = 16; o > 0; o >>= 1) lm = fmaxf(lm, __shfl_xor_sync(0xffffffffu, lm, o));
  if ((tid & 31) == 0) atomicMax((unsigned *)&s_lmax, __float_as_uint(lm));
  // inverse triangles, one column per thread: threads [0, jb) Uinv, [64, 64 + jb) Linv
  if (tid < jb) {
    const int c = tid;
    for (int r = c; r >= 0; --r) {
      T s = (r == c) ? (T)1 : (T)0;
      for (int p = r + 1; p <= c; ++p) s -= a[r * NP_LD + p] * inv[p * NP_LD + c];
      inv[r * NP_LD + c] = s / a[r * NP_LD + r];
    }
  } else if (tid >= NP_NB && tid < NP_NB + jb) {
    const int c = tid - NP_NB;
    linv[c * NP_LD + c] = (T)1;
    for (int r = c + 1; r < jb; ++r) {
      T s = (T)0;
      for (int p = c; p < r; ++p) s -= a[r * NP_LD + p] * linv[p * NP_LD + c];
      linv[r * NP_LD + c] = s;
    }
  }
  __syncthreads();
  for (int e = tid; e < jb * jb; e += NP_T) {
    const int r = e % jb, c = e / jb;
    A[(size_t)(k + r) + (size_t)(k + c) * lda] = a[r * NP_LD + c];
    Uinv[r + (size_t)c * NP_NB] = r <= c ? inv[r * NP_LD + c] : (T)0;
    Linv[r + (size_t)c * NP_NB] = r > c ? linv[r * NP_LD + c] : (r == c ? (T)1 : (T)0);
  }
  if (tid == 0) np_note_lmax(lmax_bits, s_lmax);
}

// 64 x 64 tiles of the panel: blocks [0, nrb) take 64 rows of A21 and write
// A21 Uinv over them; blocks [nrb, nrb + ncb) take 64 columns of A12 and
// write Linv A12.  Each thread computes a 4 x 4 piece of the tile from the
// two shared operands (the tile and the inverse triangle).
template <typename T>
__global__ void __launch_bounds__(NP_T) k_np_panel(T *A, int lda, int n, int k, int jb,
                                                   const T *Linv, const T *Uinv, int nrb,
                                                   unsigned *lmax_bits) {
  extern __shared__ __align__(16) unsigned char np_sm[];
  T *x = (T *)np_sm;            // 64 x 64 operand tile, [row][col], ld NP_LD
  T *w = x + NP_NB * NP_LD;     // 64 x 64 inverse, [row][col], ld NP_LD
  const int tid = threadIdx.x;
  const bool rows = (int)blockIdx.x < nrb;
  const int b = rows ? blockIdx.x : blockIdx.x - nrb;
  const int r0 = rows ? k + jb + NP_NB * b : k;      // first row of the tile in A
  const int c0 = rows ? k : k + jb + NP_NB * b;      // first column of the tile in A
  const int nr = rows ? min(NP_NB, n - r0) : jb;
  const int nc = rows ? jb : min(NP_NB, n - c0);
  const T *W = rows ? Uinv : Linv;
  for (int e = tid; e < NP_NB * NP_NB; e += NP_T) {
    const int r = e % NP_NB, c = e / NP_NB;
    x[r * NP_LD + c] = (r < nr && c < nc) ? A[(size_t)(r0 + r) + (size_t)(c0 + c) * lda] : (T)0;
    w[r * NP_LD + c] = (r < jb && c < jb) ? W[r + (size_t)c * NP_NB] : (T)0;
  }
  __syncthreads();
  // out = x w (rows) or w x (columns); thread (ty, tx) owns rows 4 ty .. and
  // columns 4 tx ..
  const int ty = tid / 16, tx = tid % 16;
  T acc[4][4];
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) acc[u][v] = (T)0;
  const T *L = rows ? x : w, *R = rows ? w : x;
#pragma unroll 4
  for (int p = 0; p < NP_NB; ++p) {
    T lv[4], rv[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) lv[u] = L[(4 * ty + u) * NP_LD + p];
#pragma unroll
    for (int v = 0; v < 4; ++v) rv[v] = R[p * NP_LD + 4 * tx + v];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v) acc[u][v] = fma(lv[u], rv[v], acc[u][v]);
  }
  // through shared memory back to A, coalesced along the columns
  __syncthreads();
  float lm = 0.f;
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int r = 4 * ty + u, c = 4 * tx + v;
      x[r * NP_LD + c] = acc[u][v];
      if (rows && r < nr && c < nc) lm = fmaxf(lm, (float)fabs((double)acc[u][v]));
    }
  __syncthreads();
  for (int e = tid; e < NP_NB * NP_NB; e += NP_T) {
    const int r = e % NP_NB, c = e / NP_NB;
    if (r < nr && c < nc) A[(size_t)(r0 + r) + (size_t)(c0 + c) * lda] = x[r * NP_LD + c];
  }
  if (rows) {
    for (int o = 16; o > 0; o >>= 1) lm = fmaxf(lm, __shfl_xor_sync(0xffffffffu, lm, o));
    if ((tid & 31) == 0) np_note_lmax(lmax_bits, lm);
  }
}

__global__ void k_np_ipiv(int n, int *ipiv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) ipiv[i] = i + 1;
}

static cublasStatus_t np_gemm_minus(cublasHandle_t h, int m, int n, int k, const double *A,
                                    int lda, const double *B, int ldb, double *C, int ldc) {
  const double one = 1.0, mone = -1.0;
  return cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, m, n, k, &mone, A, lda, B, ldb, &one, C, ldc);
}

int gemm_tf32_minus(cudaStream_t st, int m, int n, int k, const float *A, int lda,
                    const float *B, int ldb, float *C, int ldc);

__global__ void k_np_iota(int n, int *v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = i;
}

static cublasStatus_t np_gemm_minus(cublasHandle_t h, int m, int n, int k, const float *A,
                                    int lda, const float *B, int ldb, float *C, int ldc) {
  const float one = 1.f, mone = -1.f;
  return cublasSgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, m, n, k, &mone, A, lda, B, ldb, &one, C, ldc);
}

template <typename T>
int lu_getrf_nopiv(cublasHandle_t cb, cudaStream_t st, LuWork &w, int n, T *A, int lda,
                   int *ipiv, int gemm_update, int *perm, float *lmax) {
  *lmax = 0.f;
  if (n <= 0) return DUST_OK;
  // inverse triangles of every diagonal block are kept (Linv then Uinv per
  // block) for lu_getrs_nopiv
  const size_t tri = (size_t)NP_NB * NP_NB;
  const int nblk_ = (n + NP_NB - 1) / NP_NB;
  DUST_TRY(devbuf_grow(w.np, 256 + 2 * tri * sizeof(T) * (size_t)nblk_));
  unsigned *bits = (unsigned *)w.np.p;
  T *inv0 = (T *)((char *)w.np.p + 256);
  DUST_CUDA(cudaMemsetAsync(bits, 0, sizeof(unsigned), st));
  const int smd = 3 * NP_NB * NP_LD * (int)sizeof(T), smp = 2 * NP_NB * NP_LD * (int)sizeof(T);
  static bool attr = false;  // per element type
  if (!attr) {
    DUST_CUDA(cudaFuncSetAttribute(k_np_diag<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smd));
    DUST_CUDA(cudaFuncSetAttribute(k_np_panel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smp));
    attr = true;
  }
  CUBLAS_CHECK(cublasSetStream(cb, st));
  for (int k = 0; k < n; k += NP_NB) {
    const int jb = std::min(NP_NB, n - k), m2 = n - k - jb;
    T *Linv = inv0 + 2 * tri * (size_t)(k / NP_NB), *Uinv = Linv + tri;
    k_np_diag<T><<<1, NP_T, smd, st>>>(A, lda, k, jb, Linv, Uinv, bits);
    if (m2 > 0) {
      const int nrb = (m2 + NP_NB - 1) / NP_NB;
      k_np_panel<T><<<2 * nrb, NP_T, smp, st>>>(A, lda, n, k, jb, Linv, Uinv, nrb, bits);
      T *L21 = A + (k + jb) + (size_t)k * lda, *U12 = A + k + (size_t)(k + jb) * lda,
        *A22 = A + (k + jb) + (size_t)(k + jb) * lda;
      if (sizeof(T) == 4 && gemm_update == 1) {
        DUST_TRY(gemm_tf32_minus(st, m2, m2, jb, (const float *)L21, lda, (const float *)U12,
                                 lda, (float *)A22, lda));
      } else {
        CUBLAS_CHECK(np_gemm_minus(cb, m2, m2, jb, L21, lda, U12, lda, A22, lda));
      }
    }
  }
  if (ipiv) k_np_ipiv<<<(n + 255) / 256, 256, 0, st>>>(n, ipiv);
  if (perm) k_np_iota<<<(n + 255) / 256, 256, 0, st>>>(n, perm);
  DUST_CUDA(cudaGetLastError());
  unsigned hb = 0;
  DUST_CUDA(cudaMemcpyAsync(&hb, bits, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  DUST_CUDA(cudaStreamSynchronize(st));
  unsigned tmp = hb;
  memcpy(lmax, &tmp, sizeof(float));
  return DUST_OK;
}

// Block substitution with the kept inverse triangles: one launch per 64-row
// block i (forward: i ascending with Linv, backward: descending with Uinv).
// Every CTA of the launch recomputes Y_i = Inv_i B_i (64 x 64 by 64 x NP_RC,
// from B's block i, which no CTA of the launch writes), and then updates its
// 64 rows of the not yet solved part, B_r -= A_(r,i) Y_i; CTA 0 also stores
// Y_i into X.  Grid: (row tiles, RHS chunks of NP_RC columns).
#define NP_RC 32
template <typename T, bool FWD>
__global__ void __launch_bounds__(NP_T) k_np_subst(const T *A, int lda, int n, int nrhs,
                                                   int i, const T *Inv, T *B, int ldb, T *X,
                                                   int ldx) {
  extern __shared__ __align__(16) unsigned char np_sm[];
  T *w = (T *)np_sm;                // 64 x 64 inverse, [row][col], ld NP_LD
  T *b = w + NP_NB * NP_LD;         // 64 x NP_RC block i of B, [row][col]
  T *y = b + NP_NB * (NP_RC + 1);   // 64 x NP_RC Y_i
  T *l = y + NP_NB * (NP_RC + 1);   // 64 x 64 coupling tile A_(r,i), [row][col]
  const int tid = threadIdx.x;
  const int k = i * NP_NB, jb = min(NP_NB, n - k);
  const int c0 = blockIdx.y * NP_RC, nc = min(NP_RC, nrhs - c0);
  const T *W = Inv + 2 * (size_t)NP_NB * NP_NB * i + (FWD ? 0 : (size_t)NP_NB * NP_NB);
  for (int e = tid; e < NP_NB * NP_NB; e += NP_T) {
    const int r = e % NP_NB, c = e / NP_NB;
    w[r * NP_LD + c] = (r < jb && c < jb) ? W[r + (size_t)c * NP_NB] : (T)0;
  }
  for (int e = tid; e < NP_NB * NP_RC; e += NP_T) {
    const int r = e % NP_NB, c = e / NP_NB;
    b[r * (NP_RC + 1) + c] = (r < jb && c < nc) ? B[(size_t)(k + r) + (size_t)(c0 + c) * ldb] : (T)0;
  }
  __syncthreads();
  // Y_i = Inv_i B_i: thread (r, c-phase) computes y[r][c] for c = cp, cp + 8, ...
  {
    const int r = tid % NP_NB, cp = tid / NP_NB;
    for (int c = cp; c < NP_RC; c += NP_T / NP_NB) {
      T acc = (T)0;
      for (int p = 0; p < NP_NB; ++p) acc = fma(w[r * NP_LD + p], b[p * (NP_RC + 1) + c], acc);
      y[r * (NP_RC + 1) + c] = acc;
    }
  }
  __syncthreads();
  if (blockIdx.x == 0)
    for (int e = tid; e < NP_NB * NP_RC; e += NP_T) {
      const int r = e % NP_NB, c = e / NP_NB;
      if (r < jb && c < nc) X[(size_t)(k + r) + (size_t)(c0 + c) * ldx] = y[r * (NP_RC + 1) + c];
    }
  // rows still to solve: below the block (forward) or above it (backward)
  const int nrest = FWD ? n - k - jb : k;
  const int ntile = (nrest + NP_NB - 1) / NP_NB;
  if ((int)blockIdx.x >= ntile) return;
  const int r0 = FWD ? k + jb + NP_NB * blockIdx.x : NP_NB * blockIdx.x;
  const int nr = min(NP_NB, (FWD ? n : k) - r0);
  for (int e = tid; e < NP_NB * NP_NB; e += NP_T) {
    const int r = e % NP_NB, c = e / NP_NB;
    l[r * NP_LD + c] = (r < nr && c < jb) ? A[(size_t)(r0 + r) + (size_t)(k + c) * lda] : (T)0;
  }
  __syncthreads();
  {
    const int r = tid % NP_NB, cp = tid / NP_NB;
    if (r < nr)
      for (int c = cp; c < nc; c += NP_T / NP_NB) {
        T acc = (T)0;
        for (int p = 0; p < NP_NB; ++p) acc = fma(l[r * NP_LD + p], y[p * (NP_RC + 1) + c], acc);
        B[(size_t)(r0 + r) + (size_t)(c0 + c) * ldb] -= acc;
      }
  }
}

template <typename T>
int lu_getrs_nopiv(cudaStream_t st, LuWork &w, int n, int nrhs, const T *A, int lda, T *B,
                   int ldb) {
  if (n <= 0 || nrhs <= 0) return DUST_OK;
  const int nb = (n + NP_NB - 1) / NP_NB;
  const T *inv0 = (const T *)((const char *)w.np.p + 256);
  const size_t xb = (size_t)n * nrhs * sizeof(T);
  DUST_TRY(devbuf_grow(w.np_x, xb));
  T *X = (T *)w.np_x.p;
  const int sm = (2 * NP_NB * NP_LD + 2 * NP_NB * (NP_RC + 1)) * (int)sizeof(T);
  static bool attr = false;  // per element type
  if (!attr) {
    DUST_CUDA(cudaFuncSetAttribute(k_np_subst<T, true>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    DUST_CUDA(cudaFuncSetAttribute(k_np_subst<T, false>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    attr = true;
  }
  const unsigned gy = (unsigned)((nrhs + NP_RC - 1) / NP_RC);
  // L Y = B: Y into X
  for (int i = 0; i < nb; ++i) {
    const int below = n - (i + 1) * NP_NB;
    const unsigned gx = (unsigned)std::max(1, (below + NP_NB - 1) / NP_NB);
    k_np_subst<T, true><<<dim3(gx, gy), NP_T, sm, st>>>(A, lda, n, nrhs, i, inv0, B, ldb, X, n);
  }
  // U X = Y: X back into B
  for (int i = nb - 1; i >= 0; --i) {
    const unsigned gx = (unsigned)std::max(1, i);
    k_np_subst<T, false><<<dim3(gx, gy), NP_T, sm, st>>>(A, lda, n, nrhs, i, inv0, X, n, B, ldb);
  }
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}

template int lu_getrs_nopiv<double>(cudaStream_t, LuWork &, int, int, const double *, int,
                                    double *, int);
template int lu_getrs_nopiv<float>(cudaStream_t, LuWork &, int, int, const float *, int, float *,
                                   int);
template int lu_getrf_nopiv<double>(cublasHandle_t, cudaStream_t, LuWork &, int, double *, int,
                                    int *, int, int *, float *);
template int lu_getrf_nopiv<float>(cublasHandle_t, cudaStream_t, LuWork &, int, float *, int,
                                   int *, int, int *, float *);
