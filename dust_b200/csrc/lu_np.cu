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
//   for each outer panel of NP_NBO columns, for each block column k (NP_NB
//   wide) in it:
//     k_np_diag   one CTA: unpivoted LU of the diagonal block in shared
//                 memory, its inverse triangles Linv (unit lower) and Uinv
//                 (upper) by substitution, max |l| of the block;
//     k_np_panel  L21 = A21 Uinv (row tiles, down to n) and U12 = Linv A12
//                 (column tiles, inside the outer panel), 64 x 64
//                 register-tiled products, max |l| of L21;
//     update      of the outer panel's own columns;
//   then the outer panel's U12 right of it (forward substitution over its
//   blocks with Linv) and the trailing update A22 -= L21 U12 of inner
//   dimension NP_NBO (tcgen05 TF32 GEMM for FP32, DGEMM for FP64), which
//   streams the trailing matrix a quarter as often as NP_NB-wide steps.
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
#define NP_NBO 256  // outer panel width (a multiple of NP_NB)
#define NP_T 256
#define NP_LD (NP_NB + 1)

__device__ __forceinline__ void np_note_lmax(unsigned *bits, float v) {
  atomicMax(bits, __float_as_uint(v));
}

// Diagonal block.  Threads 0..63 hold one column each in registers (the
// steps are unrolled, so every row index is a constant).  At step j the
// owner of column j scales its rows below j by the reciprocal of the pivot
// (as dgetf2 does) and publishes the multipliers in shared memory (two
// buffers, so one barrier per step), and every later column subtracts its
// row-j element times them.  The factored block then goes to shared memory
// and the inverse triangles are solved one column per thread, Uinv by
// threads 0..63 (back substitution) and Linv by threads 64..127 (forward
// substitution), reading the factors as broadcasts; columns of the inverse
// are zero above (Linv) or below (Uinv) the diagonal by the recurrences
// themselves.  The block's LU, max |l| and the inverses go to global memory.
#define NPD_T 128
template <typename T>
__global__ void __launch_bounds__(NPD_T) k_np_diag(T *A, int lda, int k, int jb, T *Linv,
                                                   T *Uinv, unsigned *lmax_bits) {
  extern __shared__ __align__(16) unsigned char np_sm[];
  T *a = (T *)np_sm;                   // the block, [row][col], ld NP_LD
  T *inv = a + NP_NB * NP_LD;          // Uinv, [row][col]
  T *linv = inv + NP_NB * NP_LD;       // Linv, [row][col]
  __shared__ T s_l[2][NP_NB];
  __shared__ T s_rd[NP_NB];            // 1 / U(r, r)
  const int tid = threadIdx.x;
  for (int e = tid; e < NP_NB * NP_NB; e += NPD_T) {
    const int i = e % NP_NB, c = e / NP_NB;
    a[i * NP_LD + c] = (i < jb && c < jb) ? A[(size_t)(k + i) + (size_t)(k + c) * lda]
                                          : (i == c ? (T)1 : (T)0);
  }
  __syncthreads();
  float lm = 0.f;
  bool zero = false;
  {
    const int t = tid;  // column (threads >= 64 only pass the barriers)
    T col[NP_NB];
#pragma unroll
    for (int r = 0; r < NP_NB; ++r) col[r] = t < NP_NB ? a[r * NP_LD + t] : (T)0;
#pragma unroll
    for (int j = 0; j < NP_NB; ++j) {
      if (j < jb) {
        if (t == j) {
          const T piv = col[j];
          if (piv == (T)0) zero = true;
          const T rinv = (T)1 / piv;
#pragma unroll
          for (int r = j + 1; r < NP_NB; ++r) {
            col[r] *= rinv;
            s_l[j & 1][r] = col[r];
            if (r < jb) lm = fmaxf(lm, (float)fabs((double)col[r]));
          }
        }
        __syncthreads();
        if (t > j && t < NP_NB) {
          const T u = col[j];
#pragma unroll
          for (int r = j + 1; r < NP_NB; ++r) col[r] = fma(-s_l[j & 1][r], u, col[r]);
        }
      }
    }
    __syncthreads();
    if (t < NP_NB)
#pragma unroll
      for (int r = 0; r < NP_NB; ++r) a[r * NP_LD + t] = col[r];
  }
  if (zero) lm = INFINITY;
  for (int o = 16; o > 0; o >>= 1) lm = fmaxf(lm, __shfl_xor_sync(0xffffffffu, lm, o));
  if ((tid & 31) == 0) np_note_lmax(lmax_bits, lm);
  __syncthreads();
  if (tid < NP_NB) s_rd[tid] = (T)1 / a[tid * NP_LD + tid];
  __syncthreads();
  {
    T x[NP_NB];
    if (tid < NP_NB) {
      // Uinv column c: U x = e_c, rows from the bottom
      const int c = tid;
#pragma unroll
      for (int r = NP_NB - 1; r >= 0; --r) {
        T acc = (r == c) ? (T)1 : (T)0;
#pragma unroll
        for (int p = r + 1; p < NP_NB; ++p) acc = fma(-a[r * NP_LD + p], x[p], acc);
        x[r] = acc * s_rd[r];
      }
#pragma unroll
      for (int r = 0; r < NP_NB; ++r) inv[r * NP_LD + c] = x[r];
    } else if (tid < 2 * NP_NB) {
      // Linv column c: L x = e_c (unit diagonal), rows from the top
      const int c = tid - NP_NB;
#pragma unroll
      for (int r = 0; r < NP_NB; ++r) {
        T acc = (r == c) ? (T)1 : (T)0;
#pragma unroll
        for (int p = 0; p < r; ++p) acc = fma(-a[r * NP_LD + p], x[p], acc);
        x[r] = acc;
      }
#pragma unroll
      for (int r = 0; r < NP_NB; ++r) linv[r * NP_LD + c] = x[r];
    }
  }
  __syncthreads();
  for (int e = tid; e < jb * jb; e += NPD_T) {
    const int r = e % jb, c = e / jb;
    A[(size_t)(k + r) + (size_t)(k + c) * lda] = a[r * NP_LD + c];
    Uinv[r + (size_t)c * NP_NB] = r <= c ? inv[r * NP_LD + c] : (T)0;
    Linv[r + (size_t)c * NP_NB] = r > c ? linv[r * NP_LD + c] : (r == c ? (T)1 : (T)0);
  }
}

// 64 x 64 tiles of the panel: blocks [0, nrb) take 64 rows of A21 (rows
// below the block, to n) and write A21 Uinv over them; blocks [nrb, nrb + ncb)
// take 64 columns of A12 (rows of the block, columns [cbeg, cend)) and write
// Linv A12.  Each thread computes a 4 x 4 piece of the tile from the two
// shared operands (the tile and the inverse triangle).
template <typename T>
__global__ void __launch_bounds__(NP_T) k_np_panel(T *A, int lda, int n, int k, int jb,
                                                   const T *Linv, const T *Uinv, int nrb,
                                                   int cbeg, int cend, unsigned *lmax_bits) {
  extern __shared__ __align__(16) unsigned char np_sm[];
  T *x = (T *)np_sm;            // 64 x 64 operand tile, [row][col], ld NP_LD
  T *w = x + NP_NB * NP_LD;     // 64 x 64 inverse, [row][col], ld NP_LD
  const int tid = threadIdx.x;
  const bool rows = (int)blockIdx.x < nrb;
  const int b = rows ? blockIdx.x : blockIdx.x - nrb;
  const int r0 = rows ? k + jb + NP_NB * b : k;      // first row of the tile in A
  const int c0 = rows ? k : cbeg + NP_NB * b;        // first column of the tile in A
  const int nr = rows ? min(NP_NB, n - r0) : jb;
  const int nc = rows ? jb : min(NP_NB, cend - c0);
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
  // C -= A B (m x nn, inner kk) on the tensor cores (FP32) or DGEMM
  auto update = [&](int m, int nn, int kk, const T *Am, const T *Bm, T *Cm) -> int {
    if (m <= 0 || nn <= 0 || kk <= 0) return DUST_OK;
    if (sizeof(T) == 4 && gemm_update == 1)
      return gemm_tf32_minus(st, m, nn, kk, (const float *)Am, lda, (const float *)Bm, lda,
                             (float *)Cm, lda);
    CUBLAS_CHECK(np_gemm_minus(cb, m, nn, kk, Am, lda, Bm, lda, Cm, lda));
    return DUST_OK;
  };
  auto at = [&](int r, int c) { return A + r + (size_t)c * lda; };
  // two levels: outer panels of NP_NBO columns factored in NP_NB steps that
  // update only the panel's own columns; then the panel's U12 (its unit lower
  // block's forward substitution, with the kept inverse triangles) and one
  // trailing update of inner dimension NP_NBO
  for (int K = 0; K < n; K += NP_NBO) {
    const int Ke = std::min(K + NP_NBO, n);
    for (int k = K; k < Ke; k += NP_NB) {
      const int jb = std::min(NP_NB, n - k), m2 = n - k - jb, wc = Ke - k - jb;
      T *Linv = inv0 + 2 * tri * (size_t)(k / NP_NB), *Uinv = Linv + tri;
      k_np_diag<T><<<1, NPD_T, smd, st>>>(A, lda, k, jb, Linv, Uinv, bits);
      const int nrb = (m2 + NP_NB - 1) / NP_NB, ncb = (wc + NP_NB - 1) / NP_NB;
      if (nrb + ncb > 0)
        k_np_panel<T><<<nrb + ncb, NP_T, smp, st>>>(A, lda, n, k, jb, Linv, Uinv, nrb, k + jb,
                                                     Ke, bits);
      DUST_TRY(update(m2, wc, jb, at(k + jb, k), at(k, k + jb), at(k + jb, k + jb)));
    }
    if (Ke < n) {
      const int ncb = (n - Ke + NP_NB - 1) / NP_NB;
      for (int k = K; k < Ke; k += NP_NB) {
        const T *Linv = inv0 + 2 * tri * (size_t)(k / NP_NB);
        k_np_panel<T><<<ncb, NP_T, smp, st>>>(A, lda, n, k, NP_NB, Linv, Linv, 0, Ke, n, bits);
        DUST_TRY(update(Ke - k - NP_NB, n - Ke, NP_NB, at(k + NP_NB, k), at(k, Ke),
                        at(k + NP_NB, Ke)));
      }
      DUST_TRY(update(n - Ke, n - Ke, Ke - K, at(Ke, K), at(K, Ke), at(Ke, Ke)));
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

// Block substitution with the kept inverse triangles, one cooperative launch
// per triangle (forward: blocks i ascending with Linv; backward: descending
// with Uinv).  At step i every CTA computes Y_i = Inv_i B_i for a chunk of
// NP_NB right-hand sides (B's block i is final: every earlier step ended at a
// grid barrier) and then updates its share of the 64-row tiles not yet
// solved, B_r -= A_(r,i) Y_i; CTA 0 stores Y_i into X.  The grid barrier
// spins with an iteration limit and raises the error word instead of
// hanging; every CTA then stops at the same step.
#define NP_SPIN_LIMIT (1ll << 24)

__device__ __forceinline__ bool np_grid_barrier(unsigned *bar, unsigned G, int *err) {
  __syncthreads();
  __shared__ int s_fail;
  if (threadIdx.x == 0) {
    s_fail = 0;
    volatile unsigned *vgen = bar + 1;
    const unsigned g0 = *vgen;
    __threadfence();
    const unsigned arrived = atomicAdd(bar, 1u);
    if (arrived == G - 1u) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      long long it = 0;
      while (*vgen == g0) {
        if (++it > NP_SPIN_LIMIT || *(volatile int *)err) {
          atomicExch(err, 1);
          s_fail = 1;
          break;
        }
        if (it > 64) __nanosleep(32);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return s_fail == 0;
}

// out (64 x 64) of thread (ty, tx): rows 4 ty .., columns 4 tx .. of L R, both
// [row][col] with ld NP_LD in shared memory
template <typename T>
__device__ __forceinline__ void np_mm64(const T *L, const T *R, int ty, int tx, T (&acc)[4][4]) {
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) acc[u][v] = (T)0;
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
}

template <typename T, bool FWD>
__global__ void __launch_bounds__(NP_T) k_np_subst(const T *A, int lda, int n, int nrhs,
                                                   const T *Inv, T *B, int ldb, T *X, int ldx,
                                                   unsigned *bar, int *err) {
  extern __shared__ __align__(16) unsigned char np_sm[];
  T *w = (T *)np_sm;               // Inv_i
  T *b = w + NP_NB * NP_LD;        // B_i (a chunk of right-hand sides)
  T *y = b + NP_NB * NP_LD;        // Y_i
  T *l = y + NP_NB * NP_LD;        // A_(r,i) of the CTA's first tile
  T *o = l + NP_NB * NP_LD;        // the update of a tile
  const int tid = threadIdx.x, ty = tid / 16, tx = tid % 16;
  const unsigned G = gridDim.x;
  const int nb = (n + NP_NB - 1) / NP_NB;
  // the inverse triangle and the first coupling tile of a step depend only
  // on the factors, so they are loaded before the grid barrier that ends the
  // previous step; only B's block i waits for it
  auto step_of = [&](int s) { return FWD ? s : nb - 1 - s; };
  auto load_inv_tile = [&](int s, T *lt) {
    const int i = step_of(s), k = i * NP_NB, jb = min(NP_NB, n - k);
    const T *W = Inv + 2 * (size_t)NP_NB * NP_NB * i + (FWD ? 0 : (size_t)NP_NB * NP_NB);
    const int nrest = FWD ? n - k - jb : k;
    const int ntile = (nrest + NP_NB - 1) / NP_NB;
    const int tile = blockIdx.x;
    const int r0 = FWD ? k + jb + NP_NB * tile : NP_NB * tile;
    const int nr = tile < ntile ? min(NP_NB, (FWD ? n : k) - r0) : 0;
    for (int e = tid; e < NP_NB * NP_NB; e += NP_T) {
      const int r = e % NP_NB, c = e / NP_NB;
      w[r * NP_LD + c] = (r < jb && c < jb) ? W[r + (size_t)c * NP_NB] : (T)0;
      lt[r * NP_LD + c] = (r < nr && c < jb) ? A[(size_t)(r0 + r) + (size_t)(k + c) * lda] : (T)0;
    }
  };
  load_inv_tile(0, l);
  for (int s = 0; s < nb; ++s) {
    const int i = step_of(s);
    const int k = i * NP_NB, jb = min(NP_NB, n - k);
    const int nrest = FWD ? n - k - jb : k;
    const int ntile = (nrest + NP_NB - 1) / NP_NB;
    const bool busy = blockIdx.x == 0 || (int)blockIdx.x < ntile;
    for (int c0 = 0; c0 < nrhs && busy; c0 += NP_NB) {
      const int nc = min(NP_NB, nrhs - c0);
      __syncthreads();
      for (int e = tid; e < NP_NB * NP_NB; e += NP_T) {
        const int r = e % NP_NB, c = e / NP_NB;
        // B changes between steps on other SMs: read it past L1
        b[r * NP_LD + c] =
            (r < jb && c < nc) ? __ldcg(B + (size_t)(k + r) + (size_t)(c0 + c) * ldb) : (T)0;
      }
      __syncthreads();
      T acc[4][4];
      np_mm64(w, b, ty, tx, acc);
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) y[(4 * ty + u) * NP_LD + 4 * tx + v] = acc[u][v];
      __syncthreads();
      if (blockIdx.x == 0)
        for (int e = tid; e < NP_NB * NP_NB; e += NP_T) {
          const int r = e % NP_NB, c = e / NP_NB;
          if (r < jb && c < nc) X[(size_t)(k + r) + (size_t)(c0 + c) * ldx] = y[r * NP_LD + c];
        }
      for (int tile = blockIdx.x; tile < ntile; tile += G) {
        const int r0 = FWD ? k + jb + NP_NB * tile : NP_NB * tile;
        const int nr = min(NP_NB, (FWD ? n : k) - r0);
        T *lt = l;
        if (tile != (int)blockIdx.x) {
          // a further tile of this CTA: its coupling block is loaded here
          lt = o;
          __syncthreads();
          for (int e = tid; e < NP_NB * NP_NB; e += NP_T) {
            const int r = e % NP_NB, c = e / NP_NB;
            lt[r * NP_LD + c] =
                (r < nr && c < jb) ? A[(size_t)(r0 + r) + (size_t)(k + c) * lda] : (T)0;
          }
          __syncthreads();
        }
        np_mm64(lt, y, ty, tx, acc);
        // through shared memory, then coalesced along the columns
        __syncthreads();
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int v = 0; v < 4; ++v) o[(4 * ty + u) * NP_LD + 4 * tx + v] = acc[u][v];
        __syncthreads();
        for (int e = tid; e < NP_NB * NP_NB; e += NP_T) {
          const int r = e % NP_NB, c = e / NP_NB;
          if (r < nr && c < nc) {
            T *bp = B + (size_t)(r0 + r) + (size_t)(c0 + c) * ldb;
            *bp = __ldcg(bp) - o[r * NP_LD + c];
          }
        }
      }
    }
    __syncthreads();
    if (s + 1 < nb) load_inv_tile(s + 1, l);
    if (!np_grid_barrier(bar, G, err)) return;
  }
}

template <typename T>
int lu_getrs_nopiv(cudaStream_t st, LuWork &w, int n, int nrhs, const T *A, int lda, T *B,
                   int ldb) {
  if (n <= 0 || nrhs <= 0) return DUST_OK;
  const T *inv0 = (const T *)((const char *)w.np.p + 256);
  const size_t xb = (size_t)n * nrhs * sizeof(T);
  DUST_TRY(devbuf_grow(w.np_x, xb + 256));
  T *X = (T *)((char *)w.np_x.p + 256);
  unsigned *bar = (unsigned *)w.np_x.p;  // arrivals, generation, error word
  int *err = (int *)(bar + 2);
  const int sm = 5 * NP_NB * NP_LD * (int)sizeof(T);
  static int G = 0;  // co-resident CTAs, per element type
  if (G == 0) {
    DUST_CUDA(cudaFuncSetAttribute(k_np_subst<T, true>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    DUST_CUDA(cudaFuncSetAttribute(k_np_subst<T, false>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    int dev = 0, nsm = 0, per = 0;
    DUST_CUDA(cudaGetDevice(&dev));
    DUST_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    DUST_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_np_subst<T, true>, NP_T, sm));
    G = std::max(1, nsm * std::max(per, 1));
  }
  const int nb = (n + NP_NB - 1) / NP_NB;
  const int g = std::min(G, std::max(1, nb - 1));
  DUST_CUDA(cudaMemsetAsync(bar, 0, 16, st));
  // L Y = B: Y into X; U X = Y: X back into B
  int ldn = n;
  {
    void *args[] = {(void *)&A, (void *)&lda, (void *)&n, (void *)&nrhs, (void *)&inv0,
                    (void *)&B, (void *)&ldb, (void *)&X, (void *)&ldn, (void *)&bar, (void *)&err};
    DUST_CUDA(cudaLaunchCooperativeKernel((void *)k_np_subst<T, true>, dim3(g), dim3(NP_T), args,
                                          sm, st));
  }
  {
    void *args[] = {(void *)&A, (void *)&lda, (void *)&n, (void *)&nrhs, (void *)&inv0,
                    (void *)&X, (void *)&ldn, (void *)&B, (void *)&ldb, (void *)&bar, (void *)&err};
    DUST_CUDA(cudaLaunchCooperativeKernel((void *)k_np_subst<T, false>, dim3(g), dim3(NP_T), args,
                                          sm, st));
  }
  int herr = 0;
  DUST_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  DUST_CUDA(cudaStreamSynchronize(st));
  return herr ? DUST_ERR_TIMEOUT : DUST_OK;
}

template int lu_getrs_nopiv<double>(cudaStream_t, LuWork &, int, int, const double *, int,
                                    double *, int);
template int lu_getrs_nopiv<float>(cudaStream_t, LuWork &, int, int, const float *, int, float *,
                                   int);
template int lu_getrf_nopiv<double>(cublasHandle_t, cudaStream_t, LuWork &, int, double *, int,
                                    int *, int, int *, float *);
template int lu_getrf_nopiv<float>(cublasHandle_t, cudaStream_t, LuWork &, int, float *, int,
                                   int *, int, int *, float *);
