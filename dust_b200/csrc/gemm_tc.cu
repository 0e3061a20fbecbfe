// gemm_tc.cu -- FP32 trailing-update GEMM of the mixed-precision LU:
// C -= A B (column-major).  This first version is a shared-memory tiled
// CUDA-core kernel; the tensor-core (tcgen05) kernel replaces it.
#include "dust_common.cuh"

#define TG_BM 64
#define TG_BN 64
#define TG_BK 16

__global__ void __launch_bounds__(256) k_sgemm_minus(int m, int n, int k, const float *A,
                                                     int lda, const float *B, int ldb,
                                                     float *C, int ldc) {
  __shared__ float sA[TG_BK][TG_BM + 4];
  __shared__ float sB[TG_BK][TG_BN + 4];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int bm = blockIdx.x * TG_BM, bn = blockIdx.y * TG_BN;
  float acc[4][4] = {};
  for (int k0 = 0; k0 < k; k0 += TG_BK) {
    for (int t = threadIdx.x; t < TG_BK * TG_BM; t += 256) {
      int r = t % TG_BM, c = t / TG_BM;
      int gr = bm + r, gc = k0 + c;
      sA[c][r] = (gr < m && gc < k) ? A[(size_t)gr + (size_t)gc * lda] : 0.f;
    }
    for (int t = threadIdx.x; t < TG_BK * TG_BN; t += 256) {
      int r = t % TG_BK, c = t / TG_BK;
      int gr = k0 + r, gc = bn + c;
      sB[r][c] = (gr < k && gc < n) ? B[(size_t)gr + (size_t)gc * ldb] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < TG_BK; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = sA[kk][tx + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = sB[kk][ty + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int gr = bm + tx + 16 * i, gc = bn + ty + 16 * j;
      if (gr < m && gc < n) C[(size_t)gr + (size_t)gc * ldc] -= acc[i][j];
    }
}

int gemm_tf32_minus(cudaStream_t st, int m, int n, int k, const float *A, int lda,
                    const float *B, int ldb, float *C, int ldc) {
  if (m <= 0 || n <= 0 || k <= 0) return DUST_OK;
  dim3 grd((m + TG_BM - 1) / TG_BM, (n + TG_BN - 1) / TG_BN);
  k_sgemm_minus<<<grd, 256, 0, st>>>(m, n, k, A, lda, B, ldb, C, ldc);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}
