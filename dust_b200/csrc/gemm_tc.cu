// gemm_tc.cu -- tensor-core (tcgen05, sm_100a) GEMM for the trailing updates
// of the mixed-precision LU:  C -= A B  (column-major FP32 operands read as
// TF32, FP32 accumulation in tensor memory).
//
// One CTA computes a 128 x 128 tile of C with 128 threads:
//  * A (128 x K) and B (K x 128) tiles are staged by all threads through
//    two shared-memory stages of BK = 32 in the canonical K-major,
//    no-swizzle UMMA layout (8-row x 16-byte core matrices; SBO = 128 B
//    between 8-row groups, LBO = 2 KiB between 16-byte K chunks);
//  * one elected thread issues tcgen05.mma.kind::tf32 (M = 128, N = 128,
//    K = 8 per instruction) into a 128-column TMEM accumulator and commits
//    each stage to an mbarrier, so the next stage loads while the tensor
//    core works;
//  * every wait on an mbarrier is bounded: on timeout the kernel raises an
//    error flag, waits (bounded) for its own MMAs, frees its TMEM and
//    returns;
//  * the epilogue reads the accumulator with tcgen05.ld (each warp its 32
//    TMEM lanes) and subtracts it from C with coalesced column stores.
#include <cuda.h>

#include "dust_common.cuh"
#include "fmm_internal.h"
#include "tc_common.cuh"

#define TC_BM 128
#define TC_BN 128
#define TC_BK 32
#define TC_THREADS 128
#define TC_STAGE_BYTES (TC_BM * TC_BK * 4 + TC_BN * TC_BK * 4)  // 32 KiB

// byte offset of element (row r, k) in a K-major no-swizzle tile of 128 rows
__device__ __forceinline__ uint32_t kmaj_off(int r, int k) {
  return (uint32_t)((k >> 2) * 2048 + (r >> 3) * 128 + (r & 7) * 16 + (k & 3) * 4);
}

__global__ void __launch_bounds__(TC_THREADS) k_gemm_tf32_minus(int m, int n, int k, const float *A,
                                                                int lda, const float *B, int ldb,
                                                                float *C, int ldc, int *err,
                                                                float sign) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  __shared__ __align__(8) uint64_t s_mbar[2];
  __shared__ uint32_t s_tmem;
  unsigned char *sm = (unsigned char *)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int gm0 = blockIdx.x * TC_BM, gn0 = blockIdx.y * TC_BN;
  const int nk = (k + TC_BK - 1) / TC_BK;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&s_tmem)),
                 "r"(TC_BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_mbar[0])));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_mbar[1])));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = s_tmem;

  // stage loader: A rows gm0.., k cols; B cols gn0.., k rows
  auto load_stage = [&](int kt, int s) {
    unsigned char *sa = sm + s * TC_STAGE_BYTES;
    unsigned char *sb = sa + TC_BM * TC_BK * 4;
    const int k0 = kt * TC_BK;
    // A: 128 rows x 32 k; column k of the tile is contiguous in global
    for (int e = tid; e < TC_BM * TC_BK; e += TC_THREADS) {
      int r = e & (TC_BM - 1), kk = e >> 7;
      int gr = gm0 + r, gk = k0 + kk;
      float v = (gr < m && gk < k) ? A[(size_t)gr + (size_t)gk * lda] : 0.f;
      *(float *)(sa + kmaj_off(r, kk)) = v;
    }
    // B: 128 columns (n) x 32 k; each column's k run is contiguous
    for (int e = tid; e < TC_BN * (TC_BK / 4); e += TC_THREADS) {
      int c = e / (TC_BK / 4), kq = (e % (TC_BK / 4)) * 4;
      int gc = gn0 + c, gk = k0 + kq;
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (gc < n) {
        const float *bp = B + (size_t)gc * ldb + gk;
        if (gk + 3 < k) {
          v.x = bp[0];
          v.y = bp[1];
          v.z = bp[2];
          v.w = bp[3];
        } else {
          if (gk < k) v.x = bp[0];
          if (gk + 1 < k) v.y = bp[1];
          if (gk + 2 < k) v.z = bp[2];
        }
      }
      *(float4 *)(sb + kmaj_off(c, kq)) = v;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  };

  // tf32 x tf32 -> f32, M = 128, N = 128, both K-major
  const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_BN >> 3) << 17) |
                         ((uint32_t)(TC_BM >> 4) << 24);
  bool ok = true;
  if (nk > 0) load_stage(0, 0);
  __syncthreads();
  for (int kt = 0; kt < nk; ++kt) {
    const int s = kt & 1;
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t sa = smem_u32(sm + s * TC_STAGE_BYTES);
      const uint32_t sb = sa + TC_BM * TC_BK * 4;
      for (int j = 0; j < TC_BK / 8; ++j) {
        // K elements 8j .. 8j+7 = 16-byte chunks 2j, 2j+1
        uint64_t ad = make_sdesc(sa + 2 * j * 2048, 2048, 128);
        uint64_t bd = make_sdesc(sb + 2 * j * 2048, 2048, 128);
        uint32_t acc = (kt > 0 || j > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(
                tmem),
            "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
      }
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
              smem_u32(&s_mbar[s])));
    }
    if (kt + 1 < nk) {
      const int s1 = s ^ 1;
      // the stage is free once the MMAs of tile kt-1 (its last use) are done
      if (kt >= 1 && !mbar_wait(smem_u32(&s_mbar[s1]), (uint32_t)(((kt - 1) >> 1) & 1))) ok = false;
      load_stage(kt + 1, s1);
    }
    __syncthreads();
  }
  if (nk > 0 && !mbar_wait(smem_u32(&s_mbar[(nk - 1) & 1]), (uint32_t)(((nk - 1) >> 1) & 1)))
    ok = false;
  // CTA-uniform: the tcgen05.ld below must run convergently in every warp
  const int all_ok = __syncthreads_and(ok ? 1 : 0);
  if (!all_ok) {
    if (tid == 0) atomicExch(err, 1);
    // give the MMAs still in flight a second bounded wait before TMEM is freed
    if (nk > 0) mbar_wait(smem_u32(&s_mbar[(nk - 1) & 1]), (uint32_t)(((nk - 1) >> 1) & 1));
  }
  asm volatile("tcgen05.fence::after_thread_sync;");
  // epilogue: warp w owns TMEM lanes 32w .. 32w+31 = tile rows
  if (all_ok && nk > 0) {
    const int r = warp * 32 + lane, gr = gm0 + r;
    for (int c0 = 0; c0 < TC_BN; c0 += 8) {
      uint32_t v[8];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
            "=r"(v[7])
          : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (gr < m)
        for (int j = 0; j < 8; ++j) {
          int gc = gn0 + c0 + j;
          if (gc < n) C[(size_t)gr + (size_t)gc * ldc] += sign * __uint_as_float(v[j]);
        }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_BN));
}

// ---------------------------------------------------------------------------
// TMA-fed pipelined variant (used when both operands are 16-byte aligned with
// leading dimensions that are multiples of 4 floats).
//
//  * tile 128 x 256 of C per CTA, BK = 32, TP_STAGES stages of 48 KiB;
//  * A (column-major, M contiguous) is loaded MN-major: four TMA boxes of
//    32 (M) x 32 (K) floats with the 128-byte swizzle, i.e. the canonical
//    MN-major SW128 layout (128-byte rows along M, 8-row K groups 1 KiB
//    apart = SBO, 32-element M groups 4 KiB apart = LBO);
//  * B (column-major, K contiguous) is loaded K-major: one TMA box of
//    32 (K) x 256 (N) floats with the 128-byte swizzle (8-row N groups
//    1 KiB apart = SBO); the K step of an instruction advances the start
//    address by 32 bytes inside the swizzle atom;
//  * warp 0 lane 0 produces (TMA, mbarrier expect-tx), warp 1 lane 0 issues
//    tcgen05.mma (M = 128, N = 256, K = 8) and commits each stage back to
//    its empty barrier; the accumulator lives in 256 TMEM columns;
//  * every wait is bounded; on timeout the kernel flags the error, waits
//    (bounded) for the copies and MMAs it issued, frees TMEM and returns.
#define TP_BM 128
#define TP_BN 256
#define TP_BK 32
#define TP_STAGES 4
#define TP_A_BYTES (TP_BM * TP_BK * 4)  // 16 KiB
#define TP_B_BYTES (TP_BN * TP_BK * 4)  // 32 KiB
#define TP_STAGE_BYTES (TP_A_BYTES + TP_B_BYTES)
// MN-major TF32 operands use the 128-byte swizzle with 32-byte atomicity
// (UMMA layout type 1; TMA CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B): 128-byte
// rows along M, 4-row K groups of 512 B (SBO), 32-element M groups one
// 4 KiB box apart (LBO)
#ifndef TP_A_MN_LAYOUT
#define TP_A_MN_LAYOUT 1
#endif
#ifndef TP_A_MN_LBO
#define TP_A_MN_LBO 4096
#endif
#ifndef TP_A_MN_SBO
#define TP_A_MN_SBO 512
#endif
#ifndef TP_A_MN_TMA_SWIZZLE
#define TP_A_MN_TMA_SWIZZLE CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B
#endif

__device__ __forceinline__ uint64_t make_sdesc_sw(uint32_t saddr, uint32_t lbo, uint32_t sbo,
                                                  uint32_t layout) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version (sm_100)
  d |= (uint64_t)layout << 61;  // 2 = 128-byte swizzle, 1 = 128-byte with 32-byte atoms
  return d;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y,
                                            uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, "
      "{%2, %3}], [%4];" ::"r"(dst),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(mbar)
      : "memory");
}

// AK: A stored K-major (row-major M x K, i.e. the transpose is column-major)
// and loaded like B; otherwise A is column-major and loaded MN-major.
template <bool AK>
__global__ void __launch_bounds__(TC_THREADS, 1)
    k_gemm_tf32_tma(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                    int m, int n, int k, float *C, int ldc, int *err, float sign) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  __shared__ __align__(8) uint64_t s_full[TP_STAGES], s_empty[TP_STAGES], s_done;
  __shared__ uint32_t s_tmem;
  __shared__ int s_fail, s_issued, s_consumed;
  unsigned char *sm = (unsigned char *)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int gm0 = blockIdx.x * TP_BM, gn0 = blockIdx.y * TP_BN;
  const int nk = (k + TP_BK - 1) / TP_BK;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&s_tmem)),
                 "r"(TP_BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 32) {
    for (int s = 0; s < TP_STAGES; ++s) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_full[s])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_empty[s])));
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_done)));
    asm volatile("fence.mbarrier_init.release.cluster;");
    s_fail = 0;
    s_issued = 0;
    s_consumed = 0;
  }
  if (tid == 64) {
    asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&tmA) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&tmB) : "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = s_tmem;
  const uint32_t sbase = smem_u32(sm);

  if (warp == 0 && lane == 0) {
    // producer
    int kt = 0;
    for (; kt < nk; ++kt) {
      const int s = kt % TP_STAGES;
      if (kt >= TP_STAGES &&
          !mbar_wait(smem_u32(&s_empty[s]), (uint32_t)(((kt / TP_STAGES) - 1) & 1))) {
        atomicExch(&s_fail, 1);
        break;
      }
      if (*(volatile int *)&s_fail) break;
      const uint32_t fb = smem_u32(&s_full[s]);
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb),
                   "r"((uint32_t)TP_STAGE_BYTES)
                   : "memory");
      const uint32_t sa = sbase + s * TP_STAGE_BYTES;
      if (AK)
        tma_load_2d(sa, &tmA, kt * TP_BK, gm0, fb);
      else
        for (int i = 0; i < TP_BM / 32; ++i)
          tma_load_2d(sa + i * 4096, &tmA, gm0 + 32 * i, kt * TP_BK, fb);
      tma_load_2d(sa + TP_A_BYTES, &tmB, kt * TP_BK, gn0, fb);
    }
    s_issued = kt;
  } else if (warp == 1 && lane == 0) {
    // MMA issuer: tf32 x tf32 -> f32, M = 128, N = 256, A MN-major, B K-major
    const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((AK ? 0u : 1u) << 15) |
                           ((uint32_t)(TP_BN >> 3) << 17) | ((uint32_t)(TP_BM >> 4) << 24);
    int kt = 0;
    for (; kt < nk; ++kt) {
      const int s = kt % TP_STAGES;
      if (!mbar_wait(smem_u32(&s_full[s]), (uint32_t)((kt / TP_STAGES) & 1))) {
        atomicExch(&s_fail, 1);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t sa = sbase + s * TP_STAGE_BYTES, sb = sa + TP_A_BYTES;
#pragma unroll
      for (int j = 0; j < TP_BK / 8; ++j) {
        const uint64_t ad = AK ? make_sdesc_sw(sa + j * 32, 16, 1024, 2)
                               : make_sdesc_sw(sa + j * 1024, TP_A_MN_LBO, TP_A_MN_SBO,
                                               TP_A_MN_LAYOUT);
        const uint64_t bd = make_sdesc_sw(sb + j * 32, 16, 1024, 2);
        const uint32_t acc = (kt > 0 || j > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(
                tmem),
            "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
      }
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
              smem_u32(&s_empty[s])));
    }
    s_consumed = kt;
    // completes once every MMA issued above has finished
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            smem_u32(&s_done)));
  }
  __syncwarp();
  bool ok = mbar_wait(smem_u32(&s_done), 0u);
  const int all_ok = __syncthreads_and(ok && !*(volatile int *)&s_fail);
  if (!all_ok) {
    if (tid == 0) {
      atomicExch(err, 1);
      // copies issued but never consumed: wait (bounded) for them to land
      for (int kt = s_consumed; kt < s_issued; ++kt)
        mbar_wait(smem_u32(&s_full[kt % TP_STAGES]), (uint32_t)((kt / TP_STAGES) & 1));
    }
    if (!ok) mbar_wait(smem_u32(&s_done), 0u);
  }
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (all_ok && nk > 0) {
    const int r = warp * 32 + lane, gr = gm0 + r;
    for (int c0 = 0; c0 < TP_BN; c0 += 16) {
      if (gn0 + c0 >= n) break;  // warp-uniform
      uint32_t v[16];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
          "%11, %12, %13, %14, %15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
            "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
            "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
      // the 16 loads of C are issued back to back, then the 16 stores
      float cv[16];
      float *cp = C + (size_t)gr + (size_t)(gn0 + c0) * ldc;
      const int ncol = min(16, n - gn0 - c0);
#pragma unroll
      for (int j = 0; j < 16; ++j) cv[j] = (gr < m && j < ncol) ? __ldcg(cp + (size_t)j * ldc) : 0.f;
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int j = 0; j < 16; ++j)
        if (gr < m && j < ncol) __stcg(cp + (size_t)j * ldc, cv[j] + sign * __uint_as_float(v[j]));
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TP_BN));
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}

// 2-D FP32 map of a column-major (rows x cols, ld) matrix, box (32 rows x
// box_cols), zero fill out of bounds
static bool encode_cm(CUtensorMap *map, const float *p, int rows, int cols, int ld, int box_cols,
                      CUtensorMapSwizzle swz) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {(cuuint64_t)rows, (cuuint64_t)cols};
  cuuint64_t strides[1] = {(cuuint64_t)ld * 4};
  cuuint32_t box[2] = {32u, (cuuint32_t)box_cols};
  cuuint32_t es[2] = {1u, 1u};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void *)p, dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

static DevBuf g_tc_err;

template <bool AK>
static int launch_tma(cudaStream_t st, const CUtensorMap &ta, const CUtensorMap &tb, int m, int n,
                      int k, float *C, int ldc, float sign) {
  const int smem_t = TP_STAGES * TP_STAGE_BYTES + 1024;
  static bool attr_t = false;
  if (!attr_t) {
    DUST_CUDA(cudaFuncSetAttribute(k_gemm_tf32_tma<AK>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, smem_t));
    attr_t = true;
  }
  dim3 grd((m + TP_BM - 1) / TP_BM, (n + TP_BN - 1) / TP_BN);
  k_gemm_tf32_tma<AK><<<grd, TC_THREADS, smem_t, st>>>(ta, tb, m, n, k, C, ldc,
                                                       (int *)g_tc_err.p, sign);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}

// C += sign * At^T B with At (k x m, column-major, ldat): A given K-major
int gemm_tf32_acc_tn(cudaStream_t st, int m, int n, int k, const float *At, int ldat,
                     const float *B, int ldb, float *C, int ldc, float sign) {
  if (m <= 0 || n <= 0 || k <= 0) return DUST_OK;
  if (!g_tc_err.p) {
    DUST_TRY(devbuf_grow(g_tc_err, 16));
    DUST_CUDA(cudaMemset(g_tc_err.p, 0, 16));
  }
  if ((uintptr_t)At % 16 || (uintptr_t)B % 16 || ldat % 4 || ldb % 4) return DUST_ERR_BAD_ARG;
  CUtensorMap ta, tb;
  if (!encode_cm(&ta, At, k, m, ldat, TP_BM, CU_TENSOR_MAP_SWIZZLE_128B) ||
      !encode_cm(&tb, B, k, n, ldb, TP_BN, CU_TENSOR_MAP_SWIZZLE_128B))
    return DUST_ERR_CUDA;
  return launch_tma<true>(st, ta, tb, m, n, k, C, ldc, sign);
}

// C += sign * A B
int gemm_tf32_acc(cudaStream_t st, int m, int n, int k, const float *A, int lda, const float *B,
                  int ldb, float *C, int ldc, float sign) {
  if (m <= 0 || n <= 0 || k <= 0) return DUST_OK;
  if (!g_tc_err.p) {
    DUST_TRY(devbuf_grow(g_tc_err, 16));
    DUST_CUDA(cudaMemset(g_tc_err.p, 0, 16));
  }
  const bool aligned = ((uintptr_t)A % 16 == 0) && ((uintptr_t)B % 16 == 0) && lda % 4 == 0 &&
                       ldb % 4 == 0;
  if (aligned) {
    CUtensorMap ta, tb;
    if (encode_cm(&ta, A, m, k, lda, TP_BK, TP_A_MN_TMA_SWIZZLE) &&
        encode_cm(&tb, B, k, n, ldb, TP_BN, CU_TENSOR_MAP_SWIZZLE_128B))
      return launch_tma<false>(st, ta, tb, m, n, k, C, ldc, sign);
  }
  const int smem = 2 * TC_STAGE_BYTES + 1024;
  static bool attr = false;
  if (!attr) {
    DUST_CUDA(cudaFuncSetAttribute(k_gemm_tf32_minus, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   smem));
    attr = true;
  }
  dim3 grd((m + TC_BM - 1) / TC_BM, (n + TC_BN - 1) / TC_BN);
  k_gemm_tf32_minus<<<grd, TC_THREADS, smem, st>>>(m, n, k, A, lda, B, ldb, C, ldc,
                                                   (int *)g_tc_err.p, sign);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}

int gemm_tf32_minus(cudaStream_t st, int m, int n, int k, const float *A, int lda,
                    const float *B, int ldb, float *C, int ldc) {
  return gemm_tf32_acc(st, m, n, k, A, lda, B, ldb, C, ldc, -1.0f);
}

int gemm_tf32_error(cudaStream_t st) {
  if (!g_tc_err.p) return DUST_OK;
  int h = 0;
  DUST_CUDA(cudaMemcpyAsync(&h, g_tc_err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  DUST_CUDA(cudaStreamSynchronize(st));
  return h ? DUST_ERR_TIMEOUT : DUST_OK;
}

extern "C" int dust_tc_gemm_tf32_minus(int m, int n, int k, const float *A, int lda,
                                       const float *B, int ldb, float *C, int ldc, void *stream) {
  if (m < 0 || n < 0 || k < 0 || (m && n && k && (!A || !B || !C))) return DUST_ERR_BAD_ARG;
  if (lda < m || ldb < k || ldc < m) return DUST_ERR_BAD_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  DUST_TRY(gemm_tf32_minus(st, m, n, k, A, lda, B, ldb, C, ldc));
  return gemm_tf32_error(st);
}
