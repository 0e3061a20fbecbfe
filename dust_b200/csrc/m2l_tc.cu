// m2l_tc.cu -- multipole-to-local translation of levels >= 2 on the tensor
// cores (FP32C mode, multipole degree <= 4).
//
// M2L_multipole (src/fmm/mod_multipole.f90:282-356) in the scaled form of
// m2l.cu:  g(m') = (-1)^|m'| / m'! * sum_n Dhat(m'+n) x ahat(n).  For one
// offset o between target and source cell the map ahat -> g is fixed, and
// the cross product splits into six scalar products per component pair:
//   g_x += A_z B_y - A_y B_z,  g_y += A_x B_z - A_z B_x,  g_z += A_y B_x - A_x B_y
// with A_c[t][n] = ahat_c(n) of the source of target t at offset o and
// B_d[m'][n] = Dhat_d(m'+n) of offset o.  A CTA takes 128 targets of one
// level and octant class (they share the 189 offsets of their interaction
// lists, mod_octree.f90:440-476) as the M = 128 rows of tcgen05.mma
// (kind::tf32, N = 64 outputs m', K = 40 monomials n) and accumulates the
// three g components in TMEM over all offsets.
//
// Precision: 3xTF32.  Each FP32 operand is split into its TF32 rounding and
// the FP32 remainder, and a product is Ah Bh + Ah Bl + Al Bh, which keeps
// about FP32 accuracy; the tables are split from their FP64 values.
//
// Roles (448 threads):
//  warps 0-7  producers: per offset look up the 128 source cells (empty,
//             inactive or missing ones give zero rows) and copy their
//             pre-split coefficients (TF32 high part, FP32 remainder) with
//             cp.async into the canonical no-swizzle K-major layout, one
//             (component, split) per stage, four stages in rotation;
//  warps 8-11 drain the TMEM accumulators to FP64 (one TMEM lane quarter =
//             32 targets per warp, all columns per thread) every MT_GROUP
//             offsets while the tensor core runs the next group, and at the
//             end add the rescaled locals to the FP64 b and g;
//  warp 12    lane 0 issues the 90 tcgen05.mma of an offset and commits;
//  warp 13    lane 0 streams the offset's table image (61,440 B, prepared
//             once per level in the operand layout) with one bulk copy.
// Offsets where no target of the CTA has a source are skipped altogether.
// Every mbarrier wait is bounded: a role that gives up raises a CTA flag
// that stops the others; the kernel then reports through `err`, waits
// (bounded) for its copies and MMAs, frees TMEM and returns.
#include <cstring>
#include <vector>

#include "dust_common.cuh"
#include "fmm_internal.h"
#include "tc_common.cuh"

#define MT_M 128
#define MT_K 40
#define MT_N 64
#define MT_KCH (MT_K / 4)
#define MT_ASPLIT (MT_KCH * 2048)  // one split of an A buffer: 128 rows x 40
#define MT_BSPLIT (MT_KCH * 1024)  // one split of one component table: 64 rows
#define MT_BCOMP (2 * MT_BSPLIT)
#define MT_BIMG (3 * MT_BCOMP)  // one offset: 3 components x (high, low)
#define MT_SMEM (2 * MT_BIMG + 4 * MT_ASPLIT + 1024)  // 2 table images, 4 A stages
#define MT_NCAND 216

// byte offsets in the canonical K-major no-swizzle layouts (core matrices of
// 8 rows x 16 B; 8-row groups 128 B apart; K chunks of 4 floats one
// row-count x 16 B apart)
__host__ __device__ inline uint32_t mt_aoff(int r, int k) {
  return (uint32_t)((k >> 2) * 2048 + (r >> 3) * 128 + (r & 7) * 16 + (k & 3) * 4);
}
__host__ __device__ inline uint32_t mt_boff(int r, int k) {
  return (uint32_t)((k >> 2) * 1024 + (r >> 3) * 128 + (r & 7) * 16 + (k & 3) * 4);
}

// table image of one level: for each of the 343 offsets in [-3,3]^3, per
// component d the high and low TF32 parts of B_d[m'][n] = Dhat_d(m'+n)
__global__ void k_m2l_tc_image(const double *dtab, const uint16_t *isum, int nD, int nm, int nm1,
                               int nout, float *img) {
  size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)343 * 3 * MT_N * MT_K) return;
  const int n = (int)(e % MT_K), r = (int)((e / MT_K) % MT_N), c = (int)((e / (MT_K * MT_N)) % 3);
  const size_t tab = e / (3 * MT_N * MT_K);
  double v = 0.0;
  if (r < nout && n < nm) v = dtab[((size_t)tab * nD + isum[(size_t)n * nm1 + r]) * 3 + c];
  const float hi = tf32_rna((float)v);
  const float lo = (float)(v - (double)hi);
  char *base = (char *)img + tab * MT_BIMG + (size_t)c * MT_BCOMP;
  *(float *)(base + mt_boff(r, n)) = hi;
  *(float *)(base + MT_BSPLIT + mt_boff(r, n)) = lo;
}

// scaled source coefficients ahat(n, c) = a(n, c) / (n! h^|n|) of the active
// cells of levels >= 2 in FP32, split for 3xTF32 into the TF32 rounding and
// the FP32 remainder: [cell][c][hi, lo][40] (zero beyond nm)
__global__ void k_scale_a_tc(FmmDev d, uint32_t c0, uint32_t nact, float *out) {
  size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t tot = (size_t)(nact - c0) * 3 * MT_K;
  if (e >= tot) return;
  const uint32_t ci = c0 + (uint32_t)(e / (3 * MT_K));
  const int r = (int)(e % (3 * MT_K)), c = r / MT_K, nn = r % MT_K;
  float v = 0.f;
  if (nn < d.nm) {
    int ni, nj, nk;
    mono_exp(nn, ni, nj, nk);
    const int l = d.act_lev[ci];
    double hi = 1.0 / d.G.csize[l], hp = 1.0;
    for (int q = 0; q < ni + nj + nk; ++q) hp *= hi;
    v = (float)(d.A[(size_t)ci * 3 * d.nm + 3 * nn + c] * d.inv_fact[nn] * hp);
  }
  const float hv = tf32_rna(v);
  float *o = out + (size_t)(ci - c0) * 6 * MT_K + 2 * c * MT_K + nn;
  o[0] = hv;
  o[MT_K] = v - hv;
}

struct MtCand {
  int ox, oy, oz;
  bool adj;
};
__device__ __forceinline__ MtCand mt_cand(int cand, int bx, int by, int bz) {
  MtCand m;
  m.ox = cand % 6 - 2 - bx;
  m.oy = (cand / 6) % 6 - 2 - by;
  m.oz = cand / 36 - 2 - bz;
  m.adj = abs(m.ox) <= 1 && abs(m.oy) <= 1 && abs(m.oz) <= 1;
  return m;
}

// Interaction lists of every batch: src[b][cand][r] = the active non-empty
// source cell of target r at candidate offset cand (or -1), mask[b] = the
// candidates with a source for some target; also counts the M2L pairs.
__global__ void k_m2l_tc_lists(FmmDev d, const int4 *batches, const uint32_t *list, int *src,
                               uint32_t *mask) {
  const int4 bd = batches[blockIdx.x];
  const int l = bd.x, q = bd.y, t0 = bd.z, cnt = bd.w;
  const int bx = q & 1, by = (q >> 1) & 1, bz = (q >> 2) & 1;
  const int r = threadIdx.x, lane = r & 31;
  const uint32_t lo_l = d.G.lev_off[l];
  const int sh = 3 * (d.G.ll - l);
  __shared__ uint32_t s_mask[7];
  if (r < 7) s_mask[r] = 0;
  __syncthreads();
  int ti = -1000, tj = -1000, tk = -1000;
  if (r < cnt) cart_of_key(d.G, l, d.act_key[list[t0 + r]], ti, tj, tk);
  int *out = src + (size_t)blockIdx.x * MT_NCAND * MT_M;
  unsigned long long npairs = 0;
  for (int w = 0; w < 7; ++w) {
    uint32_t bits = 0;
    for (int b = 0; b < 32; ++b) {
      const int cand = w * 32 + b;
      if (cand >= MT_NCAND) break;
      const MtCand m = mt_cand(cand, bx, by, bz);
      int sc = -1;
      if (!m.adj && r < cnt) {
        const int si = ti + m.ox, sj = tj + m.oy, sk = tk + m.oz;
        if (cart_in(d.G, l, si, sj, sk)) {
          const uint32_t skey = key_of(d.G, l, si, sj, sk);
          if ((d.flags[lo_l + skey] & FL_ACTIVE) &&
              d.cstart[(skey + 1u) << sh] > d.cstart[skey << sh])
            sc = (int)d.cidx[lo_l + skey];
        }
      }
      out[(size_t)cand * MT_M + r] = sc;
      if (sc >= 0) {
        bits |= 1u << b;
        ++npairs;
      }
    }
    bits = __reduce_or_sync(0xffffffffu, bits);
    if (lane == 0 && bits) atomicOr(&s_mask[w], bits);
  }
  for (int o = 16; o > 0; o >>= 1) npairs += __shfl_xor_sync(0xffffffffu, npairs, o);
  if (lane == 0 && d.counters && npairs) atomicAdd((unsigned long long *)d.counters, npairs);
  __syncthreads();
  if (r < 7) mask[(size_t)blockIdx.x * 8 + r] = s_mask[r];
}

#define MT_NOUT 56  // output monomials of the drain and epilogue (nout <= 56)

// Drain of one accumulator set (the FP32 sums of a group of offsets): the
// drain warp's TMEM lane quarter holds its 32 targets, the thread is target
// row r; all 3 x nout sums are added in FP64 to the CTA's scratch
// scr[e][m'][r] (stored, not added, for the first group), a layout in which
// a warp's 32 targets are contiguous.  16 columns per tcgen05.ld, their 16
// FP64 partial sums loaded together.
__device__ __forceinline__ void mt_drain(uint32_t tmem, int quarter, int set, int r, int nout,
                                         bool first, double *__restrict__ scr) {
  const uint32_t base = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(set * 256);
#pragma unroll 1
  for (int e = 0; e < 3; ++e) {
#pragma unroll 1
    for (int j0 = 0; j0 < nout; j0 += 16) {
      uint32_t v[16];
      const uint32_t a = base + (uint32_t)(e * MT_N + j0);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, "
          "%10, %11, %12, %13, %14, %15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
            "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
            "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(a));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      double *sc = scr + ((size_t)e * nout + j0) * MT_M + r;
      double o[16];
#pragma unroll
      for (int j = 0; j < 16; ++j)
        o[j] = (!first && j0 + j < nout) ? sc[(size_t)j * MT_M] : 0.0;
#pragma unroll
      for (int j = 0; j < 16; ++j)
        if (j0 + j < nout) sc[(size_t)j * MT_M] = o[j] + (double)__uint_as_float(v[j]);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
}

// adds the CTA's scratch sums, rescaled, to target row r's b and g (once)
__device__ __forceinline__ void mt_epilogue(const FmmDev &d, int r, uint32_t ci, int nout,
                                            const double *s_sc, const double *__restrict__ scr) {
  const int nm = d.nm, nm1 = d.nm1;
  double *__restrict__ gx = d.Gx + (size_t)ci * 3 * nm1;
  double *__restrict__ bb = d.B + (size_t)ci * 3 * nm;
  for (int mo = 0; mo < nout; ++mo) {
    for (int e = 0; e < 3; ++e) {
      const double val = s_sc[mo] * scr[((size_t)e * nout + mo) * MT_M + r];
      if (d.use_vs) gx[3 * mo + e] += val;
      if (mo < nm) bb[3 * mo + e] += val;
    }
  }
}

// Roles: MT_PW producer warps, 4 drain warps (warps MT_PW .. MT_PW + 3, one
// TMEM lane quarter each: MT_PW is a multiple of 4), the MMA issuer and the
// table loader.
#define MT_PW 8
#define MT_P (MT_PW * 32)
#define MT_DRAIN0 MT_PW
#define MT_MMAW (MT_PW + 4)
#define MT_TMAW (MT_PW + 5)
#define MT_THREADS2 ((MT_PW + 6) * 32)
// A stages: one (component, split) of 128 rows x 40 monomials each; a
// producer keeps MT_LAG stages of copies in flight before it publishes one
#define MT_NS 4
#define MT_LAG 2
#define MT_ITEMS ((MT_M * MT_KCH) / MT_P)  // 16-byte chunks per producer and stage
static_assert((MT_M * MT_KCH) % MT_P == 0 && MT_PW % 4 == 0 && MT_LAG < MT_NS, "layout");
// offsets accumulated in one TMEM set before it is drained to FP64 (the
// tensor core's FP32 accumulation truncates, so its runs are kept short)
#ifndef MT_GROUP
#define MT_GROUP 4
#endif

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"((uint64_t)src)
               : "memory");
}

// One CTA = up to 128 targets of one level and octant class.  Sources are
// the pre-split coefficients ahat2[cell][c][hi, lo][40] (TF32-rounded high
// part and FP32 remainder of the FP32 scaled coefficient), copied with
// cp.async into MT_NS rotating stages of one (component, split) each; per
// offset the six stages feed 90 tcgen05.mma (for source component c: the
// high part with the table's high and low parts, the low part with the
// table's high part, for the two output components its cross product
// reaches).  The accumulators of MT_GROUP offsets are drained to FP64 by
// dedicated warps while the next group runs.
__global__ void __launch_bounds__(MT_THREADS2, 1)
    k_m2l_tc(FmmDev d, const int4 *batches, const uint32_t *list, const int *srcl,
             const uint32_t *maskl, const float *img, const float *ahat2, uint32_t c0, int nout,
             double *scratch, unsigned long long *err) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  __shared__ __align__(8) uint64_t s_bfull[2], s_bempty[2], s_afull[MT_NS], s_aempty[MT_NS];
  __shared__ __align__(8) uint64_t s_cfull[2], s_cempty[2], s_done;
  __shared__ uint32_t s_tmem;
  __shared__ int s_fail, s_bissued, s_bconsumed;
  __shared__ uint32_t s_mask[7];
  __shared__ double s_sc[MT_N];
  unsigned char *sm = (unsigned char *)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
  unsigned char *sB = sm, *sA = sm + 2 * MT_BIMG;
  const int4 bd = batches[blockIdx.x];
  const int l = bd.x, q = bd.y, t0 = bd.z, cnt = bd.w;
  const int bx = q & 1, by = (q >> 1) & 1, bz = (q >> 2) & 1;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int *src = srcl + (size_t)blockIdx.x * MT_NCAND * MT_M;
  double *scr = scratch + (size_t)blockIdx.x * 3 * nout * MT_M;
  volatile int *fail = &s_fail;

  if (warp == MT_MMAW) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&s_tmem)),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == MT_TMAW * 32) {
    for (int b = 0; b < 2; ++b) {
      mbar_init(&s_bfull[b], 1);
      mbar_init(&s_bempty[b], 1);
      mbar_init(&s_cfull[b], 1);
      mbar_init(&s_cempty[b], 128);
    }
    for (int b = 0; b < MT_NS; ++b) {
      mbar_init(&s_afull[b], MT_P);
      mbar_init(&s_aempty[b], 1);
    }
    mbar_init(&s_done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;");
    s_fail = 0;
    s_bissued = 0;
    s_bconsumed = 0;
  }
  if (tid < 7) s_mask[tid] = maskl[(size_t)blockIdx.x * 8 + tid];
  if (tid >= MT_M && tid < MT_M + MT_N) {
    const int mo = tid - MT_M;
    double sc = 0.0;
    if (mo < nout) {
      int oi, oj, ok;
      mono_exp(mo, oi, oj, ok);
      double hi = 1.0 / d.G.csize[l], hp = 1.0;
      for (int e = 0; e < oi + oj + ok + 2; ++e) hp *= hi;
      sc = (((oi + oj + ok) & 1) ? -1.0 : 1.0) * d.inv_fact[mo] * hp;
    }
    s_sc[mo] = sc;
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = s_tmem;
  int ntot = 0;  // offsets with a source for some target of the CTA
  for (int w = 0; w < 7; ++w) ntot += __popc(s_mask[w]);

  if (warp < MT_PW) {
    // ------------------------------------------------------------ producers
    // next candidate offset after `c` with a source for some target (216 = none)
    auto next_cand = [&](int c) {
      for (int w = (c + 1) >> 5; w < 7; ++w) {
        uint32_t bits = s_mask[w];
        if (w == ((c + 1) >> 5)) bits &= ~0u << ((c + 1) & 31);
        if (bits) return w * 32 + __ffs(bits) - 1;
      }
      return MT_NCAND;
    };
    int u = 0;
    bool ok = true;
    int cand = next_cand(-1);
    int sidx_next[MT_ITEMS];
#pragma unroll
    for (int i = 0; i < MT_ITEMS; ++i)
      sidx_next[i] =
          cand < MT_NCAND ? __ldg(src + (size_t)cand * MT_M + (tid + MT_P * i) / MT_KCH) : -1;
    while (cand < MT_NCAND && ok) {
      int sidx[MT_ITEMS];
#pragma unroll
      for (int i = 0; i < MT_ITEMS; ++i) sidx[i] = sidx_next[i];
      const int ncand = next_cand(cand);
#pragma unroll
      for (int i = 0; i < MT_ITEMS; ++i)
        sidx_next[i] =
            ncand < MT_NCAND ? __ldg(src + (size_t)ncand * MT_M + (tid + MT_P * i) / MT_KCH) : -1;
      for (int cs = 0; cs < 6 && ok; ++cs, ++u) {
        const int buf = u % MT_NS;
        if (u >= MT_NS &&
            !mbar_wait_f(smem_u32(&s_aempty[buf]), (uint32_t)((u / MT_NS - 1) & 1), fail)) {
          ok = false;
          break;
        }
        const uint32_t abase = smem_u32(sA + buf * MT_ASPLIT);
        const int c = cs >> 1, sp = cs & 1;
#pragma unroll
        for (int i = 0; i < MT_ITEMS; ++i) {
          const int item = tid + MT_P * i, rr = item / MT_KCH, kc = item % MT_KCH;
          const uint32_t dst = abase + mt_aoff(rr, 4 * kc);
          if (sidx[i] >= 0) {
            cp_async16(dst, ahat2 + (size_t)(sidx[i] - (int)c0) * 6 * MT_K + (2 * c + sp) * MT_K +
                                4 * kc);
          } else {
            asm volatile("st.shared.v4.u32 [%0], {%1, %1, %1, %1};" ::"r"(dst), "r"(0u)
                         : "memory");
          }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
        if (u >= MT_LAG) {
          // the copies of stage u - MT_LAG have landed: publish it
          asm volatile("cp.async.wait_group %0;" ::"n"(MT_LAG) : "memory");
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          mbar_arrive(&s_afull[(u - MT_LAG) % MT_NS]);
        }
      }
      cand = ncand;
    }
    // publish the stages still in flight (on every path: the copies land
    // whether or not a consumer is left)
    asm volatile("cp.async.wait_all;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (ok)
      for (int v = (u > MT_LAG ? u - MT_LAG : 0); v < u; ++v) mbar_arrive(&s_afull[v % MT_NS]);
  } else if (warp < MT_DRAIN0 + 4) {
    // --------------------------------------------------------------- drains
    const int quarter = warp & 3;
    const int r = quarter * 32 + lane;
    const int ngroups = (ntot + MT_GROUP - 1) / MT_GROUP;
    bool ok = true;
    for (int g = 0; g < ngroups && ok; ++g) {
      if (!mbar_wait_f(smem_u32(&s_cfull[g & 1]), (uint32_t)((g >> 1) & 1), fail)) {
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;");
      mt_drain(tmem, quarter, g & 1, r, nout, g == 0, scr);
      mbar_arrive(&s_cempty[g & 1]);
    }
    if (ok && ngroups > 0 && r < cnt) mt_epilogue(d, r, list[t0 + r], nout, s_sc, scr);
  } else if (warp == MT_MMAW && lane == 0) {
    // ---------------------------------------------------------- MMA issuer
    const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(MT_N >> 3) << 17) |
                           ((uint32_t)(MT_M >> 4) << 24);
    int u = 0, oi = 0;
    bool ok = true;
    uint32_t started = 0;  // bit e: accumulator e written in this group
    for (int cand = 0; cand < MT_NCAND && ok && !*fail; ++cand) {
      if (!((s_mask[cand >> 5] >> (cand & 31)) & 1u)) continue;
      const int sb = oi & 1, g = oi / MT_GROUP, set = g & 1;
      if (!mbar_wait_f(smem_u32(&s_bfull[sb]), (uint32_t)((oi >> 1) & 1), fail)) break;
      s_bconsumed = oi + 1;
      if (oi % MT_GROUP == 0) {
        // the set is free once group g - 2 has been drained
        if (g >= 2 &&
            !mbar_wait_f(smem_u32(&s_cempty[set]), (uint32_t)(((g >> 1) - 1) & 1), fail))
          break;
        started = 0;
      }
      const uint32_t bbase = smem_u32(sB + sb * MT_BIMG);
      for (int cs = 0; cs < 6; ++cs, ++u) {
        const int buf = u % MT_NS;
        if (!mbar_wait_f(smem_u32(&s_afull[buf]), (uint32_t)((u / MT_NS) & 1), fail)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;");
        const uint32_t as = smem_u32(sA + buf * MT_ASPLIT);
        const int c = cs >> 1, sp = cs & 1;
        for (int pp = 0; pp < 2; ++pp) {
          // source component c feeds two accumulators e with table component
          // dd and sign:  c = x: (y, D_z, +) (z, D_y, -);  c = y: (x, D_z, -)
          // (z, D_x, +);  c = z: (x, D_y, +) (y, D_x, -)
          const int e = pp == 0 ? (c == 0 ? 1 : 0) : (c == 2 ? 1 : 2);
          const int dd = pp == 0 ? (c == 2 ? 1 : 2) : (c == 0 ? 1 : 0);
          const uint32_t neg = pp == 0 ? (c == 1 ? 1u : 0u) : (c == 1 ? 0u : 1u);
          const uint32_t id = idesc | (neg << 13);
          const uint32_t bcomp = bbase + dd * MT_BCOMP;
          // 3xTF32: the high stage meets the table's high and low parts,
          // the low stage the table's high part
          for (int tb = 0; tb < (sp == 0 ? 2 : 1); ++tb) {
            const uint32_t bs = bcomp + (tb == 1 ? MT_BSPLIT : 0);
#pragma unroll
            for (int j = 0; j < MT_K / 8; ++j) {
              umma_tf32(tmem + (uint32_t)(set * 256 + e * MT_N),
                        make_sdesc(as + j * 4096, 2048, 128),
                        make_sdesc(bs + j * 2048, 1024, 128), id, (started >> e) & 1u);
              started |= 1u << e;
            }
          }
        }
        umma_commit(&s_aempty[buf]);
      }
      if (!ok) break;
      umma_commit(&s_bempty[sb]);
      if (oi % MT_GROUP == MT_GROUP - 1 || oi == ntot - 1) umma_commit(&s_cfull[set]);
      ++oi;
    }
    umma_commit(&s_done);
  } else if (warp == MT_TMAW && lane == 0) {
    // ---------------------------------------------------------- table loader
    const char *limg = (const char *)img + (size_t)(l - 2) * 343 * MT_BIMG;
    int oi = 0;
    for (int cand = 0; cand < MT_NCAND && !*fail; ++cand) {
      if (!((s_mask[cand >> 5] >> (cand & 31)) & 1u)) continue;
      const MtCand m = mt_cand(cand, bx, by, bz);
      const int sb = oi & 1;
      if (oi >= 2 &&
          !mbar_wait_f(smem_u32(&s_bempty[sb]), (uint32_t)(((oi >> 1) - 1) & 1), fail))
        break;
      const int tab = (m.ox + 3) + 7 * ((m.oy + 3) + 7 * (m.oz + 3));
      mbar_expect_tx(&s_bfull[sb], MT_BIMG);
      bulk_g2s(smem_u32(sB + sb * MT_BIMG), limg + (size_t)tab * MT_BIMG, MT_BIMG, &s_bfull[sb]);
      s_bissued = ++oi;
    }
  }
  __syncthreads();
  const bool okd = mbar_wait(smem_u32(&s_done), 0u);
  const int all_ok = __syncthreads_and(okd && !*fail);
  if (!all_ok) {
    if (tid == 0) {
      atomicExch(err, 1ull);
      // table copies issued but never consumed: let them land (bounded)
      for (int k = s_bconsumed; k < s_bissued; ++k)
        mbar_wait(smem_u32(&s_bfull[k & 1]), (uint32_t)((k >> 1) & 1));
    }
    if (!okd) mbar_wait(smem_u32(&s_done), 0u);
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == MT_MMAW)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
}

static inline unsigned nblk_tc(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

bool m2l_tc_usable(const dust_octree *o) {
  const int nout = o->prm.vortstretch ? o->nm1 : o->nm;
  return o->prm.precision == DUST_PREC_FP32C && o->nm <= MT_K && nout <= MT_NOUT &&
         o->G.ll >= 2;
}

int m2l_tc_tables(dust_octree *o) {
  if (!m2l_tc_usable(o)) return DUST_OK;
  const int nout = o->prm.vortstretch ? o->nm1 : o->nm;
  const size_t per = (size_t)343 * MT_BIMG;
  DUST_TRY(devbuf_grow(o->m2l_img, per * (size_t)(o->G.ll - 1)));
  for (int l = 2; l <= o->G.ll; ++l) {
    size_t tot = (size_t)343 * 3 * MT_N * MT_K;
    k_m2l_tc_image<<<nblk_tc(tot, 256), 256>>>((const double *)o->dtabs[l].p,
                                                (const uint16_t *)o->idxsum.p, o->nD, o->nm,
                                                o->nm1, nout,
                                                (float *)((char *)o->m2l_img.p + per * (l - 2)));
  }
  DUST_CUDA(cudaGetLastError());
  DUST_CUDA(cudaDeviceSynchronize());
  return DUST_OK;
}

size_t m2l_tc_ahat_bytes(size_t ncells) { return ncells * 6 * MT_K * 4; }

int m2l_tc_scale_sources(dust_octree *o, FmmDev &d, cudaStream_t st) {
  uint32_t c0 = o->ahat_c0, nact = (uint32_t)o->n_active;
  size_t tot = (size_t)(nact - c0) * 3 * MT_K;
  if (tot == 0) return DUST_OK;
  k_scale_a_tc<<<nblk_tc(tot, 256), 256, 0, st>>>(d, c0, nact, (float *)o->ahat.p);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}

int m2l_tc_run(dust_octree *o, FmmDev &d, cudaStream_t st) {
  const int nout = o->prm.vortstretch ? o->nm1 : o->nm;
  std::vector<int4> bs;
  int start = 0;
  for (int k = 0; k < 8 * (DUST_MAXLEV + 1); ++k) {
    const int c = o->m2l_cnt[k];
    const int l = k >> 3, q = k & 7;
    if (l >= 2)
      for (int b = 0; b < c; b += MT_M) bs.push_back(make_int4(l, q, start + b, std::min(MT_M, c - b)));
    start += c;
  }
  if (bs.empty()) return DUST_OK;
  const size_t nb = bs.size();
  DUST_TRY(devbuf_grow(o->m2l_bat, nb * sizeof(int4)));
  const size_t scr_b = nb * 3 * (size_t)nout * MT_M * 8;
  DUST_TRY(devbuf_grow(o->m2l_src, scr_b + nb * (MT_NCAND * MT_M * 4 + 8 * 4)));
  double *scr = (double *)o->m2l_src.p;
  int *srcl = (int *)((char *)o->m2l_src.p + scr_b);
  uint32_t *maskl = (uint32_t *)(srcl + nb * MT_NCAND * MT_M);
  DUST_CUDA(cudaMemcpyAsync(o->m2l_bat.p, bs.data(), nb * sizeof(int4), cudaMemcpyHostToDevice,
                            st));
  k_m2l_tc_lists<<<(unsigned)nb, MT_M, 0, st>>>(d, (const int4 *)o->m2l_bat.p, o->m2l_list, srcl,
                                                 maskl);
  const int smem = MT_SMEM;
  static bool attr = false;
  if (!attr) {
    DUST_CUDA(cudaFuncSetAttribute(k_m2l_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr = true;
  }
  // counters[2] is the kernel's timeout flag (cleared with the counters)
  o->kev_m2l = o->timing;
  if (o->timing) cudaEventRecord(o->ev[6], st);
  k_m2l_tc<<<(unsigned)nb, MT_THREADS2, smem, st>>>(
      d, (const int4 *)o->m2l_bat.p, o->m2l_list, srcl, maskl, (const float *)o->m2l_img.p,
      (const float *)o->ahat.p, o->ahat_c0, nout, scr, (unsigned long long *)(d.counters + 2));
  if (o->timing) cudaEventRecord(o->ev[7], st);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}
