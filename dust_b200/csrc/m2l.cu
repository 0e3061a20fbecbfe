// m2l.cu -- batched multipole-to-local translation (levels >= 2).
//
// M2L_multipole (src/fmm/mod_multipole.f90:282-356) in the form
//   g(m') = (-1)^|m'| / m'!  sum_n  Dhat(m'+n) x ahat(n),  |m'| <= p+1,
// Dhat = k! D(k) of compute_der_ker (:388-450), ahat(n) = a(n)/n!.
//
// Work decomposition.  The targets of a level are the non-empty active
// cells, grouped by their position in the parent (octant class q = key & 7):
// all targets of one class share the same 189 interaction offsets
// (children of the parent's 26 neighbours that are not adjacent,
// mod_octree.f90:440-476).  A CTA takes NB targets of one class and its
// warps share out the 189 offsets (details at k_m2l_batch).
//
// Scaling: with h the cell size of the level, the tables hold
// Shat(s) h^(|s|+1) and the sources a(n) / (n! h^|n|), so both stay of order
// one at every level and degree; the output is rescaled by h^-(|m'|+2).
//
// FP32C: tables and source coefficients in FP32, each offset's partial sums
// in FP32, accumulated across offsets in FP64.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>
#include <type_traits>
#include <vector>

#include "dust_common.cuh"
#include "fmm_internal.h"

#define M2L_T 256
#define M2L_GQ 4

struct M2LTabs {
  const void *t[DUST_MAXLEV + 1];  // per-level dimensionless tables
};

// One CTA per batch descriptor (level, class, first target, count); the
// batches of all levels >= 2 run in one launch (M2L of different levels is
// independent; L2L follows level by level).
//
// Scalar form.  The vector kernel of compute_der_ker is a gradient: with
// Shat(j) = d^j phi the plain derivatives of the scalar kernel
// phi = 1 / (4 pi sqrt(r^2 + delta^2)), Dhat(k)_c = -Shat(k + e_c), so
//   (sum_n Dhat(m'+n) x ahat(n))_x = L_y(m'+e_z) - L_z(m'+e_y)   (and cyclic),
//   L_c(j) = sum_n Shat(j+n) ahat_c(n),   1 <= |j| <= p+2 (p+1 without
// stretching).  Three scalar sums per offset replace the cross products: at
// p = 4, 83 x 35 x 3 FMAs instead of 56 x 35 x 6, and one 4-byte table read
// per (j, n) instead of a 16-byte (x y z) one.  The L_c(j) of a target are
// summed over its offsets in FP64 (shared memory) and turned into the
// outputs once, at the end.
//
// Inside a CTA the warps are independent: warp w takes offsets w, w+W, ...;
// lane i looks up the source of target i at that offset, the present ones
// are compacted with a ballot, the warp stages the offset's scalar table and
// (in chunks of up to TCX <= M2L_TC) the present sources in its own
// shared-memory slice -- sources as [n][component][slot], so the values of
// consecutive targets are one vector load -- and evaluates them with
// __syncwarp only.  A chunk of kc targets runs the register tile of 1, 2, 4
// or 8 targets (3-4 and 5-8 with zero sources in the spare slots).  In the
// tile lane i owns the indices j of slots s0..s0+SLP-1 (j-index 32 s + i);
// per source monomial n it reads SLP table entries at the positions of
// j + n (index table jsum: the three positions of one pass in one 8-byte
// word per lane) and, per component, the chunk's source values,
// for SLP x 3 x tile FMAs (packed f32x2 over target pairs in FP32).  The
// chunk's sums go to the CTA's FP64 accumulators with shared-memory atomics.
#define M2L_TC 8
#define M2L_MAXW 8
#define M2L_SLP 3

template <typename T>
struct M2LVec {
  T x, y, z;
};
template <typename T>
__device__ __forceinline__ M2LVec<T> m2l_ld(const T *p);
template <>
__device__ __forceinline__ M2LVec<float> m2l_ld<float>(const float *p) {
  const float4 v = __ldg((const float4 *)p);
  return {v.x, v.y, v.z};
}
template <>
__device__ __forceinline__ M2LVec<double> m2l_ld<double>(const double *p) {
  const double2 a = __ldg((const double2 *)p);
  return {a.x, a.y, __ldg(p + 2)};
}

// count entries (a multiple of 16 bytes) from global to shared memory
__device__ __forceinline__ void m2l_copyv(float *dst, const float *src, int count, int lane) {
  for (int e = lane; e < count / 4; e += 32)
    *(float4 *)(dst + 4 * e) = __ldg((const float4 *)(src + 4 * e));
}
__device__ __forceinline__ void m2l_copyv(double *dst, const double *src, int count, int lane) {
  for (int e = lane; e < count / 2; e += 32)
    *(double2 *)(dst + 2 * e) = __ldg((const double2 *)(src + 2 * e));
}

// acc[s][c][t] += S(j_s + n) a_c(n) of target t over the source monomials n
template <typename T, int SLP, int TCc>
__device__ __forceinline__ void m2l_tile(const T *__restrict__ sS, const T *__restrict__ sA,
                                         const uint2 *__restrict__ jq, int nm, int s0, int nJ,
                                         int TCX, int lane, const int *tl,
                                         int kreal, double *__restrict__ s_acc) {
  constexpr bool PK = std::is_same<T, float>::value && TCc >= 2;
  constexpr int NA = PK ? TCc / 2 : TCc;
  using Acc = typename std::conditional<PK, float2, T>::type;
  Acc acc[SLP][3][NA];
#pragma unroll
  for (int s = 0; s < SLP; ++s)
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int t = 0; t < NA; ++t) {
        if constexpr (PK) acc[s][c][t] = make_float2(0.f, 0.f);
        else acc[s][c][t] = (T)0;
      }
  const uint2 *jr = jq + lane;
#pragma unroll 2
  for (int n = 0; n < nm; ++n) {
    const uint2 w = jr[(size_t)n * 32];
    T S[SLP];
    S[0] = sS[w.x & 0xffffu];
    if constexpr (SLP >= 2) S[1] = sS[w.x >> 16];
    if constexpr (SLP >= 3) S[2] = sS[w.y & 0xffffu];
    const T *a = sA + (size_t)n * 3 * TCX;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if constexpr (PK) {
        float2 A[NA];
        if constexpr (TCc >= 4) {
#pragma unroll
          for (int q = 0; q < TCc / 4; ++q) {
            const float4 v = *(const float4 *)(a + c * TCX + 4 * q);
            A[2 * q] = make_float2(v.x, v.y);
            A[2 * q + 1] = make_float2(v.z, v.w);
          }
        } else {
          A[0] = *(const float2 *)(a + c * TCX);
        }
#pragma unroll
        for (int s = 0; s < SLP; ++s) {
          const float2 S2 = make_float2(S[s], S[s]);
#pragma unroll
          for (int t = 0; t < NA; ++t) acc[s][c][t] = __ffma2_rn(S2, A[t], acc[s][c][t]);
        }
      } else {
#pragma unroll
        for (int t = 0; t < TCc; ++t) {
          const T A = a[c * TCX + t];
#pragma unroll
          for (int s = 0; s < SLP; ++s) acc[s][c][t] = fma(S[s], A, acc[s][c][t]);
        }
      }
    }
  }
#pragma unroll
  for (int s = 0; s < SLP; ++s) {
    const int j = (s0 + s) * 32 + lane;
    if (j >= nJ) continue;
#pragma unroll
    for (int t = 0; t < TCc; ++t) {
      if (t >= kreal) break;  // zero-padded slots of the tile
      double *acc_t = s_acc + (size_t)tl[t] * 3 * nJ + j;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        double v;
        if constexpr (PK) v = (t & 1) ? (double)acc[s][c][t >> 1].y : (double)acc[s][c][t >> 1].x;
        else v = (double)acc[s][c][t];
        atomicAdd(acc_t + (size_t)c * nJ, v);
      }
    }
  }
}

// all slot passes of one chunk (up to M2L_SLP slots per pass); SLC > 0: the
// kernel's slot count is SLC (one pass, compiled alone), 0: any count
template <typename T, int TCc, int SLC>
__device__ __forceinline__ void m2l_chunk(const T *sS, const T *sA, const uint2 *jsum, int nm,
                                          int SL, int nJ, int TCX, int lane, const int *tl,
                                          int kreal, double *s_acc) {
  if constexpr (SLC > 0) {
    m2l_tile<T, SLC, TCc>(sS, sA, jsum, nm, 0, nJ, TCX, lane, tl, kreal, s_acc);
  } else {
    for (int s0 = 0; s0 < SL; s0 += M2L_SLP) {
      const int r = SL - s0;
      const uint2 *jq = jsum + (size_t)(s0 / M2L_SLP) * nm * 32;
      if (r >= 3)
        m2l_tile<T, 3, TCc>(sS, sA, jq, nm, s0, nJ, TCX, lane, tl, kreal, s_acc);
      else if (r == 2)
        m2l_tile<T, 2, TCc>(sS, sA, jq, nm, s0, nJ, TCX, lane, tl, kreal, s_acc);
      else
        m2l_tile<T, 1, TCc>(sS, sA, jq, nm, s0, nJ, TCX, lane, tl, kreal, s_acc);
    }
  }
}

template <typename T, int SLC>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 2 : 1)
    k_m2l_batch(FmmDev d, const int4 *batches, const uint32_t *list, int NB, int NW, int TCX,
                M2LTabs tabs, const T *ahat, uint32_t ahat_cell0, const uint2 *jsum_g, int SL,
                int nJ, int P, int jsum_smem) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int nm = d.nm;
  const int nout = d.use_vs ? d.nm1 : d.nm;
  const int4 bd = batches[blockIdx.x];
  const int l = bd.x, q = bd.y, t0 = bd.z, cnt = bd.w;
  const T *stab = (const T *)tabs.t[l];
  double *s_acc = (double *)smraw;                        // NB x 3 x nJ
  int *s_tc = (int *)(s_acc + (size_t)NB * 3 * nJ);      // NB x 3 target carts
  // passes x nm x 32 index words (optional)
  uint2 *s_js = (uint2 *)(((uintptr_t)(s_tc + 3 * NB) + 15) & ~(uintptr_t)15);
  const size_t jsz = jsum_smem ? (size_t)((SL + M2L_SLP - 1) / M2L_SLP) * nm * 32 : 0;
  const uint2 *jsum = jsum_smem ? s_js : jsum_g;
  T *s_w = (T *)(((uintptr_t)(s_js + jsz) + 15) & ~(uintptr_t)15);
  // per warp, in T, rounded to 16 bytes (vector copies into every slice)
  const size_t wslice = ((size_t)P + (size_t)TCX * 3 * nm + 3) / 4 * 4;
  __shared__ double s_hp[2 * DUST_MAXP + 6];  // (1/h)^d
  __shared__ int s_src[M2L_MAXW][M2L_TC];     // source cells of the warp's chunk
  __shared__ int s_tl[M2L_MAXW][M2L_TC];      // and their targets (batch index)
  const int bx = q & 1, by = (q >> 1) & 1, bz = (q >> 2) & 1;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t lo_l = d.G.lev_off[l];
  const int sh = 3 * (d.G.ll - l);
  if (tid == 0) {
    double hi = 1.0 / d.G.csize[l], v = 1.0;
    for (int e = 0; e < 2 * DUST_MAXP + 6; ++e, v *= hi) s_hp[e] = v;
  }
  for (int t = tid; t < NB; t += NW * 32) {
    int i = -1000, j = -1000, k = -1000;
    if (t < cnt) cart_of_key(d.G, l, d.act_key[list[t0 + t]], i, j, k);
    s_tc[3 * t] = i;
    s_tc[3 * t + 1] = j;
    s_tc[3 * t + 2] = k;
  }
  for (int e = tid; e < NB * 3 * nJ; e += NW * 32) s_acc[e] = 0.0;
  for (int e = tid; e < (int)jsz; e += NW * 32) s_js[e] = jsum_g[e];
  __syncthreads();
  T *sS = s_w + (size_t)warp * wslice;
  T *sA = sS + P;
  unsigned long long npairs = 0;
  const int L = 3, W = 2 * L + 1;
  // The warp's offsets are looked up M2L_GQ at a time: for every target the
  // source cell's flags, particle range and index are loaded without
  // branches (predicated on the cell lying in the box), so the loads of the
  // M2L_GQ offsets are in flight together instead of one dependent chain per
  // offset.
  for (int cb = warp; cb < 216; cb += NW * M2L_GQ) {
    int srcq[M2L_GQ][2];
#pragma unroll
    for (int g = 0; g < M2L_GQ; ++g) {
      const int cand = cb + g * NW;
      const int ox = cand % 6 - 2 - bx, oy = (cand / 6) % 6 - 2 - by, oz = cand / 36 - 2 - bz;
      const bool valid = cand < 216 && !(abs(ox) <= 1 && abs(oy) <= 1 && abs(oz) <= 1);
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        // NB <= 64 targets: lane i looks at targets i and 32 + i
        const int t = lane + 32 * h;
        const int si = s_tc[3 * (t < NB ? t : 0)] + ox, sj = s_tc[3 * (t < NB ? t : 0) + 1] + oy,
                  sk = s_tc[3 * (t < NB ? t : 0) + 2] + oz;
        const bool ok = valid && t < cnt && cart_in(d.G, l, si, sj, sk);
        const uint32_t skey = ok ? key_of(d.G, l, si, sj, sk) : 0u;
        const uint8_t f = ok ? d.flags[lo_l + skey] : (uint8_t)0;
        const uint32_t a0 = ok ? d.cstart[skey << sh] : 0u;
        const uint32_t a1 = ok ? d.cstart[(skey + 1u) << sh] : 0u;
        const uint32_t cx = ok ? d.cidx[lo_l + skey] : 0u;
        srcq[g][h] = (ok && (f & FL_ACTIVE) && a1 > a0) ? (int)cx : -1;
      }
    }
#pragma unroll 1
    for (int g = 0; g < M2L_GQ; ++g) {
      const int cand = cb + g * NW;
      if (cand >= 216) break;
      const int ox = cand % 6 - 2 - bx, oy = (cand / 6) % 6 - 2 - by, oz = cand / 36 - 2 - bz;
      // (selects, not a dynamically indexed array, keep srcq in registers)
      int src[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        int v = srcq[0][h];
#pragma unroll
        for (int q2 = 1; q2 < M2L_GQ; ++q2) v = (g == q2) ? srcq[q2][h] : v;
        src[h] = v;
      }
      const unsigned msk0 = __ballot_sync(0xffffffffu, src[0] >= 0),
                     msk1 = __ballot_sync(0xffffffffu, src[1] >= 0);
      if (!(msk0 | msk1)) continue;
      npairs += __popc(msk0) + __popc(msk1);
      const int tab = (ox + L) + W * ((oy + L) + W * (oz + L));
      __syncwarp();
      m2l_copyv(sS, stab + (size_t)tab * P, P, lane);
      // the present targets of both halves in chunks of up to TCX; a chunk of
      // 3-4 (5-8) runs the 4- (8-) target tile with zero sources in the spare
      // slots, which costs less than splitting it (every tile re-reads the
      // offset's table entries)
      unsigned long long m = (unsigned long long)msk0 | ((unsigned long long)msk1 << 32);
      while (m) {
        const int kc = min(__popcll(m), TCX);
        const int tile = kc <= 2 ? kc : kc <= 4 ? 4 : 8;
        int *tl = s_tl[warp];
#pragma unroll
        for (int c = 0; c < M2L_TC; ++c) {
          if (c >= kc) break;
          const int t = __ffsll((long long)m) - 1;
          m &= m - 1;
          const int sc_ = __shfl_sync(0xffffffffu, t >= 32 ? src[1] : src[0], t & 31);
          if (lane == 0) s_src[warp][c] = sc_, tl[c] = t;
        }
        __syncwarp();
        // sources of the chunk as [n][component][slot]; spare slots zero
        for (int w = lane; w < tile * nm; w += 32) {
          const int c = w / nm, e = w - c * nm;
          T *dst = sA + (size_t)e * 3 * TCX + c;
          if (c < kc) {
            const M2LVec<T> v =
                m2l_ld(ahat + ((size_t)(s_src[warp][c] - ahat_cell0) * nm + e) * 4);
            dst[0] = v.x;
            dst[TCX] = v.y;
            dst[2 * TCX] = v.z;
          } else {
            dst[0] = dst[TCX] = dst[2 * TCX] = (T)0;
          }
        }
        __syncwarp();
        if (tile == 8) m2l_chunk<T, 8, SLC>(sS, sA, jsum, nm, SL, nJ, TCX, lane, tl, kc, s_acc);
        else if (tile == 4) m2l_chunk<T, 4, SLC>(sS, sA, jsum, nm, SL, nJ, TCX, lane, tl, kc, s_acc);
        else if (tile == 2) m2l_chunk<T, 2, SLC>(sS, sA, jsum, nm, SL, nJ, TCX, lane, tl, kc, s_acc);
        else m2l_chunk<T, 1, SLC>(sS, sA, jsum, nm, SL, nJ, TCX, lane, tl, kc, s_acc);
        __syncwarp();
      }
    }
  }
  __syncthreads();
  if (lane == 0 && d.counters) atomicAdd((unsigned long long *)d.counters, npairs);
  // outputs: (sum_n Dhat(m'+n) x ahat(n)) from the L_c(j), rescaled
  for (int e = tid; e < cnt * nout; e += NW * 32) {
    const int t = e / nout, mo = e - t * nout;
    int oi, oj, ok;
    mono_exp(mo, oi, oj, ok);
    const double sc =
        (((oi + oj + ok) & 1) ? -1.0 : 1.0) * d.inv_fact[mo] * s_hp[oi + oj + ok + 2];
    const double *Lx = s_acc + (size_t)t * 3 * nJ, *Ly = Lx + nJ, *Lz = Ly + nJ;
    const int jx = mono_idx(oi + 1, oj, ok) - 1, jy = mono_idx(oi, oj + 1, ok) - 1,
              jz = mono_idx(oi, oj, ok + 1) - 1;
    const double g[3] = {Ly[jz] - Lz[jy], Lz[jx] - Lx[jz], Lx[jy] - Ly[jx]};
    const uint32_t ci = list[t0 + t];
    if (d.use_vs) {
      double *gx = d.Gx + (size_t)ci * 3 * d.nm1;
      for (int c = 0; c < 3; ++c) gx[3 * mo + c] += sc * g[c];
    }
    if (mo < nm) {
      double *bb = d.B + (size_t)ci * 3 * nm;
      for (int c = 0; c < 3; ++c) bb[3 * mo + c] += sc * g[c];
    }
  }
}

// ahat'(n) = a(n) / (n! h^|n|) for every active cell of levels >= 2
template <typename T>
__global__ void k_scale_a(FmmDev d, uint32_t c0, uint32_t nact, T *out) {
  size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int w = 3 * d.nm;
  size_t tot = (size_t)(nact - c0) * w;
  if (e >= tot) return;
  uint32_t ci = c0 + (uint32_t)(e / w);
  int r = (int)(e % w), nn = r / 3, ni, nj, nk;
  mono_exp(nn, ni, nj, nk);
  int l = d.act_lev[ci];
  double hi = 1.0 / d.G.csize[l], hp = 1.0;
  for (int q = 0; q < ni + nj + nk; ++q) hp *= hi;
  // padded [cell][nm][4] (x y z 0), so a monomial is one 16- or 32-byte load
  T *o4 = out + (size_t)(ci - c0) * 4 * d.nm + 4 * nn;
  o4[r % 3] = (T)(d.A[(size_t)ci * w + r] * d.inv_fact[nn] * hp);
  if (r % 3 == 2) o4[3] = (T)0;
}

// class keys of the active cells of levels >= 2: (level << 3 | key & 7) for
// non-empty cells and for empty leaves that hold evaluation points, 0xff for
// the other empty ones (dropped)
__global__ void k_m2l_keys(FmmDev d, uint32_t c0, uint32_t nact, uint32_t *keys,
                           uint32_t *vals, int *hist) {
  uint32_t ci = c0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (ci >= nact) return;
  int l = d.act_lev[ci];
  uint32_t key = d.act_key[ci];
  int sh = 3 * (d.G.ll - l);
  bool ne = d.cstart[(key + 1u) << sh] > d.cstart[key << sh] ||
            (d.flags[d.G.lev_off[l] + key] & FL_PTS);
  uint32_t k = ne ? (uint32_t)((l << 3) | (key & 7)) : 0xffu;
  keys[ci - c0] = k;
  vals[ci - c0] = ci;
  if (ne) atomicAdd(hist + k, 1);
}

static inline unsigned nblk(size_t n, int t) { return (unsigned)((n + t - 1) / t); }


int m2l_batch_tables(dust_octree *o) {
  // dimensionless scalar tables T(s) = Shat(s) h^(|s|+1), |s| <= 2p+2, for
  // the batched kernel (FP64 and FP32 copies), read off the vector tables:
  // Dhat(k)_c h^(|k|+2) = -Shat(k + e_c) h^(|k + e_c|+1).  Entry 0 (s = 0,
  // never used by a sum) is zero: the index table points the spare lanes of
  // the last slot there.
  const int p = o->p, nD = o->nD;
  const int nS = n_mon(2 * p + 2);
  const int P = (nS + 3) / 4 * 4;
  const int jmax = o->prm.vortstretch ? p + 2 : p + 1;
  const int nJ = n_mon(jmax) - 1, SL = (nJ + 31) / 32, nm = n_mon(p);
  o->m2l_nJ = nJ;
  o->m2l_SL = SL;
  o->m2l_P = P;
  std::vector<int> deg(nD);
  for (int q = 0; q < nD; ++q) {
    int i, j, k;
    mono_exp(q, i, j, k);
    deg[q] = i + j + k;
  }
  // source of entry s: (vector entry s - e_c, component c) for the first c
  // with s_c >= 1
  std::vector<int> sq(nS, -1), scomp(nS, 0);
  for (int s = 1; s < nS; ++s) {
    int i, j, k;
    mono_exp(s, i, j, k);
    if (i >= 1) sq[s] = mono_idx(i - 1, j, k), scomp[s] = 0;
    else if (j >= 1) sq[s] = mono_idx(i, j - 1, k), scomp[s] = 1;
    else sq[s] = mono_idx(i, j, k - 1), scomp[s] = 2;
  }
  for (int l = 2; l <= o->G.ll; ++l) {
    const size_t n = (size_t)343 * nD * 3, nt = (size_t)343 * P;
    DUST_TRY(devbuf_grow(o->dtabs[l], nt * 8));
    DUST_TRY(devbuf_grow(o->dtab32[l], nt * 4));
    std::vector<double> h(n), t64(nt, 0.0);
    std::vector<float> t32(nt, 0.f);
    DUST_CUDA(cudaMemcpy(h.data(), o->dtab[l].p, n * 8, cudaMemcpyDeviceToHost));
    const double cs = o->G.csize[l];
    std::vector<double> hp(2 * DUST_MAXP + 6, 1.0);
    for (size_t e = 1; e < hp.size(); ++e) hp[e] = hp[e - 1] * cs;
    for (size_t off = 0; off < 343; ++off)
      for (int s = 1; s < nS; ++s) {
        const int q = sq[s];
        const double v = -h[(off * nD + q) * 3 + scomp[s]] * hp[deg[q] + 2];
        t64[off * P + s] = v;
        t32[off * P + s] = (float)v;
      }
    DUST_CUDA(cudaMemcpy(o->dtabs[l].p, t64.data(), nt * 8, cudaMemcpyHostToDevice));
    DUST_CUDA(cudaMemcpy(o->dtab32[l].p, t32.data(), nt * 4, cudaMemcpyHostToDevice));
  }
  // jsum[pass][n][lane] (4 x u16) = indices of j + n for the pass's slots
  // s = 3 pass + 0..2, j the monomial of index 1 + 32 s + lane (0: spare lane)
  const int npass = (SL + M2L_SLP - 1) / M2L_SLP;
  std::vector<uint16_t> js((size_t)npass * nm * 32 * 4, 0);
  for (int nn = 0; nn < nm; ++nn) {
    int ni, nj, nk;
    mono_exp(nn, ni, nj, nk);
    for (int jj = 0; jj < nJ; ++jj) {
      int ji, jj2, jk;
      mono_exp(jj + 1, ji, jj2, jk);
      const int sl = jj / 32, lane = jj % 32, pass = sl / M2L_SLP, w = sl % M2L_SLP;
      js[(((size_t)pass * nm + nn) * 32 + lane) * 4 + w] =
          (uint16_t)mono_idx(ji + ni, jj2 + nj, jk + nk);
    }
  }
  DUST_TRY(devbuf_grow(o->jsum, js.size() * 2));
  DUST_CUDA(cudaMemcpy(o->jsum.p, js.data(), js.size() * 2, cudaMemcpyHostToDevice));
  return DUST_OK;
}

// Runs M2L for all levels >= 2 (level 1 is handled by the per-target kernel).
// `before_level(l)` style ordering: L2L into level l must already be done, so
// the caller invokes this per level.
int m2l_prepare(dust_octree *o, FmmDev &d, cudaStream_t st) {
  const int ll = o->G.ll;
  uint32_t c0 = (uint32_t)o->act_off[2 <= ll ? 2 : ll + 1];
  uint32_t nact = (uint32_t)o->n_active;
  uint32_t m = nact > c0 ? nact - c0 : 0;
  o->m2l_list = nullptr;
  memset(o->m2l_cnt, 0, sizeof(o->m2l_cnt));
  if (m == 0) return DUST_OK;
  DUST_TRY(devbuf_grow(o->m2l_buf, (size_t)m * 16 + 4096));
  uint32_t *k_in = (uint32_t *)o->m2l_buf.p, *v_in = k_in + m, *k_out = v_in + m,
           *v_out = k_out + m;
  int *hist = (int *)(v_out + m);
  DUST_CUDA(cudaMemsetAsync(hist, 0, 256 * sizeof(int), st));
  k_m2l_keys<<<nblk(m, 256), 256, 0, st>>>(d, c0, nact, k_in, v_in, hist);
  size_t tb = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tb, k_in, k_out, v_in, v_out, (int)m, 0, 8, st);
  DUST_TRY(devbuf_grow(o->cub_tmp, tb));
  DUST_CUDA(cub::DeviceRadixSort::SortPairs(o->cub_tmp.p, tb, k_in, k_out, v_in, v_out, (int)m,
                                            0, 8, st));
  int h[256];
  DUST_CUDA(cudaMemcpyAsync(h, hist, sizeof(h), cudaMemcpyDeviceToHost, st));
  DUST_CUDA(cudaStreamSynchronize(st));
  memcpy(o->m2l_cnt, h, sizeof(int) * 8 * (DUST_MAXLEV + 1));
  o->m2l_list = v_out;
  // pre-scaled source coefficients of all active cells of levels >= 2
  bool f32 = o->prm.precision == DUST_PREC_FP32C;
  size_t ab = (size_t)m * 4 * o->nm * (f32 ? 4 : 8) + 256;
  DUST_TRY(devbuf_grow(o->ahat, ab));
  o->ahat_c0 = c0;
  return DUST_OK;
}

// fills the pre-scaled coefficients once the upward pass is complete
int m2l_scale_sources(dust_octree *o, FmmDev &d, cudaStream_t st) {
  if (!o->m2l_list) return DUST_OK;
  uint32_t c0 = o->ahat_c0, nact = (uint32_t)o->n_active;
  size_t tot = (size_t)(nact - c0) * 3 * o->nm;
  if (tot == 0) return DUST_OK;
  if (o->prm.precision == DUST_PREC_FP32C)
    k_scale_a<float><<<nblk(tot, 256), 256, 0, st>>>(d, c0, nact, (float *)o->ahat.p);
  else
    k_scale_a<double><<<nblk(tot, 256), 256, 0, st>>>(d, c0, nact, (double *)o->ahat.p);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}
struct M2LLaunch {
  unsigned grid;
  int NW;
  size_t sm;
  cudaStream_t st;
  int NB, TCX, SL, nJ, P, jsum_smem;
};

template <typename T, int SLC>
static int m2l_launch(const M2LLaunch &L, FmmDev &d, const dust_octree *o, const M2LTabs &tabs,
                      const T *ahat, const uint2 *js) {
  if (L.sm > 48 * 1024)
    DUST_CUDA(cudaFuncSetAttribute(k_m2l_batch<T, SLC>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.sm));
  k_m2l_batch<T, SLC><<<L.grid, L.NW * 32, L.sm, L.st>>>(
      d, (const int4 *)o->m2l_bat.p, o->m2l_list, L.NB, L.NW, L.TCX, tabs, ahat, o->ahat_c0, js,
      L.SL, L.nJ, L.P, L.jsum_smem);
  return DUST_OK;
}

// slot counts 1-3 (degrees p <= 4 with stretching) get a kernel of their own
template <typename T>
static int m2l_launch_sl(const M2LLaunch &L, FmmDev &d, const dust_octree *o,
                         const M2LTabs &tabs, const T *ahat, const uint2 *js) {
  switch (L.SL) {
    case 1: return m2l_launch<T, 1>(L, d, o, tabs, ahat, js);
    case 2: return m2l_launch<T, 2>(L, d, o, tabs, ahat, js);
    case 3: return m2l_launch<T, 3>(L, d, o, tabs, ahat, js);
    default: return m2l_launch<T, 0>(L, d, o, tabs, ahat, js);
  }
}

int m2l_all_levels(dust_octree *o, FmmDev &d, cudaStream_t st) {
  if (!o->m2l_list) return DUST_OK;
  // batch size and warps: the largest that fit, two CTAs per SM when
  // possible, else one
  const bool f32 = o->prm.precision == DUST_PREC_FP32C;
  const size_t esz = f32 ? 4 : 8;
  const int nm = o->nm, nJ = o->m2l_nJ, SL = o->m2l_SL, P = o->m2l_P;
  int NB = 8, NW = 2, TCX = M2L_TC;
  bool found = false;
  const size_t jsb = (size_t)((SL + M2L_SLP - 1) / M2L_SLP) * nm * 32 * 8;
  const int jsum_smem = jsb <= 16 * 1024 ? 1 : 0;
  const size_t isb = jsum_smem ? jsb + 32 : 32;  // (+ two 16-byte alignments)
  auto wsl = [&](int tc) { return esz * (((size_t)P + (size_t)tc * 3 * nm + 3) / 4 * 4); };
  const int nbs[4] = {64, 48, 32, 16}, nws[5] = {8, 6, 4, 2, 1};
  // FP64 tiles stop at 4 targets (registers)
  const int tcs_f32[3] = {8, 4, 2}, tcs_f64[3] = {4, 2, 2};
  const int *tcs = f32 ? tcs_f32 : tcs_f64;
  auto smem_of = [&](int nb, int nw, int tc) {
    return (size_t)nb * 3 * nJ * 8 + (size_t)nb * 12 + isb + (size_t)nw * wsl(tc);
  };
  // two CTAs of >= 4 warps per SM when possible, else one CTA (high
  // degrees: fewer warps, shorter chunks)
  for (size_t cap : {(size_t)110 * 1024, (size_t)220 * 1024})
    for (int c = 0; c < 3 && !found; ++c)
      for (int b = 0; b < 5 && !found; ++b)
        for (int a = 0; a < 4 && !found; ++a)
          if (smem_of(nbs[a], nws[b], tcs[c]) <= cap && (nws[b] >= 4 || cap > 110 * 1024)) {
            NB = nbs[a];
            NW = nws[b];
            TCX = tcs[c];
            found = true;
          }
  if (!found) return DUST_ERR_CAPACITY;
  std::vector<int4> bs;
  int start = 0;
  for (int k = 0; k < 8 * (DUST_MAXLEV + 1); ++k) {
    int c = o->m2l_cnt[k];
    int l = k >> 3, q = k & 7;
    if (l >= 2)
      for (int b = 0; b < c; b += NB) bs.push_back(make_int4(l, q, start + b, std::min(NB, c - b)));
    start += c;
  }
  if (bs.empty()) return DUST_OK;
  DUST_TRY(devbuf_grow(o->m2l_bat, bs.size() * sizeof(int4)));
  DUST_CUDA(cudaMemcpyAsync(o->m2l_bat.p, bs.data(), bs.size() * sizeof(int4),
                            cudaMemcpyHostToDevice, st));
  const size_t sm = smem_of(NB, NW, TCX);
  M2LTabs tabs;
  for (int l = 0; l <= DUST_MAXLEV; ++l)
    tabs.t[l] = (l >= 2 && l <= o->G.ll) ? (f32 ? o->dtab32[l].p : o->dtabs[l].p) : nullptr;
  const unsigned grid = (unsigned)bs.size();
  const uint2 *js = (const uint2 *)o->jsum.p;
  o->kev_m2l = o->timing;
  if (o->timing) cudaEventRecord(o->ev[6], st);
  M2LLaunch L{grid, NW, sm, st, NB, TCX, SL, nJ, P, jsum_smem};
  if (f32) DUST_TRY(m2l_launch_sl<float>(L, d, o, tabs, (const float *)o->ahat.p, js));
  else DUST_TRY(m2l_launch_sl<double>(L, d, o, tabs, (const double *)o->ahat.p, js));
  if (o->timing) cudaEventRecord(o->ev[7], st);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}
