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
// mod_octree.f90:440-476).  A CTA takes NB targets of one class and loops
// over the 189 offsets; per offset it stages the offset's Dhat table once
// (shared by all NB targets) and the NB source multipoles (zero where the
// source cell is missing, inactive or empty) in shared memory.  A thread
// owns a 4-target x 2-output register tile, so each n-step loads 6 table
// values and 12 source values for 48 FMAs.  Accumulators stay in registers
// across the offsets; the result is added once to the cell's b and g.
//
// Scaling: with h the cell size of the level, the tables hold
// Dhat(k) h^(|k|+2) and the sources a(n) / (n! h^|n|), so both stay of order
// one at every level and degree; the output is rescaled by h^-(|m'|+2).
//
// FP32C: tables and source coefficients in FP32, each offset's partial sums
// in FP32, accumulated across offsets in FP64.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>
#include <vector>

#include "dust_common.cuh"
#include "fmm_internal.h"

#define M2L_T 256

struct M2LTabs {
  const void *t[DUST_MAXLEV + 1];  // per-level dimensionless tables
};

// One CTA per batch descriptor (level, class, first target, count); the
// batches of all levels >= 2 run in one launch (M2L of different levels is
// independent; L2L follows level by level).
//
// Inside a CTA the warps are independent: warp w takes offsets w, w+W, ...;
// lane i looks up the source of target i at that offset, the present ones
// are compacted with a ballot, the warp stages the offset's table and (in
// chunks of up to TCX <= M2L_TC) the present sources in its own shared-memory slice
// and evaluates them with __syncwarp only.  A chunk of kc targets runs the
// register tile of the largest power of two <= kc (8, 4, 2, 1), so no lane
// computes for an absent target.  In the tile a lane owns the outputs
// m' = mb + lane and mb + 32 + lane for every target of the chunk: per
// source monomial n it reads two table entries (Dx, Dy, Dz) at m' + n and,
// per target, the source's (ax, ay, az), each as one vector load, for
// 6 FMAs per (target, output).  The chunk's sums (over the nm source
// monomials of one offset, in T) go to the CTA's FP64 accumulators with
// shared-memory atomics.
#define M2L_TC 8
#define M2L_GQ 4
template <typename T>
struct M2LVec {
  T x, y, z;
};
template <typename T>
__device__ __forceinline__ M2LVec<T> m2l_ld(const T *p);
template <>
__device__ __forceinline__ M2LVec<float> m2l_ld<float>(const float *p) {
  const float4 v = *(const float4 *)p;
  return {v.x, v.y, v.z};
}
template <>
__device__ __forceinline__ M2LVec<double> m2l_ld<double>(const double *p) {
  const double2 a = *(const double2 *)p;
  return {a.x, a.y, p[2]};
}

// count padded (x y z 0) entries from global to shared memory, by the warp
__device__ __forceinline__ void m2l_copy4(float *dst, const float *src, int count, int lane) {
  for (int e = lane; e < count; e += 32)
    *(float4 *)(dst + 4 * e) = __ldg((const float4 *)(src + 4 * e));
}
__device__ __forceinline__ void m2l_copy4(double *dst, const double *src, int count, int lane) {
  for (int e = lane; e < 2 * count; e += 32)
    *(double2 *)(dst + 2 * e) = __ldg((const double2 *)(src + 2 * e));
}

template <typename T, int TCc>
__device__ __forceinline__ void m2l_tile(const T *__restrict__ sD, const T *__restrict__ sA,
                                         const uint16_t *__restrict__ isum, int nm, int nm1,
                                         int nout, int lane, const int *tl, int kreal,
                                         double *__restrict__ s_acc) {
  for (int mb = 0; mb < nout; mb += 64) {
    const int m0 = mb + lane, m1 = m0 + 32;
    const int c0 = m0 < nout ? m0 : 0, c1 = m1 < nout ? m1 : 0;
    T pa[TCc][2][3];
#pragma unroll
    for (int c = 0; c < TCc; ++c)
#pragma unroll
      for (int h = 0; h < 2; ++h) pa[c][h][0] = pa[c][h][1] = pa[c][h][2] = (T)0;
#pragma unroll 2
    for (int n = 0; n < nm; ++n) {
      const M2LVec<T> D0 = m2l_ld(sD + 4 * isum[(size_t)n * nm1 + c0]);
      const M2LVec<T> D1 = m2l_ld(sD + 4 * isum[(size_t)n * nm1 + c1]);
#pragma unroll
      for (int c = 0; c < TCc; ++c) {
        const M2LVec<T> a = m2l_ld(sA + ((size_t)c * nm + n) * 4);
        pa[c][0][0] = fma(D0.y, a.z, fma(-D0.z, a.y, pa[c][0][0]));
        pa[c][0][1] = fma(D0.z, a.x, fma(-D0.x, a.z, pa[c][0][1]));
        pa[c][0][2] = fma(D0.x, a.y, fma(-D0.y, a.x, pa[c][0][2]));
        pa[c][1][0] = fma(D1.y, a.z, fma(-D1.z, a.y, pa[c][1][0]));
        pa[c][1][1] = fma(D1.z, a.x, fma(-D1.x, a.z, pa[c][1][1]));
        pa[c][1][2] = fma(D1.x, a.y, fma(-D1.y, a.x, pa[c][1][2]));
      }
    }
#pragma unroll
    for (int c = 0; c < TCc; ++c) {
      if (c >= kreal) break;  // zero-padded slots of the tile
      double *acc = s_acc + (size_t)tl[c] * nout * 3;
      if (m0 < nout)
        for (int e = 0; e < 3; ++e) atomicAdd(acc + e * nout + m0, (double)pa[c][0][e]);
      if (m1 < nout)
        for (int e = 0; e < 3; ++e) atomicAdd(acc + e * nout + m1, (double)pa[c][1][e]);
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_m2l_batch(FmmDev d, const int4 *batches,
                                                   const uint32_t *list, int NB, int NW,
                                                   int TCX, M2LTabs tabs, const T *ahat,
                                                   uint32_t ahat_cell0, int isum_smem) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int nm = d.nm, nm1 = d.nm1, nD = d.nD;
  const int nout = d.use_vs ? nm1 : nm;
  const int4 bd = batches[blockIdx.x];
  const int l = bd.x, q = bd.y, t0 = bd.z, cnt = bd.w;
  const T *dtab = (const T *)tabs.t[l];
  double *s_acc = (double *)smraw;                  // NB x nout x 3
  int *s_tc = (int *)(s_acc + (size_t)NB * nout * 3);  // NB x 3 target carts
  const size_t wslice = (size_t)4 * nD + (size_t)TCX * 4 * nm;  // per warp, in T
  uint16_t *s_isum = (uint16_t *)(s_tc + 3 * NB);  // nm x nm1 index table (optional)
  const uint16_t *isum = isum_smem ? s_isum : d.idxsum;
  const size_t isz = isum_smem ? (size_t)nm * nm1 : 0;
  T *s_w = (T *)(((uintptr_t)(s_isum + isz) + 15) & ~(uintptr_t)15);
  __shared__ double s_hp[2 * DUST_MAXP + 6];  // (1/h)^d
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
  for (int e = tid; e < NB * nout * 3; e += NW * 32) s_acc[e] = 0.0;
  for (int e = tid; e < (int)isz; e += NW * 32) s_isum[e] = d.idxsum[e];
  __syncthreads();
  T *sD = s_w + (size_t)warp * wslice;
  T *sA = sD + 4 * nD;
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
      for (int q = 1; q < M2L_GQ; ++q) v = (g == q) ? srcq[q][h] : v;
      src[h] = v;
    }
    unsigned msk[2] = {__ballot_sync(0xffffffffu, src[0] >= 0),
                       __ballot_sync(0xffffffffu, src[1] >= 0)};
    if (!(msk[0] | msk[1])) continue;
    npairs += __popc(msk[0]) + __popc(msk[1]);
    const int tab = (ox + L) + W * ((oy + L) + W * (oz + L));
    const T *Dg = dtab + (size_t)tab * nD * 4;
    __syncwarp();
    m2l_copy4(sD, Dg, nD, lane);
    // the present targets of both halves in chunks of up to TCX; a chunk of
    // 3-4 (5-8) runs the 4- (8-) target tile with zero sources in the spare
    // slots, which costs less than splitting it (every tile re-reads the
    // offset's table entries for its outputs)
    unsigned long long m = (unsigned long long)msk[0] | ((unsigned long long)msk[1] << 32);
    while (m) {
      const int kc = min(__popcll(m), TCX);
      const int tile = kc <= 2 ? kc : kc <= 4 ? 4 : 8;
      int tl[M2L_TC];
      for (int c = 0; c < kc; ++c) {
        const int t = __ffsll((long long)m) - 1;
        m &= m - 1;
        tl[c] = t;
        const int sc_ = __shfl_sync(0xffffffffu, t >= 32 ? src[1] : src[0], t & 31);
        m2l_copy4(sA + (size_t)c * nm * 4, ahat + (size_t)(sc_ - ahat_cell0) * 4 * nm, nm, lane);
      }
      for (int c = kc; c < tile; ++c)
        for (int e = lane; e < 4 * nm; e += 32) sA[(size_t)c * nm * 4 + e] = (T)0;
      __syncwarp();
      if (tile == 8) m2l_tile<T, 8>(sD, sA, isum, nm, nm1, nout, lane, tl, kc, s_acc);
      else if (tile == 4) m2l_tile<T, 4>(sD, sA, isum, nm, nm1, nout, lane, tl, kc, s_acc);
      else if (tile == 2) m2l_tile<T, 2>(sD, sA, isum, nm, nm1, nout, lane, tl, kc, s_acc);
      else m2l_tile<T, 1>(sD, sA, isum, nm, nm1, nout, lane, tl, kc, s_acc);
      __syncwarp();
    }
    }
  }
  __syncthreads();
  if (lane == 0 && d.counters) atomicAdd((unsigned long long *)d.counters, npairs);
  for (int e = tid; e < cnt * nout; e += NW * 32) {
    const int t = e / nout, mo = e - t * nout;
    int oi, oj, ok;
    mono_exp(mo, oi, oj, ok);
    const double sc =
        (((oi + oj + ok) & 1) ? -1.0 : 1.0) * d.inv_fact[mo] * s_hp[oi + oj + ok + 2];
    const uint32_t ci = list[t0 + t];
    const double *acc = s_acc + (size_t)t * nout * 3;
    if (d.use_vs) {
      double *g = d.Gx + (size_t)ci * 3 * nm1;
      for (int c = 0; c < 3; ++c) g[3 * mo + c] += sc * acc[c * nout + mo];
    }
    if (mo < nm) {
      double *bb = d.B + (size_t)ci * 3 * nm;
      for (int c = 0; c < 3; ++c) bb[3 * mo + c] += sc * acc[c * nout + mo];
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
  // dimensionless tables Dhat(k) h^(|k|+2) for the batched kernel, FP64 and
  // FP32 copies
  int nD = o->nD;
  std::vector<int> deg(nD);
  for (int q = 0; q < nD; ++q) {
    int i, j, k;
    mono_exp(q, i, j, k);
    deg[q] = i + j + k;
  }
  // padded [343 offsets][nD][4] (x y z 0): one vector load per entry
  for (int l = 2; l <= o->G.ll; ++l) {
    size_t n = (size_t)343 * nD * 3, n4 = (size_t)343 * nD * 4;
    DUST_TRY(devbuf_grow(o->dtabs[l], n4 * 8));
    DUST_TRY(devbuf_grow(o->dtab32[l], n4 * 4));
    std::vector<double> h(n), h4(n4, 0.0);
    DUST_CUDA(cudaMemcpy(h.data(), o->dtab[l].p, n * 8, cudaMemcpyDeviceToHost));
    double cs = o->G.csize[l];
    std::vector<double> hp(2 * DUST_MAXP + 6, 1.0);
    for (size_t e = 1; e < hp.size(); ++e) hp[e] = hp[e - 1] * cs;
    std::vector<float> f(n4, 0.f);
    for (size_t i = 0; i < n; ++i) {
      size_t q = (i / 3) % nD;
      size_t j = (i / 3) * 4 + i % 3;
      h4[j] = h[i] * hp[deg[q] + 2];
      f[j] = (float)h4[j];
    }
    DUST_CUDA(cudaMemcpy(o->dtabs[l].p, h4.data(), n4 * 8, cudaMemcpyHostToDevice));
    DUST_CUDA(cudaMemcpy(o->dtab32[l].p, f.data(), n4 * 4, cudaMemcpyHostToDevice));
  }
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

int m2l_all_levels(dust_octree *o, FmmDev &d, cudaStream_t st) {
  if (!o->m2l_list) return DUST_OK;
  // batch size and warps: the largest that fit, two CTAs per SM when
  // possible, else one
  bool f32 = o->prm.precision == DUST_PREC_FP32C;
  size_t esz = f32 ? 4 : 8;
  int nout = o->prm.vortstretch ? o->nm1 : o->nm;
  int NB = 8, NW = 2, TCX = M2L_TC;
  bool found = false;
  const int isum_smem = (size_t)o->nm * o->nm1 * 2 <= 16 * 1024 ? 1 : 0;
  const size_t isb = isum_smem ? (size_t)o->nm * o->nm1 * 2 + 16 : 0;
  auto wsl = [&](int tc) { return esz * ((size_t)4 * o->nD + (size_t)tc * 4 * o->nm); };
  const int nbs[4] = {64, 48, 32, 16}, nws[5] = {8, 6, 4, 2, 1}, tcs[3] = {8, 4, 2};
  auto smem_of = [&](int nb, int nw, int tc) {
    return (size_t)nb * nout * 24 + (size_t)nb * 12 + 32 + isb + (size_t)nw * wsl(tc);
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
  size_t sm = smem_of(NB, NW, TCX);
  M2LTabs tabs;
  for (int l = 0; l <= DUST_MAXLEV; ++l)
    tabs.t[l] = (l >= 2 && l <= o->G.ll) ? (f32 ? o->dtab32[l].p : o->dtabs[l].p) : nullptr;
  unsigned grid = (unsigned)bs.size();
  o->kev_m2l = o->timing;
  if (o->timing) cudaEventRecord(o->ev[6], st);
  if (f32) {
    if (sm > 48 * 1024)
      DUST_CUDA(cudaFuncSetAttribute(k_m2l_batch<float>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_m2l_batch<float><<<grid, NW * 32, sm, st>>>(d, (const int4 *)o->m2l_bat.p, o->m2l_list,
                                                NB, NW, TCX, tabs, (const float *)o->ahat.p, o->ahat_c0,
                                                isum_smem);
  } else {
    if (sm > 48 * 1024)
      DUST_CUDA(cudaFuncSetAttribute(k_m2l_batch<double>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_m2l_batch<double><<<grid, NW * 32, sm, st>>>(d, (const int4 *)o->m2l_bat.p, o->m2l_list,
                                                 NB, NW, TCX, tabs, (const double *)o->ahat.p,
                                                 o->ahat_c0, isum_smem);
  }
  if (o->timing) cudaEventRecord(o->ev[7], st);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}
