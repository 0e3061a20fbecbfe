// direct.cu -- the O(N*M) direct sums of the step:
//   * elements -> particles (apply_multipole's element loop,
//     src/fmm/mod_octree.f90:1350-1373) fused with the wind and the scatter
//     of all FMM outputs to the caller's particle order;
//   * particles (+ end vortices) -> collocation points (get_vort_vel,
//     src/aeroel/mod_surfpan.f90:962-977, mod_vortlatt.f90:676-693).
//
// Far field.  When a point lies beyond the far-field radius of both the
// doublet (far_field_ratio_doublet * max edge) and the source (10 * max
// edge), the reference evaluates velocity_calc_doublet's dipole and
// velocity_calc_sou_surfpan's point-source formulas in the panel's tangent
// frame (mod_doublet.f90:199-212, mod_surfpan.f90:285-291).  Summed as
// compute_vel_surfpan does (vdou*mag - vsou*sigma) they are exactly
//   v = (A / r^3) [ r (3 mu (r.n) / r^2 + sigma) - mu n ],   mu = mag,
// which is evaluated here with one reciprocal square root (the frame
// vectors cancel algebraically; only rounding differs).  Nearer pairs use
// the reference's full formulas (elements.cuh) in FP64.
//
// Precision.  FP64 everywhere in the plain mode.  In the FP32C mode the far
// field runs in FP32 on coordinates taken relative to a reference point of
// the CTA's particle tile (so no large-coordinate cancellation); partial
// sums over one tile of sources are FP32 and are added into FP64
// accumulators tile by tile; near pairs stay FP64 (listed by the FP32
// kernel and evaluated apart from it, k_elem_far / k_elem_near).
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>

#include "dust_common.cuh"
#include "elements.cuh"
#include "fmm_internal.h"

static inline unsigned nblk(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

struct FFRec {  // far-field record of a panel (double)
  double c[3], n[3];
  double amu, asig;  // area*mag, area*sig
  double ff2;        // squared radius beyond which both far fields apply
  double pad;
};

__global__ void k_ffrec(const PanelGeo *pg, int n, double ff_dou, FFRec *out) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const PanelGeo &p = pg[j];
  FFRec r;
  for (int d = 0; d < 3; ++d) {
    r.c[d] = p.cen[d];
    r.n[d] = p.nor[d];
  }
  r.amu = p.area * p.mag;
  bool sp = p.kind == DUST_ELEM_SURFPAN;
  // compute_vel_surfpan adds -vsou*sig and the far-field vsou is -A r/r^3
  r.asig = sp ? p.area * p.sig : 0.0;
  double f = sp ? fmax(ff_dou, 10.0) : ff_dou;
  r.ff2 = (f * p.max_edge) * (f * p.max_edge);
  r.pad = 0.0;
  out[j] = r;
}

// exact reference evaluation of one panel (x 4 pi)
__device__ inline void near_pan(const RegParams &rp, const PanelGeo *pg, int j,
                                const double *pos, double *v) {
  vel_pan_near(rp, pg[j], pos, v);
}

// FP64 element sums (plain mode): far field by the closed form above, near
// pairs by the reference's formulas; then end vortices, wind and the scatter
// of all outputs to the caller's order.
//
// EO_PPT particles per thread against shared-memory tiles of EO_LOAD panels
// (far-field records, FP64).  The loader threads test each panel against the
// bounding box of the CTA's particles: a sub-tile of EO_TILE panels that
// lies beyond the far-field radius of the whole box runs the far formula
// without a per-pair test (the box distance is formed with the per-pair
// test's own operation order, so rounding, being monotone, cannot make the
// box call far a pair the per-pair test calls near).  In the other sub-tiles
// each pair is tested; the near pairs of a particle are marked in a bit mask
// and evaluated after the sub-tile's far loop, in panel order, so the sums
// are deterministic.  The reciprocal square root of the far formula is the
// FP32 approximation refined by one second-order Newton-Raphson
// (Householder) step in FP64: with y0 = x^-1/2 (1 + d) and e = 1 - x y0^2,
// y = y0 (1 + e/2 + 3 e^2/8) has relative error O(d^3), below the FP64
// rounding for |d| < 2^-21.
#define EO_PPT 2
#define EO_T 128
#define EO_NP (EO_T * EO_PPT)
#define EO_TILE 16
#define EO_SUB 4
#define EO_LOAD (EO_TILE * EO_SUB)
#define EO_PK 12  // nm x/y/z, mn x/y/z, -c x/y/z, as, ff2, pad
static_assert(EO_LOAD <= EO_T && EO_LOAD % 32 == 0 && EO_TILE <= 32, "staging layout");

__device__ __forceinline__ float rsqrt_approx(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// x^-1/2 for a normal FP32-range x > 0
__device__ __forceinline__ double rsqrt_hh(double x) {
  const double y = (double)rsqrt_approx((float)x);
  const double e = fma(-x * y, y, 1.0);
  return fma(y * e, fma(0.375, e, 0.5), y);
}

__global__ void __launch_bounds__(EO_T) k_elem_out(FmmDev d, ElemDev e, const FFRec *ff,
                                                   double *vel, double *str, double *rot) {
  __shared__ __align__(16) double s_pk[EO_LOAD][EO_PK];
  __shared__ unsigned s_nearw[EO_LOAD / 32];
  __shared__ double s_box[EO_T / 32][6];
  const size_t n = d.n;
  const uint32_t t0 = blockIdx.x * EO_NP;
  const int tid = threadIdx.x;
  double pos[EO_PPT][3], v[EO_PPT][3];
  bool act[EO_PPT];
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
#pragma unroll
  for (int i = 0; i < EO_PPT; ++i) {
    const uint32_t t = t0 + tid + i * EO_T;
    act[i] = t < n;
    const uint32_t tt = act[i] ? t : t0;
    for (int c = 0; c < 3; ++c) {
      pos[i][c] = d.P[(size_t)c * n + tt];
      lo[c] = fmin(lo[c], pos[i][c]);
      hi[c] = fmax(hi[c], pos[i][c]);
      v[i][c] = 0.0;
    }
  }
  // bounding box of the CTA's particles
#pragma unroll
  for (int c = 0; c < 3; ++c)
    for (int o = 16; o > 0; o >>= 1) {
      lo[c] = fmin(lo[c], __shfl_xor_sync(0xffffffffu, lo[c], o));
      hi[c] = fmax(hi[c], __shfl_xor_sync(0xffffffffu, hi[c], o));
    }
  if ((tid & 31) == 0)
    for (int c = 0; c < 3; ++c) s_box[tid >> 5][c] = lo[c], s_box[tid >> 5][3 + c] = hi[c];
  __syncthreads();
  for (int w = 0; w < EO_T / 32; ++w)
    for (int c = 0; c < 3; ++c) lo[c] = fmin(lo[c], s_box[w][c]), hi[c] = fmax(hi[c], s_box[w][3 + c]);
  const int ntot = e.nbody + e.nwake;
  for (int p0 = 0; p0 < ntot; p0 += EO_LOAD) {
    __syncthreads();
    bool near_box = false;
    if (tid < EO_LOAD) {
      double *pk = s_pk[tid];
      if (p0 + tid < ntot) {
        const FFRec &r = ff[p0 + tid];
        for (int c = 0; c < 3; ++c) {
          pk[c] = 3.0 * r.amu * r.n[c];
          pk[3 + c] = -r.amu * r.n[c];
          pk[6 + c] = -r.c[c];
        }
        pk[9] = r.asig;
        pk[10] = r.ff2;
        // box distance in the per-pair test's operation order
        double q[3];
        for (int c = 0; c < 3; ++c) {
          const double a = lo[c] - r.c[c], b = hi[c] - r.c[c];
          q[c] = a > 0.0 ? a : (b < 0.0 ? b : 0.0);
        }
        const double d2 = fma(q[0], q[0], fma(q[1], q[1], q[2] * q[2]));
        near_box = !(d2 > r.ff2);
      } else {
        // padding: no strength, far away
        for (int c = 0; c < 11; ++c) pk[c] = 0.0;
        pk[6] = -1.0e6;
      }
      pk[11] = 0.0;
    }
    const unsigned nb = __ballot_sync(0xffffffffu, near_box);
    if ((tid & 31) == 0 && tid < EO_LOAD) s_nearw[tid >> 5] = nb;
    __syncthreads();
    const int nsub = min(EO_SUB, (ntot - p0 + EO_TILE - 1) / EO_TILE);
    for (int sb = 0; sb < nsub; ++sb) {
      const int qs = sb * EO_TILE;
      const bool near_sub = (s_nearw[qs >> 5] >> (qs & 31)) & ((1u << EO_TILE) - 1u);
      unsigned nmask[EO_PPT];
#pragma unroll
      for (int i = 0; i < EO_PPT; ++i) nmask[i] = 0u;
#pragma unroll 4
      for (int q = 0; q < EO_TILE; ++q) {
        const double2 *pk = (const double2 *)s_pk[qs + q];
        const double2 A = pk[0], B = pk[1], C = pk[2], D = pk[3], E = pk[4], F = pk[5];
        // A = (nmx, nmy), B = (nmz, mnx), C = (mny, mnz), D = (-cx, -cy), E = (-cz, as), F = (ff2, 0)
#pragma unroll
        for (int i = 0; i < EO_PPT; ++i) {
          const double rx = pos[i][0] + D.x, ry = pos[i][1] + D.y, rz = pos[i][2] + E.x;
          const double r2 = fma(rx, rx, fma(ry, ry, rz * rz));
          const bool far = !near_sub || r2 > F.x;
          if (far) {
            const double ir = rsqrt_hh(r2);
            const double ir2 = ir * ir;
            const double k3 = ir2 * ir;
            const double rn = fma(rx, A.x, fma(ry, A.y, rz * B.x));
            const double coef = fma(rn, ir2, E.y);
            v[i][0] = fma(k3, fma(coef, rx, B.y), v[i][0]);
            v[i][1] = fma(k3, fma(coef, ry, C.x), v[i][1]);
            v[i][2] = fma(k3, fma(coef, rz, C.y), v[i][2]);
          } else {
            nmask[i] |= 1u << q;
          }
        }
      }
      if (near_sub) {
#pragma unroll
        for (int i = 0; i < EO_PPT; ++i) {
          unsigned m = act[i] ? nmask[i] : 0u;
          while (m) {
            const int q = __ffs(m) - 1;
            m &= m - 1u;
            const int j = p0 + qs + q;
            const PanelGeo *pg = j < e.nbody ? e.body + j : e.wake + (j - e.nbody);
            double u[3];
            vel_pan_near(e.rp, *pg, pos[i], u);
            for (int c = 0; c < 3; ++c) v[i][c] += u[c];
          }
        }
      }
    }
  }
  const double k4pi = 1.0 / (4.0 * DUST_PI);
#pragma unroll
  for (int i = 0; i < EO_PPT; ++i) {
    if (!act[i]) continue;
    for (int q = 0; q < e.nline; ++q) {
      double u[3];
      vel_line(e.rp, e.lines[q], pos[i], u);
      for (int c = 0; c < 3; ++c) v[i][c] += u[c];
    }
    const uint32_t t = t0 + tid + i * EO_T;
    const uint32_t ip = d.perm[t];
    for (int c = 0; c < 3; ++c) {
      vel[3 * (size_t)ip + c] = d.out[(size_t)c * n + t] + v[i][c] * k4pi + d.u_inf[c];
      if (str) str[3 * (size_t)ip + c] = (d.use_vs || d.use_vd) ? d.out[(size_t)(3 + c) * n + t] : 0.0;
      if (rot) rot[3 * (size_t)ip + c] = (d.use_vs && d.use_df) ? d.out[(size_t)(6 + c) * n + t] : 0.0;
    }
  }
}

// FP32C element sums, far and near pairs in separate kernels.
//
// k_elem_far runs the far-field test and formula in FP32 for EF2_PPT
// particles per thread against a shared-memory tile of EF2_TILE panels; the
// tile's partial sums are FP32, added into FP64 per tile.  A pair that is
// not clearly far (threshold widened by 1e-4 so a pair far in FP32 is far in
// FP64) is queued in shared memory and the queue is appended to a global list
// of near pairs.  k_elem_near evaluates that list with the reference's exact
// FP64 formulas (vel_pan_near), one pair per thread, and k_elem_fin adds the end
// vortices and writes the outputs in the caller's order.  Keeping the heavy
// FP64 formulas out of the FP32 kernel keeps its register count, and so its
// occupancy, at the level of the far-field arithmetic.
//
// Most tiles lie beyond the far-field radius of every particle of the CTA:
// the loader threads test each panel against the bounding box of the CTA's
// particles (with a further 1e-4 margin, so the box test never calls far a
// pair the per-pair test would queue) and such tiles run a loop without the
// per-pair test.  A tile shorter than EF2_TILE is padded with null panels
// (no strength, 1e6 away) so both loops are fully unrolled.
#ifndef EF2_PPT
#define EF2_PPT 2
#endif
#define EF2_T 128
#define EF2_NP (EF2_T * EF2_PPT)
#define EF2_TILE 16  // panels per FP32 partial sum and per near-queue check
#ifndef EF2_SUB
#define EF2_SUB 4  // sub-tiles staged per barrier pair
#endif
#define EF2_LOAD (EF2_TILE * EF2_SUB)
#define EF2_QCAP (EF2_NP * EF2_TILE)  // one tile's worst case
static_assert(EF2_LOAD % 32 == 0 && EF2_LOAD <= EF2_T && EF2_SUB <= 32, "staging layout");
static_assert(EF2_NP <= 1024, "local particle index is packed in 10 bits");

struct NearPair {
  uint32_t t, j;  // particle (sorted order), panel
};

__device__ __forceinline__ void ef2_flush(const uint32_t *s_q, int qn, uint32_t t0,
                                          unsigned long long *count, NearPair *list,
                                          unsigned long long cap, unsigned long long *s_base) {
  if (threadIdx.x == 0) *s_base = atomicAdd(count, (unsigned long long)qn);
  __syncthreads();
  const unsigned long long base = *s_base;
  for (int k = threadIdx.x; k < qn; k += EF2_T) {
    const unsigned long long at = base + (unsigned long long)k;
    if (at < cap) {
      const uint32_t en = s_q[k];
      list[at] = NearPair{t0 + (en & 0x3ffu), en >> 10};
    }
  }
}

// far-field term of a panel at r = p - c, added to acc:
//   nm = 3 A mu n, mn = -A mu n, as = A sigma:
//   acc += (1/r^3) (r (r.nm / r^2 + as) + mn)
__device__ __forceinline__ void ef2_term(float rx, float ry, float rz, float r2, float nmx,
                                         float nmy, float nmz, float mnx, float mny, float mnz,
                                         float as, float *acc) {
  const float ir = rsqrt_approx(r2);
  const float ir2 = ir * ir;
  const float k3 = ir2 * ir;
  const float rn = fmaf(rx, nmx, fmaf(ry, nmy, rz * nmz));
  const float coef = fmaf(rn, ir2, as);
  acc[0] = fmaf(k3, fmaf(coef, rx, mnx), acc[0]);
  acc[1] = fmaf(k3, fmaf(coef, ry, mny), acc[1]);
  acc[2] = fmaf(k3, fmaf(coef, rz, mnz), acc[2]);
}

// The same term for two panels at once in packed FP32 (f32x2) arithmetic.
__device__ __forceinline__ void ef2_term2(float2 px, float2 py, float2 pz, float2 ncx, float2 ncy,
                                          float2 ncz, float2 nmx, float2 nmy, float2 nmz,
                                          float2 mnx, float2 mny, float2 mnz, float2 as,
                                          float2 *acc) {
  const float2 rx = __fadd2_rn(px, ncx), ry = __fadd2_rn(py, ncy), rz = __fadd2_rn(pz, ncz);
  const float2 r2 = __ffma2_rn(rx, rx, __ffma2_rn(ry, ry, __fmul2_rn(rz, rz)));
  const float2 ir = make_float2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
  const float2 ir2 = __fmul2_rn(ir, ir);
  const float2 k3 = __fmul2_rn(ir2, ir);
  const float2 rn = __ffma2_rn(rx, nmx, __ffma2_rn(ry, nmy, __fmul2_rn(rz, nmz)));
  const float2 coef = __ffma2_rn(rn, ir2, as);
  acc[0] = __ffma2_rn(k3, __ffma2_rn(coef, rx, mnx), acc[0]);
  acc[1] = __ffma2_rn(k3, __ffma2_rn(coef, ry, mny), acc[1]);
  acc[2] = __ffma2_rn(k3, __ffma2_rn(coef, rz, mnz), acc[2]);
}

// Shared-memory tile: panels in pairs (q, q+1); the ten values of a pair
// (-cx, -cy, -cz, nm x/y/z, mn x/y/z, as) are stored interleaved, value k of
// panel q at [q / 2][2 k + q % 2], so five float4 loads give the ten float2
// operands of ef2_term2.
#define EF2_PK 20

__global__ void __launch_bounds__(EF2_T) k_elem_far(FmmDev d, ElemDev e, const FFRec *ff,
                                                    double *farv, unsigned long long *count,
                                                    NearPair *list, unsigned long long cap) {
  __shared__ __align__(16) float s_pk[EF2_LOAD / 2][EF2_PK];
  __shared__ float s_ff[EF2_LOAD];  // widened ff2
  __shared__ unsigned s_nearw[EF2_LOAD / 32];
  __shared__ uint32_t s_q[EF2_QCAP];  // (panel << 10) | local particle
  __shared__ float s_box[EF2_T / 32][6];
  __shared__ int s_qn;
  __shared__ unsigned long long s_base;
  const size_t n = d.n;
  const uint32_t t0 = blockIdx.x * EF2_NP;
  const int tid = threadIdx.x;
  const double ref[3] = {d.P[t0], d.P[n + t0], d.P[2 * n + t0]};
  float px[EF2_PPT], py[EF2_PPT], pz[EF2_PPT];
  bool act[EF2_PPT];
  double v[EF2_PPT][3];
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
#pragma unroll
  for (int i = 0; i < EF2_PPT; ++i) {
    const uint32_t t = t0 + tid + i * EF2_T;
    act[i] = t < n;
    double pos[3] = {ref[0], ref[1], ref[2]};
    if (act[i])
      for (int c = 0; c < 3; ++c) pos[c] = d.P[(size_t)c * n + t];
    px[i] = (float)(pos[0] - ref[0]);
    py[i] = (float)(pos[1] - ref[1]);
    pz[i] = (float)(pos[2] - ref[2]);
    if (act[i]) {
      lo[0] = fminf(lo[0], px[i]), hi[0] = fmaxf(hi[0], px[i]);
      lo[1] = fminf(lo[1], py[i]), hi[1] = fmaxf(hi[1], py[i]);
      lo[2] = fminf(lo[2], pz[i]), hi[2] = fmaxf(hi[2], pz[i]);
    }
    v[i][0] = v[i][1] = v[i][2] = 0.0;
  }
  // bounding box of the CTA's particles
#pragma unroll
  for (int c = 0; c < 3; ++c)
    for (int o = 16; o > 0; o >>= 1) {
      lo[c] = fminf(lo[c], __shfl_xor_sync(0xffffffffu, lo[c], o));
      hi[c] = fmaxf(hi[c], __shfl_xor_sync(0xffffffffu, hi[c], o));
    }
  if ((tid & 31) == 0)
    for (int c = 0; c < 3; ++c) s_box[tid >> 5][c] = lo[c], s_box[tid >> 5][3 + c] = hi[c];
  if (tid == 0) s_qn = 0;
  __syncthreads();
  for (int w = 0; w < EF2_T / 32; ++w)
    for (int c = 0; c < 3; ++c)
      lo[c] = fminf(lo[c], s_box[w][c]), hi[c] = fmaxf(hi[c], s_box[w][3 + c]);
  const int ntot = e.nbody + e.nwake;
  for (int p0 = 0; p0 < ntot; p0 += EF2_LOAD) {
    __syncthreads();
    // stage EF2_LOAD panels (EF2_SUB sub-tiles) with one barrier pair
    bool near_box = false;
    if (tid < EF2_LOAD) {
      float val[10] = {-1.0e6f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      float ffw = 0.f;
      if (p0 + tid < ntot) {
        const FFRec &r = ff[p0 + tid];
        const float cx = (float)(r.c[0] - ref[0]), cy = (float)(r.c[1] - ref[1]),
                    cz = (float)(r.c[2] - ref[2]);
        ffw = (float)r.ff2 * 1.0001f;
        const float a3 = (float)(3.0 * r.amu);
        val[0] = -cx, val[1] = -cy, val[2] = -cz;
        for (int c = 0; c < 3; ++c) {
          val[3 + c] = a3 * (float)r.n[c];
          val[6 + c] = (float)(-r.amu * r.n[c]);
        }
        val[9] = (float)r.asig;
        const float dx = fmaxf(fmaxf(lo[0] - cx, cx - hi[0]), 0.f);
        const float dy = fmaxf(fmaxf(lo[1] - cy, cy - hi[1]), 0.f);
        const float dz = fmaxf(fmaxf(lo[2] - cz, cz - hi[2]), 0.f);
        near_box = !(fmaf(dx, dx, fmaf(dy, dy, dz * dz)) > ffw * 1.0001f);
      }
      for (int k = 0; k < 10; ++k) s_pk[tid >> 1][2 * k + (tid & 1)] = val[k];
      s_ff[tid] = ffw;
    }
    // near flag of each sub-tile, one bit per sub-tile
    const unsigned nb = __ballot_sync(0xffffffffu, near_box);
    if ((tid & 31) == 0 && tid < EF2_LOAD) s_nearw[tid >> 5] = nb;
    __syncthreads();
    unsigned near_bits = 0;
#pragma unroll
    for (int w = 0; w < EF2_LOAD / 32; ++w) {
      const unsigned bw = s_nearw[w];
#pragma unroll
      for (int sb = 0; sb < 32 / EF2_TILE; ++sb)
        if ((bw >> (sb * EF2_TILE)) & ((1u << EF2_TILE) - 1u)) near_bits |= 1u << (w * (32 / EF2_TILE) + sb);
    }
    const int nsub = min(EF2_SUB, (ntot - p0 + EF2_TILE - 1) / EF2_TILE);
    for (int sb = 0; sb < nsub; ++sb) {
      const int q0 = p0 + sb * EF2_TILE;
      double tv[EF2_PPT][3];
      if (!((near_bits >> sb) & 1u)) {
        float2 acc[EF2_PPT][3];
#pragma unroll
        for (int i = 0; i < EF2_PPT; ++i) acc[i][0] = acc[i][1] = acc[i][2] = make_float2(0.f, 0.f);
#pragma unroll
        for (int pr = 0; pr < EF2_TILE / 2; ++pr) {
          const float *pk = s_pk[sb * (EF2_TILE / 2) + pr];
          const float4 A = *(const float4 *)&pk[0], B = *(const float4 *)&pk[4],
                       C = *(const float4 *)&pk[8], D = *(const float4 *)&pk[12],
                       E = *(const float4 *)&pk[16];
#pragma unroll
          for (int i = 0; i < EF2_PPT; ++i)
            ef2_term2(make_float2(px[i], px[i]), make_float2(py[i], py[i]),
                      make_float2(pz[i], pz[i]), make_float2(A.x, A.y), make_float2(A.z, A.w),
                      make_float2(B.x, B.y), make_float2(B.z, B.w), make_float2(C.x, C.y),
                      make_float2(C.z, C.w), make_float2(D.x, D.y), make_float2(D.z, D.w),
                      make_float2(E.x, E.y), make_float2(E.z, E.w), acc[i]);
        }
#pragma unroll
        for (int i = 0; i < EF2_PPT; ++i)
          for (int c = 0; c < 3; ++c) tv[i][c] = (double)acc[i][c].x + (double)acc[i][c].y;
      } else {
        // the queue must hold one sub-tile's worst case: flush first if not
        // (the near bits are the same in every thread, so are these barriers)
        __syncthreads();
        if (s_qn > EF2_QCAP - EF2_NP * EF2_TILE) {
          ef2_flush(s_q, s_qn, t0, count, list, cap, &s_base);
          __syncthreads();
          if (tid == 0) s_qn = 0;
          __syncthreads();
        }
        float acc[EF2_PPT][3];
#pragma unroll
        for (int i = 0; i < EF2_PPT; ++i) acc[i][0] = acc[i][1] = acc[i][2] = 0.f;
#pragma unroll 2
        for (int q = 0; q < EF2_TILE; ++q) {
          const int ql = sb * EF2_TILE + q;
          const float *pk = &s_pk[ql >> 1][ql & 1];
          const float ffw = s_ff[ql];
#pragma unroll
          for (int i = 0; i < EF2_PPT; ++i) {
            const float rx = px[i] + pk[0], ry = py[i] + pk[2], rz = pz[i] + pk[4];
            const float r2 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
            if (r2 > ffw) {
              ef2_term(rx, ry, rz, r2, pk[6], pk[8], pk[10], pk[12], pk[14], pk[16], pk[18],
                       acc[i]);
            } else if (act[i]) {
              const int slot = atomicAdd(&s_qn, 1);
              s_q[slot] = ((uint32_t)(q0 + q) << 10) | (uint32_t)(tid + i * EF2_T);
            }
          }
        }
#pragma unroll
        for (int i = 0; i < EF2_PPT; ++i)
          for (int c = 0; c < 3; ++c) tv[i][c] = (double)acc[i][c];
      }
#pragma unroll
      for (int i = 0; i < EF2_PPT; ++i)
        for (int c = 0; c < 3; ++c) v[i][c] += tv[i][c];
    }
  }
  __syncthreads();
  ef2_flush(s_q, s_qn, t0, count, list, cap, &s_base);
#pragma unroll
  for (int i = 0; i < EF2_PPT; ++i) {
    if (!act[i]) continue;
    const uint32_t t = t0 + tid + i * EF2_T;
    for (int c = 0; c < 3; ++c) farv[(size_t)c * n + t] = v[i][c];
  }
}

// the queued near pairs, exact FP64 (one pair per thread)
#ifndef EN_MINB
#define EN_MINB 8
#endif
__global__ void __launch_bounds__(128, EN_MINB) k_elem_near(FmmDev d, ElemDev e, const unsigned long long *count,
                            const NearPair *list, unsigned long long cap, double *farv) {
  const unsigned long long nq = min(*count, cap);
  const size_t n = d.n;
  for (unsigned long long k = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; k < nq;
       k += (unsigned long long)gridDim.x * blockDim.x) {
    const NearPair np = list[k];
    const double pos[3] = {d.P[np.t], d.P[n + np.t], d.P[2 * n + np.t]};
    const PanelGeo *pg = (int)np.j < e.nbody ? e.body + np.j : e.wake + (np.j - e.nbody);
    double u[3];
    vel_pan_near(e.rp, *pg, pos, u);
    for (int c = 0; c < 3; ++c) atomicAdd(farv + (size_t)c * n + np.t, u[c]);
  }
}

// end vortices, wind, FMM outputs; scatter to the caller's order
// End vortices in FP32 (k_elem_fin): segment (v0, v1) of circulation mag at
// a point p.  With a = p - v0,
// b = p - v1, e the unit direction and c = e x a (so |c| = h, the distance
// to the line, without the cancellation of a - (a.e) e), the reference's
// ((L - ai)/|b| + ai/|a|) c / h^2 is used while the projection ai = a.e lies
// on the segment (both terms positive), and the equivalent
// L c (|a| + |b|) / (|a||b|(|a||b| + a.b)) beyond its ends (a.b > 0 there), so
// neither form cancels.  Inside the Rankine core the result is scaled by
// h^2 / (r_rankine L)^2 as in the reference's core formula.
__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void line_vel_f(const double *vv, const float *q, const double *pos,
                                           float rr2, float rc, float *u) {
  // vv: v0 (3), v1 (3) in FP64; q: e (3), L, mag, 1 / (r_rankine L)^2.  a and
  // b are formed in FP64 and rounded once, so their accuracy does not depend
  // on the spread of the CTA's particles.  Distances and quotients by the
  // approximate reciprocal (square root) instructions.
  const float ax = (float)(pos[0] - vv[0]), ay = (float)(pos[1] - vv[1]),
              az = (float)(pos[2] - vv[2]);
  const float bx = (float)(pos[0] - vv[3]), by = (float)(pos[1] - vv[4]),
              bz = (float)(pos[2] - vv[5]);
  const float L = q[3];
  const float a2 = fmaf(ax, ax, fmaf(ay, ay, az * az));
  const float b2 = fmaf(bx, bx, fmaf(by, by, bz * bz));
  const float ira = rsqrt_approx(a2), irb = rsqrt_approx(b2);
  const float ra = a2 * ira, rb = b2 * irb;
  const float ai = fmaf(ax, q[0], fmaf(ay, q[1], az * q[2]));
  const float cx = q[1] * az - q[2] * ay, cy = q[2] * ax - q[0] * az, cz = q[0] * ay - q[1] * ax;
  const float hi2 = fmaf(cx, cx, fmaf(cy, cy, cz * cz));
  float f;
  if (ai > 0.f && ai < L) {
    f = hi2 > 0.f ? fmaf(L - ai, irb, ai * ira) * rcp_approx(hi2) : 0.f;
  } else {
    const float ab = fmaf(ax, bx, fmaf(ay, by, az * bz));
    const float den = ra * rb * fmaf(ra, rb, ab);
    f = den > 0.f ? L * (ra + rb) * rcp_approx(den) : 0.f;
  }
  if (!(hi2 > rr2 * L * L)) {
    // Rankine core (or the cutoff around the end points)
    f = (ra > L * rc && rb > L * rc) ? f * hi2 * q[5] : 0.f;
  }
  f *= q[4];
  u[0] = f * cx;
  u[1] = f * cy;
  u[2] = f * cz;
}

#define EL_T 128
#define EL_TILE 64
__global__ void __launch_bounds__(EL_T) k_elem_fin(FmmDev d, ElemDev e, const double *farv,
                                                   double *vel, double *str, double *rot) {
  __shared__ double s_v[EL_TILE][6];
  __shared__ float s_l[EL_TILE][6];
  const uint32_t t0 = blockIdx.x * EL_T, t = t0 + threadIdx.x;
  const size_t n = d.n;
  const bool act = t < n;
  double pos[3] = {0.0, 0.0, 0.0};
  if (act)
    for (int c = 0; c < 3; ++c) pos[c] = d.P[(size_t)c * n + t];
  const float rr2 = (float)(e.rp.r_rankine * e.rp.r_rankine), rc = (float)e.rp.r_cutoff;
  double w[3] = {0.0, 0.0, 0.0};
  if (act)
    for (int c = 0; c < 3; ++c) w[c] = farv[(size_t)c * n + t];
  for (int q0 = 0; q0 < e.nline; q0 += EL_TILE) {
    const int m = min(EL_TILE, e.nline - q0);
    __syncthreads();
    if (threadIdx.x < m) {
      const LineGeo &L = e.lines[q0 + threadIdx.x];
      float *q = s_l[threadIdx.x];
      for (int c = 0; c < 3; ++c) {
        s_v[threadIdx.x][c] = L.ver[0][c];
        s_v[threadIdx.x][3 + c] = L.ver[1][c];
        q[c] = (float)L.edge_uni[c];
      }
      q[3] = (float)L.edge_len;
      q[4] = (float)L.mag;
      const double rl = e.rp.r_rankine * L.edge_len;
      q[5] = (float)(1.0 / (rl * rl));
    }
    __syncthreads();
    float a[3] = {0.f, 0.f, 0.f};
    for (int k = 0; k < m; ++k) {
      float u[3];
      line_vel_f(s_v[k], s_l[k], pos, rr2, rc, u);
      a[0] += u[0];
      a[1] += u[1];
      a[2] += u[2];
    }
    for (int c = 0; c < 3; ++c) w[c] += (double)a[c];
  }
  if (!act) return;
  const double k4pi = 1.0 / (4.0 * DUST_PI);
  const uint32_t ip = d.perm[t];
  for (int c = 0; c < 3; ++c) {
    vel[3 * (size_t)ip + c] = d.out[(size_t)c * n + t] + w[c] * k4pi + d.u_inf[c];
    if (str) str[3 * (size_t)ip + c] = (d.use_vs || d.use_vd) ? d.out[(size_t)(3 + c) * n + t] : 0.0;
    if (rot) rot[3 * (size_t)ip + c] = (d.use_vs && d.use_df) ? d.out[(size_t)(6 + c) * n + t] : 0.0;
  }
}

// FP32C path: far kernel, (grow and redo if the near list overflowed), near
// kernel, outputs
static int elem_output_split(FmmDev &d, const ElemDev &e, const FFRec *ff, DevBuf &work,
                             size_t &near_cap, double *vel, double *str, double *rot,
                             cudaStream_t st, cudaEvent_t *kev, bool *kev_done) {
  const size_t n = d.n;
  if (near_cap == 0) near_cap = std::max<size_t>(1 << 20, n * 96);
  for (int attempt = 0; attempt < 3; ++attempt) {
    const size_t off_l = (n * 24 + 255) / 256 * 256 + 256;
    DUST_TRY(devbuf_grow(work, off_l + near_cap * sizeof(NearPair)));
    double *farv = (double *)work.p;
    unsigned long long *count = (unsigned long long *)((char *)work.p + off_l - 256);
    NearPair *list = (NearPair *)((char *)work.p + off_l);
    DUST_CUDA(cudaMemsetAsync(count, 0, 8, st));
    if (kev) cudaEventRecord(kev[0], st);
    k_elem_far<<<nblk(n, EF2_NP), EF2_T, 0, st>>>(d, e, ff, farv, count, list,
                                                    (unsigned long long)near_cap);
    if (kev) {
      cudaEventRecord(kev[1], st);
      if (kev_done) *kev_done = true;
    }
    unsigned long long h = 0;
    DUST_CUDA(cudaMemcpyAsync(&h, count, 8, cudaMemcpyDeviceToHost, st));
    DUST_CUDA(cudaStreamSynchronize(st));
    if (h > near_cap) {
      near_cap = (size_t)(h + h / 4 + 1024);
      continue;
    }
    if (h > 0) {
      const unsigned grid = (unsigned)std::min<unsigned long long>((h + 127) / 128, 148ull * 64);
      k_elem_near<<<grid, 128, 0, st>>>(d, e, count, list, (unsigned long long)near_cap, farv);
    }
    k_elem_fin<<<nblk(n, EL_T), EL_T, 0, st>>>(d, e, farv, vel, str, rot);
    DUST_CUDA(cudaGetLastError());
    return DUST_OK;
  }
  return DUST_ERR_CAPACITY;
}

int elem_output_device(FmmDev &d, const ElemDev &e, DevBuf &ffbuf, DevBuf &work,
                       size_t &near_cap, int precision, double *vel, double *str, double *rot,
                       cudaStream_t st, cudaEvent_t *kev, bool *kev_done) {
  if (kev_done) *kev_done = false;
  int ntot = e.nbody + e.nwake;
  DUST_TRY(devbuf_grow(ffbuf, sizeof(FFRec) * (size_t)std::max(ntot, 1)));
  FFRec *ff = (FFRec *)ffbuf.p;
  if (e.nbody) k_ffrec<<<nblk(e.nbody, 128), 128, 0, st>>>(e.body, e.nbody, e.rp.ff_dou, ff);
  if (e.nwake)
    k_ffrec<<<nblk(e.nwake, 128), 128, 0, st>>>(e.wake, e.nwake, e.rp.ff_dou, ff + e.nbody);
  if (d.n > 0) {
    // the near-pair queue packs the panel index in 22 bits
    if (precision == DUST_PREC_FP32C && ntot < (1 << 22))
      return elem_output_split(d, e, ff, work, near_cap, vel, str, rot, st, kev, kev_done);
    else
      k_elem_out<<<nblk(d.n, EO_NP), EO_T, 0, st>>>(d, e, ff, vel, str, rot);
  }
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}

// ---------------------------------------------------------------- uvort
// Grid: (point blocks) x (particle chunks); each CTA sums one chunk of
// particles for 128 points and adds its partial sums atomically.
#define UV2_T 128
#define UV2_TILE 128

// FP64 uvort (plain mode): particles in the caller's order, UVD_PPT points
// per thread (consecutive CTA slices of UV2_T points) against a shared tile
// of (x, y, z, r_v^2, alpha, w = x x alpha) records; the reciprocal square
// root as in k_elem_out (FP32 seed, one Householder step in FP64).  With
// c = rho^-3 the tile's sum is
//   sum_q c_q (p - x_q) x alpha_q = p x (sum_q c_q alpha_q) - sum_q c_q w_q,
// two 3-vector FMA accumulations per pair instead of a cross product and its
// accumulation; in FP64 the difference of the two sums costs at most about
// 1e-13 relative for a point very close to a particle.
#define UVD_PPT 4
__global__ void __launch_bounds__(UV2_T) k_uvort(int npts, const double *pts, int n,
                                                 const double *cen, const double *dir,
                                                 const double *mag, const double *rv,
                                                 int chunk, double *uv) {
  __shared__ __align__(16) double s_q[UV2_TILE][10];
  const int t0 = blockIdx.x * UV2_T * UVD_PPT + threadIdx.x;
  const int q_lo = blockIdx.y * chunk, q_hi = min(n, q_lo + chunk);
  double pos[UVD_PPT][3], v[UVD_PPT][3];
#pragma unroll
  for (int i = 0; i < UVD_PPT; ++i) {
    const int t = t0 + i * UV2_T;
    for (int c = 0; c < 3; ++c) {
      pos[i][c] = t < npts ? pts[3 * (size_t)t + c] : 0.0;
      v[i][c] = 0.0;
    }
  }
  for (int q0 = q_lo; q0 < q_hi; q0 += UV2_TILE) {
    __syncthreads();
    const int q = q0 + threadIdx.x;
    const int m = min(UV2_TILE, q_hi - q0);
    if (threadIdx.x < m) {
      const double mg = mag[q], r = rv[q];
      double *w = s_q[threadIdx.x];
      const double x = cen[3 * (size_t)q], y = cen[3 * (size_t)q + 1], z = cen[3 * (size_t)q + 2];
      const double ax = mg * dir[3 * (size_t)q], ay = mg * dir[3 * (size_t)q + 1],
                   az = mg * dir[3 * (size_t)q + 2];
      w[0] = x, w[1] = y, w[2] = z, w[3] = r * r;
      w[4] = ax, w[5] = ay, w[6] = az;
      w[7] = y * az - z * ay, w[8] = z * ax - x * az, w[9] = x * ay - y * ax;
    }
    __syncthreads();
    double A[UVD_PPT][3], W[UVD_PPT][3];
#pragma unroll
    for (int i = 0; i < UVD_PPT; ++i)
      for (int c = 0; c < 3; ++c) A[i][c] = W[i][c] = 0.0;
#pragma unroll 2
    for (int u = 0; u < m; ++u) {
      const double2 *w = (const double2 *)s_q[u];
      const double2 X = w[0], Y = w[1], Z = w[2], P = w[3], Q = w[4];
      // X = (x, y), Y = (z, r_v^2), Z = (ax, ay), P = (az, wx), Q = (wy, wz)
#pragma unroll
      for (int i = 0; i < UVD_PPT; ++i) {
        const double dx = pos[i][0] - X.x, dy = pos[i][1] - X.y, dz = pos[i][2] - Y.x;
        const double r2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, Y.y)));
        const double ir = rsqrt_hh(r2);
        const double c = ir * ir * ir;
        A[i][0] = fma(c, Z.x, A[i][0]);
        A[i][1] = fma(c, Z.y, A[i][1]);
        A[i][2] = fma(c, P.x, A[i][2]);
        W[i][0] = fma(c, P.y, W[i][0]);
        W[i][1] = fma(c, Q.x, W[i][1]);
        W[i][2] = fma(c, Q.y, W[i][2]);
      }
    }
    // velocity kernel coefficient is -1/rho^3
#pragma unroll
    for (int i = 0; i < UVD_PPT; ++i) {
      v[i][0] -= pos[i][1] * A[i][2] - pos[i][2] * A[i][1] - W[i][0];
      v[i][1] -= pos[i][2] * A[i][0] - pos[i][0] * A[i][2] - W[i][1];
      v[i][2] -= pos[i][0] * A[i][1] - pos[i][1] * A[i][0] - W[i][2];
    }
  }
  const double k4pi = 1.0 / (4.0 * DUST_PI);
#pragma unroll
  for (int i = 0; i < UVD_PPT; ++i) {
    const int t = t0 + i * UV2_T;
    if (t < npts)
      for (int c = 0; c < 3; ++c) atomicAdd(uv + 3 * (size_t)t + c, v[i][c] * k4pi);
  }
}

// FP64 uvort fused with the particles' term of the pressure equation
// (assemble_pressure_sys, src/linsys/mod_pressure_equation.f90:170-186):
// both sums run over the same (point, particle) pairs and share the
// difference, rho^2 and rho^-3, so the pressure term adds four FMAs per pair
// to k_uvort's nineteen FP64 operations instead of a second pass over the
// particles.  pt[i] = sum_q (x_q - p_i) . (dir_q x vel_q) mag_q rho^-3.
__global__ void __launch_bounds__(UV2_T) k_uvort_pres(int npts, const double *pts, int n,
                                                      const double *cen, const double *dir,
                                                      const double *mag, const double *rv,
                                                      const double *vel, int chunk, double *uv,
                                                      double *pt) {
  __shared__ __align__(16) double s_q[UV2_TILE][14];
  const int t0 = blockIdx.x * UV2_T * UVD_PPT + threadIdx.x;
  const int q_lo = blockIdx.y * chunk, q_hi = min(n, q_lo + chunk);
  double pos[UVD_PPT][3], v[UVD_PPT][3], pr[UVD_PPT];
#pragma unroll
  for (int i = 0; i < UVD_PPT; ++i) {
    const int t = t0 + i * UV2_T;
    for (int c = 0; c < 3; ++c) {
      pos[i][c] = t < npts ? pts[3 * (size_t)t + c] : 0.0;
      v[i][c] = 0.0;
    }
    pr[i] = 0.0;
  }
  for (int q0 = q_lo; q0 < q_hi; q0 += UV2_TILE) {
    __syncthreads();
    const int q = q0 + threadIdx.x;
    const int m = min(UV2_TILE, q_hi - q0);
    if (threadIdx.x < m) {
      const double mg = mag[q], r = rv[q];
      double *w = s_q[threadIdx.x];
      const double x = cen[3 * (size_t)q], y = cen[3 * (size_t)q + 1], z = cen[3 * (size_t)q + 2];
      const double dx_ = dir[3 * (size_t)q], dy_ = dir[3 * (size_t)q + 1],
                   dz_ = dir[3 * (size_t)q + 2];
      const double ax = mg * dx_, ay = mg * dy_, az = mg * dz_;
      const double vx = vel[3 * (size_t)q], vy = vel[3 * (size_t)q + 1],
                   vz = vel[3 * (size_t)q + 2];
      w[0] = x, w[1] = y, w[2] = z, w[3] = r * r;
      w[4] = ax, w[5] = ay, w[6] = az;
      w[7] = y * az - z * ay, w[8] = z * ax - x * az, w[9] = x * ay - y * ax;
      // -(mag dir x vel): the pair term is (p - x_q) . (-w)
      w[10] = -mg * (dy_ * vz - dz_ * vy);
      w[11] = -mg * (dz_ * vx - dx_ * vz);
      w[12] = -mg * (dx_ * vy - dy_ * vx);
      w[13] = 0.0;
    }
    __syncthreads();
    double A[UVD_PPT][3], W[UVD_PPT][3], Pq[UVD_PPT];
#pragma unroll
    for (int i = 0; i < UVD_PPT; ++i) {
      for (int c = 0; c < 3; ++c) A[i][c] = W[i][c] = 0.0;
      Pq[i] = 0.0;
    }
#pragma unroll 2
    for (int u = 0; u < m; ++u) {
      const double2 *w = (const double2 *)s_q[u];
      const double2 X = w[0], Y = w[1], Z = w[2], P = w[3], Q = w[4], R = w[5], S = w[6];
      // X = (x, y), Y = (z, r_v^2), Z = (ax, ay), P = (az, wx), Q = (wy, wz),
      // R = (-ux, -uy), S = (-uz, 0), u = mag dir x vel
#pragma unroll
      for (int i = 0; i < UVD_PPT; ++i) {
        const double dx = pos[i][0] - X.x, dy = pos[i][1] - X.y, dz = pos[i][2] - Y.x;
        const double r2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, Y.y)));
        const double ir = rsqrt_hh(r2);
        const double c = ir * ir * ir;
        A[i][0] = fma(c, Z.x, A[i][0]);
        A[i][1] = fma(c, Z.y, A[i][1]);
        A[i][2] = fma(c, P.x, A[i][2]);
        W[i][0] = fma(c, P.y, W[i][0]);
        W[i][1] = fma(c, Q.x, W[i][1]);
        W[i][2] = fma(c, Q.y, W[i][2]);
        Pq[i] = fma(c, fma(dx, R.x, fma(dy, R.y, dz * S.x)), Pq[i]);
      }
    }
#pragma unroll
    for (int i = 0; i < UVD_PPT; ++i) {
      v[i][0] -= pos[i][1] * A[i][2] - pos[i][2] * A[i][1] - W[i][0];
      v[i][1] -= pos[i][2] * A[i][0] - pos[i][0] * A[i][2] - W[i][1];
      v[i][2] -= pos[i][0] * A[i][1] - pos[i][1] * A[i][0] - W[i][2];
      pr[i] += Pq[i];
    }
  }
  const double k4pi = 1.0 / (4.0 * DUST_PI);
#pragma unroll
  for (int i = 0; i < UVD_PPT; ++i) {
    const int t = t0 + i * UV2_T;
    if (t < npts) {
      for (int c = 0; c < 3; ++c) atomicAdd(uv + 3 * (size_t)t + c, v[i][c] * k4pi);
      atomicAdd(pt + t, pr[i]);
    }
  }
}

// FP32C uvort on particles sorted along a Morton curve: a tile of 128
// consecutive particles is spatially compact, so coordinates relative to the
// tile's first particle are small and are rounded to FP32 once per tile.
__global__ void k_uv_keys(int n, const double *cen, double x0, double y0, double z0,
                          double inv_h, uint32_t *keys, uint32_t *vals) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  double c[3] = {cen[3 * (size_t)q] - x0, cen[3 * (size_t)q + 1] - y0, cen[3 * (size_t)q + 2] - z0};
  uint32_t k[3];
  for (int d = 0; d < 3; ++d) {
    double v = c[d] * inv_h;
    k[d] = v <= 0.0 ? 0u : (v >= 1023.0 ? 1023u : (uint32_t)v);
  }
  keys[q] = spread3(k[0]) | (spread3(k[1]) << 1) | (spread3(k[2]) << 2);
  vals[q] = (uint32_t)q;
}

// sorted block: x y z (double), ax ay az s2 (float)
__global__ void k_uv_gather(int n, const uint32_t *perm, const double *cen, const double *dir,
                            const double *mag, const double *rv, double *X, float *F) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  uint32_t q = perm[t];
  double m = mag[q];
  for (int d = 0; d < 3; ++d) {
    X[(size_t)d * n + t] = cen[3 * (size_t)q + d];
    F[(size_t)d * n + t] = (float)(m * dir[3 * (size_t)q + d]);
  }
  F[(size_t)3 * n + t] = (float)(rv[q] * rv[q]);
}

// UV2_PPT points per thread (consecutive CTA slices of UV2_T points)
#ifndef UV2_PPT
#define UV2_PPT 4
#endif
__global__ void __launch_bounds__(UV2_T) k_uvort_sorted(int npts, const double *pts, int n,
                                                        const double *X, const float *F,
                                                        int chunk, double *uv) {
  // one tile of particles per pass, coordinates relative to the tile's first
  // particle (rounded to FP32 once), d = p - x_q and the cross product
  // d x alpha_q formed per pair, so a point close to a particle loses
  // nothing to cancellation.  Pairs of particles (q, q+1) are evaluated
  // together in packed FP32 (f32x2): their ten values (-x, -y, -z, core^2,
  // alpha, -alpha) are stored interleaved, value k of particle q at
  // [q / 2][2 k + q % 2].  Partial sums over the tile in FP32, added into
  // FP64 per tile.
  __shared__ __align__(16) float s_pk[UV2_TILE / 2][20];
  __shared__ double s_ref[3];
  int t[UV2_PPT];
  double pos[UV2_PPT][3], v[UV2_PPT][3];
#pragma unroll
  for (int i = 0; i < UV2_PPT; ++i) {
    t[i] = (blockIdx.x * UV2_PPT + i) * UV2_T + threadIdx.x;
    for (int c = 0; c < 3; ++c) {
      pos[i][c] = t[i] < npts ? pts[3 * (size_t)t[i] + c] : 0.0;
      v[i][c] = 0.0;
    }
  }
  const int q_lo = blockIdx.y * chunk, q_hi = min(n, q_lo + chunk);
  for (int q0 = q_lo; q0 < q_hi; q0 += UV2_TILE) {
    __syncthreads();
    const int q = q0 + threadIdx.x;
    const int m = min(UV2_TILE, q_hi - q0);
    if (threadIdx.x < 3) s_ref[threadIdx.x] = X[(size_t)threadIdx.x * n + q0];
    __syncthreads();
    if (threadIdx.x < UV2_TILE) {
      // particles beyond the chunk: far away (1e6), no strength
      float val[10] = {-1.0e6f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      if (threadIdx.x < m) {
        const float ax = F[q], ay = F[(size_t)n + q], az = F[2 * (size_t)n + q];
        val[0] = (float)(s_ref[0] - X[q]);
        val[1] = (float)(s_ref[1] - X[(size_t)n + q]);
        val[2] = (float)(s_ref[2] - X[2 * (size_t)n + q]);
        val[3] = F[(size_t)3 * n + q];
        val[4] = ax, val[5] = ay, val[6] = az;
        val[7] = -ax, val[8] = -ay, val[9] = -az;
      }
      for (int k = 0; k < 10; ++k) s_pk[threadIdx.x >> 1][2 * k + (threadIdx.x & 1)] = val[k];
    }
    __syncthreads();
    float px[UV2_PPT], py[UV2_PPT], pz[UV2_PPT];
    float2 V[UV2_PPT][3];
#pragma unroll
    for (int i = 0; i < UV2_PPT; ++i) {
      px[i] = (float)(pos[i][0] - s_ref[0]);
      py[i] = (float)(pos[i][1] - s_ref[1]);
      pz[i] = (float)(pos[i][2] - s_ref[2]);
      for (int c = 0; c < 3; ++c) V[i][c] = make_float2(0.f, 0.f);
    }
    const int mp = (m + 1) >> 1;
#pragma unroll 2
    for (int u = 0; u < mp; ++u) {
      const float4 P0 = *(const float4 *)&s_pk[u][0], P1 = *(const float4 *)&s_pk[u][4],
                   P2 = *(const float4 *)&s_pk[u][8], P3 = *(const float4 *)&s_pk[u][12],
                   P4 = *(const float4 *)&s_pk[u][16];
      const float2 nx = make_float2(P0.x, P0.y), ny = make_float2(P0.z, P0.w),
                   nz = make_float2(P1.x, P1.y), s2 = make_float2(P1.z, P1.w),
                   ax = make_float2(P2.x, P2.y), ay = make_float2(P2.z, P2.w),
                   az = make_float2(P3.x, P3.y), mx = make_float2(P3.z, P3.w),
                   my = make_float2(P4.x, P4.y), mz = make_float2(P4.z, P4.w);
#pragma unroll
      for (int i = 0; i < UV2_PPT; ++i) {
        const float2 dx = __fadd2_rn(make_float2(px[i], px[i]), nx),
                     dy = __fadd2_rn(make_float2(py[i], py[i]), ny),
                     dz = __fadd2_rn(make_float2(pz[i], pz[i]), nz);
        const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, s2)));
        const float2 ir = make_float2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
        const float2 c = __fmul2_rn(__fmul2_rn(ir, ir), ir);
        const float2 cx = __fmul2_rn(c, dx), cy = __fmul2_rn(c, dy), cz = __fmul2_rn(c, dz);
        // c (d x alpha)
        V[i][0] = __ffma2_rn(cy, az, __ffma2_rn(cz, my, V[i][0]));
        V[i][1] = __ffma2_rn(cz, ax, __ffma2_rn(cx, mz, V[i][1]));
        V[i][2] = __ffma2_rn(cx, ay, __ffma2_rn(cy, mx, V[i][2]));
      }
    }
    // velocity kernel coefficient is -1/rho^3
#pragma unroll
    for (int i = 0; i < UV2_PPT; ++i)
      for (int c = 0; c < 3; ++c) v[i][c] -= (double)(V[i][c].x + V[i][c].y);
  }
  const double k4pi = 1.0 / (4.0 * DUST_PI);
#pragma unroll
  for (int i = 0; i < UV2_PPT; ++i)
    if (t[i] < npts)
      for (int c = 0; c < 3; ++c) atomicAdd(uv + 3 * (size_t)t[i] + c, v[i][c] * k4pi);
}

// sorted block of the fused pass: x y z (double); ax ay az s2 -wx -wy -wz
// (float) with w = mag (dir x vel) formed in FP64 and rounded once
__global__ void k_uvp_gather(int n, const uint32_t *perm, const double *cen, const double *dir,
                             const double *mag, const double *rv, const double *vel, double *X,
                             float *F) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  uint32_t q = perm[t];
  const double m = mag[q];
  const double dx = dir[3 * (size_t)q], dy = dir[3 * (size_t)q + 1], dz = dir[3 * (size_t)q + 2];
  const double vx = vel[3 * (size_t)q], vy = vel[3 * (size_t)q + 1], vz = vel[3 * (size_t)q + 2];
  for (int d = 0; d < 3; ++d) X[(size_t)d * n + t] = cen[3 * (size_t)q + d];
  F[t] = (float)(m * dx);
  F[(size_t)n + t] = (float)(m * dy);
  F[2 * (size_t)n + t] = (float)(m * dz);
  F[3 * (size_t)n + t] = (float)(rv[q] * rv[q]);
  F[4 * (size_t)n + t] = (float)(-m * (dy * vz - dz * vy));
  F[5 * (size_t)n + t] = (float)(-m * (dz * vx - dx * vz));
  F[6 * (size_t)n + t] = (float)(-m * (dx * vy - dy * vx));
}

// k_uvort_sorted with the pressure equation's particle term at the same
// points in the same pass (the FP32C counterpart of k_uvort_pres): per pair
// the difference, rho^-3 and the cross product of uvort, and d . (-w) rho^-3
// for the pressure term; 13 values per particle, interleaved in pairs
// as in k_uvort_sorted (value k of particle q at [q / 2][2 k + q % 2]).
__global__ void __launch_bounds__(UV2_T) k_uvort_pres_sorted(int npts, const double *pts, int n,
                                                             const double *X, const float *F,
                                                             int chunk, double *uv, double *pt) {
  __shared__ __align__(16) float s_pk[UV2_TILE / 2][28];
  __shared__ double s_ref[3];
  int t[UV2_PPT];
  double pos[UV2_PPT][3], v[UV2_PPT][3], pr[UV2_PPT];
#pragma unroll
  for (int i = 0; i < UV2_PPT; ++i) {
    t[i] = (blockIdx.x * UV2_PPT + i) * UV2_T + threadIdx.x;
    for (int c = 0; c < 3; ++c) {
      pos[i][c] = t[i] < npts ? pts[3 * (size_t)t[i] + c] : 0.0;
      v[i][c] = 0.0;
    }
    pr[i] = 0.0;
  }
  const int q_lo = blockIdx.y * chunk, q_hi = min(n, q_lo + chunk);
  for (int q0 = q_lo; q0 < q_hi; q0 += UV2_TILE) {
    __syncthreads();
    const int q = q0 + threadIdx.x;
    const int m = min(UV2_TILE, q_hi - q0);
    if (threadIdx.x < 3) s_ref[threadIdx.x] = X[(size_t)threadIdx.x * n + q0];
    __syncthreads();
    if (threadIdx.x < UV2_TILE) {
      // particles beyond the chunk: far away (1e6), no strength
      float val[14] = {-1.0e6f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      if (threadIdx.x < m) {
        const float ax = F[q], ay = F[(size_t)n + q], az = F[2 * (size_t)n + q];
        val[0] = (float)(s_ref[0] - X[q]);
        val[1] = (float)(s_ref[1] - X[(size_t)n + q]);
        val[2] = (float)(s_ref[2] - X[2 * (size_t)n + q]);
        val[3] = F[(size_t)3 * n + q];
        val[4] = ax, val[5] = ay, val[6] = az;
        val[7] = -ax, val[8] = -ay, val[9] = -az;
        val[10] = F[(size_t)4 * n + q];
        val[11] = F[(size_t)5 * n + q];
        val[12] = F[(size_t)6 * n + q];
      }
      for (int k = 0; k < 14; ++k) s_pk[threadIdx.x >> 1][2 * k + (threadIdx.x & 1)] = val[k];
    }
    __syncthreads();
    float px[UV2_PPT], py[UV2_PPT], pz[UV2_PPT];
    float2 V[UV2_PPT][3], W[UV2_PPT];
#pragma unroll
    for (int i = 0; i < UV2_PPT; ++i) {
      px[i] = (float)(pos[i][0] - s_ref[0]);
      py[i] = (float)(pos[i][1] - s_ref[1]);
      pz[i] = (float)(pos[i][2] - s_ref[2]);
      for (int c = 0; c < 3; ++c) V[i][c] = make_float2(0.f, 0.f);
      W[i] = make_float2(0.f, 0.f);
    }
    const int mp = (m + 1) >> 1;
#pragma unroll 2
    for (int u = 0; u < mp; ++u) {
      const float4 P0 = *(const float4 *)&s_pk[u][0], P1 = *(const float4 *)&s_pk[u][4],
                   P2 = *(const float4 *)&s_pk[u][8], P3 = *(const float4 *)&s_pk[u][12],
                   P4 = *(const float4 *)&s_pk[u][16], P5 = *(const float4 *)&s_pk[u][20],
                   P6 = *(const float4 *)&s_pk[u][24];
      const float2 nx = make_float2(P0.x, P0.y), ny = make_float2(P0.z, P0.w),
                   nz = make_float2(P1.x, P1.y), s2 = make_float2(P1.z, P1.w),
                   ax = make_float2(P2.x, P2.y), ay = make_float2(P2.z, P2.w),
                   az = make_float2(P3.x, P3.y), mx = make_float2(P3.z, P3.w),
                   my = make_float2(P4.x, P4.y), mz = make_float2(P4.z, P4.w),
                   wx = make_float2(P5.x, P5.y), wy = make_float2(P5.z, P5.w),
                   wz = make_float2(P6.x, P6.y);
#pragma unroll
      for (int i = 0; i < UV2_PPT; ++i) {
        const float2 dx = __fadd2_rn(make_float2(px[i], px[i]), nx),
                     dy = __fadd2_rn(make_float2(py[i], py[i]), ny),
                     dz = __fadd2_rn(make_float2(pz[i], pz[i]), nz);
        const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, s2)));
        const float2 ir = make_float2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
        const float2 c = __fmul2_rn(__fmul2_rn(ir, ir), ir);
        const float2 cx = __fmul2_rn(c, dx), cy = __fmul2_rn(c, dy), cz = __fmul2_rn(c, dz);
        // c (d x alpha)
        V[i][0] = __ffma2_rn(cy, az, __ffma2_rn(cz, my, V[i][0]));
        V[i][1] = __ffma2_rn(cz, ax, __ffma2_rn(cx, mz, V[i][1]));
        V[i][2] = __ffma2_rn(cx, ay, __ffma2_rn(cy, mx, V[i][2]));
        // c d . (-w): the pair term (x_q - p) . w rho^-3
        W[i] = __ffma2_rn(cx, wx, __ffma2_rn(cy, wy, __ffma2_rn(cz, wz, W[i])));
      }
    }
#pragma unroll
    for (int i = 0; i < UV2_PPT; ++i) {
      // velocity kernel coefficient is -1/rho^3
      for (int c = 0; c < 3; ++c) v[i][c] -= (double)(V[i][c].x + V[i][c].y);
      pr[i] += (double)(W[i].x + W[i].y);
    }
  }
  const double k4pi = 1.0 / (4.0 * DUST_PI);
#pragma unroll
  for (int i = 0; i < UV2_PPT; ++i)
    if (t[i] < npts) {
      for (int c = 0; c < 3; ++c) atomicAdd(uv + 3 * (size_t)t[i] + c, v[i][c] * k4pi);
      atomicAdd(pt + t[i], pr[i]);
    }
}

__global__ void k_uvort_lines(int npts, const double *pts, ElemDev e, double *uv) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts) return;
  double pos[3] = {pts[3 * (size_t)t], pts[3 * (size_t)t + 1], pts[3 * (size_t)t + 2]};
  double v[3] = {0, 0, 0};
  for (int q = 0; q < e.nline; ++q) {
    double u[3];
    vel_line(e.rp, e.lines[q], pos, u);
    for (int c = 0; c < 3; ++c) v[c] += u[c];
  }
  const double k4pi = 1.0 / (4.0 * DUST_PI);
  for (int c = 0; c < 3; ++c) atomicAdd(uv + 3 * (size_t)t + c, v[c] * k4pi);
}

void points_lines_add(int npts, const double *pts, const ElemDev &lines, double *uv,
                      cudaStream_t st) {
  if (npts > 0 && lines.nline > 0)
    k_uvort_lines<<<nblk(npts, 128), 128, 0, st>>>(npts, pts, lines, uv);
}

// Morton order of n particles over the octree box of prm (keys of 10 bits
// per axis): *perm (in scratch, from offset 0) receives the particle index
// of every sorted position; *used the scratch bytes taken.
size_t morton_perm_bytes(int n, cudaStream_t st) {
  const size_t N = (size_t)std::max(n, 1);
  size_t tb = 0;
  uint32_t *dummy = nullptr;
  cub::DeviceRadixSort::SortPairs(nullptr, tb, dummy, dummy, dummy, dummy, n, 0, 30, st);
  return (16 * N + 255) / 256 * 256 + (tb + 255) / 256 * 256;
}

int morton_perm(const dust_fmm_params *prm, int n, const double *cen, DevBuf &scratch,
                uint32_t **perm, size_t *used, cudaStream_t st) {
  const size_t N = (size_t)std::max(n, 1);
  size_t tb = 0;
  uint32_t *dummy = nullptr;
  cub::DeviceRadixSort::SortPairs(nullptr, tb, dummy, dummy, dummy, dummy, n, 0, 30, st);
  const size_t off_t = (16 * N + 255) / 256 * 256;
  DUST_TRY(devbuf_grow(scratch, off_t + tb + 256));
  char *b = (char *)scratch.p;
  uint32_t *k_in = (uint32_t *)b, *v_in = k_in + N, *k_out = v_in + N, *v_out = k_out + N;
  const double hbox =
      prm->box_length * std::max(prm->n_box[0], std::max(prm->n_box[1], prm->n_box[2]));
  if (n > 0) {
    k_uv_keys<<<nblk(n, 256), 256, 0, st>>>(n, cen, prm->origin[0], prm->origin[1],
                                             prm->origin[2], 1024.0 / hbox, k_in, v_in);
    DUST_CUDA(cub::DeviceRadixSort::SortPairs(b + off_t, tb, k_in, k_out, v_in, v_out, n, 0, 30,
                                              st));
  }
  *perm = v_out;
  *used = off_t + (tb + 255) / 256 * 256;
  return DUST_OK;
}

int points_uvort_run(const dust_fmm_params *prm, int n_pts, const double *pts, int n,
                     const double *cen, const double *dir, const double *mag, const double *rv,
                     const ElemDev &lines, DevBuf &scratch, double *uv, cudaStream_t st) {
  if (n_pts <= 0) return DUST_OK;
  DUST_CUDA(cudaMemsetAsync(uv, 0, (size_t)n_pts * 24, st));
  if (n > 0) {
    // point blocks: UV2_T points (UV2_T * UV2_PPT for the sorted FP32 kernel)
    const bool srt = prm->precision == DUST_PREC_FP32C;
    int pb = (int)nblk(n_pts, UV2_T * (srt ? UV2_PPT : UVD_PPT));
    // enough CTAs for every SM several times over; chunks of whole tiles
    int want = std::max(1, (148 * 8 + pb - 1) / pb);
    int chunk = (n + want - 1) / want;
    chunk = std::max(UV2_TILE, (chunk + UV2_TILE - 1) / UV2_TILE * UV2_TILE);
    int nch = (n + chunk - 1) / chunk;
    dim3 grd(pb, nch);
    if (prm->precision == DUST_PREC_FP32C) {
      // Morton-sort the particles over the octree box (order only matters
      // for accuracy of the tile-relative FP32 coordinates)
      size_t N = (size_t)n;
      size_t tb = 0;
      uint32_t *dummy = nullptr;
      cub::DeviceRadixSort::SortPairs(nullptr, tb, dummy, dummy, dummy, dummy, n, 0, 30, st);
      size_t off_f = (16 * N + 255) / 256 * 256;
      size_t off_x = off_f + (16 * N + 255) / 256 * 256;
      size_t off_t = off_x + (24 * N + 255) / 256 * 256;
      DUST_TRY(devbuf_grow(scratch, off_t + tb + 256));
      char *b = (char *)scratch.p;
      uint32_t *k_in = (uint32_t *)b, *v_in = k_in + N, *k_out = v_in + N, *v_out = k_out + N;
      float *F = (float *)(b + off_f);
      double *X = (double *)(b + off_x);
      double hbox = prm->box_length * std::max(prm->n_box[0], std::max(prm->n_box[1], prm->n_box[2]));
      k_uv_keys<<<nblk(n, 256), 256, 0, st>>>(n, cen, prm->origin[0], prm->origin[1],
                                               prm->origin[2], 1024.0 / hbox, k_in, v_in);
      DUST_CUDA(cub::DeviceRadixSort::SortPairs(b + off_t, tb, k_in, k_out, v_in, v_out, n, 0, 30,
                                                st));
      k_uv_gather<<<nblk(n, 256), 256, 0, st>>>(n, v_out, cen, dir, mag, rv, X, F);
      k_uvort_sorted<<<grd, UV2_T, 0, st>>>(n_pts, pts, n, X, F, chunk, uv);
    } else {
      k_uvort<<<grd, UV2_T, 0, st>>>(n_pts, pts, n, cen, dir, mag, rv, chunk, uv);
    }
  }
  if (lines.nline > 0) k_uvort_lines<<<nblk(n_pts, 128), 128, 0, st>>>(n_pts, pts, lines, uv);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}

// ------------------------------------------------- uvort without allocation
// dust_points_uvort_device_noalloc: the same sums as dust_points_uvort_device
// (same kernels, same order of operations) for callers that must not
// allocate device memory during a step.  Its only scratch (end-vortex
// geometry, and in the FP32C mode the Morton keys, the sorted particle copy
// and the radix-sort work space) lives in the fixed array below, reserved
// when the library is loaded.
static __device__ __align__(256) unsigned char g_uv_noalloc[DUST_UVORT_NOALLOC_SCRATCH];

__global__ void k_line_build(int n, const double *ver, const double *mag, LineGeo *out);

static inline size_t round256(size_t b) { return (b + 255) / 256 * 256; }

extern "C" int dust_points_uvort_device_noalloc(const dust_fmm_params *prm, int n_pts,
                                                const double *pts, int n, const double *cen,
                                                const double *dir, const double *mag,
                                                const double *r_vortex,
                                                const dust_lines *end_vort, double *uvort,
                                                void *stream) {
  if (!uvort_args_ok(prm, n_pts, pts, n, cen, dir, mag, r_vortex, end_vort, uvort))
    return DUST_ERR_BAD_ARG;
  if (n_pts == 0) return DUST_OK;
  const int nl = end_vort ? end_vort->n : 0;
  const bool f32 = prm->precision == DUST_PREC_FP32C && n > 0;
  const size_t N = (size_t)n;
  // scratch layout: [LineGeo x nl][keys/vals 16N][F 16N][X 24N][sort work]
  const size_t off_p = round256(sizeof(LineGeo) * (size_t)nl);
  const size_t off_f = off_p + (f32 ? round256(16 * N) : 0);
  const size_t off_x = off_f + (f32 ? round256(16 * N) : 0);
  const size_t off_t = off_x + (f32 ? round256(24 * N) : 0);
  char msg[160];
  if (off_t > DUST_UVORT_NOALLOC_SCRATCH) {
    snprintf(msg, sizeof(msg), "uvort no-alloc scratch: %zu bytes needed, %u available", off_t,
             (unsigned)DUST_UVORT_NOALLOC_SCRATCH);
    dust_set_last_error(msg, __FILE__, __LINE__);
    return DUST_ERR_CAPACITY;
  }
  size_t tb = 0;
  if (f32) {
    uint32_t *dummy = nullptr;
    DUST_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, dummy, dummy, dummy, dummy, n, 0, 30,
                                              (cudaStream_t)stream));
  }
  const size_t need = off_t + round256(tb);
  if (need > DUST_UVORT_NOALLOC_SCRATCH) {
    snprintf(msg, sizeof(msg), "uvort no-alloc scratch: %zu bytes needed, %u available", need,
             (unsigned)DUST_UVORT_NOALLOC_SCRATCH);
    dust_set_last_error(msg, __FILE__, __LINE__);
    return DUST_ERR_CAPACITY;
  }
  // the array's device address in the current device's context, looked up on
  // every call (nothing cached: a context reset reloads the module)
  void *sym = nullptr;
  DUST_CUDA(cudaGetSymbolAddress(&sym, g_uv_noalloc));
  char *b = (char *)sym;
  cudaStream_t st = (cudaStream_t)stream;
  ElemDev e;
  memset(&e, 0, sizeof(e));
  e.rp = reg_params(prm);
  e.nline = nl;
  e.lines = (const LineGeo *)b;
  if (nl > 0) k_line_build<<<nblk(nl, 128), 128, 0, st>>>(nl, end_vort->ver, end_vort->mag,
                                                          (LineGeo *)b);
  DUST_CUDA(cudaMemsetAsync(uvort, 0, (size_t)n_pts * 24, st));
  if (n > 0) {
    int pb = (int)nblk(n_pts, UV2_T * (f32 ? UV2_PPT : UVD_PPT));
    int want = std::max(1, (148 * 8 + pb - 1) / pb);
    int chunk = (n + want - 1) / want;
    chunk = std::max(UV2_TILE, (chunk + UV2_TILE - 1) / UV2_TILE * UV2_TILE);
    int nch = (n + chunk - 1) / chunk;
    dim3 grd(pb, nch);
    if (f32) {
      uint32_t *k_in = (uint32_t *)(b + off_p), *v_in = k_in + N, *k_out = v_in + N,
               *v_out = k_out + N;
      float *F = (float *)(b + off_f);
      double *X = (double *)(b + off_x);
      double hbox =
          prm->box_length * std::max(prm->n_box[0], std::max(prm->n_box[1], prm->n_box[2]));
      k_uv_keys<<<nblk(n, 256), 256, 0, st>>>(n, cen, prm->origin[0], prm->origin[1],
                                               prm->origin[2], 1024.0 / hbox, k_in, v_in);
      DUST_CUDA(cub::DeviceRadixSort::SortPairs(b + off_t, tb, k_in, k_out, v_in, v_out, n, 0, 30,
                                                st));
      k_uv_gather<<<nblk(n, 256), 256, 0, st>>>(n, v_out, cen, dir, mag, r_vortex, X, F);
      k_uvort_sorted<<<grd, UV2_T, 0, st>>>(n_pts, pts, n, X, F, chunk, uvort);
    } else {
      k_uvort<<<grd, UV2_T, 0, st>>>(n_pts, pts, n, cen, dir, mag, r_vortex, chunk, uvort);
    }
  }
  if (nl > 0) k_uvort_lines<<<nblk(n_pts, 128), 128, 0, st>>>(n_pts, pts, e, uvort);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}

// ------------------------------------- uvort with the pressure particle term
// dust_points_uvort_pressure_device: the uvort sum of
// dust_points_uvort_device and the pressure equation's particle term in one
// pass, FP64 (k_uvort_pres) or FP32C on Morton-sorted particles
// (k_uvort_pres_sorted); the end vortices go to uvort as before.
// end-vortex records and the FP32C pass's sorted particles (one host thread)
static DevBuf g_uvp_raw, g_uvp_geo, g_uvp_sort;

// the fused pass on device arrays, end vortices already built into e
static int uvort_pressure_run(const dust_fmm_params *prm, int n_pts, const double *pts, int n,
                              const double *cen, const double *dir, const double *mag,
                              const double *r_vortex, const double *vel, const ElemDev &e,
                              double *uvort, double *pterm, cudaStream_t st) {
  DUST_CUDA(cudaMemsetAsync(uvort, 0, (size_t)n_pts * 24, st));
  DUST_CUDA(cudaMemsetAsync(pterm, 0, (size_t)n_pts * 8, st));
  if (n > 0 && prm->precision == DUST_PREC_FP32C) {
    // particles along a Morton curve, then the packed FP32 fused pass
    const size_t N = (size_t)n;
    size_t tb = 0;
    uint32_t *dummy = nullptr;
    DUST_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, dummy, dummy, dummy, dummy, n, 0, 30,
                                              st));
    const size_t off_f = round256(16 * N), off_x = off_f + round256(28 * N),
                 off_t = off_x + round256(24 * N);
    DUST_TRY(devbuf_grow(g_uvp_sort, off_t + round256(tb)));
    char *b = (char *)g_uvp_sort.p;
    uint32_t *k_in = (uint32_t *)b, *v_in = k_in + N, *k_out = v_in + N, *v_out = k_out + N;
    float *F = (float *)(b + off_f);
    double *X = (double *)(b + off_x);
    const double hbox =
        prm->box_length * std::max(prm->n_box[0], std::max(prm->n_box[1], prm->n_box[2]));
    k_uv_keys<<<nblk(n, 256), 256, 0, st>>>(n, cen, prm->origin[0], prm->origin[1],
                                             prm->origin[2], 1024.0 / hbox, k_in, v_in);
    DUST_CUDA(cub::DeviceRadixSort::SortPairs(b + off_t, tb, k_in, k_out, v_in, v_out, n, 0, 30,
                                              st));
    k_uvp_gather<<<nblk(n, 256), 256, 0, st>>>(n, v_out, cen, dir, mag, r_vortex, vel, X, F);
    const int pb = (int)nblk(n_pts, UV2_T * UV2_PPT);
    const int want = std::max(1, (148 * 8 + pb - 1) / pb);
    int chunk = (n + want - 1) / want;
    chunk = std::max(UV2_TILE, (chunk + UV2_TILE - 1) / UV2_TILE * UV2_TILE);
    const int nch = (n + chunk - 1) / chunk;
    k_uvort_pres_sorted<<<dim3(pb, nch), UV2_T, 0, st>>>(n_pts, pts, n, X, F, chunk, uvort,
                                                         pterm);
  } else if (n > 0) {
    const int pb = (int)nblk(n_pts, UV2_T * UVD_PPT);
    const int want = std::max(1, (148 * 8 + pb - 1) / pb);
    int chunk = (n + want - 1) / want;
    chunk = std::max(UV2_TILE, (chunk + UV2_TILE - 1) / UV2_TILE * UV2_TILE);
    const int nch = (n + chunk - 1) / chunk;
    k_uvort_pres<<<dim3(pb, nch), UV2_T, 0, st>>>(n_pts, pts, n, cen, dir, mag, r_vortex, vel,
                                                  chunk, uvort, pterm);
  }
  points_lines_add(n_pts, pts, e, uvort, st);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}

static bool uvort_pressure_args_ok(const dust_fmm_params *prm, int n_pts, const double *pts,
                                   int n, const double *cen, const double *dir,
                                   const double *mag, const double *r_vortex, const double *vel,
                                   const dust_lines *end_vort, const double *uvort,
                                   const double *pterm) {
  if (!uvort_args_ok(prm, n_pts, pts, n, cen, dir, mag, r_vortex, end_vort, uvort)) return false;
  if (n_pts > 0 && !pterm) return false;
  if (n > 0 && !vel) return false;
  return true;
}

extern "C" int dust_points_uvort_pressure_device(const dust_fmm_params *prm, int n_pts,
                                                 const double *pts, int n, const double *cen,
                                                 const double *dir, const double *mag,
                                                 const double *r_vortex, const double *vel,
                                                 const dust_lines *end_vort, double *uvort,
                                                 double *pterm, void *stream) {
  if (!uvort_pressure_args_ok(prm, n_pts, pts, n, cen, dir, mag, r_vortex, vel, end_vort, uvort,
                              pterm))
    return DUST_ERR_BAD_ARG;
  if (n_pts == 0) return DUST_OK;
  cudaStream_t st = (cudaStream_t)stream;
  ElemDev e;
  DUST_TRY(elem_build_device(nullptr, nullptr, end_vort, prm->u_inf, reg_params(prm), false,
                             g_uvp_raw, g_uvp_geo, e, st));
  return uvort_pressure_run(prm, n_pts, pts, n, cen, dir, mag, r_vortex, vel, e, uvort, pterm,
                            st);
}

// Host arrays: inputs copied to a staging buffer kept across calls (one host
// thread), outputs copied back.
static DevBuf g_uvp_stage;

extern "C" int dust_points_uvort_pressure(const dust_fmm_params *prm, int n_pts,
                                          const double *pts, int n, const double *cen,
                                          const double *dir, const double *mag,
                                          const double *r_vortex, const double *vel,
                                          const dust_lines *end_vort, double *uvort,
                                          double *pterm) {
  if (!uvort_pressure_args_ok(prm, n_pts, pts, n, cen, dir, mag, r_vortex, vel, end_vort, uvort,
                              pterm))
    return DUST_ERR_BAD_ARG;
  if (n_pts == 0) return DUST_OK;
  cudaStream_t st = 0;
  ElemDev e;
  DUST_TRY(elem_build_device(nullptr, nullptr, end_vort, prm->u_inf, reg_params(prm), true,
                             g_uvp_raw, g_uvp_geo, e, st));
  const size_t P = (size_t)n_pts, N = (size_t)n;
  const size_t o_u = round256(24 * P), o_t = o_u + round256(24 * P), o_c = o_t + round256(8 * P);
  const size_t o_d = o_c + round256(24 * N), o_m = o_d + round256(24 * N),
               o_r = o_m + round256(8 * N), o_v = o_r + round256(8 * N),
               end = o_v + round256(24 * N);
  DUST_TRY(devbuf_grow(g_uvp_stage, end));
  char *b = (char *)g_uvp_stage.p;
  double *dp = (double *)b, *du = (double *)(b + o_u), *dt = (double *)(b + o_t);
  double *dc = (double *)(b + o_c), *dd = (double *)(b + o_d), *dm = (double *)(b + o_m),
         *dr = (double *)(b + o_r), *dv = (double *)(b + o_v);
  DUST_CUDA(cudaMemcpyAsync(dp, pts, 24 * P, cudaMemcpyHostToDevice, st));
  if (n > 0) {
    DUST_CUDA(cudaMemcpyAsync(dc, cen, 24 * N, cudaMemcpyHostToDevice, st));
    DUST_CUDA(cudaMemcpyAsync(dd, dir, 24 * N, cudaMemcpyHostToDevice, st));
    DUST_CUDA(cudaMemcpyAsync(dm, mag, 8 * N, cudaMemcpyHostToDevice, st));
    DUST_CUDA(cudaMemcpyAsync(dr, r_vortex, 8 * N, cudaMemcpyHostToDevice, st));
    DUST_CUDA(cudaMemcpyAsync(dv, vel, 24 * N, cudaMemcpyHostToDevice, st));
  }
  DUST_TRY(uvort_pressure_run(prm, n_pts, dp, n, dc, dd, dm, dr, dv, e, du, dt, st));
  DUST_CUDA(cudaMemcpyAsync(uvort, du, 24 * P, cudaMemcpyDeviceToHost, st));
  DUST_CUDA(cudaMemcpyAsync(pterm, dt, 8 * P, cudaMemcpyDeviceToHost, st));
  DUST_CUDA(cudaStreamSynchronize(st));
  return DUST_OK;
}
