// panel_wake.cu -- the panel wake behind the trailing edges and the particles
// it sheds, device resident (the panel part of t_wake,
// src/aeroel/mod_wake.f90:160-296):
//   initialize_wake  :468-512   first two rows of points
//   load_wake        :597-778   state of a result file (restart)
//   update_wake      :884-892   first-row intensities from the solution
//                    :894-939   velocities at the wake points
//                                (compute_vel_from_all, :2109-2150), rows
//                                moved, points_end of a full wake
//                    :1128-1176 length grown, end_pan_idou, intensities
//                                shifted one row back
//   complete_wake    :1247-1292 first two rows from the trailing edge
//                    :1797-2010 shedding (classical and refine_wake)
//                    :2091-2103 end vortices of a full wake
// plus the live-particle list of prepare_wake (:804-846) and the scatter of
// per-live-particle outputs back to the particle slots.
//
// Layout: points pts[row][point][3] (rows 0..n_wake_panels), point
// velocities pvel (same), intensities idou[row][stripe], the wake panels'
// vertices wver[row * n_stripes + stripe][4][3] (the reference's pan_p
// order) rebuilt whenever the rows change, end vortices ever[stripe][2][3].
// The per-stripe work is small (one thread per stripe or point); the wake
// point velocities reuse the element and particle direct-sum kernels.  The
// arithmetic of the bookkeeping and shedding kernels follows the reference's
// expressions in order with explicitly rounded intrinsics (no fused
// multiply-adds), as the CPU restatement evaluates them.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>
#include <vector>

#include "dust_common.cuh"
#include "fmm_internal.h"

static inline unsigned nblk(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

__device__ __forceinline__ double nrm3(double x, double y, double z) {
  return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
}

struct dust_wake {
  dust_wake_params p;
  int len = 1;            // pan_wake_len
  int len_geo = 1;        // rows whose panel geometry is current
  bool full = false;      // full_panels
  bool attached = false;  // end vortices attached (their mag pointers associated)
  std::vector<int> h_ii, h_gen;
  double *pts = nullptr, *pold = nullptr, *pvel = nullptr, *idou = nullptr;
  double *last = nullptr, *endi = nullptr, *pend = nullptr;
  double *wver = nullptr, *ever = nullptr;
  double *qpts = nullptr, *qvel = nullptr, *qtmp = nullptr;  // wake-point velocities
  int *ii = nullptr, *neigh = nullptr, *neigh_o = nullptr, *gen = nullptr;
  int *nver4 = nullptr;
  // shedding work: per stripe sub-particle counts and offsets, candidates
  int *nsub = nullptr, *soff = nullptr, *cand_ok = nullptr, *cand_rank = nullptr;
  double *cand = nullptr;  // per candidate: pos(3), area, partvec(3), n_sub, p1, p2
  int cand_cap = 0;
  DevBuf sel;              // per-stripe shedding records
  DevBuf slots, sel_work, cnt, scan_tmp;  // free-slot list and scan work
  DevBuf geo, raw;         // element records of the update
};

// -------------------------------------------------------------- kernels
// first two rows of points: initialize_wake :484-512 (normalised == 0: the
// unnormalised form below min_vel_at_te) / complete_wake :1258-1282
__global__ void k_wake_te_rows(int npt, double *pts, const double *te_pts, const double *te_dir,
                               const double *te_sc, const double *te_vel, double ux, double uy,
                               double uz, double dt, double nd, double minvel, int normalised) {
  int ip = blockIdx.x * blockDim.x + threadIdx.x;
  if (ip >= npt) return;
  double w0 = ux, w1 = uy, w2 = uz;
  if (te_vel) {
    w0 = __dsub_rn(w0, te_vel[3 * ip]);
    w1 = __dsub_rn(w1, te_vel[3 * ip + 1]);
    w2 = __dsub_rn(w2, te_vel[3 * ip + 2]);
  }
  const double w = nrm3(w0, w1, w2);
  const double *d = te_dir + 3 * ip;
  const double dn = nrm3(d[0], d[1], d[2]);
  const double sc = te_sc[ip];
  for (int c = 0; c < 3; ++c) {
    const double r1 = te_pts[3 * ip + c];
    double a;
    if (w > minvel) {
      a = __ddiv_rn(__dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(d[c], sc), w), dt), nd), dn);
    } else {
      a = __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(d[c], sc), minvel), dt), nd);
      if (normalised) a = __ddiv_rn(a, dn);
    }
    pts[3 * ip + c] = r1;
    pts[3 * ((size_t)npt + ip) + c] = __dadd_rn(r1, a);
  }
}

// panel vertices of rows 0..len-1 (p1, p2 of the row, p2, p1 of the next,
// :1285-1289) and, for a full wake, the end vortices on row len (:2096-2100)
__global__ void k_wake_geo(int ns, int npt, int len, int full, const int *ii, const double *pts,
                           double *wver, double *ever) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (len + 1) * ns) return;
  int r = t / ns, iw = t % ns;
  int p1 = ii[2 * iw] - 1, p2 = ii[2 * iw + 1] - 1;
  if (r < len) {
    double *v = wver + 12 * (size_t)t;
    const double *a = pts + 3 * ((size_t)r * npt + p1), *b = pts + 3 * ((size_t)r * npt + p2);
    const double *c = pts + 3 * ((size_t)(r + 1) * npt + p2);
    const double *d = pts + 3 * ((size_t)(r + 1) * npt + p1);
    for (int k = 0; k < 3; ++k) {
      v[k] = a[k];
      v[3 + k] = b[k];
      v[6 + k] = c[k];
      v[9 + k] = d[k];
    }
  } else if (full) {
    double *e = ever + 6 * (size_t)iw;
    const double *a = pts + 3 * ((size_t)len * npt + p1), *b = pts + 3 * ((size_t)len * npt + p2);
    for (int k = 0; k < 3; ++k) {
      e[k] = a[k];
      e[3 + k] = b[k];
    }
  }
}

// update_wake :884-892
__global__ void k_wake_first_row(int ns, const int *gen, const double *res, double *idou) {
  int iw = blockIdx.x * blockDim.x + threadIdx.x;
  if (iw >= ns) return;
  int g1 = gen[2 * iw], g2 = gen[2 * iw + 1];
  idou[iw] = g2 > 0 ? __dsub_rn(res[g1 - 1], res[g2 - 1]) : res[g1 - 1];
}

// the source rows of the wake-point velocities: rows ipan - 2 for ipan =
// 3..np (1-based), then row len for points_end
__global__ void k_wake_gather_rows(int npt, int r0, int nrows, int extra_row, const double *pts,
                                   double *q) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int nr = nrows + (extra_row >= 0 ? 1 : 0);
  if (t >= nr * npt) return;
  int k = t / npt, ip = t % npt;
  int row = k < nrows ? r0 + k : extra_row;
  for (int c = 0; c < 3; ++c) q[3 * (size_t)t + c] = pts[3 * ((size_t)row * npt + ip) + c];
}

// rows moved (:917-937) and points_end (:944-955)
__global__ void k_wake_move(int npt, int nrows, int extra_row, const double *pold,
                            const double *qvel, double *pts, double *pvel, double *pend,
                            double dt, double nd) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int nr = nrows + (extra_row >= 0 ? 1 : 0);
  if (t >= nr * npt) return;
  int k = t / npt, ip = t % npt;
  const double *v = qvel + 3 * (size_t)t;
  if (k < nrows) {
    int ipan = 3 + k;  // 1-based row written; its source is row ipan - 1
    size_t dst = 3 * ((size_t)(ipan - 1) * npt + ip), src = 3 * ((size_t)(ipan - 2) * npt + ip);
    for (int c = 0; c < 3; ++c) {
      pvel[dst + c] = v[c];
      double a = ipan != 3 ? __dmul_rn(__dmul_rn(v[c], dt), nd) : __dmul_rn(v[c], dt);
      pts[dst + c] = __dadd_rn(pold[src + c], a);
    }
  } else {
    size_t src = 3 * ((size_t)extra_row * npt + ip);
    for (int c = 0; c < 3; ++c)
      pend[3 * ip + c] = __dadd_rn(pold[src + c], __dmul_rn(__dmul_rn(v[c], dt), nd));
  }
}

// :1169-1176: end_pan_idou = last row, intensities shifted one row back
__global__ void k_wake_shift(int ns, int len, double *idou, double *endi) {
  int iw = blockIdx.x * blockDim.x + threadIdx.x;
  if (iw >= ns) return;
  endi[iw] = idou[(size_t)(len - 1) * ns + iw];
  for (int r = len - 1; r >= 1; --r) idou[(size_t)r * ns + iw] = idou[(size_t)(r - 1) * ns + iw];
}

__global__ void k_add3(int n, double *a, const double *b) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < 3 * n) a[t] = __dadd_rn(a[t], b[t]);
}

// ---------------------------------------------------------------- shedding
struct ShedParams {
  int ns, npt, nm, refine, k_refine;
  double lo[3], hi[3];
  double k_vortex_rad, vortex_rad;
};

__device__ __forceinline__ double ave_side(const double *endi, const int *neigh,
                                           const int *neigh_o, int iw, int side) {
  int nb = neigh[2 * iw + side];
  if (nb > 0)
    return __ddiv_rn(__dsub_rn(endi[iw], __dmul_rn((double)neigh_o[2 * iw + side], endi[nb - 1])),
                     2.0);
  return endi[iw];
}

// Pass 1, one thread per stripe: the circulation vector of the stripe's
// shed vorticity (:1804-1842), last_pan_idou <- end_pan_idou, and the number
// of sub-particles (1 for the classical branch, n_chord x n_span with
// refine_wake, :1846-1864).
__global__ void k_shed_stripes(ShedParams sp, const int *ii, const int *neigh, const int *neigh_o,
                               const double *pts, const double *pend, const double *endi,
                               double *last, double *stripe /* [ns][8] */, int *nsub) {
  int iw = blockIdx.x * blockDim.x + threadIdx.x;
  if (iw >= sp.ns) return;
  const int p1 = ii[2 * iw] - 1, p2 = ii[2 * iw + 1] - 1;
  const double *r1 = pts + 3 * ((size_t)sp.nm * sp.npt + p1);
  const double *r2 = pts + 3 * ((size_t)sp.nm * sp.npt + p2);
  const double *e1 = pend + 3 * p1, *e2 = pend + 3 * p2;
  double pv[3] = {0.0, 0.0, 0.0}, d[3];
  // left side
  for (int c = 0; c < 3; ++c) d[c] = __dsub_rn(r1[c], e1[c]);
  const double chord_side_len = nrm3(d[0], d[1], d[2]);
  double ave = ave_side(endi, neigh, neigh_o, iw, 0);
  for (int c = 0; c < 3; ++c) pv[c] = __dadd_rn(pv[c], __dmul_rn(d[c], ave));
  // right side
  for (int c = 0; c < 3; ++c) d[c] = __dadd_rn(-r2[c], e2[c]);
  ave = ave_side(endi, neigh, neigh_o, iw, 1);
  for (int c = 0; c < 3; ++c) pv[c] = __dadd_rn(pv[c], __dmul_rn(d[c], ave));
  // end side
  for (int c = 0; c < 3; ++c) d[c] = __dsub_rn(e1[c], e2[c]);
  const double span_side_len = nrm3(d[0], d[1], d[2]);
  ave = __dsub_rn(endi[iw], last[iw]);
  last[iw] = endi[iw];
  for (int c = 0; c < 3; ++c) pv[c] = __dadd_rn(pv[c], __dmul_rn(d[c], ave));
  int n_chord = 1, n_span = 1;
  double step_chord = 0.0, step_span = 0.0;
  if (sp.refine) {
    const double kr = (double)sp.k_refine;
    if (chord_side_len >= span_side_len) {
      n_chord = (int)ceil(__ddiv_rn(chord_side_len, __ddiv_rn(span_side_len, kr)));
      n_span = sp.k_refine;
      step_chord = __ddiv_rn(chord_side_len, (double)n_chord);
      step_span = __ddiv_rn(span_side_len, (double)n_span);
    } else {
      n_chord = sp.k_refine;
      n_span = (int)ceil(__ddiv_rn(span_side_len, __ddiv_rn(chord_side_len, kr)));
      step_chord = __ddiv_rn(chord_side_len, (double)n_chord);
      step_span = __ddiv_rn(span_side_len, (double)n_span);
    }
  }
  double *s = stripe + 8 * (size_t)iw;
  s[0] = pv[0];
  s[1] = pv[1];
  s[2] = pv[2];
  s[3] = (double)n_chord;
  s[4] = (double)n_span;
  s[5] = step_chord;
  s[6] = step_span;
  nsub[iw] = n_chord * n_span;
}

// Pass 2, one thread per sub-particle: position, area, box test
// (:1866-1873, :1927-1934).
__global__ void k_shed_candidates(ShedParams sp, int ncand, const int *ii, const double *pts,
                                  const double *pend, const double *stripe, const int *soff,
                                  double *cand /* [ncand][6] */, int *ok) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ncand) return;
  // stripe of this candidate: the last stripe whose offset is <= t
  int lo = 0, hi = sp.ns - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (soff[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  const int iw = lo, j = t - soff[iw];
  const double *s = stripe + 8 * (size_t)iw;
  const int p1 = ii[2 * iw] - 1, p2 = ii[2 * iw + 1] - 1;
  const double *r1 = pts + 3 * ((size_t)sp.nm * sp.npt + p1);
  const double *r2 = pts + 3 * ((size_t)sp.nm * sp.npt + p2);
  const double *e1 = pend + 3 * p1, *e2 = pend + 3 * p2;
  double pos[3], area;
  if (sp.refine) {
    const int n_chord = (int)s[3], n_span = (int)s[4];
    const int ic = j / n_span + 1, is = j % n_span + 1;
    const double fc = __ddiv_rn(__dsub_rn((double)ic, 0.5), (double)n_chord);
    const double fs = __ddiv_rn(__dsub_rn((double)is, 0.5), (double)n_span);
    for (int c = 0; c < 3; ++c)
      pos[c] = __dadd_rn(__dadd_rn(r1[c], __dmul_rn(fc, __dsub_rn(e1[c], r1[c]))),
                         __dmul_rn(fs, __dsub_rn(r2[c], r1[c])));
    area = __dmul_rn(s[5], s[6]);
  } else {
    for (int c = 0; c < 3; ++c)
      pos[c] = __ddiv_rn(__dadd_rn(__dadd_rn(__dadd_rn(e1[c], e2[c]), r1[c]), r2[c]), 4.0);
    double a[3], b[3];
    for (int c = 0; c < 3; ++c) {
      a[c] = __dsub_rn(e1[c], r2[c]);
      b[c] = __dsub_rn(e2[c], r2[c]);
    }
    const double x = __dsub_rn(__dmul_rn(a[1], b[2]), __dmul_rn(a[2], b[1]));
    const double y = __dsub_rn(__dmul_rn(a[2], b[0]), __dmul_rn(a[0], b[2]));
    const double z = __dsub_rn(__dmul_rn(a[0], b[1]), __dmul_rn(a[1], b[0]));
    area = nrm3(x, y, z);
  }
  bool in = true;
  for (int c = 0; c < 3; ++c) in = in && pos[c] >= sp.lo[c] && pos[c] <= sp.hi[c];
  double *o = cand + 6 * (size_t)t;
  o[0] = pos[0];
  o[1] = pos[1];
  o[2] = pos[2];
  o[3] = area;
  o[4] = (double)iw;
  o[5] = sp.refine ? __dmul_rn(s[3], s[4]) : 0.0;
  ok[t] = in ? 1 : 0;
}

// Pass 3: the accepted candidate of rank r takes the r-th free slot (the
// reference's search from k, :1876-1880, fills the lowest free slots in
// candidate order).
__global__ void k_shed_write(ShedParams sp, int ncand, const int *ok, const int *rank,
                             const int *slots, const double *cand, const double *stripe,
                             const int *ii, const double *pvel, double *cen, double *dir,
                             double *mag, double *rv, double *vel, int *free_flag) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ncand || !ok[t]) return;
  const int ip = slots[rank[t]];
  const double *o = cand + 6 * (size_t)t;
  const int iw = (int)o[4];
  const double *s = stripe + 8 * (size_t)iw;
  const double pn = nrm3(s[0], s[1], s[2]);
  free_flag[ip] = 0;
  mag[ip] = sp.refine ? __ddiv_rn(pn, o[5]) : pn;
  for (int c = 0; c < 3; ++c) {
    dir[3 * (size_t)ip + c] = pn > 1.0e-13 ? __ddiv_rn(s[c], pn) : s[c];
    cen[3 * (size_t)ip + c] = o[c];
  }
  rv[ip] = sp.k_vortex_rad >= 1e-10 ? __dmul_rn(sp.k_vortex_rad, __dsqrt_rn(__dmul_rn(2.0, o[3])))
                                     : sp.vortex_rad;
  if (vel) {
    const int p1 = ii[2 * iw] - 1, p2 = ii[2 * iw + 1] - 1;
    const double *v1 = pvel + 3 * ((size_t)sp.nm * sp.npt + p1);
    const double *v2 = pvel + 3 * ((size_t)sp.nm * sp.npt + p2);
    for (int c = 0; c < 3; ++c) vel[3 * (size_t)ip + c] = __dmul_rn(0.5, __dadd_rn(v1[c], v2[c]));
  }
}

// ------------------------------------------------- index selection (scan)
// Indices i < n with (flag[i] == 0) == want_zero, in order, written to out;
// the count to *count.  Two block-level passes around a device-wide scan of
// the block counts.
#define SEL_T 512
__global__ void __launch_bounds__(SEL_T) k_sel_count(int n, const int *flag, int want_zero,
                                                      int *bcount) {
  typedef cub::BlockReduce<int, SEL_T> BR;
  __shared__ typename BR::TempStorage tmp;
  int i = blockIdx.x * SEL_T + threadIdx.x;
  int v = (i < n && ((flag[i] == 0) == (want_zero != 0))) ? 1 : 0;
  int s = BR(tmp).Sum(v);
  if (threadIdx.x == 0) bcount[blockIdx.x] = s;
}

__global__ void __launch_bounds__(SEL_T) k_sel_write(int n, const int *flag, int want_zero,
                                                      const int *boff, int cap, int *out,
                                                      int *count, int nblocks) {
  typedef cub::BlockScan<int, SEL_T> BS;
  __shared__ typename BS::TempStorage tmp;
  int i = blockIdx.x * SEL_T + threadIdx.x;
  int v = (i < n && ((flag[i] == 0) == (want_zero != 0))) ? 1 : 0;
  int r;
  BS(tmp).ExclusiveSum(v, r);
  r += boff[blockIdx.x];
  if (v && r < cap) out[r] = i;
  if (blockIdx.x == nblocks - 1 && threadIdx.x == SEL_T - 1) *count = r + v;
}

// select_indices: out[0..*count) (count on the device, capped at cap for
// the writes); work grows as needed
static int select_indices(int n, const int *flag, int want_zero, int cap, int *out, int *count,
                          DevBuf &work, cudaStream_t st) {
  int nb = (int)nblk((size_t)std::max(n, 1), SEL_T);
  size_t tb = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tb, (int *)nullptr, (int *)nullptr, nb, st);
  size_t need = 2 * (size_t)nb * sizeof(int) + tb + 512;
  DUST_TRY(devbuf_grow(work, need));
  int *bc = (int *)work.p, *bo = bc + nb;
  void *tmp = (void *)(((uintptr_t)(bo + nb) + 255) & ~(uintptr_t)255);
  if (n == 0) {
    DUST_CUDA(cudaMemsetAsync(count, 0, sizeof(int), st));
    return DUST_OK;
  }
  k_sel_count<<<nb, SEL_T, 0, st>>>(n, flag, want_zero, bc);
  DUST_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, bc, bo, nb, st));
  k_sel_write<<<nb, SEL_T, 0, st>>>(n, flag, want_zero, bo, cap, out, count, nb);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}

// ----------------------------------------------------- live particle list
__global__ void k_live_gather(int n, const int *idx, const double *cen, const double *dir,
                              const double *mag, const double *rv, double *lc, double *ld,
                              double *lm, double *lr) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  int s = idx[t];
  for (int c = 0; c < 3; ++c) {
    lc[3 * (size_t)t + c] = cen[3 * (size_t)s + c];
    ld[3 * (size_t)t + c] = dir[3 * (size_t)s + c];
  }
  lm[t] = mag[s];
  lr[t] = rv[s];
}

__global__ void k_live_scatter(int n, const int *idx, const double *a, const double *b,
                               const double *c, double *A, double *B, double *Cc) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * n) return;
  int i = t / 3, k = t % 3;
  size_t d = 3 * (size_t)idx[i] + k;
  if (a) A[d] = a[t];
  if (b) B[d] = b[t];
  if (c) Cc[d] = c[t];
}

// selection work and count of the live-list entry point (one host thread)
static DevBuf g_live_work, g_live_cnt;

extern "C" int dust_particles_live_device(int n_slots, const int *free_flag, const double *cen,
                                          const double *dir, const double *mag,
                                          const double *r_vortex, double *lcen, double *ldir,
                                          double *lmag, double *lrv, int *idx, int *n_live,
                                          void *stream) {
  if (n_slots < 0 || !n_live) return DUST_ERR_BAD_ARG;
  if (n_slots > 0 && (!free_flag || !cen || !dir || !mag || !r_vortex || !lcen || !ldir ||
                      !lmag || !lrv || !idx))
    return DUST_ERR_BAD_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  DUST_TRY(devbuf_grow(g_live_cnt, 256));
  int *dcount = (int *)g_live_cnt.p;
  DUST_TRY(select_indices(n_slots, free_flag, 1, n_slots, idx, dcount, g_live_work, st));
  int h = 0;
  DUST_CUDA(cudaMemcpyAsync(&h, dcount, sizeof(int), cudaMemcpyDeviceToHost, st));
  DUST_CUDA(cudaStreamSynchronize(st));
  if (h > 0)
    k_live_gather<<<nblk(h, 256), 256, 0, st>>>(h, idx, cen, dir, mag, r_vortex, lcen, ldir, lmag,
                                                lrv);
  DUST_CUDA(cudaGetLastError());
  *n_live = h;
  return DUST_OK;
}

extern "C" int dust_particles_scatter_device(int n_live, const int *idx, const double *lvel,
                                             const double *lstr, const double *lrot, double *vel,
                                             double *str, double *rot, void *stream) {
  if (n_live < 0 || (n_live > 0 && !idx)) return DUST_ERR_BAD_ARG;
  if ((lvel && !vel) || (lstr && !str) || (lrot && !rot)) return DUST_ERR_BAD_ARG;
  if (n_live == 0) return DUST_OK;
  k_live_scatter<<<nblk(3 * (size_t)n_live, 256), 256, 0, (cudaStream_t)stream>>>(
      n_live, idx, lvel, lstr, lrot, vel, str, rot);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}

// ------------------------------------------------------------ entry points
static void wake_free(dust_wake *w) {
  if (!w) return;
  void *ps[] = {w->pts,  w->pold,  w->pvel,  w->idou,    w->last, w->endi,  w->pend,
                w->wver, w->ever,  w->qpts,  w->qvel,    w->qtmp, w->ii,    w->neigh,
                w->neigh_o, w->gen, w->nver4, w->nsub,   w->soff, w->cand_ok, w->cand_rank,
                w->cand};
  for (void *p : ps)
    if (p) cudaFree(p);
  devbuf_free(w->sel);
  devbuf_free(w->slots);
  devbuf_free(w->sel_work);
  devbuf_free(w->cnt);
  devbuf_free(w->scan_tmp);
  devbuf_free(w->geo);
  devbuf_free(w->raw);
  delete w;
}

static int wake_params_ok(const dust_wake_params *p) {
  if (!p || p->n_stripes <= 0 || p->n_points < 2 || p->n_wake_panels < 1) return 0;
  if (p->ndt_update_wake == 0 || !(p->dt > 0.0)) return 0;
  if (p->refine_wake && p->k_refine < 1) return 0;
  return 1;
}

template <class T>
static int dalloc(T *&p, size_t count) {
  DUST_CUDA(cudaMalloc((void **)&p, std::max(count, (size_t)1) * sizeof(T)));
  return DUST_OK;
}

extern "C" int dust_wake_create(const dust_wake_params *prm, const dust_te *te,
                                const double *te_pts, const double *te_dir,
                                const double *te_scaling, const double *te_vel, dust_wake **out) {
  if (!out || !wake_params_ok(prm) || !te || !te->ii || !te->neigh || !te->neigh_o ||
      !te->gen_elems || !te_pts || !te_dir || !te_scaling)
    return DUST_ERR_BAD_ARG;
  const int ns = prm->n_stripes, npt = prm->n_points, nm = prm->n_wake_panels;
  for (int i = 0; i < 2 * ns; ++i) {
    if (te->ii[i] < 1 || te->ii[i] > npt) return DUST_ERR_BAD_ARG;
    if (te->neigh[i] < 0 || te->neigh[i] > ns) return DUST_ERR_BAD_ARG;
    if (te->gen_elems[i] < 0) return DUST_ERR_BAD_ARG;
  }
  for (int iw = 0; iw < ns; ++iw)
    if (te->gen_elems[2 * iw] < 1) return DUST_ERR_BAD_ARG;
  dust_wake *w = new dust_wake();
  w->p = *prm;
  w->h_ii.assign(te->ii, te->ii + 2 * ns);
  w->h_gen.assign(te->gen_elems, te->gen_elems + 2 * ns);
  const size_t P = (size_t)(nm + 1) * npt * 3;
  int s = DUST_OK;
  auto A = [&](int r) {
    if (s == DUST_OK) s = r;
  };
  A(dalloc(w->pts, P));
  A(dalloc(w->pold, P));
  A(dalloc(w->pvel, P));
  A(dalloc(w->idou, (size_t)nm * ns));
  A(dalloc(w->last, ns));
  A(dalloc(w->endi, ns));
  A(dalloc(w->pend, (size_t)npt * 3));
  A(dalloc(w->wver, (size_t)nm * ns * 12));
  A(dalloc(w->ever, (size_t)ns * 6));
  A(dalloc(w->qpts, P));
  A(dalloc(w->qvel, P));
  A(dalloc(w->qtmp, P));
  A(dalloc(w->ii, 2 * (size_t)ns));
  A(dalloc(w->neigh, 2 * (size_t)ns));
  A(dalloc(w->neigh_o, 2 * (size_t)ns));
  A(dalloc(w->gen, 2 * (size_t)ns));
  A(dalloc(w->nver4, (size_t)nm * ns));
  A(dalloc(w->nsub, ns + 1));
  A(dalloc(w->soff, ns + 1));
  if (s != DUST_OK) {
    wake_free(w);
    return s;
  }
  cudaStream_t st = 0;
  std::vector<int> four((size_t)nm * ns, 4);
  double *tp = nullptr;
  if (cudaMemsetAsync(w->pts, 0, P * 8, st) != cudaSuccess ||
      cudaMemsetAsync(w->pvel, 0, P * 8, st) != cudaSuccess ||
      cudaMemsetAsync(w->idou, 0, (size_t)nm * ns * 8, st) != cudaSuccess ||
      cudaMemsetAsync(w->last, 0, (size_t)ns * 8, st) != cudaSuccess ||
      cudaMemsetAsync(w->endi, 0, (size_t)ns * 8, st) != cudaSuccess ||
      cudaMemsetAsync(w->pend, 0, (size_t)npt * 24, st) != cudaSuccess ||
      cudaMemcpyAsync(w->ii, te->ii, 8 * (size_t)ns, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(w->neigh, te->neigh, 8 * (size_t)ns, cudaMemcpyHostToDevice, st) !=
          cudaSuccess ||
      cudaMemcpyAsync(w->neigh_o, te->neigh_o, 8 * (size_t)ns, cudaMemcpyHostToDevice, st) !=
          cudaSuccess ||
      cudaMemcpyAsync(w->gen, te->gen_elems, 8 * (size_t)ns, cudaMemcpyHostToDevice, st) !=
          cudaSuccess ||
      cudaMemcpyAsync(w->nver4, four.data(), four.size() * 4, cudaMemcpyHostToDevice, st) !=
          cudaSuccess ||
      cudaMalloc((void **)&tp, (size_t)npt * (3 + 3 + 1 + 3) * 8) != cudaSuccess) {
    dust_set_last_error("wake set-up", __FILE__, __LINE__);
    wake_free(w);
    return DUST_ERR_CUDA;
  }
  double *dpts = tp, *ddir = tp + 3 * npt, *dsc = tp + 6 * npt, *dvel = tp + 7 * npt;
  bool ok = cudaMemcpyAsync(dpts, te_pts, (size_t)npt * 24, cudaMemcpyHostToDevice, st) ==
                cudaSuccess &&
            cudaMemcpyAsync(ddir, te_dir, (size_t)npt * 24, cudaMemcpyHostToDevice, st) ==
                cudaSuccess &&
            cudaMemcpyAsync(dsc, te_scaling, (size_t)npt * 8, cudaMemcpyHostToDevice, st) ==
                cudaSuccess &&
            (!te_vel || cudaMemcpyAsync(dvel, te_vel, (size_t)npt * 24, cudaMemcpyHostToDevice,
                                        st) == cudaSuccess);
  if (ok) {
    k_wake_te_rows<<<nblk(npt, 128), 128, 0, st>>>(
        npt, w->pts, dpts, ddir, dsc, te_vel ? dvel : nullptr, prm->u_inf[0], prm->u_inf[1],
        prm->u_inf[2], prm->dt, (double)prm->ndt_update_wake, prm->min_vel_at_te, 0);
    k_wake_geo<<<nblk(2 * (size_t)ns, 128), 128, 0, st>>>(ns, npt, 1, 0, w->ii, w->pts, w->wver,
                                                          w->ever);
    ok = cudaGetLastError() == cudaSuccess && cudaStreamSynchronize(st) == cudaSuccess;
  }
  cudaFree(tp);
  if (!ok) {
    dust_set_last_error("wake set-up", __FILE__, __LINE__);
    wake_free(w);
    return DUST_ERR_CUDA;
  }
  w->len = 1;
  w->len_geo = 1;
  w->full = false;
  w->attached = false;
  *out = w;
  return DUST_OK;
}

extern "C" int dust_wake_destroy(dust_wake *w) {
  wake_free(w);
  return DUST_OK;
}

extern "C" int dust_wake_elements(dust_wake *w, dust_panels *wake_pan, dust_lines *end_vort,
                                  int *n_impl, const int **impl_ind) {
  if (!w) return DUST_ERR_BAD_ARG;
  if (wake_pan) {
    memset(wake_pan, 0, sizeof(*wake_pan));
    wake_pan->n = w->len_geo * w->p.n_stripes;
    wake_pan->n_ver = w->nver4;
    wake_pan->kind = nullptr;
    wake_pan->ver = w->wver;
    wake_pan->mag = w->idou;
  }
  if (end_vort) {
    // end vortices act once complete_wake (or load_wake) of a full wake
    // has attached them; before that their mag pointers are not associated
    // and compute_vel_vortline gives 0 (src/aeroel/mod_vortline.f90:138)
    end_vort->n = w->attached ? w->p.n_stripes : 0;
    end_vort->ver = w->ever;
    end_vort->mag = w->last;
  }
  if (n_impl) *n_impl = w->p.n_stripes;
  if (impl_ind) *impl_ind = w->gen;
  return DUST_OK;
}

extern "C" int dust_wake_set_first_row_device(dust_wake *w, const double *res, void *stream) {
  if (!w || !res) return DUST_ERR_BAD_ARG;
  k_wake_first_row<<<nblk(w->p.n_stripes, 128), 128, 0, (cudaStream_t)stream>>>(
      w->p.n_stripes, w->gen, res, w->idou);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}

extern "C" int dust_wake_update_device(dust_wake *w, const dust_fmm_params *prm,
                                       const dust_panels *body, int n, const double *cen,
                                       const double *dir, const double *mag,
                                       const double *r_vortex, void *stream) {
  if (!w || !prm || n < 0 || (n > 0 && (!cen || !dir || !mag || !r_vortex)))
    return DUST_ERR_BAD_ARG;
  if (body && body->n > 0 && !body->ver) return DUST_ERR_BAD_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const int ns = w->p.n_stripes, npt = w->p.n_points, nm = w->p.n_wake_panels;
  const double dt = w->p.dt, nd = (double)w->p.ndt_update_wake;
  if (w->len == nm) w->full = true;  // :882
  const size_t P = (size_t)(nm + 1) * npt * 3;
  DUST_CUDA(cudaMemcpyAsync(w->pold, w->pts, P * 8, cudaMemcpyDeviceToDevice, st));
  // rows ipan = 3..np (1-based) from rows ipan - 2 (0-based ipan - 2), np
  // = len + 1 (+ 1 when not full); a full wake adds row len for points_end
  const int np_ = w->len + 1 + (w->full ? 0 : 1);
  const int nrows = std::max(0, np_ - 2);
  const int extra = w->full ? w->len : -1;
  const int nq = (nrows + (extra >= 0 ? 1 : 0)) * npt;
  if (nq > 0) {
    k_wake_gather_rows<<<nblk(nq, 128), 128, 0, st>>>(npt, 1, nrows, extra, w->pold, w->qpts);
    // compute_vel_from_all: body, wake panels, end vortices (+ u_inf), then
    // the particles
    dust_panels wp;
    dust_lines ev;
    dust_wake_elements(w, &wp, &ev, nullptr, nullptr);
    ElemDev e;
    DUST_TRY(elem_build_device(body, &wp, &ev, prm->u_inf, reg_params(prm), false, w->raw, w->geo,
                               e, st));
    DUST_TRY(elements_vel_points(e, nq, w->qpts, prm->u_inf, w->qvel, st));
    if (n > 0) {
      ElemDev none;
      memset(&none, 0, sizeof(none));
      none.rp = reg_params(prm);
      DUST_TRY(points_uvort_device(prm, nq, w->qpts, n, cen, dir, mag, r_vortex, none, w->qtmp,
                                   st));
      k_add3<<<nblk(3 * (size_t)nq, 256), 256, 0, st>>>(nq, w->qvel, w->qtmp);
    }
    k_wake_move<<<nblk(nq, 128), 128, 0, st>>>(npt, nrows, extra, w->pold, w->qvel, w->pts,
                                               w->pvel, w->pend, dt, nd);
  }
  // :1132-1176
  if (!w->full) w->len += 1;
  k_wake_shift<<<nblk(ns, 128), 128, 0, st>>>(ns, w->len, w->idou, w->endi);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}

extern "C" int dust_wake_complete_device(dust_wake *w, const double *te_pts,
                                         const double *te_dir, const double *te_scaling,
                                         const double *te_vel, int n_slots, double *cen,
                                         double *dir, double *mag, double *r_vortex,
                                         double *vel, int *free_flag, int *n_shed,
                                         void *stream) {
  if (!w || !te_pts || !te_dir || !te_scaling || n_slots < 0 || !n_shed) return DUST_ERR_BAD_ARG;
  if (n_slots > 0 && (!cen || !dir || !mag || !r_vortex || !free_flag)) return DUST_ERR_BAD_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const int ns = w->p.n_stripes, npt = w->p.n_points, nm = w->p.n_wake_panels;
  k_wake_te_rows<<<nblk(npt, 128), 128, 0, st>>>(
      npt, w->pts, te_pts, te_dir, te_scaling, te_vel, w->p.u_inf[0], w->p.u_inf[1],
      w->p.u_inf[2], w->p.dt, (double)w->p.ndt_update_wake, w->p.min_vel_at_te, 1);
  *n_shed = 0;
  if (w->full) {
    ShedParams sp;
    sp.ns = ns;
    sp.npt = npt;
    sp.nm = nm;
    sp.refine = w->p.refine_wake ? 1 : 0;
    sp.k_refine = w->p.k_refine;
    for (int c = 0; c < 3; ++c) {
      sp.lo[c] = w->p.box_min[c];
      sp.hi[c] = w->p.box_max[c];
    }
    sp.k_vortex_rad = w->p.k_vortex_rad;
    sp.vortex_rad = w->p.vortex_rad;
    // per-stripe record: partvec(3), n_chord, n_span, steps(2), spare
    static_assert(sizeof(double) == 8, "");
    DUST_TRY(devbuf_grow(w->sel, (size_t)ns * 8 * 8 + 256));
    double *stripe = (double *)w->sel.p;
    k_shed_stripes<<<nblk(ns, 128), 128, 0, st>>>(sp, w->ii, w->neigh, w->neigh_o, w->pts,
                                                  w->pend, w->endi, w->last, stripe, w->nsub);
    // offsets of the stripes' sub-particles (inclusive count at [ns])
    std::vector<int> hn(ns), ho(ns + 1);
    DUST_CUDA(cudaMemcpyAsync(hn.data(), w->nsub, (size_t)ns * 4, cudaMemcpyDeviceToHost, st));
    DUST_CUDA(cudaStreamSynchronize(st));
    ho[0] = 0;
    for (int i = 0; i < ns; ++i) ho[i + 1] = ho[i] + hn[i];
    const int ncand = ho[ns];
    DUST_CUDA(cudaMemcpyAsync(w->soff, ho.data(), (size_t)(ns + 1) * 4, cudaMemcpyHostToDevice,
                              st));
    if (ncand > w->cand_cap) {
      if (w->cand) cudaFree(w->cand);
      if (w->cand_ok) cudaFree(w->cand_ok);
      if (w->cand_rank) cudaFree(w->cand_rank);
      w->cand = nullptr;
      w->cand_ok = w->cand_rank = nullptr;
      w->cand_cap = 0;
      DUST_TRY(dalloc(w->cand, (size_t)ncand * 6));
      DUST_TRY(dalloc(w->cand_ok, (size_t)ncand + 1));
      DUST_TRY(dalloc(w->cand_rank, (size_t)ncand + 1));
      w->cand_cap = ncand;
    }
    if (ncand > 0) {
      k_shed_candidates<<<nblk(ncand, 128), 128, 0, st>>>(sp, ncand, w->ii, w->pts, w->pend,
                                                          stripe, w->soff, w->cand, w->cand_ok);
      // rank of each accepted candidate
      size_t tb = 0;
      cub::DeviceScan::ExclusiveSum(nullptr, tb, w->cand_ok, w->cand_rank, ncand, st);
      DUST_TRY(devbuf_grow(w->scan_tmp, tb + 256));
      DUST_CUDA(cub::DeviceScan::ExclusiveSum(w->scan_tmp.p, tb, w->cand_ok, w->cand_rank,
                                              ncand, st));
      int last_ok = 0, last_rank = 0;
      DUST_CUDA(cudaMemcpyAsync(&last_ok, w->cand_ok + ncand - 1, 4, cudaMemcpyDeviceToHost, st));
      DUST_CUDA(cudaMemcpyAsync(&last_rank, w->cand_rank + ncand - 1, 4, cudaMemcpyDeviceToHost,
                                st));
      DUST_CUDA(cudaStreamSynchronize(st));
      const int need = last_ok + last_rank;
      if (need > 0) {
        // the lowest `need` free slots, in order
        DUST_TRY(devbuf_grow(w->slots, (size_t)need * 4 + 256));
        DUST_TRY(devbuf_grow(w->cnt, 256));
        DUST_TRY(select_indices(n_slots, free_flag, 0, need, (int *)w->slots.p, (int *)w->cnt.p,
                                w->sel_work, st));
        int nfree = 0;
        DUST_CUDA(cudaMemcpyAsync(&nfree, w->cnt.p, 4, cudaMemcpyDeviceToHost, st));
        DUST_CUDA(cudaStreamSynchronize(st));
        if (nfree < need) {
          dust_set_last_error("Exceeding the maximum number of wake particles", __FILE__,
                              __LINE__);
          return DUST_ERR_CAPACITY;
        }
        k_shed_write<<<nblk(ncand, 128), 128, 0, st>>>(sp, ncand, w->cand_ok, w->cand_rank,
                                                       (const int *)w->slots.p, w->cand, stripe,
                                                       w->ii, w->pvel, cen, dir, mag, r_vortex,
                                                       vel, free_flag);
      }
      *n_shed = need;
    }
  }
  w->len_geo = w->len;
  if (w->full) w->attached = true;  // :2091-2103
  k_wake_geo<<<nblk((size_t)(w->len + 1) * ns, 128), 128, 0, st>>>(
      ns, npt, w->len, w->full ? 1 : 0, w->ii, w->pts, w->wver, w->ever);
  DUST_CUDA(cudaGetLastError());
  DUST_CUDA(cudaStreamSynchronize(st));
  return DUST_OK;
}

// velocities of the wake panels' vertices (pan_w_vel at (row, point) of
// each vertex, in the panels' vertex order) and of the end vortices'
// vertices (row len), for the pressure equation's rotational terms
__global__ void k_wake_vv(int ns, int npt, int len, int attached, const int *ii,
                          const double *pvel, double *wvv, double *evv) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (len + 1) * ns) return;
  int r = t / ns, iw = t % ns;
  int p1 = ii[2 * iw] - 1, p2 = ii[2 * iw + 1] - 1;
  const double *a = pvel + 3 * ((size_t)r * npt + p1), *b = pvel + 3 * ((size_t)r * npt + p2);
  if (r < len) {
    const double *c = pvel + 3 * ((size_t)(r + 1) * npt + p2);
    const double *d = pvel + 3 * ((size_t)(r + 1) * npt + p1);
    double *v = wvv + 12 * (size_t)t;
    for (int k = 0; k < 3; ++k) {
      v[k] = a[k];
      v[3 + k] = b[k];
      v[6 + k] = c[k];
      v[9 + k] = d[k];
    }
  } else if (attached && evv) {
    double *e = evv + 6 * (size_t)iw;
    for (int k = 0; k < 3; ++k) {
      e[k] = a[k];
      e[3 + k] = b[k];
    }
  }
}

extern "C" int dust_wake_vertex_velocities_device(dust_wake *w, double *wake_vv, double *end_vv,
                                                  void *stream) {
  if (!w || !wake_vv) return DUST_ERR_BAD_ARG;
  const int ns = w->p.n_stripes;
  k_wake_vv<<<nblk((size_t)(w->len_geo + 1) * ns, 128), 128, 0, (cudaStream_t)stream>>>(
      ns, w->p.n_points, w->len_geo, w->attached ? 1 : 0, w->ii, w->pvel, wake_vv, end_vv);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}

extern "C" int dust_wake_get_state(const dust_wake *w, int *len, double *points,
                                   double *point_vel, double *idou, double *last_idou) {
  if (!w) return DUST_ERR_BAD_ARG;
  const int ns = w->p.n_stripes, npt = w->p.n_points;
  const size_t rows = (size_t)w->len + 1;
  if (len) *len = w->len;
  if (points) DUST_CUDA(cudaMemcpy(points, w->pts, rows * npt * 24, cudaMemcpyDeviceToHost));
  if (point_vel)
    DUST_CUDA(cudaMemcpy(point_vel, w->pvel, rows * npt * 24, cudaMemcpyDeviceToHost));
  if (idou) DUST_CUDA(cudaMemcpy(idou, w->idou, (size_t)w->len * ns * 8, cudaMemcpyDeviceToHost));
  if (last_idou) DUST_CUDA(cudaMemcpy(last_idou, w->last, (size_t)ns * 8, cudaMemcpyDeviceToHost));
  return DUST_OK;
}

extern "C" int dust_wake_set_state(dust_wake *w, int len, const double *points,
                                   const double *point_vel, const double *idou,
                                   const double *last_idou) {
  if (!w || len < 1 || len > w->p.n_wake_panels || !points || !idou || !last_idou)
    return DUST_ERR_BAD_ARG;
  const int ns = w->p.n_stripes, npt = w->p.n_points;
  const size_t rows = (size_t)len + 1;
  DUST_CUDA(cudaMemcpy(w->pts, points, rows * npt * 24, cudaMemcpyHostToDevice));
  if (point_vel)
    DUST_CUDA(cudaMemcpy(w->pvel, point_vel, rows * npt * 24, cudaMemcpyHostToDevice));
  else
    DUST_CUDA(cudaMemset(w->pvel, 0, rows * npt * 24));
  DUST_CUDA(cudaMemcpy(w->idou, idou, (size_t)len * ns * 8, cudaMemcpyHostToDevice));
  DUST_CUDA(cudaMemcpy(w->last, last_idou, (size_t)ns * 8, cudaMemcpyHostToDevice));
  w->len = len;
  w->len_geo = len;
  w->full = len == w->p.n_wake_panels;  // load_wake :764
  w->attached = w->full;                 // :766-777
  k_wake_geo<<<nblk(rows * ns, 128), 128>>>(ns, npt, len, w->full ? 1 : 0, w->ii, w->pts,
                                            w->wver, w->ever);
  DUST_CUDA(cudaGetLastError());
  DUST_CUDA(cudaDeviceSynchronize());
  return DUST_OK;
}
