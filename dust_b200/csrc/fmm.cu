// fmm.cu -- octree FMM for vortex particles on sm_100a.
//
// Replaces the reference's mod_octree / mod_multipole path
// (src/fmm/mod_octree.f90:251-1429, src/fmm/mod_multipole.f90:224-450) and
// the particle kernels of src/aeroel/mod_vortpart.f90:139-336.
//
// Design (B200-first, not a translation):
//  * particles are binned at the finest level and stably radix-sorted by a
//    hierarchical Morton key, so every cell of every level owns a contiguous
//    particle range (the reference's pointer lists, mod_octree.f90:746-773
//    and 911-961, in the same order);
//  * the reference's leaf rule (npart >= min_octree_part at fixed depth,
//    siblings of leaves become leaves, :896-962) runs as one dense kernel
//    per level over Morton-ordered flag arrays; active cells and leaves are
//    compacted with device scans;
//  * multipole data live in compact per-active-cell SoA blocks;
//  * M2L evaluates the degree-(p+1) velocity local expansion g once and
//    derives the reference's gradient coefficients from it exactly,
//    c(r,:,m) = (m_r+1) g(:, m+e_r); the velocity coefficients b (degree p)
//    and g are translated with the reference's own truncations in L2L;
//  * L2P is fused into the leaf-pair P2P kernel: one CTA per leaf, the
//    near-field source ranges concatenated into one virtual index space
//    streamed through shared memory in 128-particle tiles, thread groups
//    splitting the sources of small leaves, group partials reduced through
//    shared memory.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "dust_common.cuh"
#include "elements.cuh"
#include "fmm_internal.h"

static int build_shift_tables(dust_octree *o);

// ===================================================================== host
static int grow(DevBuf &b, size_t bytes) {
  if (bytes <= b.cap) return DUST_OK;
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.cap = 0;
  size_t want = bytes + bytes / 8 + 256;
  DUST_CUDA(cudaMalloc(&b.p, want));
  b.cap = want;
  return DUST_OK;
}
void devbuf_free(DevBuf &b) {
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.cap = 0;
}
int devbuf_grow(DevBuf &b, size_t bytes) { return grow(b, bytes); }

// compute_der_ker (mod_multipole.f90:388-450) for one offset, returning
// D(3, n_mon(2p+1)) scaled by the multi-index factorial of its monomial.
static void host_der_table(int p, const double diff[3], double delta, double *Dhat) {
  int deg = 2 * p + 2;
  int nm = n_mon(deg);
  std::vector<double> bk(nm, 0.0);
  double R2 = diff[0] * diff[0] + diff[1] * diff[1] + diff[2] * diff[2] + delta * delta;
  for (int k = 0; k <= deg; ++k)
    for (int j = 0; j <= deg - k; ++j)
      for (int i = 0; i <= deg - j - k; ++i) {
        double kmod = (double)(k + j + i);
        if (i == 0 && j == 0 && k == 0) {
          bk[0] = 1.0 / (4.0 * DUST_PI * sqrt(R2));
        } else {
          double s1 = 0.0, s2 = 0.0;
          if (i >= 1) s1 += diff[0] * bk[mono_idx(i - 1, j, k)];
          if (j >= 1) s1 += diff[1] * bk[mono_idx(i, j - 1, k)];
          if (k >= 1) s1 += diff[2] * bk[mono_idx(i, j, k - 1)];
          if (i >= 2) s2 += bk[mono_idx(i - 2, j, k)];
          if (j >= 2) s2 += bk[mono_idx(i, j - 2, k)];
          if (k >= 2) s2 += bk[mono_idx(i, j, k - 2)];
          bk[mono_idx(i, j, k)] =
              1.0 / (R2 * kmod) * ((2.0 * kmod - 1.0) * s1 - (kmod - 1.0) * s2);
        }
      }
  double fact[40];
  fact[0] = 1.0;
  for (int q = 1; q < 40; ++q) fact[q] = fact[q - 1] * q;
  int nD = n_mon(2 * p + 1);
  for (int q = 0; q < nD; ++q) {
    int i, j, k;
    mono_exp(q, i, j, k);
    double f = fact[i] * fact[j] * fact[k];
    Dhat[3 * q + 0] = -(1.0 + i) * bk[mono_idx(i + 1, j, k)] * f;
    Dhat[3 * q + 1] = -(1.0 + j) * bk[mono_idx(i, j + 1, k)] * f;
    Dhat[3 * q + 2] = -(1.0 + k) * bk[mono_idx(i, j, k + 1)] * f;
  }
}

static int build_tables(dust_octree *o) {
  int p = o->p;
  int nD = n_mon(2 * p + 1);
  std::vector<double> tab;
  for (int l = 1; l <= o->G.ll; ++l) {
    int L[3];
    for (int d = 0; d < 3; ++d)
      L[d] = (l == 1) ? std::max(o->G.nbox[d], 3) : 3;
    for (int d = 0; d < 3; ++d) o->kdlen[l][d] = L[d];
    size_t nofs = (size_t)(2 * L[0] + 1) * (2 * L[1] + 1) * (2 * L[2] + 1);
    tab.assign(nofs * nD * 3, 0.0);
    size_t q = 0;
    for (int k = -L[2]; k <= L[2]; ++k)
      for (int j = -L[1]; j <= L[1]; ++j)
        for (int i = -L[0]; i <= L[0]; ++i, ++q)
          if (std::abs(i) >= 2 || std::abs(j) >= 2 || std::abs(k) >= 2) {
            double diff[3] = {o->G.csize[l] * (double)(-i), o->G.csize[l] * (double)(-j),
                              o->G.csize[l] * (double)(-k)};
            host_der_table(p, diff, o->prm.rankine_rad, &tab[q * nD * 3]);
          }
    DUST_TRY(grow(o->dtab[l], tab.size() * sizeof(double)));
    DUST_CUDA(cudaMemcpy(o->dtab[l].p, tab.data(), tab.size() * sizeof(double),
                         cudaMemcpyHostToDevice));
  }
  // index table idxsum[n * nm1 + m'] = mono_idx(m' + n), and scale tables
  int nm = n_mon(p), nm1 = n_mon(p + 1);
  std::vector<uint16_t> isum((size_t)nm * nm1);
  for (int n = 0; n < nm; ++n) {
    int a, b, c;
    mono_exp(n, a, b, c);
    for (int m = 0; m < nm1; ++m) {
      int i, j, k;
      mono_exp(m, i, j, k);
      isum[(size_t)n * nm1 + m] = (uint16_t)mono_idx(i + a, j + b, k + c);
    }
  }
  DUST_TRY(grow(o->idxsum, isum.size() * sizeof(uint16_t)));
  DUST_CUDA(cudaMemcpy(o->idxsum.p, isum.data(), isum.size() * sizeof(uint16_t),
                       cudaMemcpyHostToDevice));
  return DUST_OK;
}

static int geom_init(dust_octree *o) {
  TreeGeom &G = o->G;
  const dust_fmm_params &p = o->prm;
  memset(&G, 0, sizeof(G));
  G.ll = p.n_octree_levels;
  uint64_t off = 0;
  for (int d = 0; d < 3; ++d) {
    G.nbox[d] = p.n_box[d];
    G.xmin[d] = p.origin[d];
    G.xmax[d] = p.origin[d] + (double)p.n_box[d] * p.box_length;
  }
  for (int l = 1; l <= G.ll; ++l) {
    uint64_t nc = 1;
    for (int d = 0; d < 3; ++d) {
      G.ncl[l][d] = p.n_box[d] << (l - 1);
      nc *= (uint64_t)G.ncl[l][d];
    }
    if (nc >= (1ull << 31)) return DUST_ERR_CAPACITY;
    G.ncell[l] = (uint32_t)nc;
    G.lev_off[l] = (uint32_t)off;
    off += nc;
    if (off >= (1ull << 31)) return DUST_ERR_CAPACITY;
    G.csize[l] = (l == 1) ? p.box_length : p.box_length / (double)(1 << (l - 1));
  }
  G.lev_off[G.ll + 1] = (uint32_t)off;
  o->ncell_tot = off;
  return DUST_OK;
}

extern "C" int dust_octree_create(const dust_fmm_params *prm, dust_octree **out) {
  if (!prm || !out) return DUST_ERR_BAD_ARG;
  *out = nullptr;
  if (prm->n_octree_levels < 1 || prm->n_octree_levels > 11 ||
      prm->multipole_degree < 0 || prm->multipole_degree > DUST_MAXP ||
      prm->box_length <= 0.0 || prm->n_box[0] < 1 || prm->n_box[1] < 1 ||
      prm->n_box[2] < 1 || prm->min_octree_part < 0)
    return DUST_ERR_BAD_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return DUST_ERR_NO_DEVICE;
  dust_octree *o = new dust_octree();
  o->prm = *prm;
  o->p = prm->multipole_degree;
  o->nm = n_mon(o->p);
  o->nm1 = n_mon(o->p + 1);
  o->nD = n_mon(2 * o->p + 1);
  int st = geom_init(o);
  if (st != DUST_OK) {
    delete o;
    return st;
  }
  if (cudaStreamCreateWithFlags(&o->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete o;
    return DUST_ERR_CUDA;
  }
  for (int e = 0; e < 12; ++e) cudaEventCreate(&o->ev[e]);
  st = build_tables(o);
  if (st == DUST_OK) st = build_shift_tables(o);
  if (st == DUST_OK) st = m2l_batch_tables(o);
  if (st != DUST_OK) {
    dust_octree_destroy(o);
    return st;
  }
  *out = o;
  return DUST_OK;
}

extern "C" int dust_octree_destroy(dust_octree *o) {
  if (!o) return DUST_OK;
  cudaStreamSynchronize(o->stream);
  for (int l = 0; l <= DUST_MAXLEV; ++l) {
    devbuf_free(o->dtab[l]);
    devbuf_free(o->dtab32[l]);
    devbuf_free(o->dtabs[l]);
  }
  devbuf_free(o->m2l_buf);
  devbuf_free(o->ahat);
  devbuf_free(o->m2l_bat);
  devbuf_free(o->jsum);
  devbuf_free(o->shift);
  devbuf_free(o->ffbuf);
  devbuf_free(o->elem_work);
  DevBuf *bufs[] = {&o->idxsum, &o->keys,   &o->keys_s, &o->vals,   &o->perm,
                    &o->cnt,    &o->cstart, &o->part,   &o->flags,  &o->ind,
                    &o->cidx,   &o->lidx,   &o->act_key, &o->act_lev, &o->leaf_ci,
                    &o->mp,     &o->outs,   &o->cub_tmp, &o->small,  &o->h_in,
                    &o->h_out,  &o->h_pts,  &o->el_geo, &o->el_raw};
  for (DevBuf *b : bufs) devbuf_free(*b);
  for (int e = 0; e < 12; ++e) cudaEventDestroy(o->ev[e]);
  cudaStreamDestroy(o->stream);
  delete o;
  return DUST_OK;
}

extern "C" int dust_octree_get_stats(const dust_octree *o, dust_fmm_stats *st) {
  if (!o || !st) return DUST_ERR_BAD_ARG;
  *st = o->stats;
  return DUST_OK;
}
extern "C" int dust_octree_set_timing(dust_octree *o, int on) {
  if (!o) return DUST_ERR_BAD_ARG;
  o->timing = on != 0;
  return DUST_OK;
}

// ================================================================== kernels
__global__ void k_bin(int n, const double *__restrict__ cen, TreeGeom G,
                      uint32_t *__restrict__ keys, uint32_t *__restrict__ vals,
                      uint32_t *__restrict__ cnt, int *__restrict__ err) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  int ll = G.ll;
  double csize = G.csize[ll];
  int idx[3];
  bool bad = false;
  for (int d = 0; d < 3; ++d) {
    // idx = ceiling((cen - xmin)/csize) (mod_octree.f90:754)
    double c = ceil((cen[3 * t + d] - G.xmin[d]) / csize);
    if (!(c >= 1.0 && c <= (double)G.ncl[ll][d])) {
      bad = true;
      idx[d] = 1;
    } else {
      idx[d] = (int)c;
    }
  }
  if (bad) {
    atomicMin(err, t);
    keys[t] = 0xffffffffu;
    vals[t] = (uint32_t)t;
    return;
  }
  uint32_t key = key_of(G, ll, idx[0] - 1, idx[1] - 1, idx[2] - 1);
  keys[t] = key;
  vals[t] = (uint32_t)t;
  atomicAdd(&cnt[key], 1u);
}

// sorted SoA particle block: x y z ax ay az sigma (n each)
__global__ void k_gather(int n, const uint32_t *__restrict__ perm,
                         const double *__restrict__ cen, const double *__restrict__ dir,
                         const double *__restrict__ mag, const double *__restrict__ rv,
                         double *__restrict__ P) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  uint32_t ip = perm[t];
  double m = mag[ip];
  for (int d = 0; d < 3; ++d) {
    P[(size_t)d * n + t] = cen[3 * (size_t)ip + d];
    P[(size_t)(3 + d) * n + t] = m * dir[3 * (size_t)ip + d];
  }
  P[(size_t)6 * n + t] = rv[ip];
}

__device__ inline uint32_t cell_lo(const TreeGeom &G, const uint32_t *cstart, int l,
                                   uint32_t key) {
  return cstart[key << (3 * (G.ll - l))];
}
__device__ inline uint32_t cell_hi(const TreeGeom &G, const uint32_t *cstart, int l,
                                   uint32_t key) {
  return cstart[(key + 1u) << (3 * (G.ll - l))];
}

__global__ void k_flags_fine(TreeGeom G, const uint32_t *__restrict__ cstart, int min_part,
                             uint8_t *__restrict__ flags) {
  uint32_t key = blockIdx.x * blockDim.x + threadIdx.x;
  int ll = G.ll;
  if (key >= G.ncell[ll]) return;
  int np = (int)(cstart[key + 1] - cstart[key]);
  flags[G.lev_off[ll] + key] = (np >= min_part || ll == 1) ? (FL_LEAF | FL_ACTIVE) : 0;
}

// one upward pass of the leaf rule (mod_octree.f90:911-962) at level l
__global__ void k_flags_up(TreeGeom G, int l, const uint32_t *__restrict__ cstart,
                           int min_part, uint8_t *__restrict__ flags) {
  uint32_t key = blockIdx.x * blockDim.x + threadIdx.x;
  if (key >= G.ncell[l]) return;
  uint8_t *ch = flags + G.lev_off[l + 1] + 8u * key;
  bool got = false;
  uint8_t f[8];
  for (int c = 0; c < 8; ++c) {
    f[c] = ch[c];
    if (f[c] & (FL_LEAF | FL_BRANCH)) got = true;
  }
  if (got) {
    for (int c = 0; c < 8; ++c)
      if (!(f[c] & (FL_LEAF | FL_BRANCH))) ch[c] = FL_LEAF | FL_ACTIVE;
    flags[G.lev_off[l] + key] = FL_BRANCH | FL_ACTIVE;
  } else {
    for (int c = 0; c < 8; ++c) ch[c] = 0;
    int np = (int)(cell_hi(G, cstart, l, key) - cell_lo(G, cstart, l, key));
    flags[G.lev_off[l] + key] = (np >= min_part || l == 1) ? (FL_LEAF | FL_ACTIVE) : 0;
  }
}

// Evaluation points (panel centres) sorted into the tree as sort_particles
// sorts the panels (mod_octree.f90:776-799): the leaf above each point's
// finest cell gets FL_PTS, so that an empty leaf that holds a point still
// gets its local expansion (the particles' own M2L skips empty targets).  A
// point outside the box records its index in *err.
__global__ void k_mark_points(TreeGeom G, int npts, const double *__restrict__ pts,
                              uint8_t *__restrict__ flags, int *err) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= npts) return;
  const int ll = G.ll;
  int idx[3];
  for (int c = 0; c < 3; ++c) {
    idx[c] = (int)ceil((pts[3 * (size_t)q + c] - G.xmin[c]) / G.csize[ll]) - 1;
    if (idx[c] < 0 || idx[c] >= G.ncl[ll][c]) {
      atomicMin(err, q);
      return;
    }
  }
  for (int lv = 1; lv <= ll; ++lv) {
    const int sh = ll - lv;
    uint8_t *f = flags + G.lev_off[lv] + key_of(G, lv, idx[0] >> sh, idx[1] >> sh, idx[2] >> sh);
    if (*f & FL_LEAF) {
      *f = *f | FL_PTS;  // every writer stores the same value
      return;
    }
  }
}

__global__ void k_indicators(uint32_t ntot, const uint8_t *__restrict__ flags,
                             uint32_t *__restrict__ ia, uint32_t *__restrict__ il) {
  uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c > ntot) return;
  if (c == ntot) {
    ia[c] = 0;
    il[c] = 0;
    return;
  }
  uint8_t f = flags[c];
  ia[c] = (f & FL_ACTIVE) ? 1u : 0u;
  il[c] = (f & FL_LEAF) ? 1u : 0u;
}

__global__ void k_compact(TreeGeom G, uint32_t ntot, const uint8_t *__restrict__ flags,
                          const uint32_t *__restrict__ cidx,
                          const uint32_t *__restrict__ lidx, uint32_t *__restrict__ act_key,
                          uint8_t *__restrict__ act_lev, uint32_t *__restrict__ leaf_ci) {
  uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ntot) return;
  uint8_t f = flags[c];
  if (!(f & FL_ACTIVE)) return;
  int l = 1;
  while (l < G.ll && c >= G.lev_off[l + 1]) ++l;
  uint32_t ci = cidx[c];
  act_key[ci] = c - G.lev_off[l];
  act_lev[ci] = (uint8_t)l;
  if (f & FL_LEAF) leaf_ci[lidx[c]] = ci;
}

// per-level active offsets (scan values at level boundaries) + totals
__global__ void k_level_counts(TreeGeom G, const uint32_t *__restrict__ cidx,
                               const uint32_t *__restrict__ lidx, int64_t *__restrict__ out) {
  int l = threadIdx.x + 1;
  if (l <= G.ll + 1) out[l] = cidx[G.lev_off[l]];
  if (threadIdx.x == 0) out[0] = lidx[G.lev_off[G.ll + 1]];
}

__device__ inline double ipow_d(double x, int e) {
  double r = 1.0;
  for (int q = 0; q < e; ++q) r *= x;
  return r;
}

// P2M (leaf_M_multipole, mod_multipole.f90:224-251): one warp per leaf.
#define P2M_W 4
__global__ void __launch_bounds__(P2M_W * 32) k_p2m(FmmDev d) {
  // one warp per leaf: the leaf's particles in chunks of 32 in the warp's
  // shared memory, lanes over the output coefficients m (32 at a time); each
  // coefficient sums its particles in the same order as a serial loop
  __shared__ double sh[P2M_W][6][32];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t leaf = blockIdx.x * P2M_W + w;
  if (leaf >= d.n_leaves) return;  // warp-uniform
  uint32_t ci = d.leaf_ci[leaf];
  int l = d.act_lev[ci];
  uint32_t key = d.act_key[ci];
  int ci_, cj, ck;
  cart_of_key(d.G, l, key, ci_, cj, ck);
  double c[3];
  cell_center(d.G, l, ci_, cj, ck, c);
  uint32_t lo = cell_lo(d.G, d.cstart, l, key), hi = cell_hi(d.G, d.cstart, l, key);
  if (hi == lo) return;  // empty leaf: a = 0 (block zeroed before the pass)
  const size_t n = d.n;
  double(*sp)[32] = sh[w];
  for (int m0 = 0; m0 < d.nm; m0 += 32) {
    const int m = m0 + lane;
    int mi = 0, mj = 0, mk = 0;
    if (m < d.nm) mono_exp(m, mi, mj, mk);
    double ax = 0, ay = 0, az = 0;
    for (uint32_t s0 = lo; s0 < hi; s0 += 32) {
      const int cnt = min((int)(hi - s0), 32);
      __syncwarp();
      if (lane < cnt) {
        const uint32_t s = s0 + lane;
        sp[0][lane] = d.P[s] - c[0];
        sp[1][lane] = d.P[n + s] - c[1];
        sp[2][lane] = d.P[2 * n + s] - c[2];
        sp[3][lane] = d.P[3 * n + s];
        sp[4][lane] = d.P[4 * n + s];
        sp[5][lane] = d.P[5 * n + s];
      }
      __syncwarp();
      if (m < d.nm)
        for (int t = 0; t < cnt; ++t) {
          double pr = ipow_d(sp[0][t], mi) * ipow_d(sp[1][t], mj) * ipow_d(sp[2][t], mk);
          ax += pr * sp[3][t];
          ay += pr * sp[4][t];
          az += pr * sp[5][t];
        }
    }
    if (m < d.nm) {
      double *a = d.A + (size_t)ci * 3 * d.nm;
      a[3 * m] = ax;
      a[3 * m + 1] = ay;
      a[3 * m + 2] = az;
    }
  }
}

__device__ inline double binom_d(int n, int k) {
  double r = 1.0;
  for (int q = 1; q <= k; ++q) r = r * (double)(n - k + q) / (double)q;
  return r;
}

// M2M (mod_multipole.f90:256-278) into the active branch cells of level l.
__global__ void k_m2m(FmmDev d, int l, uint32_t act_lo) {
  uint32_t ci = act_lo + blockIdx.x;
  uint32_t key = d.act_key[ci];
  if (!(d.flags[d.G.lev_off[l] + key] & FL_BRANCH)) return;
  int m = threadIdx.x;
  if (m >= d.nm) return;
  int i, j, k;
  cart_of_key(d.G, l, key, i, j, k);
  double cp[3];
  cell_center(d.G, l, i, j, k, cp);
  int mi, mj, mk;
  mono_exp(m, mi, mj, mk);
  double acc[3] = {0, 0, 0};
  for (int ch = 0; ch < 8; ++ch) {
    uint32_t ckey = 8u * key + (uint32_t)ch;
    uint32_t cc = d.cidx[d.G.lev_off[l + 1] + ckey];
    int ii, jj, kk;
    cart_of_key(d.G, l + 1, ckey, ii, jj, kk);
    double cc3[3];
    cell_center(d.G, l + 1, ii, jj, kk, cc3);
    double dx = cc3[0] - cp[0], dy = cc3[1] - cp[1], dz = cc3[2] - cp[2];
    const double *a = d.A + (size_t)cc * 3 * d.nm;
    for (int ks = 0; ks <= mk; ++ks)
      for (int js = 0; js <= mj; ++js)
        for (int is = 0; is <= mi; ++is) {
          int s = mono_idx(is, js, ks);
          double w = binom_d(mi, is) * binom_d(mj, js) * binom_d(mk, ks) *
                     (ipow_d(dx, mi - is) * ipow_d(dy, mj - js) * ipow_d(dz, mk - ks));
          acc[0] += w * a[3 * s];
          acc[1] += w * a[3 * s + 1];
          acc[2] += w * a[3 * s + 2];
        }
  }
  double *ap = d.A + (size_t)ci * 3 * d.nm;
  ap[3 * m] = acc[0];
  ap[3 * m + 1] = acc[1];
  ap[3 * m + 2] = acc[2];
}

// ------------------------------------------------ M2M / L2L from tables
// The child-parent displacement is (+-delta, +-delta, +-delta), delta = half
// the child's cell size, with the signs given by the child's octant.  So the
// weights of M2M_multipole (mod_multipole.f90:256-278)
//   a_par(m) += sum_{s <= m} C(m,s) d^(m-s) a_child(s)
// and of L2L_multipole (:360-384)
//   b_child(m) += sum_{s >= m, |s| <= p} C(s,m) d^(s-m) b_par(s)
// are per level the same up to the sign (-1)^(sum of the exponents along the
// axes where d < 0).  The host lists, per output m, the terms (s, exponent,
// unsigned weight); the kernels apply the octant's sign.
struct ShiftTerm {
  double w;
  uint16_t s;
  uint8_t ex, ey, ez, pad[3];
};

__device__ __forceinline__ double shift_w(const ShiftTerm &t, uint32_t oct) {
  const int par = ((oct & 1u) ? 0 : t.ex) + ((oct & 2u) ? 0 : t.ey) + ((oct & 4u) ? 0 : t.ez);
  return (par & 1) ? -t.w : t.w;
}

#define SH_T 128
#define SH_W (SH_T / 32)
// M2M into the active branch cells of level l: one warp per parent, lanes
// over the output coefficient m; terms and offsets staged in shared memory,
// and each warp stages its parent's 8 children's coefficients (missing
// children as zeros) before the term loops
__global__ void __launch_bounds__(SH_T) k_m2m_t(FmmDev d, int l, uint32_t act_lo, uint32_t na,
                                                const ShiftTerm *terms, const int *off, int nterm) {
  extern __shared__ __align__(16) unsigned char shm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int w3 = 3 * d.nm;
  double *sa = (double *)shm + (size_t)warp * 8 * w3;  // [8][3 nm]
  ShiftTerm *st = (ShiftTerm *)((double *)shm + (size_t)SH_W * 8 * w3);
  int *so = (int *)(st + nterm);
  for (int e = threadIdx.x; e < nterm; e += SH_T) st[e] = terms[e];
  for (int e = threadIdx.x; e <= d.nm; e += SH_T) so[e] = off[e];
  __syncthreads();
  for (uint32_t c = blockIdx.x * SH_W + warp; c < na; c += gridDim.x * SH_W) {
    const uint32_t ci = act_lo + c;
    const uint32_t key = d.act_key[ci];
    if (!(d.flags[d.G.lev_off[l] + key] & FL_BRANCH)) continue;
    __syncwarp();
    for (int ch = 0; ch < 8; ++ch) {
      const uint32_t cc = d.cidx[d.G.lev_off[l + 1] + 8u * key + (uint32_t)ch];
      const double *a = d.A + (size_t)cc * w3;
      for (int e = lane; e < w3; e += 32) sa[ch * w3 + e] = a[e];
    }
    __syncwarp();
    for (int m = lane; m < d.nm; m += 32) {
      double acc[3] = {0, 0, 0};
      for (int ch = 0; ch < 8; ++ch) {
        const double *a = sa + ch * w3;
        for (int t = so[m]; t < so[m + 1]; ++t) {
          const double w = shift_w(st[t], (uint32_t)ch);
          const int s3 = 3 * st[t].s;
          acc[0] += w * a[s3];
          acc[1] += w * a[s3 + 1];
          acc[2] += w * a[s3 + 2];
        }
      }
      double *ap = d.A + (size_t)ci * w3;
      ap[3 * m] = acc[0];
      ap[3 * m + 1] = acc[1];
      ap[3 * m + 2] = acc[2];
    }
  }
}

// L2L into the active cells of level l (>= 2) from their parents: one warp
// per parent (an active branch cell of level l - 1), lanes over the output
// coefficient m.  The 8 children's weights differ only in sign (the octant's
// parity of the exponents), so each term's products are formed once and
// added to all 8 children's sums; the parent's b and g are staged in shared
// memory; only active children are written.  b terms (|s| <= p) and, with
// stretching, g terms (|s| <= p+1).
__device__ __forceinline__ void l2l_terms(const ShiftTerm *tt, int t0, int t1, const double *src,
                                          double (*acc)[3]) {
#pragma unroll
  for (int ch = 0; ch < 8; ++ch) acc[ch][0] = acc[ch][1] = acc[ch][2] = 0.0;
  for (int t = t0; t < t1; ++t) {
    const ShiftTerm tm = tt[t];
    const int s3 = 3 * tm.s;
    const double v0 = tm.w * src[s3], v1 = tm.w * src[s3 + 1], v2 = tm.w * src[s3 + 2];
    const unsigned px = tm.ex & 1u, py = tm.ey & 1u, pz = tm.ez & 1u;
#pragma unroll
    for (int ch = 0; ch < 8; ++ch) {
      // sign of shift_w for octant ch
      const unsigned neg = ((ch & 1) ? 0u : px) ^ ((ch & 2) ? 0u : py) ^ ((ch & 4) ? 0u : pz);
      if (neg) {
        acc[ch][0] -= v0, acc[ch][1] -= v1, acc[ch][2] -= v2;
      } else {
        acc[ch][0] += v0, acc[ch][1] += v1, acc[ch][2] += v2;
      }
    }
  }
}

__global__ void __launch_bounds__(SH_T) k_l2l_t(FmmDev d, int l, uint32_t act_lo, uint32_t na,
                                                const ShiftTerm *tb, const int *ob, int ntb,
                                                const ShiftTerm *tg, const int *og, int ntg) {
  extern __shared__ __align__(16) unsigned char shm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wb = 3 * d.nm, wg = ntg > 0 ? 3 * d.nm1 : 0;
  double *sbp = (double *)shm + (size_t)warp * (wb + wg);  // parent's b, then g
  double *sgp = sbp + wb;
  ShiftTerm *sb = (ShiftTerm *)((double *)shm + (size_t)SH_W * (wb + wg));
  ShiftTerm *sg = sb + ntb;
  int *sob = (int *)(sg + ntg);
  int *sog = sob + d.nm + 1;
  for (int e = threadIdx.x; e < ntb; e += SH_T) sb[e] = tb[e];
  for (int e = threadIdx.x; e < ntg; e += SH_T) sg[e] = tg[e];
  for (int e = threadIdx.x; e <= d.nm; e += SH_T) sob[e] = ob[e];
  for (int e = threadIdx.x; e <= d.nm1 && ntg > 0; e += SH_T) sog[e] = og[e];
  __syncthreads();
  // act_lo / na: the active cells of level l - 1 (the candidate parents)
  for (uint32_t c = blockIdx.x * SH_W + warp; c < na; c += gridDim.x * SH_W) {
    const uint32_t pc = act_lo + c;
    const uint32_t key = d.act_key[pc];
    if (!(d.flags[d.G.lev_off[l - 1] + key] & FL_BRANCH)) continue;
    uint32_t cc[8];
    unsigned live = 0;
#pragma unroll
    for (int ch = 0; ch < 8; ++ch) {
      const uint32_t ck = 8u * key + (uint32_t)ch;
      if (d.flags[d.G.lev_off[l] + ck] & FL_ACTIVE) live |= 1u << ch;
      cc[ch] = d.cidx[d.G.lev_off[l] + ck];
    }
    if (!live) continue;
    __syncwarp();
    const double *bp = d.B + (size_t)pc * wb;
    for (int e = lane; e < wb; e += 32) sbp[e] = bp[e];
    if (wg > 0) {
      const double *gp = d.Gx + (size_t)pc * wg;
      for (int e = lane; e < wg; e += 32) sgp[e] = gp[e];
    }
    __syncwarp();
    double acc[8][3];
    for (int m = lane; m < d.nm; m += 32) {
      l2l_terms(sb, sob[m], sob[m + 1], sbp, acc);
#pragma unroll
      for (int ch = 0; ch < 8; ++ch)
        if ((live >> ch) & 1u) {
          double *b = d.B + (size_t)cc[ch] * wb + 3 * m;
          b[0] += acc[ch][0], b[1] += acc[ch][1], b[2] += acc[ch][2];
        }
    }
    if (wg > 0) {
      for (int m = lane; m < d.nm1; m += 32) {
        l2l_terms(sg, sog[m], sog[m + 1], sgp, acc);
#pragma unroll
        for (int ch = 0; ch < 8; ++ch)
          if ((live >> ch) & 1u) {
            double *g = d.Gx + (size_t)cc[ch] * wg + 3 * m;
            g[0] += acc[ch][0], g[1] += acc[ch][1], g[2] += acc[ch][2];
          }
      }
    }
  }
}

static double binom_h(int n, int k) {
  double r = 1.0;
  for (int q = 1; q <= k; ++q) r = r * (double)(n - k + q) / (double)q;
  return r;
}

// term lists of one shift: up = false: s <= m (M2M, deg <= p); up = true:
// s >= m with |s| <= q (L2L of a degree-q expansion)
static void shift_terms(int nout, int q, bool up, double delta, std::vector<ShiftTerm> &t,
                        std::vector<int> &off) {
  t.clear();
  off.assign(1, 0);
  for (int m = 0; m < nout; ++m) {
    int mi, mj, mk;
    mono_exp(m, mi, mj, mk);
    for (int s = 0; s < n_mon(q); ++s) {
      int si, sj, sk;
      mono_exp(s, si, sj, sk);
      int ex, ey, ez;
      double w;
      if (!up) {
        if (si > mi || sj > mj || sk > mk) continue;
        ex = mi - si;
        ey = mj - sj;
        ez = mk - sk;
        w = binom_h(mi, si) * binom_h(mj, sj) * binom_h(mk, sk);
      } else {
        if (si < mi || sj < mj || sk < mk) continue;
        ex = si - mi;
        ey = sj - mj;
        ez = sk - mk;
        w = binom_h(si, mi) * binom_h(sj, mj) * binom_h(sk, mk);
      }
      double dp = 1.0;
      for (int e = 0; e < ex + ey + ez; ++e) dp *= delta;
      ShiftTerm x;
      memset(&x, 0, sizeof(x));
      x.w = w * dp;
      x.s = (uint16_t)s;
      x.ex = (uint8_t)ex;
      x.ey = (uint8_t)ey;
      x.ez = (uint8_t)ez;
      t.push_back(x);
    }
    off.push_back((int)t.size());
  }
}

// per level l: [0] M2M into level l, [1] L2L b into level l, [2] L2L g
static int build_shift_tables(dust_octree *o) {
  std::vector<char> blob;
  auto put = [&](const void *p, size_t n) {
    size_t at = (blob.size() + 15) / 16 * 16;
    blob.resize(at + n);
    memcpy(blob.data() + at, p, n);
    return at;
  };
  std::vector<ShiftTerm> t;
  std::vector<int> off;
  size_t at_t[DUST_MAXLEV + 1][3], at_o[DUST_MAXLEV + 1][3];
  for (int l = 1; l <= o->G.ll; ++l)
    for (int k = 0; k < 3; ++k) {
      o->shift_n[l][k] = 0;
      at_t[l][k] = at_o[l][k] = 0;
      if (k == 0 && l >= o->G.ll) continue;
      if (k > 0 && l < 2) continue;
      if (k == 0)
        shift_terms(o->nm, o->p, false, 0.5 * o->G.csize[l + 1], t, off);
      else if (k == 1)
        shift_terms(o->nm, o->p, true, 0.5 * o->G.csize[l], t, off);
      else
        shift_terms(o->nm1, o->p + 1, true, 0.5 * o->G.csize[l], t, off);
      o->shift_n[l][k] = (int)t.size();
      at_t[l][k] = put(t.data(), t.size() * sizeof(ShiftTerm));
      at_o[l][k] = put(off.data(), off.size() * sizeof(int));
    }
  DUST_TRY(devbuf_grow(o->shift, blob.size() + 16));
  DUST_CUDA(cudaMemcpy(o->shift.p, blob.data(), blob.size(), cudaMemcpyHostToDevice));
  for (int l = 1; l <= o->G.ll; ++l)
    for (int k = 0; k < 3; ++k) {
      o->shift_t[l][k] = (const char *)o->shift.p + at_t[l][k];
      o->shift_o[l][k] = (const char *)o->shift.p + at_o[l][k];
    }
  return DUST_OK;
}

static unsigned shift_grid(int64_t na) {
  int64_t w = (na + SH_T / 32 - 1) / (SH_T / 32);
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(w, 148 * 16));
}

// M2L (mod_multipole.f90:282-356): one CTA per active target cell of level
// l.  Evaluates g(m') = (-1)^|m'| / m'! sum_n Dhat(m'+n) x ahat(n) for
// |m'| <= p+1 (|m'| <= p without stretching), ahat(n) = a(n)/n!, and adds g
// into the cell's g and (|m'| <= p) b.
__global__ void k_m2l(FmmDev d, int l, uint32_t act_lo) {
  extern __shared__ double sh[];
  __shared__ int s_src[224];
  __shared__ int s_tab[224];
  __shared__ int s_n;
  double *s_a = sh;  // 3*nm
  uint32_t ci = act_lo + blockIdx.x;
  uint32_t key = d.act_key[ci];
  // an empty target cell is a leaf without particles: its local expansion
  // is evaluated only when points were sorted into it (and it has no
  // children to pass it to)
  if (cell_hi(d.G, d.cstart, l, key) == cell_lo(d.G, d.cstart, l, key) &&
      !(d.flags[d.G.lev_off[l] + key] & FL_PTS))
    return;
  int i, j, k;
  cart_of_key(d.G, l, key, i, j, k);
  const int nm = d.nm;
  const int nout = d.use_vs ? d.nm1 : d.nm;
  const int Lx = d.kdlen[l][0], Ly = d.kdlen[l][1], Lz = d.kdlen[l][2];
  if (threadIdx.x == 0) s_n = 0;
  __syncthreads();
  // interaction list (mod_octree.f90:420-476): children of the parent's 26
  // neighbours that are not adjacent, active sources only.
  const uint32_t lo_l = d.G.lev_off[l];
  if (l >= 2) {
    int pi_ = i >> 1, pj = j >> 1, pk = k >> 1;
    for (int t = threadIdx.x; t < 27 * 8; t += blockDim.x) {
      int nb = t >> 3, ch = t & 7;
      int di = nb % 3 - 1, dj = (nb / 3) % 3 - 1, dk = nb / 9 - 1;
      if (di == 0 && dj == 0 && dk == 0) continue;
      if (!cart_in(d.G, l - 1, pi_ + di, pj + dj, pk + dk)) continue;
      int si = 2 * (pi_ + di) + (ch & 1), sj = 2 * (pj + dj) + ((ch >> 1) & 1),
          sk = 2 * (pk + dk) + ((ch >> 2) & 1);
      if (abs(si - i) <= 1 && abs(sj - j) <= 1 && abs(sk - k) <= 1) continue;
      uint32_t skey = key_of(d.G, l, si, sj, sk);
      if (!(d.flags[lo_l + skey] & FL_ACTIVE)) continue;
      // an empty source has a = 0: adding it changes nothing
      if (cell_hi(d.G, d.cstart, l, skey) == cell_lo(d.G, d.cstart, l, skey)) continue;
      int q = atomicAdd(&s_n, 1);
      s_src[q] = (int)d.cidx[lo_l + skey];
      s_tab[q] = (si - i + Lx) + (2 * Lx + 1) * ((sj - j + Ly) + (2 * Ly + 1) * (sk - k + Lz));
    }
  }
  __syncthreads();
  int nsrc = s_n;
  int nlev1 = (l == 1) ? (int)d.G.ncell[1] : 0;
  if (threadIdx.x == 0 && d.counters) atomicAdd((unsigned long long *)d.counters, (unsigned long long)nsrc);
  int mo = threadIdx.x;  // output monomial
  int oi = 0, oj = 0, ok = 0;
  if (mo < nout) mono_exp(mo, oi, oj, ok);
  double acc[3] = {0, 0, 0};
  const uint16_t *isum = d.idxsum;
  for (int q = 0; q < nsrc + nlev1; ++q) {
    int src, tab;
    if (q < nsrc) {
      src = s_src[q];
      tab = s_tab[q];
    } else {
      // level 1: every non-adjacent level-1 cell
      uint32_t sk1 = (uint32_t)(q - nsrc);
      int si, sj, sk;
      cart_of_key(d.G, 1, sk1, si, sj, sk);
      if (abs(si - i) <= 1 && abs(sj - j) <= 1 && abs(sk - k) <= 1) continue;
      if (!(d.flags[lo_l + sk1] & FL_ACTIVE)) continue;
      if (cell_hi(d.G, d.cstart, 1, sk1) == cell_lo(d.G, d.cstart, 1, sk1)) continue;
      src = (int)d.cidx[lo_l + sk1];
      tab = (si - i + Lx) + (2 * Lx + 1) * ((sj - j + Ly) + (2 * Ly + 1) * (sk - k + Lz));
    }
    __syncthreads();
    const double *a = d.A + (size_t)src * 3 * nm;
    for (int t = threadIdx.x; t < 3 * nm; t += blockDim.x) s_a[t] = a[t] * d.inv_fact[t / 3];
    __syncthreads();
    if (mo < nout) {
      const double *D = d.dtab[l] + (size_t)tab * d.nD * 3;
      for (int nn = 0; nn < nm; ++nn) {
        int qd = isum[(size_t)nn * d.nm1 + mo];
        double Dx = __ldg(D + 3 * qd), Dy = __ldg(D + 3 * qd + 1), Dz = __ldg(D + 3 * qd + 2);
        double ax = s_a[3 * nn], ay = s_a[3 * nn + 1], az = s_a[3 * nn + 2];
        acc[0] += Dy * az - Dz * ay;
        acc[1] += Dz * ax - Dx * az;
        acc[2] += Dx * ay - Dy * ax;
      }
    }
  }
  if (mo < nout && (nsrc + nlev1) > 0) {
    double sc = (((oi + oj + ok) & 1) ? -1.0 : 1.0) * d.inv_fact[mo];
    if (d.use_vs) {
      double *g = d.Gx + (size_t)ci * 3 * d.nm1;
      for (int e = 0; e < 3; ++e) g[3 * mo + e] += sc * acc[e];
    }
    if (mo < nm) {
      double *b = d.B + (size_t)ci * 3 * nm;
      for (int e = 0; e < 3; ++e) b[3 * mo + e] += sc * acc[e];
    }
  }
}

// L2L (mod_multipole.f90:360-384) into the active cells of level l from
// their parents: b truncated at degree p, g at degree p+1.
__global__ void k_l2l(FmmDev d, int l, uint32_t act_lo) {
  uint32_t ci = act_lo + blockIdx.x;
  uint32_t key = d.act_key[ci];
  uint32_t pkey = key >> 3;
  uint32_t pc = d.cidx[d.G.lev_off[l - 1] + pkey];
  int i, j, k, pi_, pj, pk;
  cart_of_key(d.G, l, key, i, j, k);
  cart_of_key(d.G, l - 1, pkey, pi_, pj, pk);
  double c[3], cp[3];
  cell_center(d.G, l, i, j, k, c);
  cell_center(d.G, l - 1, pi_, pj, pk, cp);
  double dx = c[0] - cp[0], dy = c[1] - cp[1], dz = c[2] - cp[2];
  int m = threadIdx.x;
  int p = d.p;
  if (m < d.nm) {
    int mi, mj, mk;
    mono_exp(m, mi, mj, mk);
    const double *bp = d.B + (size_t)pc * 3 * d.nm;
    double acc[3] = {0, 0, 0};
    for (int ks = mk; ks <= p; ++ks)
      for (int js = mj; js <= p - ks; ++js)
        for (int is = mi; is <= p - ks - js; ++is) {
          int s = mono_idx(is, js, ks);
          double w = binom_d(is, mi) * binom_d(js, mj) * binom_d(ks, mk) *
                     (ipow_d(dx, is - mi) * ipow_d(dy, js - mj) * ipow_d(dz, ks - mk));
          acc[0] += w * bp[3 * s];
          acc[1] += w * bp[3 * s + 1];
          acc[2] += w * bp[3 * s + 2];
        }
    double *b = d.B + (size_t)ci * 3 * d.nm;
    for (int e = 0; e < 3; ++e) b[3 * m + e] += acc[e];
  }
  if (d.use_vs && m < d.nm1) {
    int mi, mj, mk;
    mono_exp(m, mi, mj, mk);
    const double *gp = d.Gx + (size_t)pc * 3 * d.nm1;
    double acc[3] = {0, 0, 0};
    int q = p + 1;
    for (int ks = mk; ks <= q; ++ks)
      for (int js = mj; js <= q - ks; ++js)
        for (int is = mi; is <= q - ks - js; ++is) {
          int s = mono_idx(is, js, ks);
          double w = binom_d(is, mi) * binom_d(js, mj) * binom_d(ks, mk) *
                     (ipow_d(dx, is - mi) * ipow_d(dy, js - mj) * ipow_d(dz, ks - mk));
          acc[0] += w * gp[3 * s];
          acc[1] += w * gp[3 * s + 1];
          acc[2] += w * gp[3 * s + 2];
        }
    double *g = d.Gx + (size_t)ci * 3 * d.nm1;
    for (int e = 0; e < 3; ++e) g[3 * m + e] += acc[e];
  }
}

// ------------------------------------------------------------- L2P + P2P
struct P2PAcc {
  double v[3], s[3], r[3], f[3];
};

// x^-1/2 for a normal FP32-range x > 0: the FP32 approximation refined by
// one second-order Newton-Raphson (Householder) step in FP64.  With
// y0 = x^-1/2 (1 + d) and e = 1 - x y0^2, y = y0 (1 + e/2 + 3 e^2/8) has
// relative error O(d^3), below the FP64 rounding for |d| < 2^-21.
__device__ __forceinline__ double p2p_rsqrt(double x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"((float)x));
  const double y = (double)r;
  const double e = fma(-x * y, y, 1.0);
  return fma(y * e, fma(0.375, e, 0.5), y);
}

// One source q acting on target p: the reference's compute_vel,
// compute_stretch, compute_rotu and compute_diffusion of source q
// (mod_vortpart.f90:139-336), 4*pi factors applied by the caller.  s2 and
// is2 are the source's r_v^2 and 1 / r_v^2.
template <bool VS, bool DF, bool VD>
__device__ __forceinline__ void p2p_pair(const double *tp, const double *ta, double qx,
                                         double qy, double qz, double qax, double qay,
                                         double qaz, double s2, double is2, P2PAcc &A) {
  double dx = tp[0] - qx, dy = tp[1] - qy, dz = tp[2] - qz;
  double r2 = dx * dx + dy * dy + dz * dz;
  double inv = p2p_rsqrt(r2 + s2);
  double inv2 = inv * inv;
  double c = -inv2 * inv;        // -1/rho^3
  double dd = -3.0 * c * inv2;   // 3/rho^5
  double cx = dy * qaz - dz * qay, cy = dz * qax - dx * qaz, cz = dx * qay - dy * qax;
  A.v[0] += c * cx;
  A.v[1] += c * cy;
  A.v[2] += c * cz;
  if (VS) {
    double vx = ta[1] * qaz - ta[2] * qay, vy = ta[2] * qax - ta[0] * qaz,
           vz = ta[0] * qay - ta[1] * qax;
    double dv = dx * vx + dy * vy + dz * vz;
    A.s[0] -= c * vx + dd * dx * dv;
    A.s[1] -= c * vy + dd * dy * dv;
    A.s[2] -= c * vz + dd * dz * dv;
    if (DF) {
      // dist x (dist x aq) = dist (dist.aq) - aq r^2
      double da = dx * qax + dy * qay + dz * qaz;
      A.r[0] += -2.0 * c * qax + dd * (dx * da - qax * r2);
      A.r[1] += -2.0 * c * qay + dd * (dy * da - qay * r2);
      A.r[2] += -2.0 * c * qaz + dd * (dz * da - qaz * r2);
    }
  }
  if (VD) {
    // (1/s^2) vol (aq - ap) eta, vol = 4/3 pi s^3, eta = 105/(8 pi)/s^3/(1+r^2/s^2)^4.5
    double t = r2 * is2 + 1.0;
    double rt = p2p_rsqrt(t);
    double rt2 = rt * rt, rt4 = rt2 * rt2;
    double w = 17.5 * is2 * (rt4 * rt4 * rt);
    A.f[0] += w * (qax - ta[0]);
    A.f[1] += w * (qay - ta[1]);
    A.f[2] += w * (qaz - ta[2]);
  }
}

struct P2PAccF {
  float v[3], s[3], r[3], f[3];
};

// FP32 form of p2p_pair on coordinates relative to the leaf centre
template <bool VS, bool DF, bool VD>
__device__ __forceinline__ void p2p_pair_f(const float *tp, const float *ta, float qx, float qy,
                                           float qz, float qax, float qay, float qaz, float s2,
                                           float is2, P2PAccF &A) {
  float dx = tp[0] - qx, dy = tp[1] - qy, dz = tp[2] - qz;
  float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
  float inv = rsqrtf(r2 + s2);
  float inv2 = inv * inv;
  float c = -inv2 * inv;
  float dd = -3.0f * c * inv2;
  float cx = dy * qaz - dz * qay, cy = dz * qax - dx * qaz, cz = dx * qay - dy * qax;
  A.v[0] = fmaf(c, cx, A.v[0]);
  A.v[1] = fmaf(c, cy, A.v[1]);
  A.v[2] = fmaf(c, cz, A.v[2]);
  if (VS) {
    float vx = ta[1] * qaz - ta[2] * qay, vy = ta[2] * qax - ta[0] * qaz,
          vz = ta[0] * qay - ta[1] * qax;
    float dv = dx * vx + dy * vy + dz * vz;
    A.s[0] -= c * vx + dd * dx * dv;
    A.s[1] -= c * vy + dd * dy * dv;
    A.s[2] -= c * vz + dd * dz * dv;
    if (DF) {
      float da = dx * qax + dy * qay + dz * qaz;
      A.r[0] += -2.0f * c * qax + dd * (dx * da - qax * r2);
      A.r[1] += -2.0f * c * qay + dd * (dy * da - qay * r2);
      A.r[2] += -2.0f * c * qaz + dd * (dz * da - qaz * r2);
    }
  }
  if (VD) {
    float t = fmaf(r2, is2, 1.0f);
    float rt = rsqrtf(t);
    float rt2 = rt * rt, rt4 = rt2 * rt2;
    float w = 17.5f * is2 * (rt4 * rt4 * rt);
    A.f[0] += w * (qax - ta[0]);
    A.f[1] += w * (qay - ta[1]);
    A.f[2] += w * (qaz - ta[2]);
  }
}

// L2P + P2P, one warp per leaf.  Leaves hold a few particles (6 on average
// in the 2M-particle full step), so a CTA per leaf would leave most lanes
// idle.  The warp lists the leaf's near field as particle ranges (the 26
// active same-level neighbours, the coarser leaf neighbours of every level
// above -- leaf_neigh, mod_octree.f90:964-988 -- and the leaf itself, at most
// 26 * DUST_MAXLEV + 1 ranges), then takes its targets 32 at a time: lanes
// are split into G = 32 / cnt groups of cnt lanes (one lane per target),
// lane (tl, grp) accumulates target tl over the sources u = grp mod G of
// each 32-source tile staged in the warp's own shared memory, and group 0
// adds the other groups' sums from shared memory.  A source is found from
// its position in the concatenated ranges by a binary search over the
// range prefix sums (walked forward tile by tile).
//   FP64: pairs by p2p_pair on absolute coordinates, summed in FP64.
//   FP32C (F32): pairs by p2p_pair_f on coordinates relative to the leaf
//   centre (differences formed in FP64, rounded once), FP32 partial sums of
//   up to 128 sources folded into FP64.
// L2P (mod_octree.f90:1171-1212) is FP64 in both.
#define P2W_WARPS 1  // one warp per CTA: leaves finish independently
#define P2W_TILE 32
#define P2W_MAXR (26 * DUST_MAXLEV + 4)
#define P2W_NV 8  // staged per source: x y z, alpha x y z, r_v^2, 1 / r_v^2
#define P2W_LQ 4  // levels whose near-field loads are issued together

template <bool VS, bool DF, bool VD, bool TV, bool F32>
__global__ void __launch_bounds__(P2W_WARPS * 32, 16) k_p2p_w(FmmDev d) {
  using R = typename std::conditional<F32, float, double>::type;
  __shared__ R s_src[P2W_WARPS][P2W_NV][P2W_TILE];
  __shared__ uint32_t s_sid[P2W_WARPS][P2W_TILE];
  __shared__ uint32_t s_rlo[P2W_WARPS][P2W_MAXR];
  __shared__ uint32_t s_rcum[P2W_WARPS][P2W_MAXR + 1];
  __shared__ double s_acc[P2W_WARPS][12][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t leaf = blockIdx.x * P2W_WARPS + w;
  if (leaf >= d.n_leaves) return;  // warp-uniform: no CTA-wide barriers below
  const uint32_t ci = d.leaf_ci[leaf];
  const int l = d.act_lev[ci];
  const uint32_t key = d.act_key[ci];
  int ci_, cj, ck;
  cart_of_key(d.G, l, key, ci_, cj, ck);
  double cc[3];
  cell_center(d.G, l, ci_, cj, ck, cc);
  const uint32_t lo = cell_lo(d.G, d.cstart, l, key), hi = cell_hi(d.G, d.cstart, l, key);
  if (hi == lo) return;
  uint32_t *rlo = s_rlo[w], *rcum = s_rcum[w];
  // near-field source ranges: same level first, then coarser levels.  The
  // flags and particle ranges of P2W_LQ levels are loaded without branches
  // (predicated on the neighbour lying in the box), so those loads are in
  // flight together rather than one dependent chain per level.
  int nr = 0;
  for (int lev0 = l; lev0 >= 1; lev0 -= P2W_LQ) {
    bool predq[P2W_LQ];
    uint32_t a0q[P2W_LQ], a1q[P2W_LQ];
#pragma unroll
    for (int q = 0; q < P2W_LQ; ++q) {
      const int lev = lev0 - q;
      const int sh = l - lev;
      const int ai = ci_ >> sh, aj = cj >> sh, ak = ck >> sh;
      const int di = lane % 3 - 1, dj = (lane / 3) % 3 - 1, dk = lane / 9 - 1;
      const bool ok = lev >= 1 && lane < 27 && lane != 13 &&
                      cart_in(d.G, lev, ai + di, aj + dj, ak + dk);
      const uint32_t nk = ok ? key_of(d.G, lev, ai + di, aj + dj, ak + dk) : 0u;
      const uint8_t f = ok ? d.flags[d.G.lev_off[lev] + nk] : (uint8_t)0;
      a0q[q] = ok ? cell_lo(d.G, d.cstart, lev, nk) : 0u;
      a1q[q] = ok ? cell_hi(d.G, d.cstart, lev, nk) : 0u;
      const bool want = (lev == l) ? (f & FL_ACTIVE) != 0 : (f & FL_LEAF) != 0;
      predq[q] = ok && want && a1q[q] > a0q[q];
    }
#pragma unroll
    for (int q = 0; q < P2W_LQ; ++q) {
      const unsigned msk = __ballot_sync(0xffffffffu, predq[q]);
      // 26 per level and l <= DUST_MAXLEV levels: the list cannot overflow
      if (predq[q] && nr + __popc(msk) < P2W_MAXR) {
        const int pos = nr + __popc(msk & ((1u << lane) - 1u));
        rlo[pos] = a0q[q];
        rcum[pos] = a1q[q] - a0q[q];
      }
      nr = min(nr + __popc(msk), P2W_MAXR - 1);
    }
  }
  __syncwarp();
  if (lane == 0) {
    rlo[nr] = lo;
    rcum[nr] = hi - lo;
    ++nr;
    uint32_t run = 0;
    for (int r = 0; r < nr; ++r) {
      const uint32_t len = rcum[r];
      rcum[r] = run;
      run += len;
    }
    rcum[nr] = run;
  }
  nr = __shfl_sync(0xffffffffu, nr, 0);  // lane 0 appended the own leaf
  __syncwarp();
  const uint32_t S = rcum[nr];
  const size_t n = d.n;
  const int nt = (int)(hi - lo), nm = d.nm, nm1 = d.nm1;
  if (lane == 0 && d.counters)
    atomicAdd((unsigned long long *)d.counters + 1, (unsigned long long)nt * (S - 1));
  const double k4pi = 1.0 / (4.0 * DUST_PI);
  const double *bl = d.B + (size_t)ci * 3 * nm, *gl = d.Gx + (size_t)ci * 3 * nm1;
  // L2P of one target (FP64): velocity and the gradient of the local field
  // (the monomials m0, m0 + ms, ... only: the caller splits the sum)
  auto l2p = [&](uint32_t ti, int m0, int ms, double *lv, double *g) {
    const double x = d.P[ti] - cc[0], y = d.P[n + ti] - cc[1], z = d.P[2 * n + ti] - cc[2];
    double px[DUST_MAXP + 1], py[DUST_MAXP + 1], pz[DUST_MAXP + 1];
    px[0] = py[0] = pz[0] = 1.0;
#pragma unroll
    for (int e = 1; e <= DUST_MAXP; ++e) {
      px[e] = px[e - 1] * x;
      py[e] = py[e - 1] * y;
      pz[e] = pz[e - 1] * z;
    }
    for (int e = 0; e < 3; ++e) lv[e] = 0.0;
    for (int e = 0; e < 9; ++e) g[e] = 0.0;
    for (int m = m0; m < nm; m += ms) {
      int mi, mj, mk;
      mono_exp(m, mi, mj, mk);
      const double pr = px[mi] * py[mj] * pz[mk];
      for (int e = 0; e < 3; ++e) lv[e] += __ldg(bl + 3 * m + e) * pr;
      if (VS) {
        const double *g0 = gl + 3 * mono_idx(mi + 1, mj, mk), *g1 = gl + 3 * mono_idx(mi, mj + 1, mk),
                     *g2 = gl + 3 * mono_idx(mi, mj, mk + 1);
        const double f0 = (mi + 1) * pr, f1 = (mj + 1) * pr, f2 = (mk + 1) * pr;
        for (int e = 0; e < 3; ++e) {
          g[0 + 3 * e] += f0 * __ldg(g0 + e);
          g[1 + 3 * e] += f1 * __ldg(g1 + e);
          g[2 + 3 * e] += f2 * __ldg(g2 + e);
        }
      }
    }
  };
  double ave_ros = 0.0;
  if (TV) {
    // leaf average of |sym(grad)|^2 from the local expansion (:1214-1230)
    double part = 0.0;
    for (int t = lane; t < nt; t += 32) {
      double lv[3], g[9];
      l2p(lo + t, 0, 1, lv, g);
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          const double sy = 0.5 * (g[a + 3 * b] + g[b + 3 * a]);
          part += sy * sy;
        }
    }
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    ave_ros = part / (double)nt;
  }
  R *fs = &s_src[w][0][0];
  double *acc = &s_acc[w][0][lane];  // this lane's 12 FP64 sums, stride 32
  for (int t0 = 0; t0 < nt; t0 += 32) {
    // G groups of cnt lanes (one lane per target) split the sources; lanes
    // beyond G * cnt idle
    const int cnt = min(32, nt - t0);
    const int TPR = cnt, G = 32 / TPR, tl = lane % TPR, grp = lane / TPR;
    const bool act = grp < G;
    const uint32_t ti = lo + t0 + (act ? tl : 0);
    R tp[3], ta[3];
    for (int q = 0; q < 3; ++q) {
      tp[q] = F32 ? (R)(d.P[(size_t)q * n + ti] - cc[q]) : (R)d.P[(size_t)q * n + ti];
      ta[q] = (R)d.P[(size_t)(3 + q) * n + ti];
    }
    // FP64 sums: in registers (FP64 pairs) or in shared memory (FP32C,
    // which keeps its registers for the FP32 partial sums)
    P2PAcc A;
    P2PAccF B;
    for (int e = 0; e < 3; ++e) {
      A.v[e] = A.s[e] = A.r[e] = A.f[e] = 0.0;
      B.v[e] = B.s[e] = B.r[e] = B.f[e] = 0.0f;
    }
    if (F32)
      for (int e = 0; e < 12; ++e) acc[32 * e] = 0.0;
    int since = 0;
    // the sources of the next tile are loaded into registers while the
    // current tile is evaluated; each lane's range index only moves forward
    // (source v = s0 + lane grows by the tile size)
    int ra = 0;
    double pf[7];
    uint32_t psid = 0;
    bool pv = false;
    auto fetch = [&](uint32_t v) {
      pv = v < S;
      if (pv) {
        while (ra + 1 < nr && rcum[ra + 1] <= v) ++ra;  // last r with rcum[r] <= v
        psid = rlo[ra] + (v - rcum[ra]);
#pragma unroll
        for (int q = 0; q < 7; ++q) pf[q] = d.P[(size_t)q * n + psid];
      }
    };
    fetch(lane);
    for (uint32_t s0 = 0; s0 < S; s0 += P2W_TILE) {
      __syncwarp();
      if (pv) {
        s_sid[w][lane] = psid;
        for (int q = 0; q < 3; ++q)
          fs[q * P2W_TILE + lane] = F32 ? (R)(pf[q] - cc[q]) : (R)pf[q];
        for (int q = 3; q < 6; ++q) fs[q * P2W_TILE + lane] = (R)pf[q];
        const double rv = pf[6];
        if constexpr (F32) {
          const float s2 = (float)rv * (float)rv;
          fs[6 * P2W_TILE + lane] = s2;
          fs[7 * P2W_TILE + lane] = VD ? __frcp_rn(s2) : 0.f;
        } else {
          const double s2 = rv * rv;
          fs[6 * P2W_TILE + lane] = s2;
          fs[7 * P2W_TILE + lane] = VD ? __drcp_rn(s2) : 0.0;
        }
      }
      __syncwarp();
      fetch(s0 + P2W_TILE + lane);
      const int m = (int)min((uint32_t)P2W_TILE, S - s0);
      if (act)
        for (int u = grp; u < m; u += G) {
          if (s_sid[w][u] == ti) continue;
          if constexpr (F32)
            p2p_pair_f<VS, DF, VD>(tp, ta, fs[u], fs[P2W_TILE + u], fs[2 * P2W_TILE + u],
                                   fs[3 * P2W_TILE + u], fs[4 * P2W_TILE + u],
                                   fs[5 * P2W_TILE + u], fs[6 * P2W_TILE + u],
                                   fs[7 * P2W_TILE + u], B);
          else
            p2p_pair<VS, DF, VD>(tp, ta, fs[u], fs[P2W_TILE + u], fs[2 * P2W_TILE + u],
                                 fs[3 * P2W_TILE + u], fs[4 * P2W_TILE + u],
                                 fs[5 * P2W_TILE + u], fs[6 * P2W_TILE + u],
                                 fs[7 * P2W_TILE + u], A);
        }
      if (F32 && (++since == 4 || s0 + P2W_TILE >= S)) {
        // FP32 partial sums of up to 128 sources folded into FP64
        since = 0;
        for (int e = 0; e < 3; ++e) {
          acc[32 * e] += (double)B.v[e];
          acc[32 * (3 + e)] += (double)B.s[e];
          acc[32 * (6 + e)] += (double)B.r[e];
          acc[32 * (9 + e)] += (double)B.f[e];
          B.v[e] = B.s[e] = B.r[e] = B.f[e] = 0.0f;
        }
      }
    }
    // combine the groups of each target (group 0's lane sums the others'
    // shared-memory sums)
    if (!F32)
      for (int e = 0; e < 3; ++e) {
        acc[32 * e] = A.v[e];
        acc[32 * (3 + e)] = A.s[e];
        acc[32 * (6 + e)] = A.r[e];
        acc[32 * (9 + e)] = A.f[e];
      }
    __syncwarp();
    double Q[12];
    for (int e = 0; e < 12; ++e) {
      Q[e] = acc[32 * e];
      if (grp == 0)
        for (int g = 1; g < G; ++g) Q[e] += acc[32 * e + g * TPR];
    }
    __syncwarp();
    // L2P (FP64) split over the groups: lane (tl, grp) sums the monomials
    // grp, grp + G, ... of its target; group 0 adds the other groups' parts
    double lv[3], g[9];
    if (act) {
      l2p(ti, grp, G, lv, g);
      for (int e = 0; e < 3; ++e) acc[32 * e] = lv[e];
      for (int e = 0; e < 9; ++e) acc[32 * (3 + e)] = g[e];
    }
    __syncwarp();
    if (act && grp == 0) {
      for (int q = 1; q < G; ++q) {
        for (int e = 0; e < 3; ++e) lv[e] += acc[32 * e + q * TPR];
        for (int e = 0; e < 9; ++e) g[e] += acc[32 * (3 + e) + q * TPR];
      }
      const double tad[3] = {d.P[3 * n + ti], d.P[4 * n + ti], d.P[5 * n + ti]};
      double ls[3] = {0, 0, 0}, lr[3] = {0, 0, 0};
      if (VS) {
        for (int e = 0; e < 3; ++e) ls[e] = tad[0] * g[e] + tad[1] * g[e + 3] + tad[2] * g[e + 6];
        if (DF) {
          lr[0] = g[1 + 6] - g[2 + 3];
          lr[1] = g[2 + 0] - g[0 + 6];
          lr[2] = g[0 + 3] - g[1 + 0];
        }
      }
      double nu = d.nu_inf;
      if (TV) {
        const double rv = d.P[6 * n + ti];
        nu += (0.11 * rv) * (0.11 * rv) * sqrt(2.0 * ave_ros);
      }
      for (int e = 0; e < 3; ++e) {
        d.out[(size_t)e * n + ti] = lv[e] + Q[e] * k4pi;
        d.out[(size_t)(3 + e) * n + ti] = ls[e] + Q[3 + e] * k4pi + (VD ? Q[9 + e] * nu : 0.0);
        d.out[(size_t)(6 + e) * n + ti] = lr[e] + Q[6 + e] * k4pi;
      }
    }
    __syncwarp();  // acc is reused by the next 32 targets
  }
}

// ======================================================== host orchestration
static inline unsigned nblk(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

static void fill_dev(dust_octree *o, FmmDev &d, int n) {
  memset(&d, 0, sizeof(d));
  d.G = o->G;
  d.n = (uint32_t)n;
  d.p = o->p;
  d.nm = o->nm;
  d.nm1 = o->nm1;
  d.nD = o->nD;
  d.use_vs = o->prm.vortstretch != 0;
  d.use_df = o->prm.divergence_filtering != 0;
  d.use_vd = o->prm.diffusion != 0;
  d.nu_inf = o->prm.nu_inf;
  for (int c = 0; c < 3; ++c) d.u_inf[c] = o->prm.u_inf[c];
  for (int l = 0; l <= DUST_MAXLEV; ++l) {
    d.dtab[l] = (const double *)o->dtab[l].p;
    for (int c = 0; c < 3; ++c) d.kdlen[l][c] = o->kdlen[l][c];
  }
  d.idxsum = (const uint16_t *)o->idxsum.p;
  // 1/m! of the multi-index m, for every monomial up to degree p+1
  for (int m = 0; m < o->nm1 && m < 224; ++m) {
    int i, j, k;
    mono_exp(m, i, j, k);
    double fi = 1, fj = 1, fk = 1;
    for (int q = 2; q <= i; ++q) fi *= q;
    for (int q = 2; q <= j; ++q) fj *= q;
    for (int q = 2; q <= k; ++q) fk *= q;
    d.inv_fact[m] = 1.0 / (fi * fj * fk);
  }
}

// Builds the tree of n device-resident particles and evaluates the FMM; the
// outputs stay in o->outs (sorted order) for the element pass.
int fmm_prepare_device(dust_octree *o, int n, const double *cen, const double *dir,
                       const double *mag, const double *rv, int n_pts, const double *pts,
                       cudaStream_t st) {
  TreeGeom &G = o->G;
  o->last_stream = st;
  const int ll = G.ll;
  const uint32_t nfine = G.ncell[ll];
  const uint32_t ntot = (uint32_t)o->ncell_tot;
  size_t N = (size_t)std::max(n, 1);
  DUST_TRY(grow(o->keys, N * 4));
  DUST_TRY(grow(o->keys_s, N * 4));
  DUST_TRY(grow(o->vals, N * 4));
  DUST_TRY(grow(o->perm, N * 4));
  DUST_TRY(grow(o->cnt, (size_t)(nfine + 1) * 4));
  DUST_TRY(grow(o->cstart, (size_t)(nfine + 1) * 4));
  DUST_TRY(grow(o->part, N * 7 * 8));
  DUST_TRY(grow(o->flags, (size_t)ntot + 1));
  DUST_TRY(grow(o->ind, (size_t)(ntot + 1) * 8));
  DUST_TRY(grow(o->cidx, (size_t)(ntot + 1) * 4));
  DUST_TRY(grow(o->lidx, (size_t)(ntot + 1) * 4));
  DUST_TRY(grow(o->small, 64 * 8));
  DUST_TRY(grow(o->outs, N * 9 * 8));
  uint32_t *keys = (uint32_t *)o->keys.p, *keys_s = (uint32_t *)o->keys_s.p;
  uint32_t *vals = (uint32_t *)o->vals.p, *perm = (uint32_t *)o->perm.p;
  uint32_t *cnt = (uint32_t *)o->cnt.p, *cstart = (uint32_t *)o->cstart.p;
  uint8_t *flags = (uint8_t *)o->flags.p;
  uint32_t *ia = (uint32_t *)o->ind.p, *il = ia + (ntot + 1);
  uint32_t *cidx = (uint32_t *)o->cidx.p, *lidx = (uint32_t *)o->lidx.p;
  int64_t *small = (int64_t *)o->small.p;
  int *err = (int *)(small + 40);

  o->kev_m2l = false;
  if (o->timing) cudaEventRecord(o->ev[0], st);
  DUST_CUDA(cudaMemsetAsync(cnt, 0, (size_t)(nfine + 1) * 4, st));
  int big = 0x7fffffff;
  DUST_CUDA(cudaMemcpyAsync(err, &big, sizeof(int), cudaMemcpyHostToDevice, st));
  if (n > 0) k_bin<<<nblk(n, 256), 256, 0, st>>>(n, cen, G, keys, vals, cnt, err);
  // radix sort (stable) by finest key; bits needed for the finest key
  int bits = 1;
  while (bits < 32 && (1ull << bits) < (uint64_t)nfine) ++bits;
  size_t tb1 = 0, tb2 = 0, tb3 = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tb1, keys, keys_s, vals, perm, n, 0, bits, st);
  cub::DeviceScan::ExclusiveSum(nullptr, tb2, cnt, cstart, (int)nfine + 1, st);
  cub::DeviceScan::ExclusiveSum(nullptr, tb3, ia, cidx, (int)ntot + 1, st);
  size_t tb = std::max(tb1, std::max(tb2, tb3));
  DUST_TRY(grow(o->cub_tmp, tb));
  if (n > 0) {
    DUST_CUDA(cub::DeviceRadixSort::SortPairs(o->cub_tmp.p, tb, keys, keys_s, vals, perm, n,
                                              0, bits, st));
  }
  DUST_CUDA(cub::DeviceScan::ExclusiveSum(o->cub_tmp.p, tb, cnt, cstart, (int)nfine + 1, st));
  double *P = (double *)o->part.p;
  if (n > 0) k_gather<<<nblk(n, 256), 256, 0, st>>>(n, perm, cen, dir, mag, rv, P);
  // leaf rule
  k_flags_fine<<<nblk(nfine, 256), 256, 0, st>>>(G, cstart, o->prm.min_octree_part, flags);
  for (int l = ll - 1; l >= 1; --l)
    k_flags_up<<<nblk(G.ncell[l], 256), 256, 0, st>>>(G, l, cstart, o->prm.min_octree_part,
                                                      flags);
  int *perr = (int *)(small + 41);
  DUST_CUDA(cudaMemcpyAsync(perr, &big, sizeof(int), cudaMemcpyHostToDevice, st));
  if (n_pts > 0) k_mark_points<<<nblk(n_pts, 128), 128, 0, st>>>(G, n_pts, pts, flags, perr);
  k_indicators<<<nblk(ntot + 1, 256), 256, 0, st>>>(ntot, flags, ia, il);
  DUST_CUDA(cub::DeviceScan::ExclusiveSum(o->cub_tmp.p, tb, ia, cidx, (int)ntot + 1, st));
  DUST_CUDA(cub::DeviceScan::ExclusiveSum(o->cub_tmp.p, tb, il, lidx, (int)ntot + 1, st));
  k_level_counts<<<1, 32, 0, st>>>(G, cidx, lidx, small);
  int64_t hsmall[DUST_MAXLEV + 3];
  int herr = 0, hperr = 0;
  DUST_CUDA(cudaMemcpyAsync(hsmall, small, sizeof(int64_t) * (ll + 2), cudaMemcpyDeviceToHost,
                            st));
  DUST_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  DUST_CUDA(cudaMemcpyAsync(&hperr, perr, sizeof(int), cudaMemcpyDeviceToHost, st));
  DUST_CUDA(cudaStreamSynchronize(st));
  if (herr != 0x7fffffff) {
    o->bad_particle = herr;
    return DUST_ERR_OUT_OF_BOX;
  }
  if (hperr != 0x7fffffff) {
    dust_set_last_error("an evaluation point lies outside the octree box", __FILE__, __LINE__);
    return DUST_ERR_OUT_OF_BOX;
  }
  o->n_leaves = hsmall[0];
  for (int l = 1; l <= ll + 1; ++l) o->act_off[l] = hsmall[l];
  o->n_active = o->act_off[ll + 1];
  const int64_t nact = o->n_active;
  DUST_TRY(grow(o->act_key, (size_t)std::max<int64_t>(nact, 1) * 4));
  DUST_TRY(grow(o->act_lev, (size_t)std::max<int64_t>(nact, 1)));
  DUST_TRY(grow(o->leaf_ci, (size_t)std::max<int64_t>(o->n_leaves, 1) * 4));
  size_t nmp = (size_t)3 * (2 * o->nm + o->nm1);
  DUST_TRY(grow(o->mp, (size_t)std::max<int64_t>(nact, 1) * nmp * 8));
  k_compact<<<nblk(ntot, 256), 256, 0, st>>>(G, ntot, flags, cidx, lidx,
                                             (uint32_t *)o->act_key.p, (uint8_t *)o->act_lev.p,
                                             (uint32_t *)o->leaf_ci.p);
  FmmDev d;
  fill_dev(o, d, n);
  d.cstart = cstart;
  d.perm = perm;
  d.P = P;
  d.flags = flags;
  d.cidx = cidx;
  d.act_key = (const uint32_t *)o->act_key.p;
  d.act_lev = (const uint8_t *)o->act_lev.p;
  d.leaf_ci = (const uint32_t *)o->leaf_ci.p;
  d.n_leaves = (uint32_t)o->n_leaves;
  double *mp = (double *)o->mp.p;
  d.A = mp;
  d.B = mp + (size_t)nact * 3 * o->nm;
  d.Gx = mp + (size_t)nact * 3 * 2 * o->nm;
  d.out = (double *)o->outs.p;
  o->dev = d;
  if (o->timing) cudaEventRecord(o->ev[1], st);
  // upward pass
  DUST_CUDA(cudaMemsetAsync(d.A, 0, (size_t)nact * 3 * (2 * o->nm + o->nm1) * 8, st));
  d.counters = (int64_t *)(small + 48);
  DUST_CUDA(cudaMemsetAsync(d.counters, 0, 4 * sizeof(int64_t), st));
  o->dev = d;
  DUST_TRY(m2l_prepare(o, d, st));
  if (o->n_leaves > 0) {
    k_p2m<<<(unsigned)((o->n_leaves + P2M_W - 1) / P2M_W), P2M_W * 32, 0, st>>>(d);
  }
  for (int l = ll - 1; l >= 1; --l) {
    int64_t na = o->act_off[l + 1] - o->act_off[l];
    if (na > 0) {
      const int nt = o->shift_n[l][0];
      const size_t shm = (size_t)SH_W * 8 * 3 * o->nm * 8 + (size_t)nt * sizeof(ShiftTerm) +
                         (size_t)(o->nm + 1) * 4;
      if (shm > 48 * 1024)
        DUST_CUDA(cudaFuncSetAttribute(k_m2m_t, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)shm));
      k_m2m_t<<<shift_grid(na), SH_T, shm, st>>>(d, l, (uint32_t)o->act_off[l], (uint32_t)na,
                                                  (const ShiftTerm *)o->shift_t[l][0],
                                                  (const int *)o->shift_o[l][0], nt);
    }
  }
  DUST_TRY(m2l_scale_sources(o, d, st));
  if (o->timing) cudaEventRecord(o->ev[2], st);
  // downward pass: M2L of every level (level 1 per target, levels >= 2 in
  // one batched launch), then L2L level by level adds the parents' final
  // local expansions (mod_octree.f90:1074-1125 in another, equivalent order:
  // both are sums of the same terms)
  int thr_m2l = (std::max(o->nm, d.use_vs ? o->nm1 : o->nm) + 31) / 32 * 32;
  {
    int64_t na1 = o->act_off[2 <= ll ? 2 : ll + 1] - o->act_off[1];
    if (na1 > 0)
      k_m2l<<<(unsigned)na1, thr_m2l, 3 * o->nm * 8, st>>>(d, 1, (uint32_t)o->act_off[1]);
  }
  DUST_TRY(m2l_all_levels(o, d, st));
  for (int l = 2; l <= ll; ++l) {
    int64_t na = o->act_off[l + 1] - o->act_off[l];
    if (na <= 0) continue;
    const int ntb = o->shift_n[l][1], ntg = d.use_vs ? o->shift_n[l][2] : 0;
    const size_t shm = (size_t)SH_W * 3 * (o->nm + (ntg > 0 ? o->nm1 : 0)) * 8 +
                       (size_t)(ntb + ntg) * sizeof(ShiftTerm) + (size_t)(o->nm + o->nm1 + 2) * 4;
    if (shm > 48 * 1024)
      DUST_CUDA(cudaFuncSetAttribute(k_l2l_t, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)shm));
    const int64_t npar = o->act_off[l] - o->act_off[l - 1];
    k_l2l_t<<<shift_grid(npar), SH_T, shm, st>>>(
        d, l, (uint32_t)o->act_off[l - 1], (uint32_t)npar, (const ShiftTerm *)o->shift_t[l][1],
        (const int *)o->shift_o[l][1], ntb, (const ShiftTerm *)o->shift_t[l][2],
        (const int *)o->shift_o[l][2], ntg);
  }
  if (o->timing) cudaEventRecord(o->ev[3], st);
  o->dev = d;
  o->prepared_n = n;
  o->prepared_pts = n_pts;
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}

// leaves: L2P + P2P of the particles with the prepared tree and expansions
int fmm_near_device(dust_octree *o, cudaStream_t st) {
  FmmDev &d = o->dev;
  o->last_stream = st;
  if (o->timing) cudaEventRecord(o->ev[10], st);
  if (o->n_leaves > 0) {
    bool vs = d.use_vs, df = d.use_df, vd = d.use_vd, tv = o->prm.turbulent_viscosity != 0;
    const bool f32 = o->prm.precision == DUST_PREC_FP32C;
    const unsigned grid = (unsigned)((o->n_leaves + P2W_WARPS - 1) / P2W_WARPS);
#define LAUNCH_P2P(A, B, C, D)                                                   \
  do {                                                                         \
    if (f32)                                                                   \
      k_p2p_w<A, B, C, D, true><<<grid, P2W_WARPS * 32, 0, st>>>(d);           \
    else                                                                       \
      k_p2p_w<A, B, C, D, false><<<grid, P2W_WARPS * 32, 0, st>>>(d);          \
  } while (0)
    if (vs && df && vd && !tv) LAUNCH_P2P(true, true, true, false);
    else if (vs && df && vd && tv) LAUNCH_P2P(true, true, true, true);
    else if (vs && df && !vd) LAUNCH_P2P(true, true, false, false);
    else if (vs && !df && vd && !tv) LAUNCH_P2P(true, false, true, false);
    else if (vs && !df && vd && tv) LAUNCH_P2P(true, false, true, true);
    else if (vs && !df && !vd) LAUNCH_P2P(true, false, false, false);
    else if (!vs && vd && !tv) LAUNCH_P2P(false, false, true, false);
    else if (!vs && vd && tv) LAUNCH_P2P(false, false, true, true);
    else LAUNCH_P2P(false, false, false, false);
#undef LAUNCH_P2P
  }
  if (o->timing) cudaEventRecord(o->ev[4], st);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}

int fmm_run_device(dust_octree *o, int n, const double *cen, const double *dir,
                   const double *mag, const double *rv, cudaStream_t st) {
  DUST_TRY(fmm_prepare_device(o, n, cen, dir, mag, rv, 0, nullptr, st));
  return fmm_near_device(o, st);
}

// ----------------------------------------------- particles -> points (FMM)
// apply_multipole_panels (mod_octree.f90:1433-1508) on the GPU: one thread
// per point.  The point is binned into the finest cell as sort_particles
// bins panel centres (:776-799) and takes the leaf above that cell (the
// leaves partition the box); its velocity is the leaf's local expansion
// (FP64 L2P of b) plus the particles of the leaf's 26 active same-level
// neighbours, of its coarser leaf neighbours (leaf_neigh) and of the leaf
// itself, summed in FP64 with the particle kernel of compute_vel
// (mod_vortpart.f90:139-155).  A point outside the octree box sets the
// error word (the reference stops there).
__global__ void k_points_fmm(FmmDev d, int npts, const double *__restrict__ pts,
                             double *__restrict__ uv, int *err) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= npts) return;
  const TreeGeom &G = d.G;
  const int ll = G.ll;
  const size_t n = d.n;
  const double pos[3] = {pts[3 * (size_t)q], pts[3 * (size_t)q + 1], pts[3 * (size_t)q + 2]};
  int idx[3];
  for (int c = 0; c < 3; ++c) {
    idx[c] = (int)ceil((pos[c] - G.xmin[c]) / G.csize[ll]) - 1;
    if (idx[c] < 0 || idx[c] >= G.ncl[ll][c]) {
      atomicMin(err, q);
      for (int e = 0; e < 3; ++e) uv[3 * (size_t)q + e] = 0.0;
      return;
    }
  }
  int l = 0, ci = 0, cj = 0, ck = 0;
  uint32_t key = 0;
  for (int lv = 1; lv <= ll; ++lv) {
    const int sh = ll - lv;
    const int a = idx[0] >> sh, b = idx[1] >> sh, c = idx[2] >> sh;
    const uint32_t k = key_of(G, lv, a, b, c);
    if (d.flags[G.lev_off[lv] + k] & FL_LEAF) {
      l = lv, ci = a, cj = b, ck = c, key = k;
      break;
    }
  }
  double v[3] = {0.0, 0.0, 0.0};
  if (l > 0) {
    const uint32_t cell = d.cidx[G.lev_off[l] + key];
    double cc[3];
    cell_center(G, l, ci, cj, ck, cc);
    const double x = pos[0] - cc[0], y = pos[1] - cc[1], z = pos[2] - cc[2];
    const double *bl = d.B + (size_t)cell * 3 * d.nm;
    for (int m = 0; m < d.nm; ++m) {
      int mi, mj, mk;
      mono_exp(m, mi, mj, mk);
      double pr = 1.0;
      for (int e = 0; e < mi; ++e) pr *= x;
      for (int e = 0; e < mj; ++e) pr *= y;
      for (int e = 0; e < mk; ++e) pr *= z;
      for (int e = 0; e < 3; ++e) v[e] += bl[3 * m + e] * pr;
    }
    const double k4pi = 1.0 / (4.0 * DUST_PI);
    auto range = [&](uint32_t lo, uint32_t hi) {
      for (uint32_t t = lo; t < hi; ++t) {
        const double dx = pos[0] - d.P[t], dy = pos[1] - d.P[n + t], dz = pos[2] - d.P[2 * n + t];
        const double ax = d.P[3 * n + t], ay = d.P[4 * n + t], az = d.P[5 * n + t],
                     s = d.P[6 * n + t];
        const double dn = sqrt(dx * dx + dy * dy + dz * dz + s * s);
        const double c = -1.0 / (dn * dn * dn) * k4pi;
        v[0] += c * (dy * az - dz * ay);
        v[1] += c * (dz * ax - dx * az);
        v[2] += c * (dx * ay - dy * ax);
      }
    };
    for (int lev = l; lev >= 1; --lev) {
      const int sh = l - lev;
      const int ai = ci >> sh, aj = cj >> sh, ak = ck >> sh;
      for (int kk = -1; kk <= 1; ++kk)
        for (int jj = -1; jj <= 1; ++jj)
          for (int ii = -1; ii <= 1; ++ii) {
            if (ii == 0 && jj == 0 && kk == 0) continue;
            if (!cart_in(G, lev, ai + ii, aj + jj, ak + kk)) continue;
            const uint32_t nk = key_of(G, lev, ai + ii, aj + jj, ak + kk);
            const uint8_t f = d.flags[G.lev_off[lev] + nk];
            if (lev == l ? !(f & FL_ACTIVE) : !(f & FL_LEAF)) continue;
            range(cell_lo(G, d.cstart, lev, nk), cell_hi(G, d.cstart, lev, nk));
          }
    }
    range(cell_lo(G, d.cstart, l, key), cell_hi(G, d.cstart, l, key));
  }
  for (int e = 0; e < 3; ++e) uv[3 * (size_t)q + e] = v[e];
}

void points_lines_add(int npts, const double *pts, const ElemDev &lines, double *uv,
                      cudaStream_t st);

int fmm_points_uvort_device(dust_octree *o, const ElemDev &lines, double *uv, cudaStream_t st) {
  const int n_pts = o->prepared_pts;
  if (o->prepared_n < 0) return DUST_ERR_BAD_ARG;
  if (n_pts <= 0) return DUST_OK;
  const double *pts = (const double *)o->h_pts.p;
  int *err = (int *)((int64_t *)o->small.p + 42);
  const int big = 0x7fffffff;
  DUST_CUDA(cudaMemcpyAsync(err, &big, sizeof(int), cudaMemcpyHostToDevice, st));
  k_points_fmm<<<nblk(n_pts, 128), 128, 0, st>>>(o->dev, n_pts, pts, uv, err);
  if (lines.nline > 0) points_lines_add(n_pts, pts, lines, uv, st);
  int herr = big;
  DUST_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  DUST_CUDA(cudaStreamSynchronize(st));
  if (herr != big) {
    dust_set_last_error("a point lies outside the octree box", __FILE__, __LINE__);
    return DUST_ERR_OUT_OF_BOX;
  }
  return DUST_OK;
}

int fmm_finish_device(dust_octree *o, int n, const ElemDev &e, double *vel, double *str,
                      double *rot, cudaStream_t st) {
  if (n > 0)
    DUST_TRY(elem_output_device(o->dev, e, o->ffbuf, o->elem_work, o->near_cap, o->prm.precision,
                                vel, str, rot, st, o->timing ? &o->ev[8] : nullptr, &o->kev_far));
  if (o->timing) cudaEventRecord(o->ev[5], st);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}

int fmm_collect_stats(dust_octree *o, int n, int64_t n_elem) {
  dust_fmm_stats &s = o->stats;
  memset(&s, 0, sizeof(s));
  cudaStreamSynchronize(o->last_stream);
  int status = DUST_OK;
  if (o->dev.counters) {
    int64_t c[4] = {0, 0, 0, 0};
    cudaMemcpy(c, o->dev.counters, sizeof(c), cudaMemcpyDeviceToHost);
    s.n_m2l_pairs = c[0];
    s.n_p2p_pairs = c[1];
    if (c[2]) status = DUST_ERR_TIMEOUT;  // a bounded wait of the tensor-core M2L gave up
  }
  s.n_particles = n;
  s.n_leaves = o->n_leaves;
  s.n_active_cells = o->n_active;
  s.n_levels = o->G.ll;
  s.n_elem_pairs = (int64_t)n * n_elem;
  if (o->timing) {
    cudaEventSynchronize(o->ev[5]);
    cudaEventElapsedTime(&s.ms_tree, o->ev[0], o->ev[1]);
    cudaEventElapsedTime(&s.ms_upward, o->ev[1], o->ev[2]);
    cudaEventElapsedTime(&s.ms_m2l, o->ev[2], o->ev[3]);
    cudaEventElapsedTime(&s.ms_p2p, o->ev[10], o->ev[4]);
    cudaEventElapsedTime(&s.ms_elems, o->ev[4], o->ev[5]);
    float t_pre = 0.f, t_post = 0.f;
    cudaEventElapsedTime(&t_pre, o->ev[0], o->ev[3]);
    cudaEventElapsedTime(&t_post, o->ev[10], o->ev[5]);
    s.ms_total = t_pre + t_post;
    if (o->kev_m2l) cudaEventElapsedTime(&s.ms_m2l_kernel, o->ev[6], o->ev[7]);
    if (o->kev_far) cudaEventElapsedTime(&s.ms_elem_far, o->ev[8], o->ev[9]);
  }
  return status;
}
