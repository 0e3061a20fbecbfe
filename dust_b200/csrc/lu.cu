// lu.cu -- blocked LU with partial pivoting (FP64 and FP32) on sm_100a.
//
// LAPACK dgetrf semantics (used by src/linsys/mod_linsys.f90:230-246 and
// :428-438): pivot = first row of maximum |a(i,j)|, ipiv 1-based, rows
// swapped across the whole matrix, L unit lower, U upper, info = first
// zero pivot.
//
// Panel factorisation (64 columns), by the panel's height:
//  * up to 2048 rows: one CTA (k_panel_1cta) holding 16- (FP32) or 8-column
//    (FP64) sub-panels in registers, two CTA barriers per column;
//  * taller panels that fit the shared memory of a cluster of 8 or 16 CTAs:
//    k_panel_cluster, one cluster barrier per column, candidates exchanged
//    through distributed shared memory;
//  * otherwise one cooperative launch of G CTAs (k_panel): CTA g keeps rows
//    [g*R, (g+1)*R) of the panel in shared memory, one grid-wide barrier per
//    column (before it every CTA publishes its local maximum and that row,
//    and the owner of the diagonal row publishes it; after it every CTA
//    selects the same pivot, performs its part of the swap from the
//    published rows and updates its rows).  Published buffers alternate
//    between two copies so a CTA one column ahead never overwrites data
//    still read.  The barrier spins with an iteration limit and raises an
//    error flag instead of hanging.
// The panel's row interchanges reach the other columns as one net
// permutation per panel (k_laswp_net); trailing updates are GEMMs (cuBLAS,
// or the tcgen05 TF32 kernel of gemm_tc.cu for FP32).
#include <climits>

#include <cooperative_groups.h>

#include "lu.cuh"

#define PAN_T 256
#define PAN_MIN_ROWS 32
#define BAR_SPIN_LIMIT (1ll << 25)

template <typename T>
struct PanelArgs {
  T *A;
  int lda, k, jb, m, G, R;
  int *ipiv, *info;
  unsigned *bar;  // [0] arrivals, [1] generation
  int *err;
  T *cval;        // [2][G]
  int *crow;      // [2][G]
  T *crowv;       // [2][G][jb]
  T *srow;        // [2][jb]
};

__device__ __forceinline__ void grid_barrier(unsigned *bar, int G, int *err) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned *vgen = bar + 1;
    unsigned g0 = *vgen;
    __threadfence();
    unsigned arrived = atomicAdd(bar, 1u);
    if (arrived == (unsigned)G - 1u) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      long long it = 0;
      while (*vgen == g0) {
        if (++it > BAR_SPIN_LIMIT) {
          atomicExch(err, 1);
          break;
        }
        if (it > 64) __nanosleep(20);
      }
    }
    __threadfence();
  }
  __syncthreads();
}

template <typename T>
__device__ __forceinline__ T ldcg(const T *p) {
  return __ldcg(p);
}

template <typename T>
__global__ void __launch_bounds__(PAN_T) k_panel(PanelArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T *sp = (T *)smraw;  // R rows x LD, row-major
  __shared__ T s_prow[128];
  __shared__ T s_wv[PAN_T / 32];
  __shared__ int s_wr[PAN_T / 32];
  __shared__ int s_p, s_gw;
  __shared__ T s_pv;
  const int g = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int NW = PAN_T / 32;
  const int jb = a.jb, LD = jb + 1;
  const int r0 = g * a.R, r1 = min(a.m, r0 + a.R), nr = max(0, r1 - r0);
  T *Ap = a.A + (size_t)a.k + (size_t)a.k * a.lda;
  for (int idx = tid; idx < nr * jb; idx += PAN_T) {
    int c = idx / nr, r = idx % nr;
    sp[r * LD + c] = Ap[(size_t)(r0 + r) + (size_t)c * a.lda];
  }
  __syncthreads();
  for (int j = 0; j < jb; ++j) {
    const int buf = j & 1;
    // local maximum of |a(r, j)| over own rows r >= j (first index on ties)
    T best = (T)-1;
    int brow = INT_MAX;
    for (int r = tid; r < nr; r += PAN_T) {
      int gr = r0 + r;
      if (gr < j) continue;
      T v = fabs(sp[r * LD + j]);
      if (v != v) v = (T)-0.5;  // NaN: still a candidate, below every number
      if (v > best || (v == best && gr < brow)) {
        best = v;
        brow = gr;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      T ov = __shfl_down_sync(0xffffffffu, best, o);
      int orr = __shfl_down_sync(0xffffffffu, brow, o);
      if (ov > best || (ov == best && orr < brow)) {
        best = ov;
        brow = orr;
      }
    }
    if (lane == 0) {
      s_wv[warp] = best;
      s_wr[warp] = brow;
    }
    __syncthreads();
    if (tid == 0) {
      T b = s_wv[0];
      int br = s_wr[0];
      for (int w = 1; w < NW; ++w)
        if (s_wv[w] > b || (s_wv[w] == b && s_wr[w] < br)) {
          b = s_wv[w];
          br = s_wr[w];
        }
      s_p = br;
      a.crow[buf * a.G + g] = br;
      a.cval[buf * a.G + g] = (br == INT_MAX) ? (T)-1 : b;
    }
    __syncthreads();
    const int mybest = s_p;
    if (mybest != INT_MAX)
      for (int c = tid; c < jb; c += PAN_T)
        a.crowv[((size_t)buf * a.G + g) * jb + c] = sp[(mybest - r0) * LD + c];
    if (j >= r0 && j < r1)
      for (int c = tid; c < jb; c += PAN_T) a.srow[buf * jb + c] = sp[(j - r0) * LD + c];
    grid_barrier(a.bar, a.G, a.err);
    // global pivot: maximum over the published candidates
    {
      T bv = (T)-1;
      int br = INT_MAX, bg = -1;
      for (int q = tid; q < a.G; q += PAN_T) {
        int rr = ldcg(a.crow + buf * a.G + q);
        T vv = ldcg(a.cval + buf * a.G + q);
        if (rr != INT_MAX && (vv > bv || (vv == bv && rr < br))) {
          bv = vv;
          br = rr;
          bg = q;
        }
      }
      for (int o = 16; o > 0; o >>= 1) {
        T ov = __shfl_down_sync(0xffffffffu, bv, o);
        int orr = __shfl_down_sync(0xffffffffu, br, o);
        int og = __shfl_down_sync(0xffffffffu, bg, o);
        if (ov > bv || (ov == bv && orr < br)) {
          bv = ov;
          br = orr;
          bg = og;
        }
      }
      __syncthreads();
      if (lane == 0) {
        s_wv[warp] = bv;
        s_wr[warp] = br;
      }
      __shared__ int s_wg[PAN_T / 32];
      if (lane == 0) s_wg[warp] = bg;
      __syncthreads();
      if (tid == 0) {
        T b = s_wv[0];
        int rr = s_wr[0], gg = s_wg[0];
        for (int w = 1; w < NW; ++w)
          if (s_wv[w] > b || (s_wv[w] == b && s_wr[w] < rr)) {
            b = s_wv[w];
            rr = s_wr[w];
            gg = s_wg[w];
          }
        s_p = rr;
        s_gw = gg;
      }
      __syncthreads();
    }
    int p = s_p, gw = s_gw;
    if (gw < 0 || gw >= a.G || p < j || p >= a.m) {
      // cannot happen while some CTA owns a row >= j; keep the indices in
      // bounds and report instead of reading outside the published buffers
      if (tid == 0) atomicExch(a.err, 2);
      gw = (j >= r0 && j < r1) ? g : 0;
      p = j;
    }
    for (int c = tid; c < jb; c += PAN_T) s_prow[c] = ldcg(a.crowv + ((size_t)buf * a.G + gw) * jb + c);
    __syncthreads();
    if (tid == 0) s_pv = s_prow[j];
    if (g == 0 && tid == 0) {
      a.ipiv[a.k + j] = a.k + p + 1;
      if (s_prow[j] == (T)0 && *a.info == 0) *a.info = a.k + j + 1;
    }
    if (p != j) {
      if (j >= r0 && j < r1)
        for (int c = tid; c < jb; c += PAN_T) sp[(j - r0) * LD + c] = s_prow[c];
      if (p >= r0 && p < r1)
        for (int c = tid; c < jb; c += PAN_T) sp[(p - r0) * LD + c] = ldcg(a.srow + buf * jb + c);
    }
    __syncthreads();
    const T pv = s_pv;
    if (pv != (T)0) {
      const T rinv = (T)1 / pv;
      for (int r = warp; r < nr; r += NW) {
        if (r0 + r <= j) continue;
        T l = sp[r * LD + j] * rinv;
        for (int c = j + 1 + lane; c < jb; c += 32) sp[r * LD + c] -= l * s_prow[c];
        __syncwarp();
        if (lane == 0) sp[r * LD + j] = l;
      }
    }
    __syncthreads();
  }
  for (int idx = tid; idx < nr * jb; idx += PAN_T) {
    int c = idx / nr, r = idx % nr;
    Ap[(size_t)(r0 + r) + (size_t)c * a.lda] = sp[r * LD + c];
  }
}

// Cluster panel factorisation: the panel's rows are split over the C CTAs
// of one thread-block cluster, each CTA keeping its rows in shared memory.
// Per column every CTA publishes its local pivot candidate (|value|, row and
// the row's jb entries) in its own shared memory, one hardware cluster
// barrier follows, and every CTA then reads the C candidates (and the
// diagonal row) through distributed shared memory and makes the same
// choice.  Published buffers alternate between two copies, so a CTA one
// column ahead never overwrites data another CTA still reads; a final
// cluster barrier keeps every CTA's shared memory alive until the last
// remote read.  No spin waits: the cluster's CTAs are co-scheduled and all
// take the same barriers.
#define CPAN_T 256

template <typename T>
struct CPanelShared {  // published per column, two copies
  T cval[2];
  int crow[2];
};

template <typename T>
__global__ void __launch_bounds__(CPAN_T) k_panel_cluster(PanelArgs<T> a) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ __align__(16) unsigned char smraw[];
  const int jb = a.jb, LD = jb + 1;
  T *sp = (T *)smraw;                        // R rows x LD, row-major
  T *s_crowv = sp + (size_t)a.R * LD;        // [2][jb] candidate row
  T *s_srow = s_crowv + 2 * jb;              // [2][jb] diagonal row (owner only)
  T *s_prow = s_srow + 2 * jb;               // [jb] pivot row (local copy)
  __shared__ CPanelShared<T> s_pub;
  __shared__ T s_wv[CPAN_T / 32];
  __shared__ int s_wr[CPAN_T / 32], s_wg[CPAN_T / 32];
  __shared__ int s_p;
  const int g = (int)cl.block_rank(), C = (int)cl.num_blocks();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int NW = CPAN_T / 32;
  const int r0 = g * a.R, r1 = min(a.m, r0 + a.R), nr = max(0, r1 - r0);
  T *Ap = a.A + (size_t)a.k + (size_t)a.k * a.lda;
  for (int c = 0; c < jb; ++c)
    for (int r = tid; r < nr; r += CPAN_T) sp[r * LD + c] = Ap[(size_t)(r0 + r) + (size_t)c * a.lda];
  __syncthreads();
  for (int j = 0; j < jb; ++j) {
    const int buf = j & 1;
    // local maximum of |a(r, j)| over own rows r >= j (first index on ties)
    T best = (T)-1;
    int brow = INT_MAX;
    for (int r = tid; r < nr; r += CPAN_T) {
      const int gr = r0 + r;
      if (gr < j) continue;
      T v = fabs(sp[r * LD + j]);
      if (v != v) v = (T)-0.5;  // NaN: still a candidate, below every number
      if (v > best || (v == best && gr < brow)) {
        best = v;
        brow = gr;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const T ov = __shfl_down_sync(0xffffffffu, best, o);
      const int orr = __shfl_down_sync(0xffffffffu, brow, o);
      if (ov > best || (ov == best && orr < brow)) {
        best = ov;
        brow = orr;
      }
    }
    if (lane == 0) {
      s_wv[warp] = best;
      s_wr[warp] = brow;
    }
    __syncthreads();
    if (tid == 0) {
      T b = s_wv[0];
      int br = s_wr[0];
      for (int w = 1; w < NW; ++w)
        if (s_wv[w] > b || (s_wv[w] == b && s_wr[w] < br)) {
          b = s_wv[w];
          br = s_wr[w];
        }
      s_p = br;
      s_pub.crow[buf] = br;
      s_pub.cval[buf] = (br == INT_MAX) ? (T)-1 : b;
    }
    __syncthreads();
    const int mybest = s_p;
    if (mybest != INT_MAX)
      for (int c = tid; c < jb; c += CPAN_T) s_crowv[buf * jb + c] = sp[(mybest - r0) * LD + c];
    if (j >= r0 && j < r1)
      for (int c = tid; c < jb; c += CPAN_T) s_srow[buf * jb + c] = sp[(j - r0) * LD + c];
    cl.sync();
    // global pivot: the maximum over the C published candidates (warp 0)
    if (warp == 0) {
      T bv = (T)-1;
      int br = INT_MAX, bg = -1;
      for (int q = lane; q < C; q += 32) {
        const CPanelShared<T> *rp = cl.map_shared_rank(&s_pub, q);
        const int rr = rp->crow[buf];
        const T vv = rp->cval[buf];
        if (rr != INT_MAX && (vv > bv || (vv == bv && rr < br))) {
          bv = vv;
          br = rr;
          bg = q;
        }
      }
      for (int o = 16; o > 0; o >>= 1) {
        const T ov = __shfl_down_sync(0xffffffffu, bv, o);
        const int orr = __shfl_down_sync(0xffffffffu, br, o);
        const int og = __shfl_down_sync(0xffffffffu, bg, o);
        if (ov > bv || (ov == bv && orr < br)) {
          bv = ov;
          br = orr;
          bg = og;
        }
      }
      if (lane == 0) {
        s_wr[0] = br;
        s_wg[0] = bg;
      }
    }
    __syncthreads();
    int p = s_wr[0], gw = s_wg[0];
    if (gw < 0 || gw >= C || p < j || p >= a.m) {
      // cannot happen while some CTA owns a row >= j; keep the indices in
      // bounds and report instead of reading outside the published buffers
      if (tid == 0) atomicExch(a.err, 2);
      gw = g;
      p = j;
    }
    const T *prow_src = cl.map_shared_rank(s_crowv, gw) + buf * jb;
    for (int c = tid; c < jb; c += CPAN_T) s_prow[c] = prow_src[c];
    if (p != j && p >= r0 && p < r1) {
      // the diagonal row j moves to row p: fetch it from its owner
      const T *srow_src = cl.map_shared_rank(s_srow, j / a.R) + buf * jb;
      for (int c = tid; c < jb; c += CPAN_T) sp[(p - r0) * LD + c] = srow_src[c];
    }
    __syncthreads();
    const T pv = s_prow[j];
    if (g == 0 && tid == 0) {
      a.ipiv[a.k + j] = a.k + p + 1;
      if (pv == (T)0 && *a.info == 0) *a.info = a.k + j + 1;
    }
    if (p != j && j >= r0 && j < r1)
      for (int c = tid; c < jb; c += CPAN_T) sp[(j - r0) * LD + c] = s_prow[c];
    __syncthreads();
    if (pv != (T)0) {
      // one thread per row (LD = jb + 1 words apart: no bank conflicts)
      const T rinv = (T)1 / pv;
      for (int r = tid; r < nr; r += CPAN_T) {
        if (r0 + r <= j) continue;
        T *row = sp + (size_t)r * LD;
        const T l = row[j] * rinv;
        row[j] = l;
#pragma unroll 4
        for (int c = j + 1; c < jb; ++c) row[c] -= l * s_prow[c];
      }
    }
    __syncthreads();
  }
  for (int c = 0; c < jb; ++c)
    for (int r = tid; r < nr; r += CPAN_T) Ap[(size_t)(r0 + r) + (size_t)c * a.lda] = sp[r * LD + c];
  cl.sync();  // no CTA leaves while another may still read its shared memory
}

// Single-CTA panel factorisation for panels of moderate height.  The CTA
// factors the panel in sub-panels of W columns; thread t keeps rows t,
// t + NT, ... (RPT of them) of the sub-panel in registers, so the rank-1
// updates of a column touch no memory and a pivot search needs only CTA
// barriers (two per column); the pivot row is exchanged through shared
// memory.  After a
// sub-panel: its row interchanges are applied to the panel's other columns
// (as one net permutation of the touched rows), U12 right of it is solved
// with its unit lower triangle, and the panel's remaining columns get the
// rank-W update from the rows still in registers.  Pivot choice, ipiv and
// info are those of the column-by-column algorithm (first maximum wins).
#define P1_T 512
#define P1_NW (P1_T / 32)
#define P1_JB 64  // widest panel

template <typename T, int W, int RPT>
__global__ void __launch_bounds__(P1_T) k_panel_1cta(PanelArgs<T> a) {
  constexpr int VEC = 16 / (int)sizeof(T);  // U12 columns per vector load
  const int m = a.m, jb = a.jb, lda = a.lda;
  __shared__ __align__(16) T s_u[W * P1_JB];  // U12 of the current sub-panel
  __shared__ T s_l11[W][W + 1];
  // per column, alternating between two copies (a column's readers finish
  // before any thread passes the next column's second barrier)
  __shared__ __align__(16) T s_prow[2][W], s_jrow[2][W];
  __shared__ T s_wv[2][P1_NW];
  __shared__ int s_wr[2][P1_NW];
  __shared__ int s_piv[W], s_pos[2 * W], s_src[2 * W];
  __shared__ int s_np;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  T *Ap = a.A + (size_t)a.k + (size_t)a.k * lda;
  T x[RPT][W];
  int par = 0;
  for (int s0 = 0; s0 < jb; s0 += W) {
    const int w = min(W, jb - s0);
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
      const int r = tid + k * P1_T;
#pragma unroll
      for (int c = 0; c < W; ++c)
        x[k][c] = (r < m && c < w) ? Ap[r + (size_t)(s0 + c) * lda] : (T)0;
    }
#pragma unroll
    for (int jj = 0; jj < W; ++jj) {
      if (jj >= w) break;
      const int j = s0 + jj;
      // maximum of |a(r, j)| over rows r >= j (first index on ties)
      T best = (T)-1;
      int brow = INT_MAX;
#pragma unroll
      for (int k = 0; k < RPT; ++k) {
        const int r = tid + k * P1_T;
        if (r >= j && r < m) {
          T v = fabs(x[k][jj]);
          if (v != v) v = (T)-0.5;  // NaN: still a candidate, below every number
          if (v > best || (v == best && r < brow)) {
            best = v;
            brow = r;
          }
        }
      }
      for (int o = 16; o > 0; o >>= 1) {
        const T ov = __shfl_xor_sync(0xffffffffu, best, o);
        const int orr = __shfl_xor_sync(0xffffffffu, brow, o);
        if (ov > best || (ov == best && orr < brow)) {
          best = ov;
          brow = orr;
        }
      }
      if (lane == 0) {
        s_wv[par][warp] = best;
        s_wr[par][warp] = brow;
      }
      __syncthreads();
      // every warp reduces the warps' candidates itself
      best = lane < P1_NW ? s_wv[par][lane] : (T)-1;
      brow = lane < P1_NW ? s_wr[par][lane] : INT_MAX;
      for (int o = 16; o > 0; o >>= 1) {
        const T ov = __shfl_xor_sync(0xffffffffu, best, o);
        const int orr = __shfl_xor_sync(0xffffffffu, brow, o);
        if (ov > best || (ov == best && orr < brow)) {
          best = ov;
          brow = orr;
        }
      }
      const int p = (brow == INT_MAX) ? j : brow;
      // rows j and p through shared memory
#pragma unroll
      for (int k = 0; k < RPT; ++k) {
        const int r = tid + k * P1_T;
        if (r == p)
#pragma unroll
          for (int c = 0; c < W; ++c) s_prow[par][c] = x[k][c];
        if (r == j)
#pragma unroll
          for (int c = 0; c < W; ++c) s_jrow[par][c] = x[k][c];
      }
      if (tid == 0) s_piv[jj] = p;
      __syncthreads();
      const T *prow = s_prow[par];
#pragma unroll
      for (int k = 0; k < RPT; ++k) {
        const int r = tid + k * P1_T;
        if (r == j)
#pragma unroll
          for (int c = 0; c < W; ++c) x[k][c] = prow[c];
        else if (r == p)
#pragma unroll
          for (int c = 0; c < W; ++c) x[k][c] = s_jrow[par][c];
      }
      const T pv = prow[jj];
      if (tid == 0) {
        a.ipiv[a.k + j] = a.k + p + 1;
        if (pv == (T)0 && *a.info == 0) *a.info = a.k + j + 1;
      }
      if (pv != (T)0) {
        const T rinv = (T)1 / pv;
#pragma unroll
        for (int k = 0; k < RPT; ++k) {
          const int r = tid + k * P1_T;
          if (r > j && r < m) {
            const T l = x[k][jj] * rinv;
            x[k][jj] = l;
#pragma unroll
            for (int c = jj + 1; c < W; ++c) x[k][c] -= l * prow[c];
          }
        }
      }
      par ^= 1;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
      const int r = tid + k * P1_T;
      if (r < m) {
#pragma unroll
        for (int c = 0; c < W; ++c)
          if (c < w) Ap[r + (size_t)(s0 + c) * lda] = x[k][c];
        if (r >= s0 && r < s0 + w)
#pragma unroll
          for (int c = 0; c < W; ++c) s_l11[r - s0][c] = x[k][c];
      }
    }
    // net permutation of the rows the sub-panel's interchanges touched:
    // position s_pos[q] receives the content of row s_src[q]
    if (tid == 0) {
      int np = 0;
      for (int jj = 0; jj < w; ++jj) {
        const int j = s0 + jj, p = s_piv[jj];
        if (p == j) continue;
        int ij = -1, ip = -1;
        for (int q = 0; q < np; ++q) {
          if (s_pos[q] == j) ij = q;
          if (s_pos[q] == p) ip = q;
        }
        if (ij < 0) {
          s_pos[np] = j;
          s_src[np] = j;
          ij = np++;
        }
        if (ip < 0) {
          s_pos[np] = p;
          s_src[np] = p;
          ip = np++;
        }
        const int t = s_src[ij];
        s_src[ij] = s_src[ip];
        s_src[ip] = t;
      }
      s_np = np;
    }
    __syncthreads();
    {
      // the other columns of the panel: at most 2W rows x (P1_JB - 1) columns
      const int np = s_np, nco = jb - w;
      T vals[(2 * W * (P1_JB - 1) + P1_T - 1) / P1_T];
      int cnt = 0;
      for (int e = tid; e < np * nco; e += P1_T) {
        const int q = e % np, ci = e / np, c = ci < s0 ? ci : ci + w;
        vals[cnt++] = Ap[s_src[q] + (size_t)c * lda];
      }
      __syncthreads();
      cnt = 0;
      for (int e = tid; e < np * nco; e += P1_T) {
        const int q = e % np, ci = e / np, c = ci < s0 ? ci : ci + w;
        Ap[s_pos[q] + (size_t)c * lda] = vals[cnt++];
      }
    }
    __syncthreads();
    const int c1 = s0 + w, nc = jb - c1;
    if (nc > 0) {
      // U12 = L11^-1 A12: one lane per column, the column in registers
      if (tid < nc) {
        T u[W];
        const size_t cb = (size_t)(c1 + tid) * lda;
#pragma unroll
        for (int i = 0; i < W; ++i) {
          if (i < w) {
            T sacc = Ap[s0 + i + cb];
#pragma unroll
            for (int q = 0; q < i; ++q) sacc -= s_l11[i][q] * u[q];
            u[i] = sacc;
            s_u[i * P1_JB + tid] = sacc;
            Ap[s0 + i + cb] = sacc;
          }
        }
      }
      __syncthreads();
      // A22 -= L21 U12 for the rows below the sub-panel, from the registers
#pragma unroll
      for (int k = 0; k < RPT; ++k) {
        const int r = tid + k * P1_T;
        if (r < c1 || r >= m) continue;
        for (int c = 0; c < nc; c += VEC) {
          T v[VEC];
#pragma unroll
          for (int e = 0; e < VEC; ++e) v[e] = c + e < nc ? Ap[r + (size_t)(c1 + c + e) * lda] : (T)0;
#pragma unroll
          for (int q = 0; q < W; ++q) {
            T uu[VEC];
            *(float4 *)uu = *(const float4 *)&s_u[q * P1_JB + c];
            const T lq = q < w ? x[k][q] : (T)0;
#pragma unroll
            for (int e = 0; e < VEC; ++e) v[e] -= lq * uu[e];
          }
#pragma unroll
          for (int e = 0; e < VEC; ++e)
            if (c + e < nc) Ap[r + (size_t)(c1 + c + e) * lda] = v[e];
        }
      }
    }
    __syncthreads();
  }
}

template <typename T, int W, int RPT>
static bool panel_1cta_try(cudaStream_t st, const PanelArgs<T> &pa, int *status) {
  if (pa.jb > P1_JB || pa.m > RPT * P1_T) return false;
  k_panel_1cta<T, W, RPT><<<1, P1_T, 0, st>>>(pa);
  *status = cudaGetLastError() == cudaSuccess ? DUST_OK : DUST_ERR_CUDA;
  return true;
}

// rows per thread from the panel height (up to 4, so panels of up to 2048
// rows), sub-panels of 16 (FP32) or 8 (FP64) columns; taller panels go to
// the cluster kernel
template <typename T>
static bool panel_1cta_launch(cudaStream_t st, const PanelArgs<T> &pa, int *status) {
  if constexpr (sizeof(T) == 4)
    return panel_1cta_try<T, 16, 2>(st, pa, status) || panel_1cta_try<T, 16, 4>(st, pa, status);
  else
    return panel_1cta_try<T, 8, 2>(st, pa, status) || panel_1cta_try<T, 8, 4>(st, pa, status);
}

// Launches the cluster panel when the panel fits in the shared memory of a
// cluster of 8 (or, where the device allows it, 16) CTAs; returns false to
// fall back to the grid-wide version.  The kernel attributes and whether a
// cluster of each size with the full shared memory can be resident are set
// up once per element type.
template <typename T>
static bool panel_cluster_launch(cudaStream_t st, PanelArgs<T> pa, int *status) {
  static int max_sm = -1;
  static bool ok[2] = {false, false};
  if (max_sm < 0) {
    int dev = 0, opt = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&opt, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    max_sm = opt - 2048;  // room for the static shared variables
    bool attrs = cudaFuncSetAttribute(k_panel_cluster<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      max_sm) == cudaSuccess;
    const bool np = attrs && cudaFuncSetAttribute(k_panel_cluster<T>,
                                                  cudaFuncAttributeNonPortableClusterSizeAllowed,
                                                  1) == cudaSuccess;
    for (int i = 0; i < 2 && attrs; ++i) {
      const int C = i == 0 ? 8 : 16;
      if (C > 8 && !np) break;
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(C);
      cfg.blockDim = dim3(CPAN_T);
      cfg.dynamicSmemBytes = (size_t)max_sm;
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = C;
      at[0].val.clusterDim.y = 1;
      at[0].val.clusterDim.z = 1;
      cfg.attrs = at;
      cfg.numAttrs = 1;
      int ncl = 0;
      ok[i] = cudaOccupancyMaxActiveClusters(&ncl, k_panel_cluster<T>, &cfg) == cudaSuccess &&
              ncl >= 1;
    }
    cudaGetLastError();
  }
  const int jb = pa.jb, m = pa.m;
  const size_t fixed = (size_t)5 * jb * sizeof(T) + 1024;
  for (int i = 0; i < 2; ++i) {
    const int C = i == 0 ? 8 : 16;
    const int R = (m + C - 1) / C;
    const size_t sm = (size_t)R * (jb + 1) * sizeof(T) + fixed;
    if (!ok[i] || sm > (size_t)max_sm) continue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C);
    cfg.blockDim = dim3(CPAN_T);
    cfg.dynamicSmemBytes = sm;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    pa.G = C;
    pa.R = R;
    *status = cudaLaunchKernelEx(&cfg, k_panel_cluster<T>, pa) == cudaSuccess ? DUST_OK
                                                                               : DUST_ERR_CUDA;
    return true;
  }
  return false;
}

template <typename T>
__global__ void k_laswp(T *A, int lda, int c0, int c1, int k1, int k2, const int *ipiv) {
  int c = c0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= c1) return;
  T *col = A + (size_t)c * lda;
  for (int i = k1; i < k2; ++i) {
    int p = ipiv[i] - 1;
    if (p != i && p >= 0 && p < lda) {
      T t = col[i];
      col[i] = col[p];
      col[p] = t;
    }
  }
}

// Row interchanges of one panel (pivots ipiv[k .. k+jb)) on the columns
// outside it, [0, k) and [k + jb, n): the jb transpositions, applied in
// order, permute at most 2 jb rows; every CTA derives that net permutation
// (position <- source row) in shared memory and moves the touched rows of
// its LW_C columns, reading them all before writing any.  CTA 0 also
// applies it to `perm` (when given), the factorisation's row permutation.
#define LW_C 32
#define LW_T 256
template <typename T>
__global__ void __launch_bounds__(LW_T) k_laswp_net(T *A, int lda, int n, int k, int jb,
                                                    const int *ipiv, int *perm) {
  extern __shared__ int s_map[];  // [n - k]: slot of a touched row, or -1
  __shared__ int s_pos[2 * P1_JB], s_src[2 * P1_JB];
  __shared__ int s_np;
  const int m = n - k, tid = threadIdx.x;
  for (int r = tid; r < m; r += LW_T) s_map[r] = -1;
  __syncthreads();
  if (tid == 0) {
    int np = 0;
    for (int jj = 0; jj < jb; ++jj) {
      const int p = ipiv[k + jj] - 1 - k;
      if (p == jj || p < 0 || p >= m) continue;
      int ij = s_map[jj], ip = s_map[p];
      if (ij < 0) {
        s_pos[np] = jj;
        s_src[np] = jj;
        s_map[jj] = ij = np++;
      }
      if (ip < 0) {
        s_pos[np] = p;
        s_src[np] = p;
        s_map[p] = ip = np++;
      }
      const int t = s_src[ij];
      s_src[ij] = s_src[ip];
      s_src[ip] = t;
    }
    s_np = np;
  }
  __syncthreads();
  const int np = s_np, ncol = n - jb;
  if (perm && blockIdx.x == 0) {
    // the running row permutation of the factorisation (for lu_getrs)
    const int pv = tid < np ? perm[k + s_src[tid]] : 0;
    __syncthreads();
    if (tid < np) perm[k + s_pos[tid]] = pv;
  }
  const int c0 = blockIdx.x * LW_C, cn = min(LW_C, ncol - c0);
  if (cn <= 0 || np == 0) return;
  constexpr int PER = (2 * P1_JB * LW_C + LW_T - 1) / LW_T;
  T v[PER];
  int cnt = 0;
  for (int e = tid; e < np * cn; e += LW_T) {
    const int q = e % np, ci = c0 + e / np, c = ci < k ? ci : ci + jb;
    v[cnt++] = A[(size_t)k + s_src[q] + (size_t)c * lda];
  }
  __syncthreads();
  cnt = 0;
  for (int e = tid; e < np * cn; e += LW_T) {
    const int q = e % np, ci = c0 + e / np, c = ci < k ? ci : ci + jb;
    A[(size_t)k + s_pos[q] + (size_t)c * lda] = v[cnt++];
  }
}

template <typename T>
void lu_laswp(cudaStream_t st, T *A, int lda, int c0, int c1, int k1, int k2,
              const int *ipiv) {
  if (c1 <= c0 || k2 <= k1) return;
  int nc = c1 - c0;
  k_laswp<T><<<(nc + 127) / 128, 128, 0, st>>>(A, lda, c0, c1, k1, k2, ipiv);
}

static cublasStatus_t trsm_(cublasHandle_t h, cublasSideMode_t s, cublasFillMode_t u,
                            cublasDiagType_t d, int m, int n, const double *A, int lda,
                            double *B, int ldb) {
  const double one = 1.0;
  return cublasDtrsm(h, s, u, CUBLAS_OP_N, d, m, n, &one, A, lda, B, ldb);
}
static cublasStatus_t trsm_(cublasHandle_t h, cublasSideMode_t s, cublasFillMode_t u,
                            cublasDiagType_t d, int m, int n, const float *A, int lda,
                            float *B, int ldb) {
  const float one = 1.0f;
  return cublasStrsm(h, s, u, CUBLAS_OP_N, d, m, n, &one, A, lda, B, ldb);
}
static cublasStatus_t gemm_minus_(cublasHandle_t h, int m, int n, int k, const double *A,
                                  int lda, const double *B, int ldb, double *C, int ldc) {
  const double mone = -1.0, one = 1.0;
  return cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, m, n, k, &mone, A, lda, B, ldb, &one, C, ldc);
}
static cublasStatus_t gemm_minus_(cublasHandle_t h, int m, int n, int k, const float *A,
                                  int lda, const float *B, int ldb, float *C, int ldc) {
  const float mone = -1.0f, one = 1.0f;
  return cublasSgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, m, n, k, &mone, A, lda, B, ldb, &one, C, ldc);
}

__global__ void k_iota(int n, int *v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = i;
}

// B(:, c) = B(perm, c) for each column: one CTA per column through shared
// memory
template <typename T>
__global__ void k_permute_rows(T *B, int ldb, int n, const int *perm) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T *s = (T *)smraw;
  T *col = B + (size_t)blockIdx.x * ldb;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s[i] = col[i];
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) col[i] = s[perm[i]];
}

// tcgen05 TF32 trailing update (gemm_tc.cu); C -= A B, FP32 column-major.
int gemm_tf32_minus(cudaStream_t st, int m, int n, int k, const float *A, int lda,
                    const float *B, int ldb, float *C, int ldc);

#define CUBLAS_OK(x)                                                      \
  do {                                                                    \
    if ((x) != CUBLAS_STATUS_SUCCESS) {                                   \
      dust_set_last_error("cuBLAS call failed", __FILE__, __LINE__);      \
      return DUST_ERR_CUDA;                                               \
    }                                                                     \
  } while (0)

template <typename T>
int lu_getrf(cublasHandle_t cb, cudaStream_t st, LuWork &w, int n, T *A, int lda,
             int *ipiv, int *info_dev, int gemm_update, int *perm) {
  if (n <= 0) return DUST_OK;
  if (perm) {
    if ((size_t)n * sizeof(int) > 200 * 1024) return DUST_ERR_BAD_ARG;
    k_iota<<<(n + 255) / 256, 256, 0, st>>>(n, perm);
  }
  const int nb = 64;
  if (w.nsm == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&w.nsm, cudaDevAttrMultiProcessorCount, dev);
    if (w.nsm <= 0) w.nsm = 1;
  }
  const int Gmax = w.nsm;
  size_t bytes = 64 + 2 * Gmax * (sizeof(T) + sizeof(int)) + 2 * (size_t)Gmax * nb * sizeof(T) +
                 2 * nb * sizeof(T) + 256;
  DUST_TRY(devbuf_grow(w.sync, bytes));
  char *base = (char *)w.sync.p;
  unsigned *bar = (unsigned *)base;
  int *err = (int *)(base + 16);
  T *cval = (T *)(base + 64);
  int *crow = (int *)(cval + 2 * Gmax);
  T *crowv = (T *)(((uintptr_t)(crow + 2 * Gmax) + 15) & ~(uintptr_t)15);
  T *srow = crowv + 2 * (size_t)Gmax * nb;
  DUST_CUDA(cudaMemsetAsync(base, 0, 64, st));
  DUST_CUDA(cudaMemsetAsync(info_dev, 0, sizeof(int), st));
  CUBLAS_OK(cublasSetStream(cb, st));
  for (int k = 0; k < n; k += nb) {
    const int jb = std::min(nb, n - k), m = n - k;
    int G = std::min(Gmax, std::max(1, (m + PAN_MIN_ROWS - 1) / PAN_MIN_ROWS));
    int R = (m + G - 1) / G;
    G = (m + R - 1) / R;
    size_t sm = (size_t)R * (jb + 1) * sizeof(T);
    if (sm > 48 * 1024)
      DUST_CUDA(cudaFuncSetAttribute(k_panel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sm));
    PanelArgs<T> pa{A, lda, k, jb, m, G, R, ipiv, info_dev, bar, err, cval, crow, crowv, srow};
    int cst = DUST_OK;
    if (panel_1cta_launch<T>(st, pa, &cst) || panel_cluster_launch<T>(st, pa, &cst)) {
      if (cst != DUST_OK) {
        dust_set_last_error("panel launch failed", __FILE__, __LINE__);
        return cst;
      }
    } else {
      void *args[] = {&pa};
      DUST_CUDA(cudaMemsetAsync(bar, 0, 8, st));
      DUST_CUDA(
          cudaLaunchCooperativeKernel((void *)k_panel<T>, dim3(G), dim3(PAN_T), args, sm, st));
    }
    if (n > jb || perm) {
      const size_t msm = (size_t)(n - k) * sizeof(int);
      static size_t opened = 48 * 1024;  // per element type
      if (msm > 200 * 1024) {
        lu_laswp<T>(st, A, lda, 0, k, k, k + jb, ipiv);
        lu_laswp<T>(st, A, lda, k + jb, n, k, k + jb, ipiv);
      } else {
        if (msm > opened) {
          DUST_CUDA(cudaFuncSetAttribute(k_laswp_net<T>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
          opened = 200 * 1024;
        }
        k_laswp_net<T><<<std::max(1, (n - jb + LW_C - 1) / LW_C), LW_T, msm, st>>>(A, lda, n, k,
                                                                                  jb, ipiv, perm);
      }
    }
    if (k + jb < n) {
      CUBLAS_OK(trsm_(cb, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_DIAG_UNIT, jb,
                      n - k - jb, A + k + (size_t)k * lda, lda, A + k + (size_t)(k + jb) * lda,
                      lda));
      int m2 = n - k - jb;
      if (gemm_update == 1 && sizeof(T) == 4) {
        DUST_TRY(gemm_tf32_minus(st, m2, m2, jb, (const float *)(A + (k + jb) + (size_t)k * lda),
                                 lda, (const float *)(A + k + (size_t)(k + jb) * lda), lda,
                                 (float *)(A + (k + jb) + (size_t)(k + jb) * lda), lda));
      } else {
        CUBLAS_OK(gemm_minus_(cb, m2, m2, jb, A + (k + jb) + (size_t)k * lda, lda,
                              A + k + (size_t)(k + jb) * lda, lda,
                              A + (k + jb) + (size_t)(k + jb) * lda, lda));
      }
    }
  }
  DUST_CUDA(cudaGetLastError());
  int herr = 0;
  DUST_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  DUST_CUDA(cudaStreamSynchronize(st));
  if (herr == 1) return DUST_ERR_TIMEOUT;
  if (herr) return DUST_ERR_CUDA;
  return DUST_OK;
}

template <typename T>
int lu_getrs(cublasHandle_t cb, cudaStream_t st, int n, int nrhs, const T *A, int lda,
             const int *ipiv, T *B, int ldb, const int *perm) {
  if (n <= 0 || nrhs <= 0) return DUST_OK;
  CUBLAS_OK(cublasSetStream(cb, st));
  const size_t psm = (size_t)n * sizeof(T);
  if (perm && psm <= 200 * 1024) {
    static size_t opened = 48 * 1024;  // per element type
    if (psm > opened) {
      DUST_CUDA(cudaFuncSetAttribute(k_permute_rows<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     200 * 1024));
      opened = 200 * 1024;
    }
    k_permute_rows<T><<<nrhs, 512, psm, st>>>(B, ldb, n, perm);
  } else {
    lu_laswp<T>(st, B, ldb, 0, nrhs, 0, n, ipiv);
  }
  CUBLAS_OK(trsm_(cb, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_DIAG_UNIT, n, nrhs, A,
                  lda, B, ldb));
  CUBLAS_OK(trsm_(cb, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_DIAG_NON_UNIT, n, nrhs,
                  A, lda, B, ldb));
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}

template int lu_getrf<double>(cublasHandle_t, cudaStream_t, LuWork &, int, double *, int, int *,
                              int *, int, int *);
template int lu_getrf<float>(cublasHandle_t, cudaStream_t, LuWork &, int, float *, int, int *,
                             int *, int, int *);
template void lu_laswp<double>(cudaStream_t, double *, int, int, int, int, int, const int *);
template void lu_laswp<float>(cudaStream_t, float *, int, int, int, int, int, const int *);
template int lu_getrs<double>(cublasHandle_t, cudaStream_t, int, int, const double *, int,
                              const int *, double *, int, const int *);
template int lu_getrs<float>(cublasHandle_t, cudaStream_t, int, int, const float *, int,
                             const int *, float *, int, const int *);
