// dust_common.cuh -- shared device helpers of the sm_100a implementation.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>

#include "../../include/dust_b200.h"

#define DUST_MAXLEV 16
#define DUST_MAXP 8
#define DUST_PI 3.14159265358979323846

// Status propagation for host code: any CUDA error becomes DUST_ERR_CUDA.
#define DUST_CUDA(call)                                                        \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      dust_set_last_error(cudaGetErrorString(e_), __FILE__, __LINE__);         \
      return DUST_ERR_CUDA;                                                    \
    }                                                                          \
  } while (0)

#define DUST_TRY(expr)                                                         \
  do {                                                                         \
    int s_ = (expr);                                                           \
    if (s_ != DUST_OK) return s_;                                              \
  } while (0)

void dust_set_last_error(const char *msg, const char *file, int line);

// ------------------------------------------------------------ monomials
// Monomial ordering of the reference (set_degree_polyexp,
// src/fmm/mod_multipole.f90:454-501): by total degree o, then i descending,
// then j descending.  Closed form of its index (0-based).
__host__ __device__ inline int mono_idx(int i, int j, int k) {
  int o = i + j + k, a = j + k;
  return o * (o + 1) * (o + 2) / 6 + a * (a + 1) / 2 + (a - j);
}
__host__ __device__ inline int n_mon(int p) { return (p + 1) * (p + 2) * (p + 3) / 6; }
__host__ __device__ inline void mono_exp(int m, int &i, int &j, int &k) {
  int o = 0;
  while ((o + 1) * (o + 2) * (o + 3) / 6 <= m) ++o;
  int r = m - o * (o + 1) * (o + 2) / 6;
  int a = 0;
  while ((a + 1) * (a + 2) / 2 <= r) ++a;
  j = a - (r - a * (a + 1) / 2);
  k = a - j;
  i = o - a;
}

// ------------------------------------------------------------ cell keys
// A cell of level l (1-based) is identified by its hierarchical key:
// level-1 box index (x fastest over n_box), then one octal digit per level
// with child number x + 2y + 4z -- the reference's child numbering
// p = ic + 2 jc + 4 kc (mod_octree.f90:344-366).  Children of key K are
// 8K .. 8K+7, so every cell at every level owns a contiguous key range of
// the finest level, and (after a stable sort by finest key) a contiguous
// range of particles.
__host__ __device__ inline uint32_t spread3(uint32_t v) {
  v &= 0x3ff;
  v = (v | (v << 16)) & 0x030000FF;
  v = (v | (v << 8)) & 0x0300F00F;
  v = (v | (v << 4)) & 0x030C30C3;
  v = (v | (v << 2)) & 0x09249249;
  return v;
}
__host__ __device__ inline uint32_t compact3(uint32_t v) {
  v &= 0x09249249;
  v = (v ^ (v >> 2)) & 0x030C30C3;
  v = (v ^ (v >> 4)) & 0x0300F00F;
  v = (v ^ (v >> 8)) & 0x030000FF;
  v = (v ^ (v >> 16)) & 0x000003FF;
  return v;
}

struct TreeGeom {
  int ll;                       // number of levels
  int nbox[3];
  double xmin[3], xmax[3];
  int ncl[DUST_MAXLEV + 1][3];  // cells per direction per level
  uint32_t ncell[DUST_MAXLEV + 1];
  uint32_t lev_off[DUST_MAXLEV + 2];  // offsets of levels in concatenated
                                      // per-cell arrays
  double csize[DUST_MAXLEV + 1];
};

__host__ __device__ inline uint32_t key_of(const TreeGeom &G, int l, int i, int j,
                                           int k) {
  int sh = l - 1;
  uint32_t m = (1u << sh) - 1u;
  uint32_t box = (uint32_t)(i >> sh) +
                 (uint32_t)G.nbox[0] * ((uint32_t)(j >> sh) + (uint32_t)G.nbox[1] *
                                                                (uint32_t)(k >> sh));
  uint32_t loc = spread3((uint32_t)i & m) | (spread3((uint32_t)j & m) << 1) |
                 (spread3((uint32_t)k & m) << 2);
  return (box << (3 * sh)) | loc;
}
__host__ __device__ inline void cart_of_key(const TreeGeom &G, int l, uint32_t key,
                                            int &i, int &j, int &k) {
  int sh = l - 1;
  uint32_t box = key >> (3 * sh);
  uint32_t loc = key & ((1u << (3 * sh)) - 1u);
  int bx = (int)(box % (uint32_t)G.nbox[0]);
  uint32_t r = box / (uint32_t)G.nbox[0];
  int by = (int)(r % (uint32_t)G.nbox[1]);
  int bz = (int)(r / (uint32_t)G.nbox[1]);
  i = (bx << sh) | (int)compact3(loc);
  j = (by << sh) | (int)compact3(loc >> 1);
  k = (bz << sh) | (int)compact3(loc >> 2);
}
// Cell centre exactly as initialize_octree computes it
// (mod_octree.f90:324-327, 358-361).
__host__ __device__ inline void cell_center(const TreeGeom &G, int l, int i, int j,
                                            int k, double *c) {
  int ijk[3] = {i + 1, j + 1, k + 1};
  for (int d = 0; d < 3; ++d) {
    double den = (l == 1) ? (double)G.nbox[d] : (double)(G.nbox[d] * (1 << (l - 1)));
    c[d] = G.xmin[d] + ((double)ijk[d] - 0.5) * (G.xmax[d] - G.xmin[d]) / den;
  }
}
__host__ __device__ inline bool cart_in(const TreeGeom &G, int l, int i, int j, int k) {
  return i >= 0 && j >= 0 && k >= 0 && i < G.ncl[l][0] && j < G.ncl[l][1] &&
         k < G.ncl[l][2];
}

#define FL_LEAF 1
#define FL_BRANCH 2
#define FL_ACTIVE 4
#define FL_PTS 8  // an empty leaf that holds evaluation points (its locals are needed)

