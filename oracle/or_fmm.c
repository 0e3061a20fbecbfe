/*
 * or_fmm.c -- oracle (test infrastructure only): restatement of the
 * reference's octree FMM for vortex particles.
 *
 *   src/fmm/mod_multipole.f90   set_degree_polyexp :454-501, nbinom :505-520,
 *                               nfact :524-537, leaf_M :224-251, M2M :256-278,
 *                               M2L :282-356, L2L :360-384, compute_der_ker
 *                               :388-450
 *   src/fmm/mod_octree.f90      initialize_octree :251-518, sort_particles
 *                               :703-996, calculate_multipole :1002-1133,
 *                               apply_multipole :1139-1429
 *   src/aeroel/mod_vortpart.f90 compute_vel :139-155, compute_stretch
 *                               :176-227, compute_rotu :236-256,
 *                               kernel_coeffs :260-297, compute_diffusion
 *                               :305-324, etaeps :328-336
 *
 * Loop orders follow the reference so that summation orders match.  The
 * particle lists of the reference (finest-cell lists filled in particle
 * order, parents concatenating children 1..8 with x fastest) equal a stable
 * sort of the particles by a hierarchical Morton key; the oracle stores
 * every cell's list as a range of that sorted order.
 */
#include "dust_oracle.h"
#include "or_internal.h"

#include <omp.h>

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define MAXLEV 12

static int g_fact_wrap = 0;
void or_set_factorial_wrap(int on) { g_fact_wrap = on; }

/* Work sampling for the timed CPU baseline: with stride s > 1, M2L runs for
 * every s-th target cell only and the apply loop (L2P, P2P, elements) for
 * every s-th leaf; the tree, P2M, M2M and L2L run in full.  The results of
 * a sampled run are incomplete and serve timing only. */
static int g_stride = 1;
static double g_times[4];
static int64_t g_sampled[2];
void or_set_sample_stride(int s) { g_stride = s > 1 ? s : 1; }
/* OpenMP threads of every oracle loop */
void or_set_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
}
/* times (s) of the last or_fmm_apply: tree (init + sort), upward (P2M +
 * M2M), M2L + L2L, apply; sampled[0] = M2L pairs evaluated, sampled[1] =
 * particles evaluated in the apply loop */
void or_last_fmm_times(double *t4, int64_t *sampled) {
  for (int i = 0; i < 4; ++i) t4[i] = g_times[i];
  sampled[0] = g_sampled[0];
  sampled[1] = g_sampled[1];
}

/* ---------------------------------------------------------------- polyexp */
typedef struct {
  int deg, n_mon;
  int n_mon_d[64];
  int *idx; /* (deg+1)^3, -1 where i+j+k > deg */
  int *pwr; /* 3*n_mon */
  int32_t fact32[64];
  int64_t fact64[64];
} pexp_t;

static int pidx(const pexp_t *P, int i, int j, int k) {
  int D = P->deg + 1;
  return P->idx[i + D * (j + D * k)];
}

/* set_degree_polyexp, mod_multipole.f90:454-501 (0-based indices) */
static void pexp_set(pexp_t *P, int deg) {
  int D = deg + 1, ipol = 0;
  P->deg = deg;
  P->idx = (int *)malloc(sizeof(int) * D * D * D);
  for (int q = 0; q < D * D * D; ++q) P->idx[q] = -1;
  for (int o = 0; o <= deg; ++o) {
    for (int i = o; i >= 0; --i)
      for (int j = o - i; j >= 0; --j) {
        int k = o - j - i;
        P->idx[i + D * (j + D * k)] = ipol++;
      }
    P->n_mon_d[o] = ipol;
  }
  P->n_mon = ipol;
  P->pwr = (int *)malloc(sizeof(int) * 3 * ipol);
  ipol = 0;
  for (int o = 0; o <= deg; ++o)
    for (int i = o; i >= 0; --i)
      for (int j = o - i; j >= 0; --j) {
        int k = o - j - i;
        P->pwr[3 * ipol + 0] = i;
        P->pwr[3 * ipol + 1] = j;
        P->pwr[3 * ipol + 2] = k;
        ++ipol;
      }
  P->fact32[0] = 1;
  P->fact64[0] = 1;
  for (int o = 1; o <= deg; ++o) {
    /* default-integer arithmetic of the reference wraps modulo 2^32 */
    P->fact32[o] = (int32_t)((uint32_t)o * (uint32_t)P->fact32[o - 1]);
    P->fact64[o] = (int64_t)o * P->fact64[o - 1];
  }
}

static void pexp_free(pexp_t *P) {
  free(P->idx);
  free(P->pwr);
}

/* nfact_polyexp :524-537 as the integer the reference holds */
static int32_t nfact32(const pexp_t *P, int i, int j, int k) {
  uint32_t r = 1;
  r *= (uint32_t)P->fact32[i];
  r *= (uint32_t)P->fact32[j];
  r *= (uint32_t)P->fact32[k];
  return (int32_t)r;
}
static int64_t nfact64(const pexp_t *P, int i, int j, int k) {
  return P->fact64[i] * P->fact64[j] * P->fact64[k];
}

/* nbinom_polyexp :505-520 */
static int nbinom(const pexp_t *P, const int m[3], const int s[3]) {
  int64_t r = 1;
  for (int d = 0; d < 3; ++d)
    r *= P->fact64[m[d]] / (P->fact64[s[d]] * P->fact64[m[d] - s[d]]);
  return (int)r;
}

/* integer power as Fortran real**integer (x**0 == 1) */
static double ipow(double x, int e) {
  double r = 1.0;
  for (int q = 0; q < e; ++q) r *= x;
  return r;
}

/* compute_der_ker, mod_multipole.f90:388-450.
 * D: [3 * n_mon_d(deg-1)] as D(3,:), Dc: [9 * n_mon_d(deg-2)] as Dc(3,3,:) */
static void der_ker(const pexp_t *Pd, const double diff[3], double delta,
                    double *D, double *Dc) {
  int deg = Pd->deg;
  double *bk = (double *)calloc(Pd->n_mon, sizeof(double));
  double R2 = diff[0] * diff[0] + diff[1] * diff[1] + diff[2] * diff[2] +
              delta * delta;
  for (int k = 0; k <= deg; ++k)
    for (int j = 0; j <= deg - k; ++j)
      for (int i = 0; i <= deg - j - k; ++i) {
        double kmod = (double)(k + j + i);
        if (i == 0 && j == 0 && k == 0) {
          bk[pidx(Pd, 0, 0, 0)] = 1.0 / (4.0 * OR_PI * sqrt(R2));
        } else {
          double s1 = 0.0, s2 = 0.0;
          if (i - 1 >= 0) s1 += diff[0] * bk[pidx(Pd, i - 1, j, k)];
          if (j - 1 >= 0) s1 += diff[1] * bk[pidx(Pd, i, j - 1, k)];
          if (k - 1 >= 0) s1 += diff[2] * bk[pidx(Pd, i, j, k - 1)];
          if (i - 2 >= 0) s2 += bk[pidx(Pd, i - 2, j, k)];
          if (j - 2 >= 0) s2 += bk[pidx(Pd, i, j - 2, k)];
          if (k - 2 >= 0) s2 += bk[pidx(Pd, i, j, k - 2)];
          bk[pidx(Pd, i, j, k)] = 1.0 / (R2 * kmod) *
                                  ((2.0 * kmod - 1.0) * s1 - (kmod - 1.0) * s2);
        }
      }
  for (int k = 0; k <= deg - 1; ++k)
    for (int j = 0; j <= deg - 1 - k; ++j)
      for (int i = 0; i <= deg - 1 - j - k; ++i) {
        int q = pidx(Pd, i, j, k);
        D[3 * q + 0] = -(1.0 + i) * bk[pidx(Pd, i + 1, j, k)];
        D[3 * q + 1] = -(1.0 + j) * bk[pidx(Pd, i, j + 1, k)];
        D[3 * q + 2] = -(1.0 + k) * bk[pidx(Pd, i, j, k + 1)];
      }
  for (int k = 0; k <= deg - 2; ++k)
    for (int j = 0; j <= deg - 2 - k; ++j)
      for (int i = 0; i <= deg - 2 - j - k; ++i) {
        int q = pidx(Pd, i, j, k);
        int qi = pidx(Pd, i + 1, j, k), qj = pidx(Pd, i, j + 1, k),
            qk = pidx(Pd, i, j, k + 1);
        for (int c = 0; c < 3; ++c) {
          Dc[9 * q + 0 * 3 + c] = -(1.0 + i) * D[3 * qi + c];
          Dc[9 * q + 1 * 3 + c] = -(1.0 + j) * D[3 * qj + c];
          Dc[9 * q + 2 * 3 + c] = -(1.0 + k) * D[3 * qk + c];
        }
      }
  free(bk);
}

/* ------------------------------------------------------------------ tree */
typedef struct {
  double *a, *b, *c; /* a(3,n_mon), b(3,n_mon), c(3,3,n_mon) column-major */
} mp_t;

typedef struct {
  int ll, p, min_part, use_vs, use_divfilt, use_vd, use_tv;
  int nbox[3];
  double xmin[3], xmax[3], box_length, delta, nu_inf;
  int ncl[MAXLEV + 1][3];
  int64_t ncell[MAXLEV + 1];
  double csize[MAXLEV + 1];
  unsigned char *fl[MAXLEV + 1]; /* bit0 leaf, bit1 branch, bit2 active */
  mp_t *mp[MAXLEV + 1];
  double *cen[MAXLEV + 1];
  int64_t *ln_cnt[MAXLEV + 1];  /* leaf_neigh count per cell */
  int64_t **ln[MAXLEV + 1];     /* leaf_neigh: (level<<40 | lin)         */
  int kdlen[MAXLEV + 1][3];
  double *D[MAXLEV + 1], *Dc[MAXLEV + 1];
  int nD, nDc;
  pexp_t pe, pd;
  /* particles */
  int64_t *cstart; /* finest key -> first sorted position; size ncell_ll+1 */
  int64_t *perm;   /* sorted position -> caller index                       */
  int64_t nleaves;
  int *leaf_lev;
  int64_t *leaf_lin;
} tree_t;

static tree_t *g_last = NULL; /* kept for or_last_tree_flags */

#define FL_LEAF 1
#define FL_BRANCH 2
#define FL_ACTIVE 4

static inline int64_t lin_of(const tree_t *T, int l, int i, int j, int k) {
  return (int64_t)i + (int64_t)T->ncl[l][0] * ((int64_t)j + (int64_t)T->ncl[l][1] * k);
}
static inline void cart_of(const tree_t *T, int l, int64_t lin, int *i, int *j,
                           int *k) {
  *i = (int)(lin % T->ncl[l][0]);
  int64_t r = lin / T->ncl[l][0];
  *j = (int)(r % T->ncl[l][1]);
  *k = (int)(r / T->ncl[l][1]);
}
static inline uint64_t spread3(uint64_t v) {
  uint64_t r = 0;
  for (int b = 0; b < 21; ++b) r |= ((v >> b) & 1ull) << (3 * b);
  return r;
}
/* hierarchical key of a cell: level-1 box, then child index x+2y+4z per
 * level (the reference's child numbering p = ic + 2 jc + 4 kc, :344-366) */
static uint64_t key_of(const tree_t *T, int l, int i, int j, int k) {
  int sh = l - 1;
  uint64_t bx = (uint64_t)(i >> sh), by = (uint64_t)(j >> sh), bz = (uint64_t)(k >> sh);
  uint64_t m = (uint64_t)((1 << sh) - 1);
  uint64_t loc = spread3((uint64_t)i & m) | (spread3((uint64_t)j & m) << 1) |
                 (spread3((uint64_t)k & m) << 2);
  uint64_t box = bx + (uint64_t)T->nbox[0] * (by + (uint64_t)T->nbox[1] * bz);
  return (box << (3 * sh)) | loc;
}
static inline void cell_range(const tree_t *T, int l, int i, int j, int k,
                              int64_t *lo, int64_t *hi) {
  uint64_t key = key_of(T, l, i, j, k);
  int sh = 3 * (T->ll - l);
  *lo = T->cstart[key << sh];
  *hi = T->cstart[(key + 1) << sh];
}

static void mp_init(const tree_t *T, mp_t *m) {
  int n = T->pe.n_mon;
  if (!m->a) {
    m->a = (double *)calloc(3 * n, sizeof(double));
    m->b = (double *)calloc(3 * n, sizeof(double));
    if (T->use_vs) m->c = (double *)calloc(9 * n, sizeof(double));
  } else {
    memset(m->a, 0, sizeof(double) * 3 * n);
    memset(m->b, 0, sizeof(double) * 3 * n);
    if (T->use_vs) memset(m->c, 0, sizeof(double) * 9 * n);
  }
}
static void mp_destroy(mp_t *m) {
  free(m->a);
  free(m->b);
  free(m->c);
  m->a = m->b = m->c = NULL;
}

static void tree_free(tree_t *T) {
  if (!T) return;
  for (int l = 1; l <= T->ll; ++l) {
    if (T->mp[l])
      for (int64_t c = 0; c < T->ncell[l]; ++c) mp_destroy(&T->mp[l][c]);
    free(T->mp[l]);
    free(T->fl[l]);
    free(T->cen[l]);
    if (T->ln[l])
      for (int64_t c = 0; c < T->ncell[l]; ++c) free(T->ln[l][c]);
    free(T->ln[l]);
    free(T->ln_cnt[l]);
    free(T->D[l]);
    free(T->Dc[l]);
  }
  free(T->cstart);
  free(T->perm);
  free(T->leaf_lev);
  free(T->leaf_lin);
  pexp_free(&T->pe);
  pexp_free(&T->pd);
  free(T);
}

/* initialize_octree, mod_octree.f90:251-518 */
static tree_t *tree_init(const dust_fmm_params *prm) {
  tree_t *T = (tree_t *)calloc(1, sizeof(tree_t));
  T->ll = prm->n_octree_levels;
  T->p = prm->multipole_degree;
  T->min_part = prm->min_octree_part;
  T->use_vs = prm->vortstretch != 0;
  T->use_divfilt = prm->divergence_filtering != 0;
  T->use_vd = prm->diffusion != 0;
  T->use_tv = prm->turbulent_viscosity != 0;
  T->nu_inf = prm->nu_inf;
  T->box_length = prm->box_length;
  T->delta = prm->rankine_rad;
  for (int d = 0; d < 3; ++d) {
    T->nbox[d] = prm->n_box[d];
    T->xmin[d] = prm->origin[d];
    T->xmax[d] = prm->origin[d] + (double)prm->n_box[d] * prm->box_length;
  }
  pexp_set(&T->pe, T->p);
  pexp_set(&T->pd, 2 * T->p + 2);
  T->nD = T->pd.n_mon_d[T->pd.deg - 1];
  T->nDc = T->pd.n_mon_d[T->pd.deg - 2];
  for (int l = 1; l <= T->ll; ++l) {
    for (int d = 0; d < 3; ++d) T->ncl[l][d] = T->nbox[d] << (l - 1);
    T->ncell[l] = (int64_t)T->ncl[l][0] * T->ncl[l][1] * T->ncl[l][2];
    T->csize[l] = (l == 1) ? T->box_length
                           : T->box_length / (double)(1 << (l - 1));
    T->fl[l] = (unsigned char *)calloc(T->ncell[l], 1);
    T->mp[l] = (mp_t *)calloc(T->ncell[l], sizeof(mp_t));
    T->cen[l] = (double *)malloc(sizeof(double) * 3 * T->ncell[l]);
    T->ln[l] = (int64_t **)calloc(T->ncell[l], sizeof(int64_t *));
    T->ln_cnt[l] = (int64_t *)calloc(T->ncell[l], sizeof(int64_t));
    for (int64_t c = 0; c < T->ncell[l]; ++c) {
      int i, j, k;
      cart_of(T, l, c, &i, &j, &k);
      int ijk[3] = {i + 1, j + 1, k + 1};
      for (int d = 0; d < 3; ++d) {
        /* cen = xmin + (idx-0.5)*(xmax-xmin)/(nbox*2**(l-1)) (:324-327, 359) */
        double den = (l == 1) ? (double)T->nbox[d]
                              : (double)(T->nbox[d] * (1 << (l - 1)));
        T->cen[l][3 * c + d] =
            T->xmin[d] + ((double)ijk[d] - 0.5) * (T->xmax[d] - T->xmin[d]) / den;
      }
    }
  }
  /* kernel derivative tables (:486-516) */
  for (int l = 1; l <= T->ll; ++l) {
    for (int d = 0; d < 3; ++d)
      T->kdlen[l][d] = (l == 1) ? (T->nbox[d] > 3 ? T->nbox[d] : 3) : 3;
    int Lx = T->kdlen[l][0], Ly = T->kdlen[l][1], Lz = T->kdlen[l][2];
    int64_t nofs = (int64_t)(2 * Lx + 1) * (2 * Ly + 1) * (2 * Lz + 1);
    T->D[l] = (double *)calloc(nofs * 3 * T->nD, sizeof(double));
    T->Dc[l] = (double *)calloc(nofs * 9 * T->nDc, sizeof(double));
    int64_t q = 0;
    for (int k = -Lz; k <= Lz; ++k)
      for (int j = -Ly; j <= Ly; ++j)
        for (int i = -Lx; i <= Lx; ++i, ++q) {
          if (abs(i) >= 2 || abs(j) >= 2 || abs(k) >= 2) {
            double diff[3] = {T->csize[l] * (double)(-i), T->csize[l] * (double)(-j),
                              T->csize[l] * (double)(-k)};
            der_ker(&T->pd, diff, T->delta, T->D[l] + q * 3 * T->nD,
                    T->Dc[l] + q * 9 * T->nDc);
          }
        }
  }
  return T;
}

static int64_t kd_index(const tree_t *T, int l, int di, int dj, int dk) {
  int Lx = T->kdlen[l][0], Ly = T->kdlen[l][1], Lz = T->kdlen[l][2];
  return (int64_t)(di + Lx) + (int64_t)(2 * Lx + 1) *
                                  ((int64_t)(dj + Ly) + (int64_t)(2 * Ly + 1) * (dk + Lz));
}

static int tree_in(const tree_t *T, int l, int i, int j, int k) {
  return i >= 0 && j >= 0 && k >= 0 && i < T->ncl[l][0] && j < T->ncl[l][1] &&
         k < T->ncl[l][2];
}

static void set_leaf(tree_t *T, int l, int64_t c) {
  T->fl[l][c] |= FL_LEAF;
  T->leaf_lev[T->nleaves] = l;
  T->leaf_lin[T->nleaves] = c;
  T->nleaves++;
  T->fl[l][c] |= FL_ACTIVE;
  mp_init(T, &T->mp[l][c]);
}
static void set_branch(tree_t *T, int l, int64_t c) {
  T->fl[l][c] |= FL_BRANCH | FL_ACTIVE;
  mp_init(T, &T->mp[l][c]);
}
static void set_inactive(tree_t *T, int l, int64_t c) {
  T->fl[l][c] &= (unsigned char)~(FL_LEAF | FL_BRANCH | FL_ACTIVE);
  mp_destroy(&T->mp[l][c]);
}

static int64_t child_lin(const tree_t *T, int l, int i, int j, int k, int ch) {
  int ic = ch & 1, jc = (ch >> 1) & 1, kc = (ch >> 2) & 1;
  return lin_of(T, l + 1, 2 * i + ic, 2 * j + jc, 2 * k + kc);
}

/* sort_particles, mod_octree.f90:703-996 (no redistribution, no panels) */
static int tree_sort(tree_t *T, int n, const double *cen) {
  int ll = T->ll;
  double csize = T->csize[ll];
  int64_t ncl = T->ncell[ll];
  uint64_t *key = (uint64_t *)malloc(sizeof(uint64_t) * (n > 0 ? n : 1));
  for (int ip = 0; ip < n; ++ip) {
    int idx[3];
    for (int d = 0; d < 3; ++d)
      idx[d] = (int)ceil((cen[3 * ip + d] - T->xmin[d]) / csize);
    for (int d = 0; d < 3; ++d)
      if (idx[d] <= 0 || idx[d] > T->ncl[ll][d]) {
        free(key);
        return DUST_ERR_OUT_OF_BOX;
      }
    key[ip] = key_of(T, ll, idx[0] - 1, idx[1] - 1, idx[2] - 1);
  }
  /* stable counting sort by finest key */
  T->cstart = (int64_t *)calloc(ncl + 1, sizeof(int64_t));
  for (int ip = 0; ip < n; ++ip) T->cstart[key[ip] + 1]++;
  for (int64_t c = 0; c < ncl; ++c) T->cstart[c + 1] += T->cstart[c];
  int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * (ncl + 1));
  memcpy(fill, T->cstart, sizeof(int64_t) * (ncl + 1));
  T->perm = (int64_t *)malloc(sizeof(int64_t) * (n > 0 ? n : 1));
  for (int ip = 0; ip < n; ++ip) T->perm[fill[key[ip]]++] = ip;
  free(fill);
  free(key);

  int64_t maxleaves = ncl;
  T->leaf_lev = (int *)malloc(sizeof(int) * maxleaves);
  T->leaf_lin = (int64_t *)malloc(sizeof(int64_t) * maxleaves);
  T->nleaves = 0;
  for (int l = 1; l <= ll; ++l) memset(T->fl[l], 0, T->ncell[l]);

  /* bottom level (:898-908) */
  for (int k = 0; k < T->ncl[ll][2]; ++k)
    for (int j = 0; j < T->ncl[ll][1]; ++j)
      for (int i = 0; i < T->ncl[ll][0]; ++i) {
        int64_t lo, hi;
        cell_range(T, ll, i, j, k, &lo, &hi);
        if ((hi - lo) >= T->min_part || ll == 1)
          set_leaf(T, ll, lin_of(T, ll, i, j, k));
      }
  /* upward (:911-962) */
  for (int l = ll - 1; l >= 1; --l)
    for (int k = 0; k < T->ncl[l][2]; ++k)
      for (int j = 0; j < T->ncl[l][1]; ++j)
        for (int i = 0; i < T->ncl[l][0]; ++i) {
          int got_l = 0, got_b = 0;
          for (int ch = 0; ch < 8; ++ch) {
            unsigned char f = T->fl[l + 1][child_lin(T, l, i, j, k, ch)];
            if (f & FL_LEAF) got_l = 1;
            if (f & FL_BRANCH) got_b = 1;
          }
          int64_t c = lin_of(T, l, i, j, k);
          if (got_l || got_b) {
            for (int ch = 0; ch < 8; ++ch) {
              int64_t cc = child_lin(T, l, i, j, k, ch);
              unsigned char f = T->fl[l + 1][cc];
              if (!(f & FL_LEAF) && !(f & FL_BRANCH)) set_leaf(T, l + 1, cc);
            }
            set_branch(T, l, c);
          } else {
            for (int ch = 0; ch < 8; ++ch)
              set_inactive(T, l + 1, child_lin(T, l, i, j, k, ch));
            int64_t lo, hi;
            cell_range(T, l, i, j, k, &lo, &hi);
            if ((hi - lo) >= T->min_part || l == 1) set_leaf(T, l, c);
          }
        }
  /* leaf neighbours (:964-988) */
  for (int l = 2; l <= ll; ++l)
    for (int k = 0; k < T->ncl[l][2]; ++k)
      for (int j = 0; j < T->ncl[l][1]; ++j)
        for (int i = 0; i < T->ncl[l][0]; ++i) {
          int64_t c = lin_of(T, l, i, j, k);
          if (!(T->fl[l][c] & FL_ACTIVE)) continue;
          int pi_ = i >> 1, pj = j >> 1, pk = k >> 1;
          int64_t pc = lin_of(T, l - 1, pi_, pj, pk);
          int64_t np = T->ln_cnt[l - 1][pc];
          int64_t *lst = (int64_t *)malloc(sizeof(int64_t) * (np + 26));
          int64_t cnt = 0;
          for (int64_t q = 0; q < np; ++q) lst[cnt++] = T->ln[l - 1][pc][q];
          for (int kc = -1; kc <= 1; ++kc)
            for (int jc = -1; jc <= 1; ++jc)
              for (int ic = -1; ic <= 1; ++ic) {
                if (ic == 0 && jc == 0 && kc == 0) continue;
                if (!tree_in(T, l - 1, pi_ + ic, pj + jc, pk + kc)) continue;
                int64_t nc = lin_of(T, l - 1, pi_ + ic, pj + jc, pk + kc);
                if (T->fl[l - 1][nc] & FL_LEAF)
                  lst[cnt++] = ((int64_t)(l - 1) << 40) | nc;
              }
          T->ln[l][c] = lst;
          T->ln_cnt[l][c] = cnt;
        }
  return DUST_OK;
}

/* leaf_M_multipole :224-251 */
static void p2m(const tree_t *T, mp_t *m, const double *ccen, int64_t lo,
                int64_t hi, const double *cen, const double *dir,
                const double *mag) {
  int nmon = T->pe.n_mon;
  for (int q = 0; q < 3 * nmon; ++q) m->a[q] = 0.0;
  for (int mm = 0; mm < nmon; ++mm) {
    const int *pw = T->pe.pwr + 3 * mm;
    for (int64_t s = lo; s < hi; ++s) {
      int64_t ip = T->perm[s];
      double pr = ipow(cen[3 * ip] - ccen[0], pw[0]) *
                  ipow(cen[3 * ip + 1] - ccen[1], pw[1]) *
                  ipow(cen[3 * ip + 2] - ccen[2], pw[2]);
      for (int d = 0; d < 3; ++d)
        m->a[3 * mm + d] += mag[ip] * pr * dir[3 * ip + d];
    }
  }
}

/* M2M_multipole :256-278 */
static void m2m(const tree_t *T, mp_t *m, const double *cen, const mp_t *ch,
                const double *ccen) {
  int nmon = T->pe.n_mon;
  for (int mm = 0; mm < nmon; ++mm) {
    const int *id = T->pe.pwr + 3 * mm;
    for (int ks = 0; ks <= id[2]; ++ks)
      for (int js = 0; js <= id[1]; ++js)
        for (int is = 0; is <= id[0]; ++is) {
          int s = pidx(&T->pe, is, js, ks);
          int sv[3] = {is, js, ks};
          double w = (double)nbinom(&T->pe, id, sv) *
                     (ipow(ccen[0] - cen[0], id[0] - is) *
                      ipow(ccen[1] - cen[1], id[1] - js) *
                      ipow(ccen[2] - cen[2], id[2] - ks));
          for (int d = 0; d < 3; ++d) m->a[3 * mm + d] += w * ch->a[3 * s + d];
        }
  }
}

static inline void cross3(const double *a, const double *b, double *r) {
  r[0] = a[1] * b[2] - a[2] * b[1];
  r[1] = a[2] * b[0] - a[0] * b[2];
  r[2] = a[0] * b[1] - a[1] * b[0];
}

/* M2L_multipole :282-356 */
static void m2l(const tree_t *T, mp_t *m, const double *D, const double *Dc,
                const mp_t *src) {
  const pexp_t *P = &T->pe, *Pd = &T->pd;
  int nmon = P->n_mon;
  for (int mm = 0; mm < nmon; ++mm) {
    const int *pm = P->pwr + 3 * mm;
    double sv[3] = {0, 0, 0}, sg[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int nn = 0; nn < nmon; ++nn) {
      const int *pn = P->pwr + 3 * nn;
      int id[3] = {pm[0] + pn[0], pm[1] + pn[1], pm[2] + pn[2]};
      int q = pidx(Pd, id[0], id[1], id[2]);
      double mult;
      if (g_fact_wrap)
        mult = (double)nfact32(Pd, id[0], id[1], id[2]) /
               (double)(int32_t)((uint32_t)nfact32(P, pm[0], pm[1], pm[2]) *
                                 (uint32_t)nfact32(P, pn[0], pn[1], pn[2]));
      else
        mult = (double)nfact64(Pd, id[0], id[1], id[2]) /
               (double)(nfact64(P, pm[0], pm[1], pm[2]) *
                        nfact64(P, pn[0], pn[1], pn[2]));
      double cr[3];
      cross3(D + 3 * q, src->a + 3 * nn, cr);
      for (int d = 0; d < 3; ++d) sv[d] = sv[d] + mult * cr[d];
      if (T->use_vs)
        for (int r = 0; r < 3; ++r) {
          cross3(Dc + 9 * q + 3 * r, src->a + 3 * nn, cr);
          /* sum_g(r,:) = sum_g(r,:) + mult*cross(Dc(:,r,q), a) */
          for (int d = 0; d < 3; ++d) sg[r + 3 * d] = sg[r + 3 * d] + mult * cr[d];
        }
    }
    double sgn = ((pm[0] + pm[1] + pm[2]) & 1) ? -1.0 : 1.0;
    for (int d = 0; d < 3; ++d) m->b[3 * mm + d] += sgn * sv[d];
    if (T->use_vs)
      for (int q = 0; q < 9; ++q) m->c[9 * mm + q] += sgn * sg[q];
  }
}

/* L2L_multipole :360-384 (c stored as c(3,3,m): [9*m + r + 3*d]) */
static void l2l(const tree_t *T, mp_t *m, const double *cen, const mp_t *par,
                const double *pcen) {
  const pexp_t *P = &T->pe;
  int nmon = P->n_mon, deg = P->deg;
  for (int mm = 0; mm < nmon; ++mm) {
    const int *id = P->pwr + 3 * mm;
    for (int ks = id[2]; ks <= deg; ++ks)
      for (int js = id[1]; js <= deg - ks; ++js)
        for (int is = id[0]; is <= deg - ks - js; ++is) {
          int s = pidx(P, is, js, ks);
          int sv[3] = {is, js, ks};
          double mult = (double)nbinom(P, sv, id) *
                        (ipow(cen[0] - pcen[0], is - id[0]) *
                         ipow(cen[1] - pcen[1], js - id[1]) *
                         ipow(cen[2] - pcen[2], ks - id[2]));
          for (int d = 0; d < 3; ++d) m->b[3 * mm + d] += mult * par->b[3 * s + d];
          if (T->use_vs)
            for (int q = 0; q < 9; ++q) m->c[9 * mm + q] += mult * par->c[9 * s + q];
        }
  }
}

/* interaction list of cell (l,i,j,k) in the reference's order (:420-476) */
static int inter_list(const tree_t *T, int l, int i, int j, int k, int *li,
                      int *lj, int *lk, int cap) {
  int n = 0;
  if (l == 1) {
    for (int kc = 0; kc < T->ncl[1][2]; ++kc)
      for (int jc = 0; jc < T->ncl[1][1]; ++jc)
        for (int ic = 0; ic < T->ncl[1][0]; ++ic)
          if (abs(ic - i) > 1 || abs(jc - j) > 1 || abs(kc - k) > 1) {
            if (n < cap) { li[n] = ic; lj[n] = jc; lk[n] = kc; }
            ++n;
          }
    return n;
  }
  int pi_ = i >> 1, pj = j >> 1, pk = k >> 1;
  for (int kc = -1; kc <= 1; ++kc)
    for (int jc = -1; jc <= 1; ++jc)
      for (int ic = -1; ic <= 1; ++ic) {
        if (ic == 0 && jc == 0 && kc == 0) continue;
        if (!tree_in(T, l - 1, pi_ + ic, pj + jc, pk + kc)) continue;
        for (int ch = 0; ch < 8; ++ch) {
          int ci = 2 * (pi_ + ic) + (ch & 1), cj = 2 * (pj + jc) + ((ch >> 1) & 1),
              ck = 2 * (pk + kc) + ((ch >> 2) & 1);
          if (abs(ci - i) > 1 || abs(cj - j) > 1 || abs(ck - k) > 1) {
            if (n < cap) { li[n] = ci; lj[n] = cj; lk[n] = ck; }
            ++n;
          }
        }
      }
  return n;
}

/* calculate_multipole :1002-1133 */
static int64_t tree_multipole(tree_t *T, const double *cen, const double *dir,
                              const double *mag) {
  int ll = T->ll;
  int64_t npairs = 0;
  double t0 = omp_get_wtime();
#pragma omp parallel for schedule(guided)
  for (int64_t lv = 0; lv < T->nleaves; ++lv) {
    int l = T->leaf_lev[lv];
    int64_t c = T->leaf_lin[lv];
    int i, j, k;
    cart_of(T, l, c, &i, &j, &k);
    int64_t lo, hi;
    cell_range(T, l, i, j, k, &lo, &hi);
    p2m(T, &T->mp[l][c], T->cen[l] + 3 * c, lo, hi, cen, dir, mag);
  }
  for (int l = ll - 1; l >= 1; --l) {
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < T->ncell[l]; ++c) {
      unsigned char f = T->fl[l][c];
      if ((f & FL_ACTIVE) && (f & FL_BRANCH)) {
        int i, j, k;
        cart_of(T, l, c, &i, &j, &k);
        for (int ch = 0; ch < 8; ++ch) {
          int64_t cc = child_lin(T, l, i, j, k, ch);
          m2m(T, &T->mp[l][c], T->cen[l] + 3 * c, &T->mp[l + 1][cc],
              T->cen[l + 1] + 3 * cc);
        }
      }
    }
  }
  g_times[1] = omp_get_wtime() - t0;
  t0 = omp_get_wtime();
  for (int l = 1; l <= ll; ++l) {
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : npairs)
    for (int64_t c = 0; c < T->ncell[l]; ++c) {
      if (!(T->fl[l][c] & FL_ACTIVE)) continue;
      if (g_stride > 1 && c % g_stride != 0) continue;
      int i, j, k;
      cart_of(T, l, c, &i, &j, &k);
      int cap = (l == 1) ? (int)T->ncell[1] : 216;
      int *li = (int *)malloc(sizeof(int) * 3 * cap);
      int n = inter_list(T, l, i, j, k, li, li + cap, li + 2 * cap, cap);
      for (int q = 0; q < n; ++q) {
        int64_t sc = lin_of(T, l, li[q], li[cap + q], li[2 * cap + q]);
        if (!(T->fl[l][sc] & FL_ACTIVE)) continue;
        int64_t kd = kd_index(T, l, li[q] - i, li[cap + q] - j, li[2 * cap + q] - k);
        m2l(T, &T->mp[l][c], T->D[l] + kd * 3 * T->nD, T->Dc[l] + kd * 9 * T->nDc,
            &T->mp[l][sc]);
        ++npairs;
      }
      free(li);
    }
    if (l < ll) {
#pragma omp parallel for schedule(dynamic)
      for (int64_t c = 0; c < T->ncell[l]; ++c) {
        if (!(T->fl[l][c] & FL_ACTIVE)) continue;
        int i, j, k;
        cart_of(T, l, c, &i, &j, &k);
        for (int ch = 0; ch < 8; ++ch) {
          int64_t cc = child_lin(T, l, i, j, k, ch);
          if (T->fl[l + 1][cc] & FL_ACTIVE)
            l2l(T, &T->mp[l + 1][cc], T->cen[l + 1] + 3 * cc, &T->mp[l][c],
                T->cen[l] + 3 * c);
        }
      }
    }
  }
  g_times[2] = omp_get_wtime() - t0;
  g_sampled[0] = npairs;
  return npairs;
}

/* kernel_coeffs :260-297 (Rosenhead) */
static inline void kernel_coeffs(double r_vort, double rr, double *c, double *d) {
  double distn = sqrt(rr * rr + r_vort * r_vort);
  *c = -1.0 / (distn * distn * distn);
  *d = 3.0 / (distn * distn * distn * distn * distn);
}
static inline double norm3(const double *v) {
  return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
}

/* the P2P contribution of source q on target p (one pass of the inner
 * loops at mod_octree.f90:1257-1348) */
static inline void p2p_pair(const tree_t *T, const double *pos, const double *alpha,
                            double nu_eff, int64_t q, const double *cen,
                            const double *dir, const double *mag,
                            const double *rv, double *vel, double *str,
                            double *rot) {
  double dist[3] = {pos[0] - cen[3 * q], pos[1] - cen[3 * q + 1],
                    pos[2] - cen[3 * q + 2]};
  double distn = norm3(dist), c, d;
  kernel_coeffs(rv[q], distn, &c, &d);
  const double *dq = dir + 3 * q;
  double mq = mag[q];
  /* compute_vel :139-155 */
  double cr[3];
  cross3(dist, dq, cr);
  for (int e = 0; e < 3; ++e) vel[e] += (c * cr[e] * mq) / (4.0 * OR_PI);
  if (T->use_vs) {
    /* compute_stretch :176-227 */
    double aq[3] = {dq[0] * mq, dq[1] * mq, dq[2] * mq}, vp[3];
    cross3(alpha, aq, vp);
    double dv = dist[0] * vp[0] + dist[1] * vp[1] + dist[2] * vp[2];
    for (int e = 0; e < 3; ++e)
      str[e] += (-(c * vp[e] + d * dist[e] * dv)) / (4.0 * OR_PI);
    if (T->use_divfilt) {
      /* compute_rotu :236-256 */
      double t1[3], t2[3];
      cross3(dist, aq, t1);
      cross3(dist, t1, t2);
      for (int e = 0; e < 3; ++e)
        rot[e] += (-2.0 * c * aq[e] + d * t2[e]) / (4.0 * OR_PI);
    }
  }
  if (T->use_vd) {
    /* compute_diffusion :305-324, etaeps :328-336 */
    double s = rv[q];
    double vol = 4.0 / 3.0 * OR_PI * s * s * s;
    double x = distn / s;
    double eta = 105.0 / (8.0 * OR_PI) / pow(x * x + 1.0, 4.5);
    eta = eta / (s * s * s);
    for (int e = 0; e < 3; ++e) {
      double df = 1.0 / (s * s) * (vol * dq[e] * mq - vol * alpha[e]) * eta;
      str[e] += df * nu_eff;
    }
  }
}

/* apply_multipole :1139-1429 */
static int64_t tree_apply(tree_t *T, int n, const double *cen, const double *dir,
                          const double *mag, const double *rv,
                          const dust_fmm_params *prm, const or_elemctx *ectx,
                          double *vel_o, double *str_o, double *rot_o) {
  const pexp_t *P = &T->pe;
  int nmon = P->n_mon;
  int64_t npairs = 0, nsampled = 0;
  (void)n;
#pragma omp parallel for schedule(dynamic) reduction(+ : npairs, nsampled)
  for (int64_t lv = 0; lv < T->nleaves; ++lv) {
    if (g_stride > 1 && lv % g_stride != 0) continue;
    int l = T->leaf_lev[lv];
    int64_t c = T->leaf_lin[lv];
    int i, j, k;
    cart_of(T, l, c, &i, &j, &k);
    int64_t lo, hi;
    cell_range(T, l, i, j, k, &lo, &hi);
    int64_t np = hi - lo;
    nsampled += np;
    const mp_t *m = &T->mp[l][c];
    const double *cc = T->cen[l] + 3 * c;
    double *velv = (double *)calloc(3 * (np > 0 ? np : 1), sizeof(double));
    double *strv = (double *)calloc(3 * (np > 0 ? np : 1), sizeof(double));
    double *rotv = (double *)calloc(3 * (np > 0 ? np : 1), sizeof(double));
    double ave_ros = 0.0;
    for (int64_t s = 0; s < np; ++s) {
      int64_t ip = T->perm[lo + s];
      const double *pos = cen + 3 * ip;
      double alpha[3] = {mag[ip] * dir[3 * ip], mag[ip] * dir[3 * ip + 1],
                         mag[ip] * dir[3 * ip + 2]};
      double v[3] = {0, 0, 0}, g[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int mm = 0; mm < nmon; ++mm) {
        const int *pw = P->pwr + 3 * mm;
        double pr = ipow(pos[0] - cc[0], pw[0]) * ipow(pos[1] - cc[1], pw[1]) *
                    ipow(pos[2] - cc[2], pw[2]);
        for (int e = 0; e < 3; ++e) v[e] = v[e] + m->b[3 * mm + e] * pr;
        if (T->use_vs)
          for (int q = 0; q < 9; ++q) g[q] = g[q] + m->c[9 * mm + q] * pr;
      }
      for (int e = 0; e < 3; ++e) velv[3 * s + e] = v[e];
      if (T->use_vs) {
        /* str = matmul(alpha, transpose(grad)): str(i) = sum_j alpha(j) grad(i,j) */
        for (int e = 0; e < 3; ++e)
          strv[3 * s + e] = alpha[0] * g[e + 0] + alpha[1] * g[e + 3] + alpha[2] * g[e + 6];
        if (T->use_divfilt) {
          /* grad(i,j) = g[i + 3j] */
          rotv[3 * s + 0] = g[1 + 6] - g[2 + 3];
          rotv[3 * s + 1] = g[2 + 0] - g[0 + 6];
          rotv[3 * s + 2] = g[0 + 3] - g[1 + 0];
        }
      }
      if (T->use_vd) {
        double acc = 0.0;
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) {
            double sym = 0.5 * (g[a + 3 * b] + g[b + 3 * a]);
            acc += sym * sym;
          }
        ave_ros += acc;
      }
    }
    if (T->use_vd && np > 0) ave_ros /= (double)np;

    for (int64_t s = 0; s < np; ++s) {
      int64_t ip = T->perm[lo + s];
      const double *pos = cen + 3 * ip;
      double alpha[3] = {mag[ip] * dir[3 * ip], mag[ip] * dir[3 * ip + 1],
                         mag[ip] * dir[3 * ip + 2]};
      double v[3] = {velv[3 * s], velv[3 * s + 1], velv[3 * s + 2]};
      double st[3] = {strv[3 * s], strv[3 * s + 1], strv[3 * s + 2]};
      double ro[3] = {rotv[3 * s], rotv[3 * s + 1], rotv[3 * s + 2]};
      double tv = T->use_tv ? (0.11 * rv[ip]) * (0.11 * rv[ip]) * sqrt(2.0 * ave_ros) : 0.0;
      double nu_eff = T->nu_inf + tv;
      /* 26 same-level neighbours */
      for (int kk = -1; kk <= 1; ++kk)
        for (int jj = -1; jj <= 1; ++jj)
          for (int ii = -1; ii <= 1; ++ii) {
            if (ii == 0 && jj == 0 && kk == 0) continue;
            if (!tree_in(T, l, i + ii, j + jj, k + kk)) continue;
            int64_t nc = lin_of(T, l, i + ii, j + jj, k + kk);
            if (!(T->fl[l][nc] & FL_ACTIVE)) continue;
            int64_t nlo, nhi;
            cell_range(T, l, i + ii, j + jj, k + kk, &nlo, &nhi);
            for (int64_t t = nlo; t < nhi; ++t) {
              p2p_pair(T, pos, alpha, nu_eff, T->perm[t], cen, dir, mag, rv, v, st, ro);
              ++npairs;
            }
          }
      /* leaf neighbours */
      int64_t nln = (l >= 2) ? T->ln_cnt[l][c] : 0;
      for (int64_t q = 0; q < nln; ++q) {
        int64_t e = T->ln[l][c][q];
        int el_ = (int)(e >> 40);
        int64_t elin = e & ((1ll << 40) - 1);
        int ei, ej, ek;
        cart_of(T, el_, elin, &ei, &ej, &ek);
        int64_t nlo, nhi;
        cell_range(T, el_, ei, ej, ek, &nlo, &nhi);
        for (int64_t t = nlo; t < nhi; ++t) {
          p2p_pair(T, pos, alpha, nu_eff, T->perm[t], cen, dir, mag, rv, v, st, ro);
          ++npairs;
        }
      }
      /* own leaf, skipping self */
      for (int64_t t = lo; t < hi; ++t) {
        if (t == lo + s) continue;
        p2p_pair(T, pos, alpha, nu_eff, T->perm[t], cen, dir, mag, rv, v, st, ro);
        ++npairs;
      }
      /* non-particle elements + wind (:1350-1373) */
      or_elements_vel_accum(prm, ectx, pos, v);
      for (int e = 0; e < 3; ++e) {
        vel_o[3 * ip + e] = v[e];
        if (str_o) str_o[3 * ip + e] = (T->use_vs || T->use_vd) ? st[e] : 0.0;
        if (rot_o) rot_o[3 * ip + e] = (T->use_vs && T->use_divfilt) ? ro[e] : 0.0;
      }
    }
    free(velv);
    free(strv);
    free(rotv);
  }
  g_sampled[1] = nsampled;
  return npairs;
}

int or_fmm_apply(const dust_fmm_params *prm, int n, const double *cen,
                 const double *dir, const double *mag, const double *r_vortex,
                 const dust_elements *elems, double *vel, double *stretch,
                 double *rotu, int64_t *counters) {
  if (!prm || n < 0 || prm->n_octree_levels < 1 ||
      prm->n_octree_levels > MAXLEV || prm->multipole_degree < 0)
    return DUST_ERR_BAD_ARG;
  double t0 = omp_get_wtime();
  tree_t *T = tree_init(prm);
  int st = tree_sort(T, n, cen);
  if (st != DUST_OK) {
    tree_free(T);
    return st;
  }
  g_times[0] = omp_get_wtime() - t0;
  int64_t m2lp = tree_multipole(T, cen, dir, mag);
  t0 = omp_get_wtime();
  or_elemctx *ectx = or_elemctx_build(elems, prm->u_inf);
  int64_t p2pp = tree_apply(T, n, cen, dir, mag, r_vortex, prm, ectx, vel,
                            stretch, rotu);
  or_elemctx_free(ectx);
  g_times[3] = omp_get_wtime() - t0;
  if (counters) {
    int64_t act = 0;
    for (int l = 1; l <= T->ll; ++l)
      for (int64_t c = 0; c < T->ncell[l]; ++c) act += (T->fl[l][c] & FL_ACTIVE) ? 1 : 0;
    counters[0] = T->nleaves;
    counters[1] = act;
    counters[2] = m2lp;
    counters[3] = p2pp;
  }
  tree_free(g_last);
  g_last = T;
  return DUST_OK;
}

/* Velocity of one vortex particle q at pos (compute_vel of t_vortpart,
 * mod_vortpart.f90:139-155, divided by 4 pi as the callers do). */
static inline void part_vel(const double *pos, int64_t q, const double *cen, const double *dir,
                            const double *mag, const double *rv, double *u) {
  double dist[3] = {pos[0] - cen[3 * q], pos[1] - cen[3 * q + 1], pos[2] - cen[3 * q + 2]};
  double distn = norm3(dist);
  double dn = sqrt(distn * distn + rv[q] * rv[q]);
  double c = -1.0 / (dn * dn * dn), cr[3];
  cross3(dist, dir + 3 * q, cr);
  for (int d = 0; d < 3; ++d) u[d] = u[d] + (c * cr[d] * mag[q]) / (4.0 * OR_PI);
}

/* apply_multipole_panels (mod_octree.f90:1433-1508): the particles' velocity
 * at points (panel centres) from the FMM -- each point is sorted into the
 * finest cell that holds it (sort_particles, :776-799) and takes the local
 * expansion of the leaf above it, then the particles of that leaf's 26
 * active same-level neighbours, of its leaf_neigh and of the leaf itself --
 * plus the end vortices by direct sum (the vortical elements get_vort_vel
 * keeps in vort_p when the particles go through the FMM, mod_wake.f90:
 * 819-845).  The reference adds the FMM part to uvort and then resets uvort
 * in get_vort_vel (mod_surfpan.f90:970); here the sum is returned. */
int or_fmm_points_uvort(const dust_fmm_params *prm, int n, const double *cen,
                        const double *dir, const double *mag, const double *r_vortex,
                        int n_pts, const double *pts, const dust_lines *end_vort,
                        double *uvort) {
  if (!prm || n < 0 || n_pts < 0 || prm->n_octree_levels < 1 ||
      prm->n_octree_levels > MAXLEV || prm->multipole_degree < 0)
    return DUST_ERR_BAD_ARG;
  tree_t *T = tree_init(prm);
  int st = tree_sort(T, n, cen);
  if (st != DUST_OK) {
    tree_free(T);
    return st;
  }
  tree_multipole(T, cen, dir, mag);
  const int ll = T->ll;
  const pexp_t *P = &T->pe;
  int nl = end_vort ? end_vort->n : 0;
  or_line_t *ls = (or_line_t *)malloc(sizeof(or_line_t) * (nl + 1));
  for (int j = 0; j < nl; ++j) or_line_build(end_vort, j, &ls[j]);
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 4)
  for (int ip = 0; ip < n_pts; ++ip) {
    const double *pos = pts + 3 * ip;
    int idx[3];
    for (int d = 0; d < 3; ++d) idx[d] = (int)ceil((pos[d] - T->xmin[d]) / T->csize[ll]);
    int out = 0;
    for (int d = 0; d < 3; ++d) out |= idx[d] <= 0 || idx[d] > T->ncl[ll][d];
    if (out) {
      bad = 1;
      continue;
    }
    /* the leaf above the finest cell */
    int l = 1, i = 0, j = 0, k = 0;
    int64_t c = -1;
    for (int lv = 1; lv <= ll; ++lv) {
      int sh = ll - lv;
      i = (idx[0] - 1) >> sh, j = (idx[1] - 1) >> sh, k = (idx[2] - 1) >> sh;
      int64_t cc = lin_of(T, lv, i, j, k);
      if (T->fl[lv][cc] & FL_LEAF) {
        l = lv;
        c = cc;
        break;
      }
    }
    double v[3] = {0, 0, 0};
    if (c >= 0) {
      const mp_t *m = &T->mp[l][c];
      const double *cc = T->cen[l] + 3 * c;
      for (int mm = 0; mm < P->n_mon; ++mm) {
        const int *pw = P->pwr + 3 * mm;
        double pr = ipow(pos[0] - cc[0], pw[0]) * ipow(pos[1] - cc[1], pw[1]) *
                    ipow(pos[2] - cc[2], pw[2]);
        for (int e = 0; e < 3; ++e) v[e] = v[e] + m->b[3 * mm + e] * pr;
      }
      for (int kk = -1; kk <= 1; ++kk)
        for (int jj = -1; jj <= 1; ++jj)
          for (int ii = -1; ii <= 1; ++ii) {
            if (ii == 0 && jj == 0 && kk == 0) continue;
            if (!tree_in(T, l, i + ii, j + jj, k + kk)) continue;
            int64_t nc = lin_of(T, l, i + ii, j + jj, k + kk);
            if (!(T->fl[l][nc] & FL_ACTIVE)) continue;
            int64_t nlo, nhi;
            cell_range(T, l, i + ii, j + jj, k + kk, &nlo, &nhi);
            for (int64_t t = nlo; t < nhi; ++t)
              part_vel(pos, T->perm[t], cen, dir, mag, r_vortex, v);
          }
      int64_t nln = (l >= 2) ? T->ln_cnt[l][c] : 0;
      for (int64_t q = 0; q < nln; ++q) {
        int64_t e = T->ln[l][c][q];
        int el_ = (int)(e >> 40);
        int64_t elin = e & ((1ll << 40) - 1);
        int ei, ej, ek;
        cart_of(T, el_, elin, &ei, &ej, &ek);
        int64_t nlo, nhi;
        cell_range(T, el_, ei, ej, ek, &nlo, &nhi);
        for (int64_t t = nlo; t < nhi; ++t)
          part_vel(pos, T->perm[t], cen, dir, mag, r_vortex, v);
      }
      int64_t lo, hi;
      cell_range(T, l, i, j, k, &lo, &hi);
      for (int64_t t = lo; t < hi; ++t) part_vel(pos, T->perm[t], cen, dir, mag, r_vortex, v);
    }
    for (int q = 0; q < nl; ++q) {
      double w[3];
      or_vel_line(prm, &ls[q], pos, w);
      for (int d = 0; d < 3; ++d) v[d] = v[d] + w[d] / (4.0 * OR_PI);
    }
    for (int d = 0; d < 3; ++d) uvort[3 * ip + d] = v[d];
  }
  free(ls);
  tree_free(T);
  return bad ? DUST_ERR_OUT_OF_BOX : DUST_OK;
}

int or_last_tree_flags(unsigned char *flags, int64_t cap) {
  if (!g_last) return DUST_ERR_BAD_ARG;
  tree_t *T = g_last;
  int64_t off = 0;
  for (int l = 1; l <= T->ll; ++l) {
    if (off + T->ncell[l] > cap) return DUST_ERR_CAPACITY;
    for (int k = 0; k < T->ncl[l][2]; ++k)
      for (int j = 0; j < T->ncl[l][1]; ++j)
        for (int i = 0; i < T->ncl[l][0]; ++i)
          flags[off + (int64_t)key_of(T, l, i, j, k)] = T->fl[l][lin_of(T, l, i, j, k)];
    off += T->ncell[l];
  }
  return DUST_OK;
}

int or_direct_particles(const dust_fmm_params *prm, int n, const double *cen,
                        const double *dir, const double *mag,
                        const double *r_vortex, int n_tgt, double *vel,
                        double *stretch, double *rotu) {
  tree_t T;
  memset(&T, 0, sizeof(T));
  T.use_vs = prm->vortstretch != 0;
  T.use_divfilt = prm->divergence_filtering != 0;
  T.use_vd = prm->diffusion != 0;
  T.nu_inf = prm->nu_inf;
#pragma omp parallel for schedule(static)
  for (int ip = 0; ip < n_tgt; ++ip) {
    const double *pos = cen + 3 * ip;
    double alpha[3] = {mag[ip] * dir[3 * ip], mag[ip] * dir[3 * ip + 1],
                       mag[ip] * dir[3 * ip + 2]};
    double v[3] = {0, 0, 0}, s[3] = {0, 0, 0}, r[3] = {0, 0, 0};
    for (int q = 0; q < n; ++q) {
      if (q == ip) continue;
      p2p_pair(&T, pos, alpha, T.nu_inf, q, cen, dir, mag, r_vortex, v, s, r);
    }
    for (int e = 0; e < 3; ++e) {
      vel[3 * ip + e] = v[e];
      if (stretch) stretch[3 * ip + e] = s[e];
      if (rotu) rotu[3 * ip + e] = r[e];
    }
  }
  return DUST_OK;
}
