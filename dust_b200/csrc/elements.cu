// elements.cu -- panel/line geometry on the device, element and particle
// direct sums (velocity at points, uvort at panel centres), and the all-pairs
// particle evaluation used as FMM truth.
//
//   element -> point velocity: compute_vel of surfpan/vortlatt/vortline
//     (mod_surfpan.f90:641-658, mod_vortlatt.f90:403-415,
//      mod_vortline.f90:126-170) as summed in apply_multipole
//     (mod_octree.f90:1350-1373)
//   particle -> panel uvort: get_vort_vel_surfpan/vortlatt
//     (mod_surfpan.f90:962-977, mod_vortlatt.f90:676-693)
#include <algorithm>
#include <cstring>

#include "dust_common.cuh"
#include "elements.cuh"
#include "fmm_internal.h"

RegParams reg_params(const dust_fmm_params *prm) {
  RegParams r;
  r.ff_dou = prm->far_field_ratio_doublet;
  r.r_rankine = prm->rankine_rad;
  r.r_cutoff = prm->cutoff_rad;
  return r;
}

static inline unsigned nblk(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

// raw (device) arrays of a panel set
struct PanRaw {
  int n;
  const int *n_ver, *kind;
  const double *ver, *mag, *ub, *uvort;
};

__global__ void k_panel_build(PanRaw r, double u0, double u1, double u2, PanelGeo *out) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= r.n) return;
  double u[3] = {u0, u1, u2};
  PanelGeo p;
  panel_build(r.ver + 12 * (size_t)j, r.n_ver ? r.n_ver[j] : 4,
              r.kind ? r.kind[j] : DUST_ELEM_VORTLATT, r.mag ? r.mag[j] : 0.0,
              r.ub ? r.ub + 3 * (size_t)j : nullptr, r.uvort ? r.uvort + 3 * (size_t)j : nullptr,
              u, p);
  out[j] = p;
}

__global__ void k_line_build(int n, const double *ver, const double *mag, LineGeo *out) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  LineGeo l;
  line_build(ver + 6 * (size_t)j, mag ? mag[j] : 0.0, l);
  out[j] = l;
}

// Copies (host case) and converts panel/line sets into device geometry
// records.  raw/geo buffers are grown and reused.
int elem_build_device(const dust_panels *body, const dust_panels *wake,
                      const dust_lines *lines, const double *u_inf, const RegParams &rp,
                      bool host_arrays, DevBuf &raw, DevBuf &geo, ElemDev &out,
                      cudaStream_t st) {
  memset(&out, 0, sizeof(out));
  out.rp = rp;
  int nb = body ? body->n : 0, nw = wake ? wake->n : 0, nl = lines ? lines->n : 0;
  if (nb < 0 || nw < 0 || nl < 0) return DUST_ERR_BAD_ARG;
  out.nbody = nb;
  out.nwake = nw;
  out.nline = nl;
  size_t gbytes = sizeof(PanelGeo) * (size_t)(nb + nw) + sizeof(LineGeo) * (size_t)nl + 256;
  DUST_TRY(devbuf_grow(geo, gbytes));
  PanelGeo *gb = (PanelGeo *)geo.p;
  PanelGeo *gw = gb + nb;
  LineGeo *gl = (LineGeo *)(gw + nw);
  out.body = gb;
  out.wake = gw;
  out.lines = gl;
  if (nb + nw + nl == 0) return DUST_OK;
  PanRaw rb{}, rw{};
  const double *lver = nullptr, *lmag = nullptr;
  if (host_arrays) {
    // pack all host arrays into one staging buffer and copy once
    auto pan_bytes = [](const dust_panels *p) -> size_t {
      if (!p || p->n == 0) return 0;
      size_t n = p->n;
      return n * 12 * 8 + (p->mag ? n * 8 : 0) + (p->ub ? n * 24 : 0) +
             (p->uvort ? n * 24 : 0) + (p->n_ver ? n * 4 : 0) + (p->kind ? n * 4 : 0) + 256;
    };
    size_t tot = pan_bytes(body) + pan_bytes(wake) + (size_t)nl * 7 * 8 + 256;
    DUST_TRY(devbuf_grow(raw, tot));
    char *base = (char *)raw.p;
    size_t off = 0;
    auto put = [&](const void *src, size_t bytes) -> const void * {
      if (!src || bytes == 0) return nullptr;
      off = (off + 15) & ~(size_t)15;
      char *dst = base + off;
      cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
      off += bytes;
      return dst;
    };
    auto put_pan = [&](const dust_panels *p, PanRaw &r) {
      r.n = p ? p->n : 0;
      if (!p || p->n == 0) return;
      size_t n = p->n;
      r.ver = (const double *)put(p->ver, n * 12 * 8);
      r.mag = (const double *)put(p->mag, n * 8);
      r.ub = (const double *)put(p->ub, n * 24);
      r.uvort = (const double *)put(p->uvort, n * 24);
      r.n_ver = (const int *)put(p->n_ver, n * 4);
      r.kind = (const int *)put(p->kind, n * 4);
    };
    put_pan(body, rb);
    put_pan(wake, rw);
    if (nl > 0) {
      lver = (const double *)put(lines->ver, (size_t)nl * 6 * 8);
      lmag = (const double *)put(lines->mag, (size_t)nl * 8);
    }
  } else {
    if (body && nb) rb = PanRaw{nb, body->n_ver, body->kind, body->ver, body->mag, body->ub, body->uvort};
    if (wake && nw) rw = PanRaw{nw, wake->n_ver, wake->kind, wake->ver, wake->mag, wake->ub, wake->uvort};
    if (nl) {
      lver = lines->ver;
      lmag = lines->mag;
    }
  }
  double u0 = u_inf ? u_inf[0] : 0.0, u1 = u_inf ? u_inf[1] : 0.0, u2 = u_inf ? u_inf[2] : 0.0;
  if (nb) k_panel_build<<<nblk(nb, 128), 128, 0, st>>>(rb, u0, u1, u2, gb);
  if (nw) k_panel_build<<<nblk(nw, 128), 128, 0, st>>>(rw, u0, u1, u2, gw);
  if (nl) k_line_build<<<nblk(nl, 128), 128, 0, st>>>(nl, lver, lmag, gl);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}

// velocity at points from all elements (x 1/4pi) + u_inf
#define EP_T 128
#define EP_TILE 16
__global__ void __launch_bounds__(EP_T) k_elements_vel(int n, const double *pts, ElemDev e,
                                                       double u0, double u1, double u2,
                                                       double *vel) {
  __shared__ PanelGeo s_p[EP_TILE];
  int t = blockIdx.x * EP_T + threadIdx.x;
  bool act = t < n;
  double pos[3] = {0, 0, 0};
  if (act)
    for (int c = 0; c < 3; ++c) pos[c] = pts[3 * (size_t)t + c];
  double v[3] = {0, 0, 0};
  int ntot = e.nbody + e.nwake;
  for (int p0 = 0; p0 < ntot; p0 += EP_TILE) {
    __syncthreads();
    int m = min(EP_TILE, ntot - p0);
    const int words = sizeof(PanelGeo) / 8;
    for (int w = threadIdx.x; w < m * words; w += EP_T) {
      int pp = w / words, ww = w % words;
      int g = p0 + pp;
      const PanelGeo *src = g < e.nbody ? e.body + g : e.wake + (g - e.nbody);
      ((double *)&s_p[pp])[ww] = ((const double *)src)[ww];
    }
    __syncthreads();
    if (act)
      for (int q = 0; q < m; ++q) {
        double u[3];
        vel_pan(e.rp, s_p[q], pos, u);
        for (int c = 0; c < 3; ++c) v[c] += u[c];
      }
  }
  if (!act) return;
  for (int q = 0; q < e.nline; ++q) {
    double u[3];
    vel_line(e.rp, e.lines[q], pos, u);
    for (int c = 0; c < 3; ++c) v[c] += u[c];
  }
  const double k4pi = 1.0 / (4.0 * DUST_PI);
  vel[3 * (size_t)t + 0] = v[0] * k4pi + u0;
  vel[3 * (size_t)t + 1] = v[1] * k4pi + u1;
  vel[3 * (size_t)t + 2] = v[2] * k4pi + u2;
}

// The same sum for a few points (the wake's points): the panels are split
// into chunks over blockIdx.y so that more than a handful of CTAs share the
// work; each chunk adds its part atomically into vel (zeroed first), the
// first chunk also the lines and u_inf.
#define EPC_PANELS 32
__global__ void __launch_bounds__(EP_T) k_elements_vel_chunk(int n, const double *pts,
                                                             ElemDev e, double u0, double u1,
                                                             double u2, double *vel) {
  __shared__ PanelGeo s_p[EP_TILE];
  const int t = blockIdx.x * EP_T + threadIdx.x;
  const bool act = t < n;
  double pos[3] = {0, 0, 0};
  if (act)
    for (int c = 0; c < 3; ++c) pos[c] = pts[3 * (size_t)t + c];
  double v[3] = {0, 0, 0};
  const int ntot = e.nbody + e.nwake;
  const int q_lo = blockIdx.y * EPC_PANELS, q_hi = min(ntot, q_lo + EPC_PANELS);
  for (int p0 = q_lo; p0 < q_hi; p0 += EP_TILE) {
    __syncthreads();
    const int m = min(EP_TILE, q_hi - p0);
    const int words = sizeof(PanelGeo) / 8;
    for (int w = threadIdx.x; w < m * words; w += EP_T) {
      const int pp = w / words, ww = w % words, g = p0 + pp;
      const PanelGeo *src = g < e.nbody ? e.body + g : e.wake + (g - e.nbody);
      ((double *)&s_p[pp])[ww] = ((const double *)src)[ww];
    }
    __syncthreads();
    if (act)
      for (int q = 0; q < m; ++q) {
        double u[3];
        vel_pan(e.rp, s_p[q], pos, u);
        for (int c = 0; c < 3; ++c) v[c] += u[c];
      }
  }
  if (!act) return;
  if (blockIdx.y == 0)
    for (int q = 0; q < e.nline; ++q) {
      double u[3];
      vel_line(e.rp, e.lines[q], pos, u);
      for (int c = 0; c < 3; ++c) v[c] += u[c];
    }
  const double k4pi = 1.0 / (4.0 * DUST_PI);
  const double w[3] = {u0, u1, u2};
  for (int c = 0; c < 3; ++c)
    atomicAdd(vel + 3 * (size_t)t + c, v[c] * k4pi + (blockIdx.y == 0 ? w[c] : 0.0));
}

int elements_vel_points(const ElemDev &e, int n, const double *pts, const double *u_inf,
                        double *vel, cudaStream_t st) {
  if (n <= 0) return DUST_OK;
  const int ntot = e.nbody + e.nwake;
  const int ny = std::max(1, (ntot + EPC_PANELS - 1) / EPC_PANELS);
  DUST_CUDA(cudaMemsetAsync(vel, 0, (size_t)n * 24, st));
  k_elements_vel_chunk<<<dim3(nblk(n, EP_T), ny), EP_T, 0, st>>>(n, pts, e, u_inf[0], u_inf[1],
                                                                  u_inf[2], vel);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}

#define UV_T 128
// All-pairs particle kernels (direct-sum truth).
__global__ void __launch_bounds__(UV_T) k_direct(int n, int ntgt, const double *cen,
                                                 const double *dir, const double *mag,
                                                 const double *rv, int vs, int df, int vd,
                                                 double nu, double *vel, double *str,
                                                 double *rot) {
  __shared__ double s[7][UV_T];
  int t = blockIdx.x * UV_T + threadIdx.x;
  bool act = t < ntgt;
  double tp[3] = {0, 0, 0}, ta[3] = {0, 0, 0};
  if (act)
    for (int c = 0; c < 3; ++c) {
      tp[c] = cen[3 * (size_t)t + c];
      ta[c] = mag[t] * dir[3 * (size_t)t + c];
    }
  double V[3] = {0, 0, 0}, Sx[3] = {0, 0, 0}, R[3] = {0, 0, 0}, F[3] = {0, 0, 0};
  for (int q0 = 0; q0 < n; q0 += UV_T) {
    __syncthreads();
    int q = q0 + threadIdx.x;
    if (q < n) {
      double m = mag[q];
      for (int c = 0; c < 3; ++c) {
        s[c][threadIdx.x] = cen[3 * (size_t)q + c];
        s[3 + c][threadIdx.x] = m * dir[3 * (size_t)q + c];
      }
      s[6][threadIdx.x] = rv[q];
    }
    __syncthreads();
    int m = min(UV_T, n - q0);
    if (act)
      for (int u = 0; u < m; ++u) {
        if (q0 + u == t) continue;
        double dx = tp[0] - s[0][u], dy = tp[1] - s[1][u], dz = tp[2] - s[2][u];
        double qax = s[3][u], qay = s[4][u], qaz = s[5][u], sq = s[6][u];
        double r2 = dx * dx + dy * dy + dz * dz;
        double s2 = sq * sq;
        double inv = rsqrt(r2 + s2), inv2 = inv * inv;
        double c = -inv2 * inv, dd = -3.0 * c * inv2;
        V[0] += c * (dy * qaz - dz * qay);
        V[1] += c * (dz * qax - dx * qaz);
        V[2] += c * (dx * qay - dy * qax);
        if (vs) {
          double vx = ta[1] * qaz - ta[2] * qay, vy = ta[2] * qax - ta[0] * qaz,
                 vz = ta[0] * qay - ta[1] * qax;
          double dv = dx * vx + dy * vy + dz * vz;
          Sx[0] -= c * vx + dd * dx * dv;
          Sx[1] -= c * vy + dd * dy * dv;
          Sx[2] -= c * vz + dd * dz * dv;
          if (df) {
            double da = dx * qax + dy * qay + dz * qaz;
            R[0] += -2.0 * c * qax + dd * (dx * da - qax * r2);
            R[1] += -2.0 * c * qay + dd * (dy * da - qay * r2);
            R[2] += -2.0 * c * qaz + dd * (dz * da - qaz * r2);
          }
        }
        if (vd) {
          double is2 = 1.0 / s2, tt = r2 * is2 + 1.0, rt = rsqrt(tt);
          double rt2 = rt * rt, rt4 = rt2 * rt2;
          double w = 17.5 * is2 * (rt4 * rt4 * rt);
          F[0] += w * (qax - ta[0]);
          F[1] += w * (qay - ta[1]);
          F[2] += w * (qaz - ta[2]);
        }
      }
  }
  if (!act) return;
  const double k4pi = 1.0 / (4.0 * DUST_PI);
  for (int c = 0; c < 3; ++c) {
    vel[3 * (size_t)t + c] = V[c] * k4pi;
    if (str) str[3 * (size_t)t + c] = Sx[c] * k4pi + (vd ? F[c] * nu : 0.0);
    if (rot) rot[3 * (size_t)t + c] = R[c] * k4pi;
  }
}

// ------------------------------------------------------------------ C ABI
namespace {
struct Scratch {
  DevBuf raw, geo, a, b;
  ~Scratch() {
    devbuf_free(raw);
    devbuf_free(geo);
    devbuf_free(a);
    devbuf_free(b);
  }
};
}  // namespace

extern "C" int dust_elements_vel(const dust_fmm_params *prm, int n_pts, const double *pts,
                                 const dust_elements *elems, double *vel) {
  if (!prm || n_pts < 0 || (n_pts > 0 && (!pts || !vel))) return DUST_ERR_BAD_ARG;
  if (n_pts == 0) return DUST_OK;
  static Scratch s;  // kept across calls (one host thread)
  cudaStream_t st = 0;
  ElemDev e;
  RegParams rp = reg_params(prm);
  DUST_TRY(elem_build_device(elems ? &elems->body : nullptr, elems ? &elems->wake : nullptr,
                             elems ? &elems->end_vort : nullptr, prm->u_inf, rp, true, s.raw,
                             s.geo, e, st));
  DUST_TRY(devbuf_grow(s.a, (size_t)n_pts * 24 * 2));
  double *dp = (double *)s.a.p, *dv = dp + 3 * (size_t)n_pts;
  DUST_CUDA(cudaMemcpyAsync(dp, pts, (size_t)n_pts * 24, cudaMemcpyHostToDevice, st));
  k_elements_vel<<<nblk(n_pts, EP_T), EP_T, 0, st>>>(n_pts, dp, e, prm->u_inf[0],
                                                     prm->u_inf[1], prm->u_inf[2], dv);
  DUST_CUDA(cudaGetLastError());
  DUST_CUDA(cudaMemcpyAsync(vel, dv, (size_t)n_pts * 24, cudaMemcpyDeviceToHost, st));
  DUST_CUDA(cudaStreamSynchronize(st));
  return DUST_OK;
}

static DevBuf g_uv_scratch;  // sort scratch of the uvort entry points (one host thread)

int points_uvort_device(const dust_fmm_params *prm, int n_pts, const double *pts, int n,
                        const double *cen, const double *dir, const double *mag,
                        const double *rv, const ElemDev &lines, double *uv, cudaStream_t st) {
  return points_uvort_run(prm, n_pts, pts, n, cen, dir, mag, rv, lines, g_uv_scratch, uv, st);
}

bool uvort_args_ok(const dust_fmm_params *prm, int n_pts, const double *pts, int n,
                   const double *cen, const double *dir, const double *mag,
                   const double *r_vortex, const dust_lines *end_vort, const double *uvort) {
  if (!prm || n_pts < 0 || n < 0) return false;
  if (end_vort && (end_vort->n < 0 || (end_vort->n > 0 && (!end_vort->ver || !end_vort->mag))))
    return false;
  if (n_pts == 0) return true;
  if (!pts || !uvort) return false;
  if (n > 0 && (!cen || !dir || !mag || !r_vortex)) return false;
  return true;
}

extern "C" int dust_points_uvort(const dust_fmm_params *prm, int n_pts, const double *pts,
                                 int n, const double *cen, const double *dir,
                                 const double *mag, const double *r_vortex,
                                 const dust_lines *end_vort, double *uvort) {
  if (!uvort_args_ok(prm, n_pts, pts, n, cen, dir, mag, r_vortex, end_vort, uvort))
    return DUST_ERR_BAD_ARG;
  if (n_pts == 0) return DUST_OK;
  static Scratch s;  // kept across calls (one host thread)
  cudaStream_t st = 0;
  ElemDev e;
  DUST_TRY(elem_build_device(nullptr, nullptr, end_vort, prm->u_inf, reg_params(prm), true,
                             s.raw, s.geo, e, st));
  size_t N = (size_t)std::max(n, 1);
  DUST_TRY(devbuf_grow(s.a, (size_t)n_pts * 24 * 2));
  DUST_TRY(devbuf_grow(s.b, N * 8 * 8));
  double *dp = (double *)s.a.p, *du = dp + 3 * (size_t)n_pts;
  double *dc = (double *)s.b.p, *dd = dc + 3 * N, *dm = dd + 3 * N, *dr = dm + N;
  DUST_CUDA(cudaMemcpyAsync(dp, pts, (size_t)n_pts * 24, cudaMemcpyHostToDevice, st));
  if (n > 0) {
    DUST_CUDA(cudaMemcpyAsync(dc, cen, (size_t)n * 24, cudaMemcpyHostToDevice, st));
    DUST_CUDA(cudaMemcpyAsync(dd, dir, (size_t)n * 24, cudaMemcpyHostToDevice, st));
    DUST_CUDA(cudaMemcpyAsync(dm, mag, (size_t)n * 8, cudaMemcpyHostToDevice, st));
    DUST_CUDA(cudaMemcpyAsync(dr, r_vortex, (size_t)n * 8, cudaMemcpyHostToDevice, st));
  }
  DUST_TRY(points_uvort_device(prm, n_pts, dp, n, dc, dd, dm, dr, e, du, st));
  DUST_CUDA(cudaMemcpyAsync(uvort, du, (size_t)n_pts * 24, cudaMemcpyDeviceToHost, st));
  DUST_CUDA(cudaStreamSynchronize(st));
  return DUST_OK;
}

extern "C" int dust_direct_particles(const dust_fmm_params *prm, int n, const double *cen,
                                     const double *dir, const double *mag,
                                     const double *r_vortex, int n_tgt, double *vel,
                                     double *stretch, double *rotu) {
  if (!prm || n < 0 || n_tgt < 0 || n_tgt > n || (n_tgt > 0 && !vel)) return DUST_ERR_BAD_ARG;
  if (n_tgt == 0) return DUST_OK;
  static Scratch s;  // kept across calls (one host thread)
  cudaStream_t st = 0;
  size_t N = (size_t)n;
  DUST_TRY(devbuf_grow(s.a, N * 8 * 8));
  DUST_TRY(devbuf_grow(s.b, (size_t)n_tgt * 9 * 8));
  double *dc = (double *)s.a.p, *dd = dc + 3 * N, *dm = dd + 3 * N, *dr = dm + N;
  double *ov = (double *)s.b.p, *os = ov + 3 * (size_t)n_tgt, *orr = os + 3 * (size_t)n_tgt;
  DUST_CUDA(cudaMemcpyAsync(dc, cen, N * 24, cudaMemcpyHostToDevice, st));
  DUST_CUDA(cudaMemcpyAsync(dd, dir, N * 24, cudaMemcpyHostToDevice, st));
  DUST_CUDA(cudaMemcpyAsync(dm, mag, N * 8, cudaMemcpyHostToDevice, st));
  DUST_CUDA(cudaMemcpyAsync(dr, r_vortex, N * 8, cudaMemcpyHostToDevice, st));
  k_direct<<<nblk(n_tgt, UV_T), UV_T, 0, st>>>(n, n_tgt, dc, dd, dm, dr, prm->vortstretch,
                                               prm->divergence_filtering, prm->diffusion,
                                               prm->nu_inf, ov, os, orr);
  DUST_CUDA(cudaGetLastError());
  DUST_CUDA(cudaMemcpyAsync(vel, ov, (size_t)n_tgt * 24, cudaMemcpyDeviceToHost, st));
  if (stretch)
    DUST_CUDA(cudaMemcpyAsync(stretch, os, (size_t)n_tgt * 24, cudaMemcpyDeviceToHost, st));
  if (rotu) DUST_CUDA(cudaMemcpyAsync(rotu, orr, (size_t)n_tgt * 24, cudaMemcpyDeviceToHost, st));
  DUST_CUDA(cudaStreamSynchronize(st));
  return DUST_OK;
}

__global__ void k_geo_out(int n, const PanelGeo *g, double *cen, double *nor, double *area) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  for (int c = 0; c < 3; ++c) {
    if (cen) cen[3 * (size_t)j + c] = g[j].cen[c];
    if (nor) nor[3 * (size_t)j + c] = g[j].nor[c];
  }
  if (area) area[j] = g[j].area;
}

extern "C" int dust_panels_geometry(const dust_panels *pan, double *cen, double *nor,
                                    double *area) {
  if (!pan || pan->n < 0) return DUST_ERR_BAD_ARG;
  if (pan->n == 0) return DUST_OK;
  static Scratch s;  // kept across calls (one host thread)
  cudaStream_t st = 0;
  ElemDev e;
  RegParams rp{10.0, 0.1, 0.001};
  DUST_TRY(elem_build_device(pan, nullptr, nullptr, nullptr, rp, true, s.raw, s.geo, e, st));
  int n = pan->n;
  DUST_TRY(devbuf_grow(s.a, (size_t)n * 7 * 8));
  double *dc = (double *)s.a.p, *dn = dc + 3 * (size_t)n, *da = dn + 3 * (size_t)n;
  k_geo_out<<<nblk(n, 128), 128, 0, st>>>(n, e.body, dc, dn, da);
  DUST_CUDA(cudaGetLastError());
  if (cen) DUST_CUDA(cudaMemcpyAsync(cen, dc, (size_t)n * 24, cudaMemcpyDeviceToHost, st));
  if (nor) DUST_CUDA(cudaMemcpyAsync(nor, dn, (size_t)n * 24, cudaMemcpyDeviceToHost, st));
  if (area) DUST_CUDA(cudaMemcpyAsync(area, da, (size_t)n * 8, cudaMemcpyDeviceToHost, st));
  DUST_CUDA(cudaStreamSynchronize(st));
  return DUST_OK;
}

extern "C" int dust_points_uvort_device(const dust_fmm_params *prm, int n_pts, const double *pts,
                                        int n, const double *cen, const double *dir,
                                        const double *mag, const double *r_vortex,
                                        const dust_lines *end_vort, double *uvort, void *stream) {
  if (!uvort_args_ok(prm, n_pts, pts, n, cen, dir, mag, r_vortex, end_vort, uvort))
    return DUST_ERR_BAD_ARG;
  if (n_pts == 0) return DUST_OK;
  cudaStream_t st = (cudaStream_t)stream;
  static thread_local Scratch s;
  ElemDev e;
  DUST_TRY(elem_build_device(nullptr, nullptr, end_vort, prm->u_inf, reg_params(prm), false,
                             s.raw, s.geo, e, st));
  DUST_TRY(points_uvort_device(prm, n_pts, pts, n, cen, dir, mag, r_vortex, e, uvort, st));
  return DUST_OK;
}

__global__ void k_centres(PanRaw r, double *cen) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= r.n) return;
  int nv = r.n_ver ? r.n_ver[j] : 4;
  for (int d = 0; d < 3; ++d) {
    double s = 0.0;
    for (int v = 0; v < nv; ++v) s += r.ver[12 * (size_t)j + 3 * v + d];
    cen[3 * (size_t)j + d] = s / (double)nv;
  }
}

extern "C" int dust_panels_centres_device(const dust_panels *pan, double *cen, void *stream) {
  if (!pan || pan->n < 0 || (pan->n > 0 && (!pan->ver || !cen))) return DUST_ERR_BAD_ARG;
  if (pan->n == 0) return DUST_OK;
  PanRaw r{pan->n, pan->n_ver, pan->kind, pan->ver, pan->mag, pan->ub, pan->uvort};
  k_centres<<<nblk(pan->n, 128), 128, 0, (cudaStream_t)stream>>>(r, cen);
  DUST_CUDA(cudaGetLastError());
  return DUST_OK;
}
