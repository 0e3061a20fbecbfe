/*
 * dust_b200.h -- C ABI of the B200 (sm_100a) implementation of DUST's
 * per-timestep aerodynamic hot path.
 *
 * The reference (DUST, Fortran 2008 + OpenMP) reaches this path through
 * module procedures of mod_octree and mod_linsys.  Every entry point below
 * replaces one of them and is meant to be bound from Fortran with
 * ISO_C_BINDING (an interface module with one BIND(C) interface per
 * function, value arguments for ints, type(c_ptr) for handles).  Arrays are
 * plain host (or, for the *_device variants, device) pointers in the
 * Fortran layout: a particle/panel coordinate array `x(3,n)` is passed as a
 * double* of length 3*n with the three components of one item contiguous.
 *
 * All calls return an int status (DUST_OK == 0).  A non-zero status maps to
 * the reference's `call error(...)` (src/general/mod_handling.f90:181).
 * Handles are not re-entrant: one handle is driven by one host thread and
 * owns one CUDA stream.  The handle-less host-array calls (dust_points_uvort,
 * dust_points_uvort_pressure, dust_particles_update, ...) keep their device
 * staging buffers across calls, so they too are called from one host thread
 * at a time.
 */
#ifndef DUST_B200_H
#define DUST_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define DUST_API __attribute__((visibility("default")))
#else
#define DUST_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define DUST_OK                0
#define DUST_ERR_CUDA          1  /* CUDA runtime / launch failure            */
#define DUST_ERR_OUT_OF_BOX    2  /* particle outside the octree box
                                     (mod_octree.f90:758-762)                 */
#define DUST_ERR_SINGULAR      3  /* zero pivot in an LU factorisation
                                     (LAPACK info>0, mod_linsys.f90:241-245)  */
#define DUST_ERR_NOT_CONVERGED 4  /* iterative solve did not reach tolerance  */
#define DUST_ERR_TIMEOUT       5  /* a bounded device wait gave up            */
#define DUST_ERR_BAD_ARG       6  /* invalid argument                         */
#define DUST_ERR_NO_DEVICE     7  /* no CUDA device / library not usable      */
#define DUST_ERR_CAPACITY      8  /* size above a documented maximum          */

/* ------------------------------------------------------- element kinds */
#define DUST_ELEM_SURFPAN  1   /* 'p': source+doublet panel, Dirichlet row
                                  (src/aeroel/mod_surfpan.f90)                */
#define DUST_ELEM_VORTLATT 2   /* 'v': vortex ring, Neumann row
                                  (src/aeroel/mod_vortlatt.f90)               */

/* ------------------------------------------------------ precision modes */
#define DUST_PREC_FP64   0     /* plain: FP64 everywhere                      */
#define DUST_PREC_FP32C  1     /* FP32 pair arithmetic on tile-relative
                                  coordinates, partial sums per tile in FP32
                                  and across tiles in FP64; M2L of levels >= 2
                                  in FP32 (SIMT, FP64 accumulation across
                                  offsets); tables, level-1 M2L, P2M, M2M,
                                  L2L, L2P and near element pairs stay FP64   */

/* Octree / FMM parameters.  One field per DUST input key
 * (src/general/mod_sim_param.f90:376-452, read at :772-804). */
typedef struct dust_fmm_params {
  double box_length;          /* box_length                                  */
  int    n_box[3];            /* n_box                                       */
  double origin[3];           /* octree_origin                               */
  int    n_octree_levels;     /* n_octree_levels                             */
  int    min_octree_part;     /* min_octree_part                             */
  int    multipole_degree;    /* multipole_degree (p)                        */
  double rankine_rad;         /* rankine_rad: M2L kernel regularisation
                                 (octree%delta, dust.f90:377) and the Rankine
                                 core of panel/line induction                 */
  double cutoff_rad;          /* cutoff_rad                                  */
  double far_field_ratio_doublet; /* far_field_ratio_doublet (10)            */
  int    vortstretch;         /* vortstretch                                 */
  int    divergence_filtering;/* divergence_filtering                        */
  int    diffusion;           /* diffusion                                   */
  int    turbulent_viscosity; /* turbulent_viscosity                         */
  double nu_inf;              /* mu_inf/rho_inf                              */
  double u_inf[3];            /* u_inf (uniform wind, mod_wind.f90:66-77)    */
  int    precision;           /* DUST_PREC_*                                 */
} dust_fmm_params;

/* A set of flat panels (quads or triangles).  Geometry is given by the
 * vertices; the derived quantities of calc_geo_data_surfpan
 * (mod_surfpan.f90:888-951) / calc_geo_data_vortlatt (mod_vortlatt.f90:
 * 601-669) are computed by the library. */
typedef struct dust_panels {
  int           n;      /* number of panels                                  */
  const int    *n_ver;  /* [n] 3 or 4                                        */
  const int    *kind;   /* [n] DUST_ELEM_*; NULL = all DUST_ELEM_VORTLATT    */
  const double *ver;    /* [12*n] ver(3,4) per panel (4th unused for tris)   */
  const double *mag;    /* [n] doublet intensity; NULL = 0                   */
  const double *ub;     /* [3*n] body velocity at the centre; NULL = 0       */
  const double *uvort;  /* [3*n] vortex-induced velocity at the centre
                           (surface-panel source strength); NULL = 0         */
} dust_panels;

/* Vortex line segments (end vortices of panel wakes, mod_vortline.f90). */
typedef struct dust_lines {
  int           n;
  const double *ver;    /* [6*n] ver(3,2) per line                           */
  const double *mag;    /* [n]                                               */
} dust_lines;

/* The non-particle vortical elements that act on particles in
 * apply_multipole (mod_octree.f90:1350-1373). */
typedef struct dust_elements {
  dust_panels body;     /* elem: implicit body elements                      */
  dust_panels wake;     /* wpan: wake panels (vortex rings)                  */
  dust_lines  end_vort; /* wvort: end vortices                               */
} dust_elements;

/* Counters of the last FMM evaluation (for logs and roofline figures). */
typedef struct dust_fmm_stats {
  int64_t n_particles;
  int64_t n_leaves;
  int64_t n_active_cells;
  int64_t n_m2l_pairs;       /* (target, active source) pairs over levels    */
  int64_t n_p2p_pairs;       /* particle pairs of the reference's near field */
  int64_t n_elem_pairs;      /* particle x element evaluations               */
  int     n_levels;
  float   ms_tree, ms_upward, ms_m2l, ms_p2p, ms_elems, ms_total;
  float   ms_m2l_kernel;     /* M2L kernel of levels >= 2 alone (k_m2l_batch) */
  float   ms_elem_far;       /* FP32 far-field element kernel alone, else 0   */
} dust_fmm_stats;

typedef struct dust_octree dust_octree;

/* ------------------------------------------------------------- octree */

/* Replaces initialize_octree (src/fmm/mod_octree.f90:251-518): builds the
 * level geometry and the per-level kernel-derivative tables
 * (compute_der_ker, src/fmm/mod_multipole.f90:388-450) on the device. */
DUST_API int dust_octree_create(const dust_fmm_params *prm, dust_octree **out);

/* Replaces destroy_octree (mod_octree.f90:691-695). */
DUST_API int dust_octree_destroy(dust_octree *oct);

/* Replaces sort_particles + calculate_multipole + apply_multipole
 * (mod_octree.f90:703-996, 1002-1133, 1139-1429) for n live particles.
 * Host arrays.  Outputs (caller order): vel(3,n) = induced velocity + wind;
 * stretch(3,n) (vortex stretching + diffusion, when either is on) and
 * rotu(3,n) (divergence-filter curl, when on); either may be NULL. */
DUST_API int dust_fmm_apply(dust_octree *oct, int n,
                   const double *cen, const double *dir, const double *mag,
                   const double *r_vortex, const dust_elements *elems,
                   double *vel, double *stretch, double *rotu);

/* Same as dust_fmm_apply with every array (including those inside *elems)
 * already resident in device memory; runs on `stream` (cudaStream_t, NULL =
 * the handle's stream) and returns without a host synchronisation when
 * `sync` == 0 (errors are then reported by the next call). */
DUST_API int dust_fmm_apply_device(dust_octree *oct, int n,
                          const double *cen, const double *dir,
                          const double *mag, const double *r_vortex,
                          const dust_elements *elems,
                          double *vel, double *stretch, double *rotu,
                          void *stream, int sync);

/* The same evaluation in the reference's two halves, so that the particles
 * enter the tree once per step and serve both the panels and themselves:
 *   dust_fmm_prepare[_device]      sort_particles + calculate_multipole of
 *                                  prepare_wake (mod_wake.f90:797-800): the
 *                                  particles and the n_pts evaluation points
 *                                  (panel centres, pts(3,n_pts), copied) are
 *                                  sorted into the tree as sort_particles
 *                                  sorts particles and panels
 *                                  (mod_octree.f90:703-799); multipoles and
 *                                  local expansions, including those of the
 *                                  empty leaves that hold points.  A particle
 *                                  or point outside the box is
 *                                  DUST_ERR_OUT_OF_BOX;
 *   dust_fmm_points_uvort[_device] apply_multipole_panels (:801,
 *                                  mod_octree.f90:1433-1508): the particles'
 *                                  velocity at the prepared points (each takes
 *                                  the local expansion of the leaf that holds
 *                                  it plus the particles of that leaf's near
 *                                  field) plus the end vortices by direct
 *                                  sum, into uvort(3,n_pts) (overwritten).
 *                                  The reference adds this to uvort and then
 *                                  discards it in get_vort_vel
 *                                  (mod_surfpan.f90:970); here it is the
 *                                  result, an approximation of
 *                                  dust_points_uvort to the FMM's accuracy;
 *   dust_fmm_finish[_device]       apply_multipole (mod_wake.f90:1115-1118):
 *                                  L2P + P2P at the prepared particles and
 *                                  the element sums, outputs as
 *                                  dust_fmm_apply (caller order).
 * points_uvort and finish need a prepared tree (DUST_ERR_BAD_ARG otherwise);
 * the tree stays valid until the next prepare or apply on the handle.  The
 * device variants run on `stream` (NULL = the handle's stream); finish
 * synchronises when `sync` != 0, points_uvort always. */
DUST_API int dust_fmm_prepare(dust_octree *oct, int n, const double *cen, const double *dir,
                              const double *mag, const double *r_vortex, int n_pts,
                              const double *pts);
DUST_API int dust_fmm_prepare_device(dust_octree *oct, int n, const double *cen,
                                     const double *dir, const double *mag,
                                     const double *r_vortex, int n_pts, const double *pts,
                                     void *stream);
DUST_API int dust_fmm_points_uvort(dust_octree *oct, const dust_lines *end_vort, double *uvort);
DUST_API int dust_fmm_points_uvort_device(dust_octree *oct, const dust_lines *end_vort,
                                          double *uvort, void *stream);
DUST_API int dust_fmm_finish(dust_octree *oct, const dust_elements *elems, double *vel,
                             double *stretch, double *rotu);
DUST_API int dust_fmm_finish_device(dust_octree *oct, const dust_elements *elems, double *vel,
                                    double *stretch, double *rotu, void *stream, int sync);

/* Counters of the last dust_fmm_apply*.  Timings are filled only when
 * `timing` was enabled with dust_octree_set_timing. */
DUST_API int dust_octree_get_stats(const dust_octree *oct, dust_fmm_stats *st);
DUST_API int dust_octree_set_timing(dust_octree *oct, int on);

/* Direct O(N^2) evaluation of the same particle kernels over all pairs
 * (the reference's P2P formulas of src/aeroel/mod_vortpart.f90:139-336
 * applied to every particle pair); used as the FMM truth.  Targets are the
 * first n_tgt particles.  Host arrays. */
DUST_API int dust_direct_particles(const dust_fmm_params *prm, int n,
                          const double *cen, const double *dir,
                          const double *mag, const double *r_vortex,
                          int n_tgt, double *vel, double *stretch,
                          double *rotu);

/* Replaces get_vort_vel_surfpan / get_vort_vel_vortlatt over all vortical
 * elements (mod_surfpan.f90:962-977, mod_vortlatt.f90:676-693, called from
 * mod_linsys.f90:295-299): uvort(3,n_pts) at the given points (panel
 * centres) induced by the n particles plus the end vortices.  Host arrays. */
DUST_API int dust_points_uvort(const dust_fmm_params *prm, int n_pts,
                      const double *pts, int n, const double *cen,
                      const double *dir, const double *mag,
                      const double *r_vortex, const dust_lines *end_vort,
                      double *uvort);

/* Device-resident variant of dust_points_uvort (all arrays, including
 * end_vort's, in device memory; stream = cudaStream_t or NULL). */
DUST_API int dust_points_uvort_device(const dust_fmm_params *prm, int n_pts,
                                      const double *pts, int n,
                                      const double *cen, const double *dir,
                                      const double *mag, const double *r_vortex,
                                      const dust_lines *end_vort, double *uvort,
                                      void *stream);

/* dust_points_uvort_device (FP64, or with prm->precision DUST_PREC_FP32C
 * packed FP32 pairs on Morton-sorted particles with FP64 sums per tile of
 * 128) together with the particles' rotational term of the pressure
 * equation at the same points
 * (assemble_pressure_sys, src/linsys/mod_pressure_equation.f90:170-186):
 *   pterm[i] = sum_q (x_q - pts_i) . (dir_q x vel_q) mag_q /
 *              (|x_q - pts_i|^2 + r_q^2)^(3/2),
 * vel(3, n) the particles' velocities, pterm[n_pts] device output.  Both
 * sums run in one pass over the (point, particle) pairs and share the
 * distance and the kernel coefficient.  Device arrays, queued on `stream`. */
DUST_API int dust_points_uvort_pressure_device(const dust_fmm_params *prm, int n_pts,
                                               const double *pts, int n, const double *cen,
                                               const double *dir, const double *mag,
                                               const double *r_vortex, const double *vel,
                                               const dust_lines *end_vort, double *uvort,
                                               double *pterm, void *stream);

/* dust_points_uvort_pressure_device on host arrays (inputs copied to a
 * device staging buffer kept across calls -- one host thread --, uvort and
 * pterm copied back): for a host code that calls get_vort_vel and
 * assemble_pressure_sys in the same step; pterm then goes to
 * dust_pressure_assemble_terms. */
DUST_API int dust_points_uvort_pressure(const dust_fmm_params *prm, int n_pts,
                                        const double *pts, int n, const double *cen,
                                        const double *dir, const double *mag,
                                        const double *r_vortex, const double *vel,
                                        const dust_lines *end_vort, double *uvort,
                                        double *pterm);

/* No counterpart in the reference.  Same result as dust_points_uvort_device
 * (same kernels and summation order) for callers that must not allocate
 * device memory during a step: a host code that hands the whole device to
 * its own pool or caching allocator (a cudaMalloc would fail or evict it), or
 * one that cannot afford the device-wide synchronisation of cudaFree inside
 * its time loop.  This entry point calls no cudaMalloc/cudaFree nor any
 * allocating library routine: its scratch (end-vortex geometry, and in the
 * FP32C mode the Morton keys, the sorted particle copy and the radix-sort
 * work space, about 56 bytes per particle plus the sort work) is a fixed
 * device array of DUST_UVORT_NOALLOC_SCRATCH bytes inside the library,
 * reserved when the library is loaded.
 *   - Sizes that need more scratch than that return DUST_ERR_CAPACITY before
 *     anything is launched; dust_last_error() names the bytes needed.  The
 *     FP64 mode needs scratch only for the end vortices (88 bytes each).
 *   - Nothing has to start at zero: the scratch is written before it is
 *     read, and uvort is overwritten (zeroed on `stream`, then summed).
 *   - The scratch is one array per device, shared by every call: calls that
 *     overlap in time (two streams, or two host threads) race on it and give
 *     wrong results.  Serialise them.
 *   - Every call looks the array's address up in the current device's
 *     context (cudaGetSymbolAddress; nothing is cached, so a context reset
 *     is harmless); the first call on a device also loads the library's
 *     device code there, so a caller that records its stream into a graph
 *     should make one call before it starts capturing.
 *   - Null pointers where data is needed (points and output with n_pts > 0,
 *     particle arrays with n > 0, end-vortex arrays with end_vort->n > 0)
 *     return DUST_ERR_BAD_ARG before anything is launched. */
#define DUST_UVORT_NOALLOC_SCRATCH (4u << 20)
DUST_API int dust_points_uvort_device_noalloc(const dust_fmm_params *prm, int n_pts,
                                              const double *pts, int n,
                                              const double *cen, const double *dir,
                                              const double *mag, const double *r_vortex,
                                              const dust_lines *end_vort, double *uvort,
                                              void *stream);

/* Panel centres (calc_geo_data) of a device-resident panel set into
 * cen(3,n) in device memory. */
DUST_API int dust_panels_centres_device(const dust_panels *pan, double *cen,
                                        void *stream);

/* Velocity induced at n_pts points by a set of panels and lines
 * (compute_vel of surfpan/vortlatt/vortline, divided by 4*pi) plus u_inf.
 * Host arrays. */
DUST_API int dust_elements_vel(const dust_fmm_params *prm, int n_pts,
                      const double *pts, const dust_elements *elems,
                      double *vel);

/* Panel centres / unit normals as computed by calc_geo_data (for callers
 * that need the collocation points).  Host arrays. */
DUST_API int dust_panels_geometry(const dust_panels *pan, double *cen, double *nor,
                         double *area);

/* --------------------------------------------------------- linear system */

typedef struct dust_linsys dust_linsys;

/* Solve modes. */
#define DUST_SOLVE_LU64      0  /* plain FP64 block LU (static LU reused +
                                   Schur update of the moving block), the
                                   reference's solve_linsys sequence          */
#define DUST_SOLVE_MIXED     1  /* FP32 LU (tensor-core trailing updates) +
                                   FP64 iterative refinement                  */
#define DUST_SOLVE_GMRES_NN  2  /* learned-preconditioned FP64 GMRES, plain LU
                                   fallback                                   */

typedef struct dust_solve_report {
  int    mode_used;       /* DUST_SOLVE_* that produced the solution         */
  int    iterations;      /* refinement / GMRES iterations                   */
  int    fell_back;       /* 1 if GMRES stalled and LU was used              */
  double residual;        /* final ||b - A x||_inf / (||A||_inf ||x||_inf);
                             GMRES: ||b - A x||_2 / ||b||_2                  */
  float  ms_factor, ms_solve;
  int    pivoted;         /* LU paths: 1 if the factorisation interchanged
                             rows (partial pivoting ran), 0 if its unpivoted
                             multipliers certified that dgetrf would not    */
} dust_solve_report;

/* Implicit wake panels (first n_impl wake panels) couple into A through
 * their generating elements (wake%pan_gen_elems_id, mod_wake.f90:150):
 * impl_ind[2*j], impl_ind[2*j+1] = 1-based element indices (0 = none). */
typedef struct dust_wake_rows {
  dust_panels  pan;       /* all wake panels, implicit ones first            */
  int          n_impl;
  const int   *impl_ind;  /* [2*n_impl]                                      */
} dust_wake_rows;

/* Replaces initialize_linsys (mod_linsys.f90:109-267) for `rank` implicit
 * elements of which the first `nstatic` do not move: builds the static rows,
 * adds the static wake, and LU-factors the static block once. */
DUST_API int dust_linsys_create(int rank, int nstatic, const dust_fmm_params *prm,
                       const dust_panels *elems, const dust_wake_rows *wake,
                       dust_linsys **out);
DUST_API int dust_linsys_destroy(dust_linsys *ls);

/* Replaces assemble_linsys (mod_linsys.f90:279-344) minus the uvort step
 * (pass elems->uvort, computed by dust_points_uvort): rebuilds the moving
 * columns of static rows, all columns of moving rows, the RHS and the wake
 * terms. */
DUST_API int dust_linsys_assemble(dust_linsys *ls, const dust_panels *elems,
                         const dust_wake_rows *wake);

/* dust_linsys_assemble with the panel arrays (and impl_ind) in device
 * memory. */
DUST_API int dust_linsys_assemble_device(dust_linsys *ls, const dust_panels *elems,
                                         const dust_wake_rows *wake);

/* Replaces solve_linsys (mod_linsys.f90:352-482).  res[rank] receives the
 * doublet intensities. */
DUST_API int dust_linsys_solve(dust_linsys *ls, int mode, double *res,
                      dust_solve_report *rep);

/* dust_linsys_solve writing res[rank] to device memory. */
DUST_API int dust_linsys_solve_device(dust_linsys *ls, int mode, double *res,
                                      dust_solve_report *rep);

/* Copies of the assembled matrix (column-major, rank x rank, BEFORE
 * factorisation of the moving part) and right-hand side, as dump_linsys
 * (mod_linsys.f90:503-524) writes them.  Either pointer may be NULL. */
DUST_API int dust_linsys_get_system(dust_linsys *ls, double *A, double *b);

/* Standalone dense solve A X = B (column-major; n x n, nrhs columns) with
 * partial-pivoting LU as LAPACK dgetrf+dgetrs (mod_linsys.f90:470-474).
 * mode: DUST_SOLVE_LU64 or DUST_SOLVE_MIXED (refined to `tol`). */
DUST_API int dust_dense_solve(int n, int nrhs, const double *A, const double *B,
                     double *X, int mode, double tol, dust_solve_report *rep);

/* dust_dense_solve on device arrays (A n x n, B and X n x nrhs, column-major,
 * leading dimension n), queued on `stream` (cudaStream_t, NULL = the legacy
 * default stream) and synchronised before return.  A is not modified: the
 * LU64 mode factors a copy, the MIXED mode only reads it (FP32 copy for the
 * factorisation, FP64 A for the residuals).  LU64 allows X == B (solved in
 * place); MIXED needs X != B.  The work areas (the factor copy, the FP32
 * matrix, pivots, refinement vectors) are kept between calls and grow with
 * the largest size seen, so repeated solves of one size allocate nothing
 * after the first; calls are serialised by a process-wide lock. */
DUST_API int dust_dense_solve_device(int n, int nrhs, const double *A, const double *B,
                                     double *X, int mode, double tol,
                                     dust_solve_report *rep, void *stream);

/* Tensor-core (tcgen05, kind::tf32) update C -= A B on device arrays
 * (column-major FP32, read as TF32, FP32 accumulation): the trailing update
 * of the mixed-precision LU (the dgemm of mod_linsys.f90:428-438 in its
 * low-precision form).  Synchronises `stream`; DUST_ERR_TIMEOUT if a bounded
 * wait inside the kernel gave up. */
DUST_API int dust_tc_gemm_tf32_minus(int m, int n, int k, const float *A, int lda,
                                     const float *B, int ldb, float *C, int ldc,
                                     void *stream);

/* ------------------------------------------------ learned preconditioner */
/* No counterpart in the reference (it refactors the moving block every step,
 * mod_linsys.f90:352-482).  A 3-layer, width-64 graph network over the
 * k-nearest-neighbour graph of the panel centres maps the current matrix to
 * a sparse approximate inverse M = (I + O) D^-1 (D = diag A, O on the graph's
 * edges).  DUST_SOLVE_GMRES_NN right-preconditions its FP64 GMRES with M, or,
 * when the system has static rows, with the block lower-triangular operator
 * that applies the FP32 inverse of the static block to the static part and M
 * to the moving part (the static inverse is built once, on first use); the
 * warm start is that operator applied to b.  Untrained (output weights zero)
 * M is Jacobi.
 * Training runs on the GPU: the loss of a stored system is
 * ||M [A Z, b] - [Z, x]||_F^2 / (n C) over 7 random +-1 probe columns Z and
 * the solution x, minimised with Adam. */
typedef struct dust_precond dust_precond;

/* Graph of n panel centres (host, 3n): each panel's k nearest others. */
DUST_API int dust_precond_create(int n, int k, const double *centres,
                                 unsigned long long seed, dust_precond **out);
DUST_API int dust_precond_destroy(dust_precond *p);
DUST_API int dust_precond_num_params(void);
DUST_API int dust_precond_get_params(const dust_precond *p, float *w, int count);
DUST_API int dust_precond_set_params(dust_precond *p, const float *w, int count);

/* Stores a training sample: `ls` assembled and not yet solved, x_dev its
 * solution (device, n doubles). */
DUST_API int dust_precond_add_sample(dust_precond *p, dust_linsys *ls,
                                     const double *x_dev, unsigned long long seed);
DUST_API int dust_precond_num_samples(const dust_precond *p);

/* Loss (and gradient, count = dust_precond_num_params()) of sample `si` at
 * the current weights; grad may be NULL. */
DUST_API int dust_precond_loss_grad(dust_precond *p, int si, float *loss,
                                    float *grad, int count);

/* The stored inputs of sample `si` (host arrays, any may be NULL):
 * x[n*8], ef[n*(k+1)*4], w[n*(k+1)], nbr[n*(k+1)], Y[n*8], T[n*8]. */
DUST_API int dust_precond_get_sample(const dust_precond *p, int si, float *x,
                                     float *ef, float *w, int *nbr, float *Y,
                                     float *T);

/* `iters` Adam steps cycling over the samples; *loss_out = mean loss of the
 * last pass. */
DUST_API int dust_precond_train(dust_precond *p, int iters, float lr,
                                float *loss_out);

/* Attaches p (NULL detaches) to the system for DUST_SOLVE_GMRES_NN. */
DUST_API int dust_linsys_set_precond(dust_linsys *ls, dust_precond *p);

/* ------------------------------------------------------ particle update */
/* Parameters of the particles' explicit Euler step in complete_wake
 * (src/aeroel/mod_wake.f90:1309-1355): dt and ndt_update_wake as
 * sim_param%dt and %ndt_update_wake, the box as wake%part_box_min/max
 * (particles_box_min/max), the switches as sim_param%use_vs, %use_vd and
 * %use_divfilt, filt_eta as sim_param%filt_eta. */
typedef struct dust_update_params {
  double dt;
  int    ndt_update_wake;
  double box_min[3], box_max[3];
  int    vortstretch;            /* use_vs                                    */
  int    diffusion;              /* use_vd                                    */
  int    divergence_filtering;   /* use_divfilt                               */
  double filt_eta;
} dust_update_params;

/* The particle loop of complete_wake (src/aeroel/mod_wake.f90:1309-1355),
 * penetration avoidance (use_pa, off by default, :1313-1318) excepted.
 * Arrays as in dust_fmm_apply: cen, dir, vel, stretch, rotu (3, n), mag (n),
 * free_flag (n; 0 = live, 1 = free slot).  For every live particle:
 *   p = cen + vel dt ndt; if p is inside the box (bounds included):
 *     cen = p, and with vortstretch or diffusion:
 *       with divergence_filtering:
 *         stretch -= filt_eta / ndt (dir mag - rotu mag / |rotu|)
 *       alpha = dir mag + stretch dt ndt; dir = alpha / |alpha| if |alpha| != 0
 *     (mag is left unchanged, as in the reference);
 *   else free_flag = 1.
 * *n_freed receives the number of particles set free (the reference
 * decrements wake%n_prt by it).  Same operation order as the reference, no
 * fused multiply-adds.  Host arrays; allocates device memory for the call. */
DUST_API int dust_particles_update(const dust_update_params *u, int n, double *cen,
                                   double *dir, const double *mag, const double *vel,
                                   double *stretch, const double *rotu, int *free_flag,
                                   int *n_freed);
/* The same on device arrays (n_freed a device int, overwritten), queued on
 * `stream` (NULL: the default stream), not synchronised; allocates nothing. */
DUST_API int dust_particles_update_device(const dust_update_params *u, int n, double *cen,
                                          double *dir, const double *mag, const double *vel,
                                          double *stretch, const double *rotu,
                                          int *free_flag, int *n_freed, void *stream);

/* ------------------------------------------------ penetration avoidance */
/* sim_param%pa_rad_mult, %pa_elrad_mult and %u_ref
 * (src/general/mod_sim_param.f90:697-702, 627-636). */
typedef struct dust_pa_params {
  double check_radius;    /* penetration_avoidance_check_radius (5.0)        */
  double element_radius;  /* penetration_avoidance_element_radius (1.5)      */
  double u_ref;           /* u_ref (default |u_inf|)                         */
} dust_pa_params;

/* complete_wake's particle loop with penetration avoidance (use_pa,
 * src/aeroel/mod_wake.f90:1312-1317): before the move, every live
 * particle's velocity goes through avoid_collision (:2350-2534) against the
 * body elements `elems` (the reference's elems_tot, in its order; surface
 * panels and vortex rings, device arrays, ub = body velocity at the centres
 * or NULL), and the corrected velocity is written back to vel (part%vel).
 * Then the step of dust_particles_update_device.  The reference's own
 * expressions are kept, including the vortex-ring branch's componentwise
 * normal distance norm2(dist * n) and its doubling of the layer thickness
 * (initially the particle's r_vortex) at every ring that passes the
 * approach test.  Device arrays, queued on `stream`; the element records
 * are built into a work buffer kept between calls (grown on first use). */
DUST_API int dust_particles_update_pa_device(const dust_update_params *u,
                                             const dust_pa_params *pa,
                                             const dust_panels *elems, int n, double *cen,
                                             double *dir, const double *mag,
                                             const double *r_vortex, double *vel,
                                             double *stretch, const double *rotu,
                                             int *free_flag, int *n_freed, void *stream);

/* The live particles of a slot array in slot order (the part_p list that
 * prepare_wake rebuilds, src/aeroel/mod_wake.f90:804-846): copies cen, dir
 * (3, n_live), mag, r_vortex (n_live) of every slot with free_flag == 0
 * into the l* arrays and its slot index into idx; *n_live (host) receives
 * the count.  Device arrays; synchronises `stream`. */
DUST_API int dust_particles_live_device(int n_slots, const int *free_flag, const double *cen,
                                        const double *dir, const double *mag,
                                        const double *r_vortex, double *lcen, double *ldir,
                                        double *lmag, double *lrv, int *idx, int *n_live,
                                        void *stream);
/* Scatters per-live-particle outputs (3, n_live) back to their slots:
 * out[idx[i]] = in[i] for each non-NULL pair.  Device arrays. */
DUST_API int dust_particles_scatter_device(int n_live, const int *idx, const double *lvel,
                                           const double *lstr, const double *lrot, double *vel,
                                           double *str, double *rot, void *stream);

/* ---------------------------------------------- panel wake and shedding */
/* The panel wake behind the trailing edges and the particles it sheds,
 * device resident: the panel part of t_wake (src/aeroel/mod_wake.f90:
 * 160-296) with initialize_wake (:331-579), load_wake (:597-778, restart),
 * update_wake (:860-1214) and complete_wake (:1222-2105).  The wake panels
 * are vortex rings of rows 1..len (len grows by one per step up to
 * n_wake_panels, then the wake is full); a full wake sheds one particle per
 * stripe per step (k_refine x n subparticles with refine_wake) into the
 * lowest free particle slots and carries an end vortex on its last row.
 * Uniform wind u_inf (variable_wind without gusts).  Not built: ring wakes
 * of actuator disks, join_te, interpolate_wake, HCAS, precice. */
typedef struct dust_wake_params {
  int    n_stripes;           /* wake%n_pan_stripes = size(te%e, 2)          */
  int    n_points;            /* wake%n_pan_points = size(te%i, 2)           */
  int    n_wake_panels;       /* n_wake_panels (wake%nmax_pan), >= 1         */
  double dt;                  /* dt                                          */
  int    ndt_update_wake;     /* ndt_update_wake                             */
  double min_vel_at_te;       /* implicit_panel_min_vel                      */
  double box_min[3], box_max[3]; /* particles_box_min / max                  */
  double vortex_rad;          /* vortex_rad                                  */
  double k_vortex_rad;        /* k_vortex_rad                                */
  int    refine_wake;         /* refine_wake                                 */
  int    k_refine;            /* k_refine                                    */
  double u_inf[3];            /* u_inf                                       */
} dust_wake_params;

/* Trailing-edge topology (t_tedge: te%ii, te%neigh, te%o, te%e, written by
 * the pre-processor, src/geo/mod_build_geo.f90:2135-2152, 2284-2289), host
 * arrays of 2*n_stripes ints, 1-based as in the reference: the two
 * trailing-edge points of each stripe, the neighbouring stripe on each side
 * (0 = none) and its orientation (+1 / -1), the generating elements
 * (0 = none). */
typedef struct dust_te {
  const int *ii;
  const int *neigh;
  const int *neigh_o;
  const int *gen_elems;
} dust_te;

typedef struct dust_wake dust_wake;

/* initialize_wake (:331-579) for the panel wake: first row of points =
 * te_pts (3, n_points; the midpoints of te%i, wake%w_start_points), second
 * row te_pts + te_dir scaling |u_inf - te_vel| dt ndt / |te_dir| (te_dir =
 * R_g pan_gen_dir, te_scaling = pan_gen_scaling, te_vel = calc_node_vel or
 * NULL for 0; below min_vel_at_te: te_dir scaling min_vel_at_te dt ndt, the
 * reference's unnormalised form at this call), len = 1, intensities 0.
 * Host arrays. */
DUST_API int dust_wake_create(const dust_wake_params *prm, const dust_te *te,
                              const double *te_pts, const double *te_dir,
                              const double *te_scaling, const double *te_vel,
                              dust_wake **out);
DUST_API int dust_wake_destroy(dust_wake *w);

/* Device views of the wake's elements for the other entry points (valid
 * until the next call on w): the wake panels of rows 1..len in the
 * reference's pan_p order (row by row, stripes in order; vortex rings, mag =
 * pan_idou), the implicit first row's generating elements (n_impl =
 * n_stripes, impl_ind 1-based, device) for dust_wake_rows, and the end
 * vortices of a full wake (n = 0 before that; mag => last_pan_idou). */
DUST_API int dust_wake_elements(dust_wake *w, dust_panels *wake_pan, dust_lines *end_vort,
                                int *n_impl, const int **impl_ind);

/* update_wake :884-892: the first row's intensities from the solution
 * (device res, 1-based gen_elems): mag(gen 1) - mag(gen 2). */
DUST_API int dust_wake_set_first_row_device(dust_wake *w, const double *res, void *stream);

/* The rest of update_wake's panel part (:894-939, :1128-1176): velocity at
 * the wake points by compute_vel_from_all (:2109-2150: the body elements
 * `body` with their intensities, the wake panels, the end vortices, the n
 * particles (device arrays) and u_inf), rows 3.. moved (the third with dt,
 * the others with dt ndt, as the reference), the extra row of a full wake
 * (points_end), then the length and the intensities shifted one row back
 * (end_pan_idou = last row).  prm supplies rankine_rad, cutoff_rad and
 * far_field_ratio_doublet.  Device arrays, queued on `stream`. */
DUST_API int dust_wake_update_device(dust_wake *w, const dust_fmm_params *prm,
                                     const dust_panels *body, int n, const double *cen,
                                     const double *dir, const double *mag,
                                     const double *r_vortex, void *stream);

/* complete_wake's panel part and shedding (:1247-1292, :1358-2010 without
 * interpolate_wake, :2091-2103): first two rows from the trailing edge (as
 * dust_wake_create, with the normalised form below min_vel_at_te), then for
 * a full wake one particle per stripe (or k_refine subparticles) at the
 * centre of the last row's far panel with circulation vector from the
 * side and end intensities, written into the lowest free slots of the
 * particle arrays (n_slots each, free_flag cleared for them; vel may be
 * NULL); *n_shed (host) receives the number shed; end vortices attached.
 * A slot shortage returns DUST_ERR_CAPACITY ("Exceeding the maximum number
 * of wake particles", :1985).  Device arrays; synchronises `stream`. */
DUST_API int dust_wake_complete_device(dust_wake *w, const double *te_pts,
                                       const double *te_dir, const double *te_scaling,
                                       const double *te_vel, int n_slots, double *cen,
                                       double *dir, double *mag, double *r_vortex,
                                       double *vel, int *free_flag, int *n_shed,
                                       void *stream);

/* Velocities of the wake panels' vertices, wake_vv[12 * len * n_stripes]
 * (pan_w_vel at each vertex's row and point, in the panels' vertex order),
 * and of the end vortices' vertices, end_vv[6 * n_stripes] (row len; may be
 * NULL; written only once the end vortices are attached): the vertex
 * velocities of assemble_pressure_sys (src/linsys/mod_pressure_equation.f90:
 * 194-223).  Device arrays. */
DUST_API int dust_wake_vertex_velocities_device(dust_wake *w, double *wake_vv, double *end_vv,
                                                void *stream);

/* State as save_status writes it (src/io/mod_dust_io.f90:355-411) and
 * load_wake reads it back (:597-778): points (len+1, n_points, 3), point
 * velocities (same), pan_idou (len, n_stripes), last_pan_idou (n_stripes);
 * host arrays, any may be NULL on get.  set_state takes len in 1..n_wake_panels
 * and marks the wake full when len == n_wake_panels (load_wake :764). */
DUST_API int dust_wake_get_state(const dust_wake *w, int *len, double *points,
                                 double *point_vel, double *idou, double *last_idou);
DUST_API int dust_wake_set_state(dust_wake *w, int len, const double *points,
                                 const double *point_vel, const double *idou,
                                 const double *last_idou);

/* ---------------------------------------------------- pressure equation */
/* The pressure integral equation of the linear-system module
 * (src/linsys/mod_pressure_equation.f90; A_pres and its static LU in
 * src/linsys/mod_linsys.f90:184-187, 250-257, 318-323).  Its unknowns are
 * the surface panels (DUST_ELEM_SURFPAN) among the system's elements, in
 * element order (static first); A_pres is their block of the influence
 * matrix before the wake correction. */
typedef struct dust_pressure dust_pressure;

/* initialize_pressure_sys (:44-79) with the static part of initialize_linsys:
 * the static block of A_pres and b_static_pres from the geometry `ls` was
 * created with, and the LU of the static block.  Call right after
 * dust_linsys_create. */
DUST_API int dust_pressure_create(dust_linsys *ls, dust_pressure **out);
DUST_API int dust_pressure_destroy(dust_pressure *p);
/* Number of surface panels and of static ones. */
DUST_API int dust_pressure_size(const dust_pressure *p, int *n_sp, int *nstatic_sp);

/* assemble_pressure_sys (:139-235) after dust_linsys_assemble of the same
 * step (its element geometry): the moving parts of A_pres, b_pres from the
 * Bernoulli sources `bern` (n_sp, device; the output of press_normvel_der,
 * :395-455; NULL = 0, as for bodies at rest) through the source-potential
 * influence (build_row_surfpan, mod_surfpan.f90:396-437), plus the
 * rotational terms of the n live particles (cen, dir, mag, r_vortex and their
 * velocities vel(3, n)), of the end vortices and of the wake panels with
 * their vertex velocities (end_vv[6 * n_end], wake_vv[12 * n_wake], e.g. from
 * dust_wake_vertex_velocities_device).  Device arrays; the kernels run on
 * `stream`, which is synchronised. */
DUST_API int dust_pressure_assemble_device(dust_pressure *p, const dust_linsys *ls,
                                           const double *bern, int n, const double *cen,
                                           const double *dir, const double *mag,
                                           const double *r_vortex, const double *vel,
                                           const dust_panels *wake, const double *wake_vv,
                                           const dust_lines *end_vort, const double *end_vv,
                                           void *stream);

/* dust_pressure_assemble_device with the particles' term already evaluated
 * at every element centre (pterm[rank], device; e.g. by
 * dust_points_uvort_pressure_device in the same pass as uvort): the term of
 * each surface panel is taken from its element's entry. */
DUST_API int dust_pressure_assemble_terms_device(dust_pressure *p, const dust_linsys *ls,
                                                 const double *bern, const double *pterm,
                                                 const dust_panels *wake, const double *wake_vv,
                                                 const dust_lines *end_vort, const double *end_vv,
                                                 void *stream);

/* solve_pressure_sys (:243-387): the block LU sequence of solve_linsys on
 * A_pres (static LU reused, Schur update and LU of the moving block, getrs);
 * res[n_sp] (device) receives the solution (the elements' pres_sol). */
DUST_API int dust_pressure_solve_device(dust_pressure *p, double *res, void *stream);

/* The same two calls on host arrays (copied to a device buffer kept by the
 * handle; the solution copied back): for host codes that keep the particles
 * in host memory. */
DUST_API int dust_pressure_assemble(dust_pressure *p, const dust_linsys *ls, const double *bern,
                                    int n, const double *cen, const double *dir,
                                    const double *mag, const double *r_vortex,
                                    const double *vel, const dust_panels *wake,
                                    const double *wake_vv, const dust_lines *end_vort,
                                    const double *end_vv);
DUST_API int dust_pressure_solve(dust_pressure *p, double *res);
/* dust_pressure_assemble_terms_device on host arrays (pterm[rank] from
 * dust_points_uvort_pressure; bern, wake, end vortices as in
 * dust_pressure_assemble). */
DUST_API int dust_pressure_assemble_terms(dust_pressure *p, const dust_linsys *ls,
                                          const double *bern, const double *pterm,
                                          const dust_panels *wake, const double *wake_vv,
                                          const dust_lines *end_vort, const double *end_vv);

/* Host copies of A_pres (n_sp x n_sp column-major; its static block holds
 * that block's LU) and b_pres after assembly and before the solve, as
 * dump_linsys_pres writes them (:462-489).  Either may be NULL. */
DUST_API int dust_pressure_get_system(dust_pressure *p, double *A, double *b);

/* ---------------------------------------------------------------- misc */
DUST_API const char *dust_status_string(int status);
DUST_API const char *dust_last_error(void); /* text of the last CUDA error seen      */
DUST_API int dust_device_ok(void);   /* DUST_OK if a usable sm_100 device is present */
/* sizeof() of the ABI structs in declaration order (dust_fmm_params,
 * dust_panels, dust_lines, dust_elements, dust_fmm_stats, dust_solve_report,
 * dust_wake_rows, dust_update_params, dust_pa_params, dust_wake_params,
 * dust_te), for binding checks; returns the
 * number of sizes. */
DUST_API int dust_abi_sizes(int64_t *out, int n);

#ifdef __cplusplus
}
#endif
#endif /* DUST_B200_H */
