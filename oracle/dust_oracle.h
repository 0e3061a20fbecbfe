/*
 * dust_oracle.h -- CPU oracle (test infrastructure only).
 *
 * A plain-C, FP64, OpenMP restatement of the reference's hot path, used
 * only by the tests, by __graft_entry__.smoke() and by bench.py's CPU
 * baseline as the checker.  The product never links or calls it.
 *
 * Reference files restated (paths inside the DUST project):
 *   src/fmm/mod_multipole.f90    polynomial tools, P2M, M2M, M2L, L2L,
 *                                kernel-derivative recurrence
 *   src/fmm/mod_octree.f90       octree geometry, leaf rule, leaf_neigh,
 *                                interaction lists, calculate/apply_multipole
 *   src/aeroel/mod_vortpart.f90  particle kernels (vel, stretch, rotu, PSE)
 *   src/aeroel/mod_doublet.f90   doublet potential / velocity
 *   src/aeroel/mod_surfpan.f90   source potential / velocity, rows
 *   src/aeroel/mod_vortlatt.f90  vortex-lattice rows
 *   src/aeroel/mod_vortline.f90  vortex line velocity
 *   src/linsys/mod_linsys.f90    static/moving block LU sequence
 *   src/linsys/mod_pressure_equation.f90  pressure integral equation
 *   src/aeroel/mod_wake.f90      particle loop of complete_wake, avoid_collision
 *
 * Parity pins: the reference is Fortran and cannot be compiled here (no
 * Fortran compiler, LAPACK or HDF5).  Its regression fixtures hold its own
 * results (tests/sym_test/static/{v,p,nl_v}/Output/ref_res_00{10,11}.h5):
 * the step-11 re-solve (particle and end-vortex uvort, both influence
 * kernels, both row builders, the wake coupling, the LU) and the step
 * 10 -> 11 wake advance (element and particle velocities, stretching,
 * diffusion, penetration avoidance, the Euler update and the shedding) are
 * checked against them (tests/test_reference_fixture.py).  The LU sequence
 * is also pinned against LAPACK (the reference's third-party solver)
 * through scipy; the FMM's multipole parts and the rest of the influence
 * kernels by analytic known answers and independent formulas (solid-angle
 * sums and the Van Oosterom-Strackee solid angle, vortex-ring and
 * straight-segment Biot-Savart laws, quadrature of the source potential,
 * the particle-pair kernel, FMM -> direct-sum convergence).
 */
#ifndef DUST_ORACLE_H
#define DUST_ORACLE_H

#include "../include/dust_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* 1 = reproduce the reference's default-integer (32-bit, wrapping)
 * factorials in the M2L weights (mod_multipole.f90:489-497, 524-537);
 * 0 (default) = exact factorials. */
void or_set_factorial_wrap(int on);

/* Full FMM evaluation: initialize_octree + sort_particles +
 * calculate_multipole + apply_multipole.  Returns DUST_* status. */
int or_fmm_apply(const dust_fmm_params *prm, int n, const double *cen,
                 const double *dir, const double *mag, const double *r_vortex,
                 const dust_elements *elems, double *vel, double *stretch,
                 double *rotu, int64_t *counters /* [4]: leaves, active,
                 m2l pairs, p2p pairs; may be NULL */);

/* Tree of the last or_fmm_apply (for structure checks):
 * per level l (1..ll) the dense flag array in Morton-key order
 * (bit0 leaf, bit1 branch, bit2 active).  flags must hold
 * sum_l prod(nbox)*8^(l-1) bytes. */
int or_last_tree_flags(unsigned char *flags, int64_t cap);

/* apply_multipole_panels: particle velocity at points from the FMM (leaf
 * local expansion + near-field particles) plus end vortices by direct sum. */
int or_fmm_points_uvort(const dust_fmm_params *prm, int n, const double *cen,
                        const double *dir, const double *mag, const double *r_vortex,
                        int n_pts, const double *pts, const dust_lines *end_vort,
                        double *uvort);

/* Direct sum of the particle kernels over all pairs (targets = first n_tgt). */
int or_direct_particles(const dust_fmm_params *prm, int n, const double *cen,
                        const double *dir, const double *mag,
                        const double *r_vortex, int n_tgt, double *vel,
                        double *stretch, double *rotu);

/* Element influence at points (compute_vel / 4pi summed + u_inf). */
int or_elements_vel(const dust_fmm_params *prm, int n_pts, const double *pts,
                    const dust_elements *elems, double *vel);

/* uvort at points from particles + end vortices (get_vort_vel_*). */
int or_points_uvort(const dust_fmm_params *prm, int n_pts, const double *pts,
                    int n, const double *cen, const double *dir,
                    const double *mag, const double *r_vortex,
                    const dust_lines *end_vort, double *uvort);

/* Single-element kernels (for unit tests).  kind = DUST_ELEM_*. */
int or_panel_geometry(const dust_panels *pan, double *cen, double *nor,
                      double *area);
double or_potential_doublet(const dust_fmm_params *prm, const dust_panels *pan,
                            int j, const double *pos);
void or_velocity_doublet(const dust_fmm_params *prm, const dust_panels *pan,
                         int j, const double *pos, double *v);
double or_potential_source(const dust_fmm_params *prm, const dust_panels *pan,
                           int j, double dou, const double *pos);
void or_velocity_source(const dust_fmm_params *prm, const dust_panels *pan,
                        int j, const double *pos, double *v);

/* Linear system: assemble (initialize_linsys + assemble_linsys without the
 * uvort step) and solve with the reference's block LU sequence.
 * A_out (rank x rank, column-major) / b_out receive the assembled system
 * before the moving-block factorisation; res the solution. */
int or_linsys_run(const dust_fmm_params *prm, int rank, int nstatic,
                  const dust_panels *elems_init, const dust_panels *elems_step,
                  const dust_wake_rows *wake_init,
                  const dust_wake_rows *wake_step,
                  double *A_out, double *b_out, double *res);

/* The two assembly halves of or_linsys_run on caller arrays (A rank x rank
 * column-major, bst nst x nst, b rank, all zero-initialised by the caller):
 * initialize_linsys's static rows and static wake, and one assemble_linsys
 * (uvort from elems->uvort).  The static LU between them is the caller's. */
void or_linsys_init(const dust_fmm_params *prm, int rank, int nst,
                    const dust_panels *elems, const dust_wake_rows *wake, double *A,
                    double *bst, double *b);
void or_linsys_step(const dust_fmm_params *prm, int rank, int nst,
                    const dust_panels *elems, const dust_wake_rows *wake, double *A,
                    const double *bst, double *b);

/* Work sampling of or_fmm_apply for the timed CPU baseline (stride 1 =
 * full evaluation) and the phase times / sampled work of the last call. */
void or_set_sample_stride(int s);
void or_set_threads(int n);
void or_last_fmm_times(double *t4, int64_t *sampled);

/* Rows `rows[0..nrows)` of the all-moving system (nstatic = 0) as
 * assemble_linsys builds them; A_rows nrows x rank row-major. */
int or_linsys_rows(const dust_fmm_params *prm, int rank, const dust_panels *elems,
                   const dust_wake_rows *wake, int nrows, const int *rows,
                   double *A_rows, double *b_rows);

/* LAPACK-equivalent dense kernels (column-major). */
int  or_dgetrf(int m, int n, double *A, int lda, int *ipiv);
void or_dgetrs(int n, int nrhs, const double *A, int lda, const int *ipiv,
               double *B, int ldb);
void or_dlaswp(int n, double *A, int lda, int k1, int k2, const int *ipiv);
void or_dtrsm_llnu(int m, int n, const double *A, int lda, double *B, int ldb);
void or_dtrsm_runn(int m, int n, const double *A, int lda, double *B, int ldb);
void or_dgemm_nn_minus(int m, int n, int k, const double *A, int lda,
                       const double *B, int ldb, double *C, int ldc);

/* The pressure integral equation of one step (mod_pressure_equation.f90,
 * the pressure parts of mod_linsys.f90 and build_row_surfpan): A_pres
 * (n_sp x n_sp column-major, n_sp = surface panels among the rank elements,
 * static first), b_pres and res_pres.  bern: Bernoulli source per surface
 * panel or NULL; particles with their velocities vel(3, n); wake panels with
 * the velocities of their four vertices wake_vv[12 * n_wake]; end vortices
 * with those of their two vertices end_vv[6 * n_end]. */
int or_pressure_run(const dust_fmm_params *prm, int rank, int nstatic,
                    const dust_panels *elems_init, const dust_panels *elems_step,
                    const double *bern, int n, const double *cen, const double *dir,
                    const double *mag, const double *r_vortex, const double *vel,
                    const dust_panels *wake, const double *wake_vv, const dust_lines *end_vort,
                    const double *end_vv, double *A_out, double *b_out, double *res);

/* The particles' term of assemble_pressure_sys alone at n_pts points. */
int or_pressure_particles(int n_pts, const double *pts, int n, const double *cen,
                          const double *dir, const double *mag, const double *r_vortex,
                          const double *vel, double *out);

/* Particle loop of complete_wake (mod_wake.f90:1309-1355), arguments as
 * dust_particles_update. */
int or_particles_update(const dust_update_params *u, int n, double *cen, double *dir,
                        const double *mag, const double *vel, double *stretch,
                        const double *rotu, int *free_flag, int *n_freed);

/* The same loop with penetration avoidance (avoid_collision,
 * mod_wake.f90:2350-2534) against the body elements `elems` (host arrays);
 * vel is overwritten with the corrected velocities. */
int or_particles_update_pa(const dust_update_params *u, const dust_pa_params *pa,
                           const dust_panels *elems, int n, double *cen, double *dir,
                           const double *mag, const double *r_vortex, double *vel,
                           double *stretch, const double *rotu, int *free_flag,
                           int *n_freed);

#ifdef __cplusplus
}
#endif
#endif
