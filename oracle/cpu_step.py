"""One timestep of the reference's hot path on the host cores (test and
benchmark infrastructure: the CPU baseline, never the product).

The reference (Fortran + OpenMP) cannot be built here, so its step is
restated: the oracle's C loops (OpenMP) for everything the reference codes
itself, and LAPACK/BLAS through scipy for what the reference hands to its
third-party LAPACK, in the reference's call sequence:

* get_vort_vel over particles + end vortices at every implicit element
  (mod_surfpan.f90:962-977, mod_vortlatt.f90:676-693) -- or_points_uvort;
* assemble_linsys (mod_linsys.f90:279-344) -- or_linsys_step;
* solve_linsys (mod_linsys.f90:352-482): dlaswp, dtrsm('L','L','N','U'),
  dtrsm('R','U','N','N'), dgemm, dgetrf of the moving block, dlaswp, pivot
  shift, dgetrs -- scipy.linalg.lapack / blas (OpenBLAS);
* the implicit wake panels' intensities (update_wake, mod_wake.f90:881-889);
* the pressure integral equation of the surface panels
  (mod_pressure_equation.f90:139-387): the particles' rotational term at the
  surface panels with the previous update's velocities (or_pressure_particles;
  the Bernoulli sources are zero for bodies at rest) and dgetrs with the
  static LU of A_pres (dust.f90:621, 641-643);
* sort_particles + calculate_multipole + apply_multipole with the element
  sums (mod_octree.f90:703-1429) -- or_fmm_apply;
* complete_wake's particle loop (mod_wake.f90:1309-1355) --
  or_particles_update.

initialize_linsys's static rows, the static LU (dgetrf) and A_pres's static
LU run once, in ``CpuStep.__init__``, outside the step.
"""
import ctypes as C
import time

import numpy as np
from scipy.linalg import blas, lapack

import oracle as O
from dust_b200 import abi


def set_threads(n):
    """Threads of the oracle's OpenMP loops and of OpenBLAS."""
    O.lib().or_set_threads(C.c_int(int(n)))
    try:
        from threadpoolctl import threadpool_limits
        threadpool_limits(limits=int(n))
    except Exception:  # pragma: no cover - threadpoolctl is optional
        pass


def _laswp_rows(M, piv0, k1, k2):
    """Row interchanges i <-> piv0[i] for i in [k1, k2) applied in order
    (LAPACK dlaswp with 0-based pivots)."""
    idx = np.arange(M.shape[0])
    for i in range(k1, k2):
        p = piv0[i]
        if p != i:
            idx[i], idx[p] = idx[p], idx[i]
    M[:] = M[idx]


def solve_linsys_lapack(A, P0, nst, b):
    """solve_linsys on the assembled A (Fortran order; the static block holds
    its LU with 0-based pivots P0[:nst]).  Returns (res, P0 of the step)."""
    n = A.shape[0]
    nmv = n - nst
    P = P0.copy()
    if nst > 0 and nmv > 0:
        Asd = np.asfortranarray(A[:nst, nst:])
        _laswp_rows(Asd, P[:nst], 0, nst)
        Lss = A[:nst, :nst]
        Asd = blas.dtrsm(1.0, Lss, Asd, side=0, lower=1, trans_a=0, diag=1, overwrite_b=1)
        Ads = np.asfortranarray(A[nst:, :nst])
        Ads = blas.dtrsm(1.0, Lss, Ads, side=1, lower=0, trans_a=0, diag=0, overwrite_b=1)
        Add = np.asfortranarray(A[nst:, nst:])
        Add = blas.dgemm(-1.0, Ads, Asd, beta=1.0, c=Add, overwrite_c=1)
        A[:nst, nst:] = Asd
        A[nst:, :nst] = Ads
        A[nst:, nst:] = Add
    if nmv > 0:
        Add = np.asfortranarray(A[nst:, nst:])
        lu, piv, info = lapack.dgetrf(Add, overwrite_a=1)
        if info != 0:
            raise RuntimeError("dgetrf info %d" % info)
        A[nst:, nst:] = lu
        P[nst:] = piv
        if nst > 0:
            Ads = np.asfortranarray(A[nst:, :nst])
            _laswp_rows(Ads, P[nst:], 0, nmv)
            A[nst:, :nst] = Ads
        P[nst:] += nst
    res, info = lapack.dgetrs(A, P, b)
    if info != 0:
        raise RuntimeError("dgetrs info %d" % info)
    return res, P


class CpuStep:
    """The full-step workload (dust_b200.synth.FullStepCase) on the host
    cores; ``step()`` returns the per-phase wall times (s)."""

    def __init__(self, case, params):
        self.case = case
        self.params = params
        c = case
        t0 = time.perf_counter()
        wk = (c.wake, c.n_impl, c.impl_ind)
        self.A, self.bst, self.b0 = O.linsys_init(params, c.rank, c.nstatic, c.elems, wk)
        if c.nstatic > 0:
            lu, piv, info = lapack.dgetrf(self.A[:c.nstatic, :c.nstatic])
            if info != 0:
                raise RuntimeError("static dgetrf info %d" % info)
            self.A[:c.nstatic, :c.nstatic] = lu
            self.P = np.zeros(c.rank, dtype=np.int32)
            self.P[:c.nstatic] = piv
        else:
            self.P = np.zeros(c.rank, dtype=np.int32)
        # A_pres: the surface panels' block of the influence matrix without
        # the wake correction (every surface panel is static here)
        self.sp = np.nonzero(c.elems.kind == abi.DUST_ELEM_SURFPAN)[0]
        if len(self.sp):
            Aw, _, _ = O.linsys_init(params, c.rank, c.nstatic, c.elems,
                                     (abi.empty_panels(), 0, None))
            self.lu_p, self.piv_p, info = lapack.dgetrf(Aw[np.ix_(self.sp, self.sp)])
            if info != 0:
                raise RuntimeError("A_pres dgetrf info %d" % info)
            del Aw
        self.vel = np.zeros((c.mag.shape[0], 3))
        from dust_b200.step import update_params_for
        self.upd = update_params_for(c, params)
        self.free = np.zeros(c.mag.shape[0], dtype=np.int32)
        self.t_init = time.perf_counter() - t0
        self.ind = c.impl_ind.astype(np.int64) - 1

    def step(self):
        c, prm = self.case, self.params
        t = {}
        t0 = time.perf_counter()
        cen_el = np.where(c.elems.n_ver[:, None] == 4, c.elems.ver.mean(axis=1),
                          c.elems.ver[:, :3].mean(axis=1))
        c.elems.uvort = O.points_uvort(prm, cen_el, c.cen, c.dir, c.mag, c.r_vortex, c.end_vort)
        t["uvort"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        b = self.b0.copy()
        O.linsys_step(prm, c.rank, c.nstatic, c.elems, (c.wake, c.n_impl, c.impl_ind), self.A,
                      self.bst, b)
        t["assemble"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        # the static block keeps its LU; the coupling blocks and the moving
        # block are rebuilt by the next assembly
        res, _ = solve_linsys_lapack(self.A, self.P, c.nstatic, b)
        t["solve"] = time.perf_counter() - t0
        if len(self.sp):
            t0 = time.perf_counter()
            bp = O.pressure_particles(np.ascontiguousarray(cen_el[self.sp]), c.cen, c.dir, c.mag,
                                      c.r_vortex, self.vel)
            self.res_pres, info = lapack.dgetrs(self.lu_p, self.piv_p, bp)
            t["pressure"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        c.elems.mag = res
        m2 = np.where(self.ind[:, 1] >= 0, res[np.maximum(self.ind[:, 1], 0)], 0.0)
        c.wake.mag = res[self.ind[:, 0]] - m2
        els = abi.elements_struct(c.elems, c.wake, c.end_vort)
        vel, st, ro, cnt = O.fmm_apply(prm, c.cen, c.dir, c.mag, c.r_vortex, els)
        t["fmm"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        cen, dir_, _, self.free, _ = O.particles_update(self.upd, c.cen, c.dir, c.mag, vel, st,
                                                        ro, self.free)
        c.cen[:], c.dir[:] = cen, dir_
        t["particles_update"] = time.perf_counter() - t0
        self.res, self.vel = res, vel
        return t
