"""Host-side mirror of the reference's mod_octree interface.

The reference (src/fmm/mod_octree.f90:78-79) exposes initialize_octree,
sort_particles, calculate_multipole, apply_multipole, apply_multipole_panels
and destroy_octree.  Here initialize_octree returns an ``Octree`` whose
``apply_multipole`` runs sort + calculate + apply in one C-ABI call
(``dust_fmm_apply``), the way the per-timestep caller uses them
(mod_wake.f90:797-801 then :1115-1118 within one step).  Errors raise
``DustError`` as the reference calls ``error`` (mod_handling.f90:181).
"""
import ctypes as C

import numpy as np

from . import abi
from ._lib import check, lib


class Octree:
    def __init__(self, params):
        self.params = params
        self._p = params.struct()
        h = C.c_void_p()
        check(lib().dust_octree_create(C.byref(self._p), C.byref(h)), "dust_octree_create")
        self._h = h

    def close(self):
        if self._h:
            lib().dust_octree_destroy(self._h)
            self._h = None

    destroy_octree = close

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_timing(self, on=True):
        check(lib().dust_octree_set_timing(self._h, int(bool(on))), "dust_octree_set_timing")

    def stats(self):
        s = abi.FmmStats()
        check(lib().dust_octree_get_stats(self._h, C.byref(s)), "dust_octree_get_stats")
        return {k: getattr(s, k) for k, _ in abi.FmmStats._fields_}

    def apply_multipole(self, cen, dir_, mag, r_vortex, elements=None,
                        want_stretch=True, want_rotu=True, out=None):
        """Velocity (incl. u_inf), stretching and div-filter curl at every
        particle, in the caller's particle order.  ``out``: optional
        (vel, stretch, rotu) host arrays (n x 3 float64, C order) to write,
        e.g. page-locked buffers reused across steps."""
        cen, dir_, mag, rv = (abi.f64(cen), abi.f64(dir_), abi.f64(mag), abi.f64(r_vortex))
        n = mag.shape[0]
        est, keep = elements if elements is not None else abi.elements_struct()
        if out is not None:
            vel, st, ro = out
            for a in (vel, st, ro):
                if a is not None and (a.dtype != np.float64 or a.shape != (n, 3)
                                      or not a.flags.c_contiguous):
                    raise ValueError("out arrays must be C-contiguous float64 (n, 3)")
        else:
            vel = np.empty((n, 3))
            st = np.empty((n, 3)) if want_stretch else None
            ro = np.empty((n, 3)) if want_rotu else None
        check(lib().dust_fmm_apply(self._h, n, abi.dptr(cen), abi.dptr(dir_), abi.dptr(mag),
                                   abi.dptr(rv), C.byref(est), abi.dptr(vel), abi.dptr(st),
                                   abi.dptr(ro)), "dust_fmm_apply")
        return vel, st, ro

    # --- the two halves (prepare_wake's octree part / update_wake's apply)
    def prepare(self, cen, dir_, mag, r_vortex, pts=None):
        """sort_particles + calculate_multipole (host arrays); ``pts`` are the
        evaluation points (panel centres) sorted into the tree with them."""
        cen, dir_, mag, rv = (abi.f64(cen), abi.f64(dir_), abi.f64(mag), abi.f64(r_vortex))
        pts = None if pts is None else abi.f64(pts).reshape(-1, 3)
        self._n = mag.shape[0]
        self._npts = 0 if pts is None else pts.shape[0]
        check(lib().dust_fmm_prepare(self._h, self._n, abi.dptr(cen), abi.dptr(dir_),
                                     abi.dptr(mag), abi.dptr(rv), self._npts, abi.dptr(pts)),
              "dust_fmm_prepare")

    def points_uvort(self, end_vort=None):
        """apply_multipole_panels: the prepared particles' velocity at the
        prepared points plus the end vortices (host arrays)."""
        ev = end_vort if end_vort is not None else abi.empty_lines()
        evs = ev.struct()
        out = np.empty((getattr(self, "_npts", 0), 3))
        check(lib().dust_fmm_points_uvort(self._h, C.byref(evs), abi.dptr(out)),
              "dust_fmm_points_uvort")
        return out

    def finish(self, elements=None, want_stretch=True, want_rotu=True, out=None):
        """apply_multipole at the prepared particles (host outputs)."""
        n = self._n
        est, keep = elements if elements is not None else abi.elements_struct()
        if out is not None:
            vel, st, ro = out
        else:
            vel = np.empty((n, 3))
            st = np.empty((n, 3)) if want_stretch else None
            ro = np.empty((n, 3)) if want_rotu else None
        check(lib().dust_fmm_finish(self._h, C.byref(est), abi.dptr(vel), abi.dptr(st),
                                    abi.dptr(ro)), "dust_fmm_finish")
        return vel, st, ro

    def apply_multipole_device(self, cen, dir_, mag, r_vortex, vel, stretch=None, rotu=None,
                               elements=None, stream=0, sync=True):
        """Device-resident variant: arguments are torch CUDA tensors (float64,
        contiguous); ``elements`` is a (struct, keep) pair whose pointers are
        device pointers."""
        n = mag.shape[0]
        vp = lambda t: C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_double)) \
            if t is not None else C.POINTER(C.c_double)()
        est = elements[0] if elements is not None else abi.elements_struct()[0]
        check(lib().dust_fmm_apply_device(self._h, int(n), vp(cen), vp(dir_), vp(mag),
                                          vp(r_vortex), C.byref(est), vp(vel), vp(stretch),
                                          vp(rotu), C.c_void_p(stream), int(bool(sync))),
              "dust_fmm_apply_device")


def initialize_octree(params):
    """initialize_octree (mod_octree.f90:251)."""
    return Octree(params)


def direct_particles(params, cen, dir_, mag, r_vortex, n_tgt=None):
    """All-pairs evaluation of the particle kernels on the GPU (FMM truth)."""
    cen, dir_, mag, rv = (abi.f64(cen), abi.f64(dir_), abi.f64(mag), abi.f64(r_vortex))
    n = mag.shape[0]
    nt = n if n_tgt is None else int(n_tgt)
    vel, st, ro = np.empty((nt, 3)), np.empty((nt, 3)), np.empty((nt, 3))
    p = params.struct()
    check(lib().dust_direct_particles(C.byref(p), n, abi.dptr(cen), abi.dptr(dir_),
                                      abi.dptr(mag), abi.dptr(rv), nt, abi.dptr(vel),
                                      abi.dptr(st), abi.dptr(ro)), "dust_direct_particles")
    return vel, st, ro


def points_uvort(params, pts, cen, dir_, mag, r_vortex, end_vort=None):
    """get_vort_vel at arbitrary points (panel centres): particles + end vortices."""
    pts = abi.f64(pts).reshape(-1, 3)
    cen, dir_, mag, rv = (abi.f64(cen), abi.f64(dir_), abi.f64(mag), abi.f64(r_vortex))
    ev = end_vort if end_vort is not None else abi.empty_lines()
    evs = ev.struct()
    out = np.empty_like(pts)
    p = params.struct()
    check(lib().dust_points_uvort(C.byref(p), pts.shape[0], abi.dptr(pts), mag.shape[0],
                                  abi.dptr(cen), abi.dptr(dir_), abi.dptr(mag), abi.dptr(rv),
                                  C.byref(evs), abi.dptr(out)), "dust_points_uvort")
    return out


def elements_vel(params, pts, elements):
    pts = abi.f64(pts).reshape(-1, 3)
    est, keep = elements
    out = np.empty_like(pts)
    p = params.struct()
    check(lib().dust_elements_vel(C.byref(p), pts.shape[0], abi.dptr(pts), C.byref(est),
                                  abi.dptr(out)), "dust_elements_vel")
    return out


def panels_geometry(panels):
    s = panels.struct()
    n = panels.n
    cen, nor, area = np.empty((n, 3)), np.empty((n, 3)), np.empty(n)
    check(lib().dust_panels_geometry(C.byref(s), abi.dptr(cen), abi.dptr(nor),
                                     abi.dptr(area)), "dust_panels_geometry")
    return cen, nor, area
