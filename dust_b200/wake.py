"""The particle loop of complete_wake (src/aeroel/mod_wake.f90:1309-1355) on
the GPU: move every live particle by vel dt ndt_update_wake, free the ones
that leave the particle box, filter the stretching term and renew the
direction (mag unchanged), as dust_particles_update in include/dust_b200.h.
"""
import ctypes as C

import numpy as np

from . import abi
from ._lib import check, lib


def complete_wake_particles(u, cen, dir_, mag, vel, stretch, rotu, free):
    """Host arrays (cen, dir, vel, stretch, rotu: (n, 3); mag: (n,); free:
    (n,) 0/1); ``u`` from abi.update_params.  Returns updated copies
    (cen, dir, stretch, free) and the number of particles set free."""
    cen, dir_, stretch = (np.array(abi.f64(a), dtype=np.float64, order="C")
                          for a in (cen, dir_, stretch))
    mag, vel, rotu = abi.f64(mag), abi.f64(vel), abi.f64(rotu)
    free = np.array(free, dtype=np.int32, order="C")
    nf = C.c_int(0)
    check(lib().dust_particles_update(C.byref(u), int(mag.shape[0]), abi.dptr(cen),
                                      abi.dptr(dir_), abi.dptr(mag), abi.dptr(vel),
                                      abi.dptr(stretch), abi.dptr(rotu),
                                      free.ctypes.data_as(C.POINTER(C.c_int)), C.byref(nf)),
          "dust_particles_update")
    return cen, dir_, stretch, free, nf.value


def complete_wake_particles_device(u, cen, dir_, mag, vel, stretch, rotu, free, n_freed,
                                   stream=0):
    """Device variant on torch CUDA tensors, in place: cen, dir, stretch
    (float64, (n, 3)), free (int32, (n,)), n_freed (int32, (1,)); queued on
    ``stream`` (an int handle, 0 = default stream), not synchronised."""
    vp = lambda t: C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_double)) \
        if t is not None else C.POINTER(C.c_double)()
    ip = lambda t: C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_int))
    check(lib().dust_particles_update_device(C.byref(u), int(mag.shape[0]), vp(cen), vp(dir_),
                                             vp(mag), vp(vel), vp(stretch), vp(rotu), ip(free),
                                             ip(n_freed), C.c_void_p(stream)),
          "dust_particles_update_device")


def _dp(t):
    """double* of a torch CUDA tensor (None -> NULL)."""
    return (C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_double)) if t is not None
            else C.POINTER(C.c_double)())


def _ip(t):
    return (C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_int)) if t is not None
            else C.POINTER(C.c_int)())


def complete_wake_particles_pa_device(u, pa, body, cen, dir_, mag, r_vortex, vel, stretch, rotu,
                                      free, n_freed, stream=0):
    """complete_wake's particle loop with penetration avoidance
    (dust_particles_update_pa_device) on torch CUDA tensors, in place; ``body``
    an abi.Panels struct of device pointers, ``pa`` from abi.pa_params."""
    check(lib().dust_particles_update_pa_device(
        C.byref(u), C.byref(pa), C.byref(body), int(mag.shape[0]), _dp(cen), _dp(dir_),
        _dp(mag), _dp(r_vortex), _dp(vel), _dp(stretch), _dp(rotu), _ip(free), _ip(n_freed),
        C.c_void_p(stream)), "dust_particles_update_pa_device")


def live_particles_device(free, cen, dir_, mag, r_vortex, lcen, ldir, lmag, lrv, idx, stream=0):
    """The live particles in slot order (prepare_wake's part_p list) into the
    l* tensors and their slot indices into idx; returns their number."""
    n = C.c_int(0)
    check(lib().dust_particles_live_device(int(free.shape[0]), _ip(free), _dp(cen), _dp(dir_),
                                           _dp(mag), _dp(r_vortex), _dp(lcen), _dp(ldir),
                                           _dp(lmag), _dp(lrv), _ip(idx), C.byref(n),
                                           C.c_void_p(stream)), "dust_particles_live_device")
    return n.value


def scatter_particles_device(n_live, idx, lvel, lstr, lrot, vel, stretch, rotu, stream=0):
    check(lib().dust_particles_scatter_device(int(n_live), _ip(idx), _dp(lvel), _dp(lstr),
                                              _dp(lrot), _dp(vel), _dp(stretch), _dp(rotu),
                                              C.c_void_p(stream)),
          "dust_particles_scatter_device")


class PanelWake:
    """The device-resident panel wake and its shedding (dust_wake_* of
    include/dust_b200.h): initialize_wake on creation, then per step
    set_first_row (update_wake :884-892), update (the rest of update_wake's
    panel part) and complete (complete_wake's rows, shedding, end vortices).

    ``prm``: abi.WakeParams; ii, neigh, neigh_o, gen: (n_stripes, 2) ints,
    1-based; te_pts, te_dir: (n_points, 3); te_scaling: (n_points,)."""

    def __init__(self, prm, ii, neigh, neigh_o, gen, te_pts, te_dir, te_scaling, te_vel=None):
        self.prm = prm
        self._te_keep = [abi.i32(np.asarray(a).reshape(-1)) for a in (ii, neigh, neigh_o, gen)]
        te = abi.Te(*[abi.iptr(a) for a in self._te_keep])
        h = C.c_void_p()
        check(lib().dust_wake_create(C.byref(prm), C.byref(te), abi.dptr(abi.f64(te_pts)),
                                     abi.dptr(abi.f64(te_dir)), abi.dptr(abi.f64(te_scaling)),
                                     abi.dptr(abi.f64(te_vel)), C.byref(h)), "dust_wake_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().dust_wake_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # pragma: no cover
            pass

    def elements(self):
        """(wake panels abi.Panels, end vortices abi.Lines, n_impl, impl_ind
        pointer): device views valid until the next call on the wake."""
        wp, ev = abi.Panels(), abi.Lines()
        ni = C.c_int(0)
        ip = C.POINTER(C.c_int)()
        check(lib().dust_wake_elements(self._h, C.byref(wp), C.byref(ev), C.byref(ni),
                                       C.byref(ip)), "dust_wake_elements")
        return wp, ev, ni.value, ip

    def set_first_row(self, res, stream=0):
        check(lib().dust_wake_set_first_row_device(self._h, _dp(res), C.c_void_p(stream)),
              "dust_wake_set_first_row_device")

    def update(self, fprm_struct, body, cen, dir_, mag, r_vortex, n=None, stream=0):
        """update_wake's panel part after the first row; ``body`` abi.Panels
        (device pointers, mag = the solution), particles: the live list."""
        nn = int(mag.shape[0]) if n is None else int(n)
        check(lib().dust_wake_update_device(self._h, C.byref(fprm_struct), C.byref(body), nn,
                                            _dp(cen), _dp(dir_), _dp(mag), _dp(r_vortex),
                                            C.c_void_p(stream)), "dust_wake_update_device")

    def complete(self, te_pts, te_dir, te_scaling, te_vel, cen, dir_, mag, r_vortex, vel, free,
                 stream=0):
        """complete_wake's panel part and shedding into the slot tensors;
        returns the number of particles shed."""
        ns = C.c_int(0)
        check(lib().dust_wake_complete_device(self._h, _dp(te_pts), _dp(te_dir), _dp(te_scaling),
                                              _dp(te_vel), int(free.shape[0]), _dp(cen),
                                              _dp(dir_), _dp(mag), _dp(r_vortex), _dp(vel),
                                              _ip(free), C.byref(ns), C.c_void_p(stream)),
              "dust_wake_complete_device")
        return ns.value

    def get_state(self):
        """(len, points (len+1, n_points, 3), point velocities, idou (len,
        n_stripes), last_pan_idou) as host arrays."""
        p = self.prm
        ln = C.c_int(0)
        check(lib().dust_wake_get_state(self._h, C.byref(ln), None, None, None, None),
              "dust_wake_get_state")
        L = ln.value
        pts = np.zeros((L + 1, p.n_points, 3))
        pv = np.zeros((L + 1, p.n_points, 3))
        idou = np.zeros((L, p.n_stripes))
        last = np.zeros(p.n_stripes)
        check(lib().dust_wake_get_state(self._h, C.byref(ln), abi.dptr(pts), abi.dptr(pv),
                                        abi.dptr(idou), abi.dptr(last)), "dust_wake_get_state")
        return L, pts, pv, idou, last

    def set_state(self, length, points, point_vel, idou, last):
        """load_wake: state of a result file."""
        check(lib().dust_wake_set_state(self._h, int(length), abi.dptr(abi.f64(points)),
                                        abi.dptr(abi.f64(point_vel)), abi.dptr(abi.f64(idou)),
                                        abi.dptr(abi.f64(last))), "dust_wake_set_state")
