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
