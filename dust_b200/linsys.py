"""Host-side mirror of the reference's mod_linsys interface.

The reference (src/linsys/mod_linsys.f90:86-87) exposes initialize_linsys,
assemble_linsys, solve_linsys, destroy_linsys and dump_linsys.  ``Linsys``
keeps those names; the matrix and its factors stay on the GPU.
"""
import ctypes as C

import numpy as np

from . import abi
from ._lib import check, lib


class Linsys:
    def __init__(self, params, rank, nstatic, elems, wake=None, n_impl=0, impl_ind=None):
        """initialize_linsys: static rows, static wake, one-time LU of the
        static block.  ``elems`` is a PanelSet of all implicit elements
        (static first); ``wake`` a PanelSet of the wake panels (implicit ones
        first) with ``impl_ind`` (n_impl, 2) 1-based generating elements."""
        self.params = params
        self.rank = int(rank)
        self.nstatic = int(nstatic)
        self._p = params.struct()
        es = elems.struct()
        wk = wake if wake is not None else abi.empty_panels()
        ws, keep = abi.wake_rows_struct(wk, n_impl, impl_ind if n_impl else np.zeros(2))
        h = C.c_void_p()
        check(lib().dust_linsys_create(self.rank, self.nstatic, C.byref(self._p), C.byref(es),
                                       C.byref(ws), C.byref(h)), "dust_linsys_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().dust_linsys_destroy(self._h)
            self._h = None

    destroy_linsys = close

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def assemble_linsys(self, elems, wake=None, n_impl=0, impl_ind=None):
        es = elems.struct()
        wk = wake if wake is not None else abi.empty_panels()
        ws, keep = abi.wake_rows_struct(wk, n_impl, impl_ind if n_impl else np.zeros(2))
        check(lib().dust_linsys_assemble(self._h, C.byref(es), C.byref(ws)),
              "dust_linsys_assemble")

    def sync(self):
        """Wait for the handle's stream (assembly is asynchronous)."""
        # dust_linsys_get_system with no outputs only synchronises the stream
        check(lib().dust_linsys_get_system(self._h, abi.dptr(None), abi.dptr(None)),
              "dust_linsys_get_system")

    def get_system(self):
        """dump_linsys: (A, b) as assembled (the static block holds its LU)."""
        A = np.empty(self.rank * self.rank)
        b = np.empty(self.rank)
        check(lib().dust_linsys_get_system(self._h, abi.dptr(A), abi.dptr(b)),
              "dust_linsys_get_system")
        return A.reshape(self.rank, self.rank).T.copy(), b

    dump_linsys = get_system

    def solve_linsys(self, mode=abi.DUST_SOLVE_LU64):
        res = np.empty(self.rank)
        rep = abi.SolveReport()
        check(lib().dust_linsys_solve(self._h, int(mode), abi.dptr(res), C.byref(rep)),
              "dust_linsys_solve")
        return res, {k: getattr(rep, k) for k, _ in abi.SolveReport._fields_}


def initialize_linsys(params, rank, nstatic, elems, wake=None, n_impl=0, impl_ind=None):
    return Linsys(params, rank, nstatic, elems, wake, n_impl, impl_ind)


def dense_solve(A, B, mode=abi.DUST_SOLVE_LU64, tol=1e-12):
    """Solve A X = B on the GPU (LU as dgetrf/dgetrs, or mixed precision)."""
    A = np.asfortranarray(np.asarray(A, dtype=np.float64))
    B = np.asarray(B, dtype=np.float64)
    vec = B.ndim == 1
    Bf = np.asfortranarray(B.reshape(A.shape[0], -1))
    n, nrhs = Bf.shape
    X = np.zeros((n, nrhs), order="F")
    rep = abi.SolveReport()
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    check(lib().dust_dense_solve(int(n), int(nrhs), dp(A), dp(Bf), dp(X), int(mode),
                                 C.c_double(tol), C.byref(rep)), "dust_dense_solve")
    out = X[:, 0].copy() if vec else np.ascontiguousarray(X)
    return out, {k: getattr(rep, k) for k, _ in abi.SolveReport._fields_}


def dense_solve_device(A, B, X, mode=abi.DUST_SOLVE_LU64, tol=1e-12, stream=None):
    """A X = B on device arrays (torch CUDA float64 tensors; A (n, n) and B, X
    (n, nrhs) in column-major storage, i.e. the transposes of C-contiguous
    (n, n) / (nrhs, n) tensors).  A is not modified.  Returns the report."""
    n = A.shape[0]
    nrhs = B.numel() // n
    rep = abi.SolveReport()
    vp = lambda t: C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_double))
    check(lib().dust_dense_solve_device(int(n), int(nrhs), vp(A), vp(B), vp(X), int(mode),
                                        C.c_double(tol), C.byref(rep),
                                        C.c_void_p(stream or 0)), "dust_dense_solve_device")
    return {k: getattr(rep, k) for k, _ in abi.SolveReport._fields_}


class Pressure:
    """The pressure integral equation of a linear system
    (dust_pressure_*: initialize_pressure_sys, assemble_pressure_sys,
    solve_pressure_sys of src/linsys/mod_pressure_equation.f90).  Create it
    right after the Linsys; per step, after the Linsys assembly, call
    assemble_device and solve_device (torch CUDA tensors)."""

    def __init__(self, ls):
        self.ls = ls
        h = C.c_void_p()
        check(lib().dust_pressure_create(ls._h, C.byref(h)), "dust_pressure_create")
        self._h = h
        nsp, nss = C.c_int(0), C.c_int(0)
        check(lib().dust_pressure_size(h, C.byref(nsp), C.byref(nss)), "dust_pressure_size")
        self.n_sp, self.nstatic_sp = nsp.value, nss.value

    def close(self):
        if getattr(self, "_h", None):
            lib().dust_pressure_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _p(t):
        return (C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_double)) if t is not None
                else C.POINTER(C.c_double)())

    def assemble_device(self, bern=None, parts=None, vel=None, wake=None, wake_vv=None,
                        end_vort=None, end_vv=None, stream=0):
        """parts = (cen, dir, mag, r_vortex) device tensors of the live
        particles, vel their velocities; wake / end_vort abi.Panels / abi.Lines
        structs of device pointers with wake_vv / end_vv device tensors."""
        P = self._p
        cen, dir_, mag, rv = parts if parts is not None else (None,) * 4
        n = int(mag.shape[0]) if mag is not None else 0
        check(lib().dust_pressure_assemble_device(
            self._h, self.ls._h, P(bern), n, P(cen), P(dir_), P(mag), P(rv), P(vel),
            C.byref(wake) if wake is not None else None, P(wake_vv),
            C.byref(end_vort) if end_vort is not None else None, P(end_vv),
            C.c_void_p(stream)), "dust_pressure_assemble_device")

    def assemble_terms_device(self, bern=None, pterm=None, wake=None, wake_vv=None,
                              end_vort=None, end_vv=None, stream=0):
        """assemble_device with the particle term already evaluated at every
        element centre (pterm, device tensor of the system's rank)."""
        P = self._p
        check(lib().dust_pressure_assemble_terms_device(
            self._h, self.ls._h, P(bern), P(pterm),
            C.byref(wake) if wake is not None else None, P(wake_vv),
            C.byref(end_vort) if end_vort is not None else None, P(end_vv),
            C.c_void_p(stream)), "dust_pressure_assemble_terms_device")

    def solve_device(self, res, stream=0):
        check(lib().dust_pressure_solve_device(self._h, self._p(res), C.c_void_p(stream)),
              "dust_pressure_solve_device")

    def assemble(self, bern=None, parts=None, vel=None):
        """Host-array variant of assemble_device (particles only)."""
        cen, dir_, mag, rv = (abi.f64(a) for a in parts) if parts is not None else (None,) * 4
        n = int(mag.shape[0]) if mag is not None else 0
        check(lib().dust_pressure_assemble(self._h, self.ls._h, abi.dptr(abi.f64(bern)), n,
                                           abi.dptr(cen), abi.dptr(dir_), abi.dptr(mag),
                                           abi.dptr(rv), abi.dptr(abi.f64(vel)), None, None,
                                           None, None), "dust_pressure_assemble")

    def assemble_terms(self, bern=None, pterm=None):
        """Host-array variant of assemble_terms_device (pterm of the system's
        rank from points_uvort_pressure)."""
        check(lib().dust_pressure_assemble_terms(self._h, self.ls._h, abi.dptr(abi.f64(bern)),
                                                 abi.dptr(abi.f64(pterm)), None, None, None,
                                                 None), "dust_pressure_assemble_terms")

    def solve(self):
        res = np.zeros(self.n_sp)
        check(lib().dust_pressure_solve(self._h, abi.dptr(res)), "dust_pressure_solve")
        return res

    def get_system(self):
        """dump_linsys_pres: (A_pres, b_pres) as assembled (host)."""
        n = self.n_sp
        A = np.empty(n * n)
        b = np.empty(n)
        check(lib().dust_pressure_get_system(self._h, abi.dptr(A), abi.dptr(b)),
              "dust_pressure_get_system")
        return A.reshape(n, n).T.copy(), b
