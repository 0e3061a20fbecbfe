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
