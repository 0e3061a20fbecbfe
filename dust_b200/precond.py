"""Learned sparse approximate inverse for the moving-body system.

Python side of the C-ABI's dust_precond_*: a graph network over the panels'
k-nearest-neighbour graph maps the current influence matrix to
M = (I + O) D^-1, the right preconditioner and warm start of the FP64 GMRES
that DUST_SOLVE_GMRES_NN runs (plain LU is the fallback).  Training samples
are systems the plain method has assembled and solved; the network trains on
the GPU with the library's own forward and backward kernels.
"""
import ctypes as C

import numpy as np

from . import abi
from ._lib import check, lib


class Precond:
    def __init__(self, centres, k=8, seed=0):
        centres = np.ascontiguousarray(centres, dtype=np.float64).reshape(-1, 3)
        self.n = centres.shape[0]
        self.k = int(k)
        h = C.c_void_p()
        check(lib().dust_precond_create(self.n, self.k, abi.dptr(centres), C.c_ulonglong(seed),
                                        C.byref(h)), "dust_precond_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().dust_precond_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def num_params():
        return int(lib().dust_precond_num_params())

    def get_params(self):
        w = np.empty(self.num_params(), dtype=np.float32)
        check(lib().dust_precond_get_params(self._h, w.ctypes.data_as(C.POINTER(C.c_float)),
                                            w.size), "dust_precond_get_params")
        return w

    def set_params(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        check(lib().dust_precond_set_params(self._h, w.ctypes.data_as(C.POINTER(C.c_float)),
                                            w.size), "dust_precond_set_params")

    def add_sample(self, linsys, x, seed=0):
        """`linsys` assembled and not yet solved; x its solution (host)."""
        import torch
        xd = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).cuda()
        torch.cuda.synchronize()
        check(lib().dust_precond_add_sample(self._h, linsys._h,
                                            C.cast(C.c_void_p(xd.data_ptr()), abi._dp),
                                            C.c_ulonglong(seed)), "dust_precond_add_sample")

    @property
    def num_samples(self):
        return int(lib().dust_precond_num_samples(self._h))

    def loss_grad(self, si, with_grad=True):
        loss = C.c_float()
        g = np.empty(self.num_params(), dtype=np.float32) if with_grad else None
        gp = g.ctypes.data_as(C.POINTER(C.c_float)) if with_grad else C.POINTER(C.c_float)()
        check(lib().dust_precond_loss_grad(self._h, int(si), C.byref(loss), gp,
                                           self.num_params()), "dust_precond_loss_grad")
        return float(loss.value), g

    def get_sample(self, si):
        """Host copies (x, ef, w, nbr, Y, T) of stored sample si."""
        n, K = self.n, self.k + 1
        x = np.empty((n, 8), np.float32)
        ef = np.empty((n, K, 4), np.float32)
        w = np.empty((n, K), np.float32)
        nbr = np.empty((n, K), np.int32)
        Y = np.empty((n, 8), np.float32)
        T = np.empty((n, 8), np.float32)
        fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
        check(lib().dust_precond_get_sample(self._h, int(si), fp(x), fp(ef), fp(w),
                                            nbr.ctypes.data_as(C.POINTER(C.c_int)), fp(Y), fp(T)),
              "dust_precond_get_sample")
        return x, ef, w, nbr, Y, T

    def train(self, iters, lr=1e-3):
        loss = C.c_float()
        check(lib().dust_precond_train(self._h, int(iters), C.c_float(lr), C.byref(loss)),
              "dust_precond_train")
        return float(loss.value)

    def attach(self, linsys):
        check(lib().dust_linsys_set_precond(linsys._h, self._h), "dust_linsys_set_precond")

    @staticmethod
    def detach(linsys):
        check(lib().dust_linsys_set_precond(linsys._h, C.c_void_p()), "dust_linsys_set_precond")


def train_for_case(case, params, angles, iters=400, lr=2e-3, k=8, seed=0):
    """Trains a Precond on the moving-body systems of ``case`` (a
    synth.FullStepCase-like object with set_angle) at the given rotor
    azimuths: each system is assembled and solved by the plain LU, then
    stored as a sample.  Returns (precond, info) and leaves the case at
    azimuth 0."""
    import time
    from .linsys import Linsys
    c = case
    t0 = time.perf_counter()
    ls = Linsys(params, c.rank, c.nstatic, c.elems, c.wake, c.n_impl, c.impl_ind)
    pc = Precond(_centres(c.elems), k=k, seed=seed)
    for q, ang in enumerate(angles):
        c.set_angle(float(ang))
        ls.assemble_linsys(c.elems, c.wake, c.n_impl, c.impl_ind)
        x, _ = ls.solve_linsys(abi.DUST_SOLVE_LU64)
        ls.assemble_linsys(c.elems, c.wake, c.n_impl, c.impl_ind)
        pc.add_sample(ls, x, seed=seed * 1000 + q)
    t1 = time.perf_counter()
    l0 = float(np.mean([pc.loss_grad(i, with_grad=False)[0] for i in range(pc.num_samples)]))
    l1 = pc.train(iters, lr)
    t2 = time.perf_counter()
    # GMRES iterations on the azimuth-0 system (not a training azimuth when
    # the caller offsets them): untrained network (Jacobi) vs trained
    c.set_angle(0.0)
    its = {}
    for name, p in (("gmres_iters_untrained", Precond(_centres(c.elems), k=k, seed=seed)),
                    ("gmres_iters_trained", pc)):
        p.attach(ls)
        ls.assemble_linsys(c.elems, c.wake, c.n_impl, c.impl_ind)
        _, rep = ls.solve_linsys(abi.DUST_SOLVE_GMRES_NN)
        its[name] = int(rep["iterations"]) if not rep["fell_back"] else None
    Precond.detach(ls)
    ls.close()
    info = {"samples": int(pc.num_samples), "iters": int(iters), "loss_untrained": l0,
            "loss_trained": l1, "s_data": round(t1 - t0, 2), "s_train": round(t2 - t1, 2)}
    info.update(its)
    return pc, info


def _centres(elems):
    """Panel centres as the library computes them (mean of the vertices)."""
    nv = elems.n_ver
    cen = elems.ver.mean(axis=1)
    tri = nv == 3
    if tri.any():
        cen[tri] = elems.ver[tri, :3].mean(axis=1)
    return cen
