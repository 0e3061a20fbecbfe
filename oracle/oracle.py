"""Python access to the CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module; the product never does.  It builds (if needed) and loads
oracle/_build/libdust_oracle.so, the C restatement of the reference's hot
path (see dust_oracle.h for the file:line map).
"""
import ctypes as C
import os
import subprocess

import numpy as np

from dust_b200 import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "libdust_oracle.so")
_lib = None


def build():
    subprocess.run(["make", "-C", _HERE, "-s"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        _lib = C.CDLL(_SO)
        L = _lib
        L.or_fmm_apply.restype = C.c_int
        L.or_direct_particles.restype = C.c_int
        L.or_elements_vel.restype = C.c_int
        L.or_points_uvort.restype = C.c_int
        L.or_fmm_points_uvort.restype = C.c_int
        L.or_potential_doublet.restype = C.c_double
        L.or_potential_source.restype = C.c_double
        L.or_dgetrf.restype = C.c_int
        L.or_linsys_run.restype = C.c_int
        L.or_linsys_rows.restype = C.c_int
        L.or_last_tree_flags.restype = C.c_int
        L.or_particles_update.restype = C.c_int
        L.or_particles_update_pa.restype = C.c_int
        L.or_pressure_run.restype = C.c_int
        L.or_pressure_particles.restype = C.c_int
    return _lib


def set_factorial_wrap(on):
    lib().or_set_factorial_wrap(C.c_int(int(on)))


def _out(n, on=True):
    return np.zeros((n, 3)) if on else None


def set_sample_stride(stride):
    """Work sampling of fmm_apply for timing (1 = full evaluation)."""
    lib().or_set_sample_stride(C.c_int(int(stride)))


def last_fmm_times():
    """Phase times (s) of the last fmm_apply -- tree, upward, M2L + L2L,
    apply -- and the sampled work (M2L pairs, particles evaluated)."""
    t = np.zeros(4)
    n = np.zeros(2, dtype=np.int64)
    lib().or_last_fmm_times(abi.dptr(t), n.ctypes.data_as(C.POINTER(C.c_int64)))
    return t, n


def fmm_apply(prm, cen, dir_, mag, rvort, elems=None):
    """FMM evaluation; returns (vel, stretch, rotu, counters)."""
    cen, dir_, mag, rvort = (abi.f64(cen), abi.f64(dir_), abi.f64(mag), abi.f64(rvort))
    n = mag.shape[0]
    est, keep = elems if elems is not None else abi.elements_struct()
    vel, st, ro = _out(n), _out(n), _out(n)
    cnt = np.zeros(4, dtype=np.int64)
    p = prm.struct()
    rc = lib().or_fmm_apply(C.byref(p), n, abi.dptr(cen), abi.dptr(dir_), abi.dptr(mag),
                            abi.dptr(rvort), C.byref(est), abi.dptr(vel), abi.dptr(st),
                            abi.dptr(ro), cnt.ctypes.data_as(C.POINTER(C.c_int64)))
    if rc != 0:
        raise RuntimeError(f"oracle or_fmm_apply status {rc}")
    return vel, st, ro, cnt


def last_tree_flags(prm):
    tot = sum(int(np.prod(prm.n_box)) * 8 ** (l - 1)
              for l in range(1, prm.n_octree_levels + 1))
    fl = np.zeros(tot, dtype=np.uint8)
    rc = lib().or_last_tree_flags(fl.ctypes.data_as(C.POINTER(C.c_ubyte)), C.c_int64(tot))
    if rc != 0:
        raise RuntimeError(f"oracle tree flags status {rc}")
    return fl


def direct_particles(prm, cen, dir_, mag, rvort, n_tgt=None):
    cen, dir_, mag, rvort = (abi.f64(cen), abi.f64(dir_), abi.f64(mag), abi.f64(rvort))
    n = mag.shape[0]
    nt = n if n_tgt is None else int(n_tgt)
    vel, st, ro = _out(nt), _out(nt), _out(nt)
    p = prm.struct()
    rc = lib().or_direct_particles(C.byref(p), n, abi.dptr(cen), abi.dptr(dir_),
                                   abi.dptr(mag), abi.dptr(rvort), nt, abi.dptr(vel),
                                   abi.dptr(st), abi.dptr(ro))
    if rc != 0:
        raise RuntimeError(f"oracle direct status {rc}")
    return vel, st, ro


def elements_vel(prm, pts, elems):
    pts = abi.f64(pts).reshape(-1, 3)
    est, keep = elems
    vel = np.zeros_like(pts)
    p = prm.struct()
    rc = lib().or_elements_vel(C.byref(p), pts.shape[0], abi.dptr(pts), C.byref(est),
                               abi.dptr(vel))
    if rc != 0:
        raise RuntimeError(f"oracle elements status {rc}")
    return vel


def points_uvort(prm, pts, cen, dir_, mag, rvort, end_vort=None):
    pts = abi.f64(pts).reshape(-1, 3)
    cen, dir_, mag, rvort = (abi.f64(cen), abi.f64(dir_), abi.f64(mag), abi.f64(rvort))
    ev = end_vort if end_vort is not None else abi.empty_lines()
    evs = ev.struct()
    out = np.zeros_like(pts)
    p = prm.struct()
    rc = lib().or_points_uvort(C.byref(p), pts.shape[0], abi.dptr(pts), mag.shape[0],
                               abi.dptr(cen), abi.dptr(dir_), abi.dptr(mag),
                               abi.dptr(rvort), C.byref(evs), abi.dptr(out))
    if rc != 0:
        raise RuntimeError(f"oracle uvort status {rc}")
    return out


def fmm_points_uvort(prm, pts, cen, dir_, mag, rvort, end_vort=None):
    """apply_multipole_panels: uvort at points from the particles' FMM plus
    the end vortices by direct sum."""
    pts = abi.f64(pts).reshape(-1, 3)
    cen, dir_, mag, rvort = (abi.f64(cen), abi.f64(dir_), abi.f64(mag), abi.f64(rvort))
    ev = end_vort if end_vort is not None else abi.empty_lines()
    evs = ev.struct()
    out = np.zeros_like(pts)
    p = prm.struct()
    rc = lib().or_fmm_points_uvort(C.byref(p), mag.shape[0], abi.dptr(cen), abi.dptr(dir_),
                                   abi.dptr(mag), abi.dptr(rvort), pts.shape[0], abi.dptr(pts),
                                   C.byref(evs), abi.dptr(out))
    if rc != 0:
        raise RuntimeError(f"oracle FMM uvort status {rc}")
    return out


def panel_geometry(pan):
    s = pan.struct()
    n = pan.n
    cen, nor, area = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n)
    lib().or_panel_geometry(C.byref(s), abi.dptr(cen), abi.dptr(nor), abi.dptr(area))
    return cen, nor, area


def potential_doublet(prm, pan, j, pos):
    s, p = pan.struct(), prm.struct()
    pos = abi.f64(pos)
    return lib().or_potential_doublet(C.byref(p), C.byref(s), int(j), abi.dptr(pos))


def velocity_doublet(prm, pan, j, pos):
    s, p = pan.struct(), prm.struct()
    pos = abi.f64(pos)
    v = np.zeros(3)
    lib().or_velocity_doublet(C.byref(p), C.byref(s), int(j), abi.dptr(pos), abi.dptr(v))
    return v


def potential_source(prm, pan, j, dou, pos):
    s, p = pan.struct(), prm.struct()
    pos = abi.f64(pos)
    return lib().or_potential_source(C.byref(p), C.byref(s), int(j), C.c_double(dou),
                                     abi.dptr(pos))


def velocity_source(prm, pan, j, pos):
    s, p = pan.struct(), prm.struct()
    pos = abi.f64(pos)
    v = np.zeros(3)
    lib().or_velocity_source(C.byref(p), C.byref(s), int(j), abi.dptr(pos), abi.dptr(v))
    return v


def dgetrf(A):
    """LU of a square matrix (returns column-major LU as (n,n) Fortran array, ipiv 1-based)."""
    A = np.asfortranarray(np.array(A, dtype=np.float64))
    n = A.shape[0]
    ipiv = np.zeros(n, dtype=np.int32)
    info = lib().or_dgetrf(n, n, A.ctypes.data_as(C.POINTER(C.c_double)), n,
                           ipiv.ctypes.data_as(C.POINTER(C.c_int)))
    return A, ipiv, info


def linsys_run(prm, rank, nstatic, elems_init, elems_step, wake_init, wake_step):
    """Assemble (init + one step) and solve; returns (A, b, res)."""
    ei, es = elems_init.struct(), elems_step.struct()
    wi, ki = abi.wake_rows_struct(*wake_init)
    ws, ks = abi.wake_rows_struct(*wake_step)
    A = np.zeros(rank * rank)
    b = np.zeros(rank)
    res = np.zeros(rank)
    p = prm.struct()
    rc = lib().or_linsys_run(C.byref(p), int(rank), int(nstatic), C.byref(ei), C.byref(es),
                             C.byref(wi), C.byref(ws), abi.dptr(A), abi.dptr(b),
                             abi.dptr(res))
    if rc != 0:
        raise RuntimeError(f"oracle linsys status {rc}")
    return A.reshape(rank, rank).T.copy(), b, res


def linsys_init(prm, rank, nstatic, elems, wake):
    """initialize_linsys's static rows and wake (no LU): returns (A, bst, b)
    with A as a Fortran-ordered (rank, rank) array."""
    es = elems.struct()
    ws, kk = abi.wake_rows_struct(*wake)
    A = np.zeros((rank, rank), order="F")
    nb = max(int(nstatic), 1)
    bst = np.zeros((nb, nb), order="F")
    b = np.zeros(rank)
    p = prm.struct()
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    lib().or_linsys_init(C.byref(p), int(rank), int(nstatic), C.byref(es), C.byref(ws), dp(A),
                         dp(bst), dp(b))
    return A, bst, b


def linsys_step(prm, rank, nstatic, elems, wake, A, bst, b):
    """assemble_linsys into A (Fortran-ordered, static block untouched) and b."""
    assert A.flags.f_contiguous and bst.flags.f_contiguous
    es = elems.struct()
    ws, kk = abi.wake_rows_struct(*wake)
    p = prm.struct()
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    lib().or_linsys_step(C.byref(p), int(rank), int(nstatic), C.byref(es), C.byref(ws), dp(A),
                         dp(bst), dp(b))


def linsys_rows(prm, elems, rows, wake=None):
    """Rows of the all-moving system (A rows (len(rows), rank), b rows)."""
    rank = elems.n
    es = elems.struct()
    wk = wake if wake is not None else (abi.empty_panels(), 0, None)
    ws, kk = abi.wake_rows_struct(*wk)
    rows = np.ascontiguousarray(rows, dtype=np.int32)
    A = np.zeros((len(rows), rank))
    b = np.zeros(len(rows))
    p = prm.struct()
    rc = lib().or_linsys_rows(C.byref(p), int(rank), C.byref(es), C.byref(ws), len(rows),
                              rows.ctypes.data_as(C.POINTER(C.c_int)), abi.dptr(A),
                              abi.dptr(b))
    if rc != 0:
        raise RuntimeError(f"oracle linsys rows status {rc}")
    return A, b


def particles_update(u, cen, dir_, mag, vel, stretch, rotu, free):
    """complete_wake's particle loop on copies; returns (cen, dir, stretch,
    free, n_freed)."""
    cen, dir_, stretch = (np.array(abi.f64(a), dtype=np.float64, order="C")
                          for a in (cen, dir_, stretch))
    mag, vel, rotu = abi.f64(mag), abi.f64(vel), abi.f64(rotu)
    free = np.array(free, dtype=np.int32, order="C")
    nf = C.c_int(0)
    rc = lib().or_particles_update(C.byref(u), mag.shape[0], abi.dptr(cen), abi.dptr(dir_),
                                   abi.dptr(mag), abi.dptr(vel), abi.dptr(stretch),
                                   abi.dptr(rotu), free.ctypes.data_as(C.POINTER(C.c_int)),
                                   C.byref(nf))
    if rc != 0:
        raise RuntimeError(f"oracle particles_update status {rc}")
    return cen, dir_, stretch, free, nf.value



def particles_update_pa(u, pa, body, cen, dir_, mag, rvort, vel, stretch, rotu, free):
    """complete_wake's particle loop with penetration avoidance against the
    panel set ``body`` (abi.PanelSet) on copies; returns (cen, dir, vel,
    stretch, free, n_freed)."""
    cen, dir_, vel, stretch = (np.array(abi.f64(a), dtype=np.float64, order="C")
                               for a in (cen, dir_, vel, stretch))
    mag, rvort, rotu = abi.f64(mag), abi.f64(rvort), abi.f64(rotu)
    free = np.array(free, dtype=np.int32, order="C")
    nf = C.c_int(0)
    bs = body.struct()
    rc = lib().or_particles_update_pa(C.byref(u), C.byref(pa), C.byref(bs), mag.shape[0],
                                      abi.dptr(cen), abi.dptr(dir_), abi.dptr(mag),
                                      abi.dptr(rvort), abi.dptr(vel), abi.dptr(stretch),
                                      abi.dptr(rotu), free.ctypes.data_as(C.POINTER(C.c_int)),
                                      C.byref(nf))
    if rc != 0:
        raise RuntimeError(f"oracle particles_update_pa status {rc}")
    return cen, dir_, vel, stretch, free, nf.value


def pressure_run(prm, rank, nstatic, elems_init, elems_step, bern, parts, vel, wake=None,
                 wake_vv=None, end_vort=None, end_vv=None):
    """The pressure integral equation of one step; returns (A_pres (n_sp,
    n_sp), b_pres, res_pres).  parts = (cen, dir, mag, r_vortex)."""
    cen, dir_, mag, rv = (abi.f64(a) for a in parts)
    vel = abi.f64(vel)
    wk = wake if wake is not None else abi.empty_panels()
    ev = end_vort if end_vort is not None else abi.empty_lines()
    ws, es = wk.struct(), ev.struct()
    ei, est = elems_init.struct(), elems_step.struct()
    nsp = int(np.sum(np.asarray(elems_step.kind) == abi.DUST_ELEM_SURFPAN))
    A = np.zeros(max(nsp, 1) ** 2)
    b = np.zeros(max(nsp, 1))
    res = np.zeros(max(nsp, 1))
    p = prm.struct()
    rc = lib().or_pressure_run(C.byref(p), int(rank), int(nstatic), C.byref(ei), C.byref(est),
                               abi.dptr(abi.f64(bern)), mag.shape[0], abi.dptr(cen),
                               abi.dptr(dir_), abi.dptr(mag), abi.dptr(rv), abi.dptr(vel),
                               C.byref(ws), abi.dptr(abi.f64(wake_vv)), C.byref(es),
                               abi.dptr(abi.f64(end_vv)), abi.dptr(A), abi.dptr(b),
                               abi.dptr(res))
    if rc != 0:
        raise RuntimeError(f"oracle pressure status {rc}")
    return A[:nsp * nsp].reshape(nsp, nsp).T.copy(), b[:nsp], res[:nsp]


def pressure_particles(pts, cen, dir_, mag, rvort, vel):
    """The particles' rotational term of the pressure equation at points."""
    pts = abi.f64(pts).reshape(-1, 3)
    cen, dir_, mag, rvort, vel = (abi.f64(a) for a in (cen, dir_, mag, rvort, vel))
    out = np.zeros(pts.shape[0])
    rc = lib().or_pressure_particles(pts.shape[0], abi.dptr(pts), mag.shape[0], abi.dptr(cen),
                                     abi.dptr(dir_), abi.dptr(mag), abi.dptr(rvort),
                                     abi.dptr(vel), abi.dptr(out))
    if rc != 0:
        raise RuntimeError(f"oracle pressure particles status {rc}")
    return out
