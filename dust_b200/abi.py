"""ctypes mirror of the structs in include/dust_b200.h.

The layouts here must match the header field by field; tests check the
sizes against the compiled library (``dust_abi_sizes``).
"""
import ctypes as C

import numpy as np

DUST_OK = 0
DUST_ERR_CUDA = 1
DUST_ERR_OUT_OF_BOX = 2
DUST_ERR_SINGULAR = 3
DUST_ERR_NOT_CONVERGED = 4
DUST_ERR_TIMEOUT = 5
DUST_ERR_BAD_ARG = 6
DUST_ERR_NO_DEVICE = 7
DUST_ERR_CAPACITY = 8

DUST_ELEM_SURFPAN = 1
DUST_ELEM_VORTLATT = 2

DUST_PREC_FP64 = 0
DUST_PREC_FP32C = 1

DUST_SOLVE_LU64 = 0
DUST_SOLVE_MIXED = 1
DUST_SOLVE_GMRES_NN = 2

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class FmmParams(C.Structure):
    _fields_ = [
        ("box_length", C.c_double),
        ("n_box", C.c_int * 3),
        ("origin", C.c_double * 3),
        ("n_octree_levels", C.c_int),
        ("min_octree_part", C.c_int),
        ("multipole_degree", C.c_int),
        ("rankine_rad", C.c_double),
        ("cutoff_rad", C.c_double),
        ("far_field_ratio_doublet", C.c_double),
        ("vortstretch", C.c_int),
        ("divergence_filtering", C.c_int),
        ("diffusion", C.c_int),
        ("turbulent_viscosity", C.c_int),
        ("nu_inf", C.c_double),
        ("u_inf", C.c_double * 3),
        ("precision", C.c_int),
    ]


class UpdateParams(C.Structure):
    """dust_update_params: the particles' Euler step of complete_wake."""
    _fields_ = [
        ("dt", C.c_double),
        ("ndt_update_wake", C.c_int),
        ("box_min", C.c_double * 3),
        ("box_max", C.c_double * 3),
        ("vortstretch", C.c_int),
        ("diffusion", C.c_int),
        ("divergence_filtering", C.c_int),
        ("filt_eta", C.c_double),
    ]


def update_params(dt, box_min, box_max, ndt_update_wake=1, vortstretch=True, diffusion=True,
                  divergence_filtering=False, filt_eta=0.0):
    u = UpdateParams()
    u.dt = float(dt)
    u.ndt_update_wake = int(ndt_update_wake)
    for d in range(3):
        u.box_min[d] = float(box_min[d])
        u.box_max[d] = float(box_max[d])
    u.vortstretch = int(bool(vortstretch))
    u.diffusion = int(bool(diffusion))
    u.divergence_filtering = int(bool(divergence_filtering))
    u.filt_eta = float(filt_eta)
    return u


class PaParams(C.Structure):
    """dust_pa_params: penetration avoidance (avoid_collision)."""
    _fields_ = [("check_radius", C.c_double), ("element_radius", C.c_double),
                ("u_ref", C.c_double)]


def pa_params(u_ref, check_radius=5.0, element_radius=1.5):
    return PaParams(float(check_radius), float(element_radius), float(u_ref))


class WakeParams(C.Structure):
    """dust_wake_params: the panel wake and its shedding."""
    _fields_ = [
        ("n_stripes", C.c_int),
        ("n_points", C.c_int),
        ("n_wake_panels", C.c_int),
        ("dt", C.c_double),
        ("ndt_update_wake", C.c_int),
        ("min_vel_at_te", C.c_double),
        ("box_min", C.c_double * 3),
        ("box_max", C.c_double * 3),
        ("vortex_rad", C.c_double),
        ("k_vortex_rad", C.c_double),
        ("refine_wake", C.c_int),
        ("k_refine", C.c_int),
        ("u_inf", C.c_double * 3),
    ]


def wake_params(n_stripes, n_points, n_wake_panels, dt, box_min, box_max, u_inf,
                vortex_rad=0.1, k_vortex_rad=1.0, min_vel_at_te=1e-8, ndt_update_wake=1,
                refine_wake=False, k_refine=1):
    w = WakeParams()
    w.n_stripes, w.n_points, w.n_wake_panels = int(n_stripes), int(n_points), int(n_wake_panels)
    w.dt, w.ndt_update_wake, w.min_vel_at_te = float(dt), int(ndt_update_wake), float(min_vel_at_te)
    for d in range(3):
        w.box_min[d], w.box_max[d], w.u_inf[d] = float(box_min[d]), float(box_max[d]), float(u_inf[d])
    w.vortex_rad, w.k_vortex_rad = float(vortex_rad), float(k_vortex_rad)
    w.refine_wake, w.k_refine = int(bool(refine_wake)), int(k_refine)
    return w


class Te(C.Structure):
    """dust_te: trailing-edge topology (1-based, 2 ints per stripe)."""
    _fields_ = [("ii", C.POINTER(C.c_int)), ("neigh", C.POINTER(C.c_int)),
                ("neigh_o", C.POINTER(C.c_int)), ("gen_elems", C.POINTER(C.c_int))]


class Panels(C.Structure):
    _fields_ = [
        ("n", C.c_int),
        ("n_ver", _ip),
        ("kind", _ip),
        ("ver", _dp),
        ("mag", _dp),
        ("ub", _dp),
        ("uvort", _dp),
    ]


class Lines(C.Structure):
    _fields_ = [("n", C.c_int), ("ver", _dp), ("mag", _dp)]


class Elements(C.Structure):
    _fields_ = [("body", Panels), ("wake", Panels), ("end_vort", Lines)]


class FmmStats(C.Structure):
    _fields_ = [
        ("n_particles", C.c_int64),
        ("n_leaves", C.c_int64),
        ("n_active_cells", C.c_int64),
        ("n_m2l_pairs", C.c_int64),
        ("n_p2p_pairs", C.c_int64),
        ("n_elem_pairs", C.c_int64),
        ("n_levels", C.c_int),
        ("ms_tree", C.c_float),
        ("ms_upward", C.c_float),
        ("ms_m2l", C.c_float),
        ("ms_p2p", C.c_float),
        ("ms_elems", C.c_float),
        ("ms_total", C.c_float),
        ("ms_m2l_kernel", C.c_float),
        ("ms_elem_far", C.c_float),
    ]


class SolveReport(C.Structure):
    _fields_ = [
        ("mode_used", C.c_int),
        ("iterations", C.c_int),
        ("fell_back", C.c_int),
        ("residual", C.c_double),
        ("ms_factor", C.c_float),
        ("ms_solve", C.c_float),
        ("pivoted", C.c_int),
    ]


class WakeRows(C.Structure):
    _fields_ = [("pan", Panels), ("n_impl", C.c_int), ("impl_ind", _ip)]


# ------------------------------------------------------------------ helpers
def dptr(a):
    """double* of a C-contiguous float64 numpy array (None -> NULL)."""
    if a is None:
        return _dp()
    assert a.dtype == np.float64 and a.flags.c_contiguous, "need contiguous float64"
    return a.ctypes.data_as(_dp)


def iptr(a):
    if a is None:
        return _ip()
    assert a.dtype == np.int32 and a.flags.c_contiguous, "need contiguous int32"
    return a.ctypes.data_as(_ip)


def f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def i32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.int32)


class PanelSet:
    """Host-side panel set (vertices ver[n,4,3], n_ver, kind, mag, ub, uvort)
    that can hand out a ``Panels`` struct whose pointers stay valid as long as
    this object lives."""

    def __init__(self, ver, n_ver=None, kind=None, mag=None, ub=None, uvort=None):
        ver = f64(ver).reshape(-1, 4, 3)
        n = ver.shape[0]
        self.ver = ver
        self.n_ver = i32(n_ver if n_ver is not None else np.full(n, 4))
        self.kind = i32(kind if kind is not None else np.full(n, DUST_ELEM_VORTLATT))
        self.mag = f64(mag)
        self.ub = None if ub is None else f64(ub).reshape(n, 3)
        self.uvort = None if uvort is None else f64(uvort).reshape(n, 3)

    @property
    def n(self):
        return self.ver.shape[0]

    def struct(self):
        return Panels(self.n, iptr(self.n_ver), iptr(self.kind), dptr(self.ver),
                      dptr(self.mag), dptr(self.ub), dptr(self.uvort))

    def subset(self, idx):
        idx = np.asarray(idx)
        g = lambda a: None if a is None else a[idx]
        return PanelSet(self.ver[idx], self.n_ver[idx], self.kind[idx], g(self.mag),
                        g(self.ub), g(self.uvort))


class LineSet:
    def __init__(self, ver, mag=None):
        self.ver = f64(ver).reshape(-1, 2, 3)
        self.mag = f64(mag if mag is not None else np.zeros(self.ver.shape[0]))

    @property
    def n(self):
        return self.ver.shape[0]

    def struct(self):
        return Lines(self.n, dptr(self.ver), dptr(self.mag))


def empty_panels():
    return PanelSet(np.zeros((0, 4, 3)))


def empty_lines():
    return LineSet(np.zeros((0, 2, 3)))


def elements_struct(body=None, wake=None, end_vort=None):
    body = body if body is not None else empty_panels()
    wake = wake if wake is not None else empty_panels()
    end_vort = end_vort if end_vort is not None else empty_lines()
    return Elements(body.struct(), wake.struct(), end_vort.struct()), (body, wake, end_vort)


def wake_rows_struct(pan, n_impl, impl_ind):
    impl = i32(np.asarray(impl_ind).reshape(-1)) if n_impl else i32(np.zeros(2))
    return WakeRows(pan.struct(), int(n_impl), iptr(impl)), (pan, impl)
