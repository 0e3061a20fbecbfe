"""dust_points_uvort_device_noalloc against dust_points_uvort_device.

The no-alloc entry point runs the same kernels in the same order from a
fixed scratch array inside the library, so its result must agree with the
allocating entry point to rounding (1e-12 relative, L2), in the FP64 and the
FP32C modes, on two calls in a row through the same scratch.  Sizes above
the scratch limit are refused with DUST_ERR_CAPACITY before any launch.

The file name keeps it last in collection order: it must pass after every
other test of the session as well as alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from dust_b200 import abi, synth
from dust_b200._lib import lib
from dust_b200.params import FmmParams

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _p(t, ctype=C.c_double):
    return C.cast(C.c_void_p(t.data_ptr()), C.POINTER(ctype))


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _case(n, n_pts, seed):
    nr = int(n * 10 / 11)
    cen, dir_, mag = synth.ring_particles(nr, n - nr, seed=seed)
    rng = np.random.default_rng(seed)
    pts = rng.uniform(-1.5, 1.5, (n_pts, 3))
    lver = np.array([[[0.0, 0.0, 0.0], [0.5, 0.5, 0.0]], [[0.2, -0.4, 0.1], [0.9, 0.3, -0.2]]])
    lmag = np.array([0.7, -0.3])
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()
    return dict(pts=dev(pts), cen=dev(cen), dir=dev(dir_), mag=dev(mag),
                rv=dev(np.full(n, 0.02)), lver=dev(lver), lmag=dev(lmag), n=n, n_pts=n_pts)


def _call(fn, prm, c, out, stream):
    lines = abi.Lines(2, _p(c["lver"]), _p(c["lmag"]))
    ps = prm.struct()
    return fn(C.byref(ps), c["n_pts"], _p(c["pts"]), c["n"], _p(c["cen"]), _p(c["dir"]),
              _p(c["mag"]), _p(c["rv"]), C.byref(lines), _p(out), C.c_void_p(stream))


@pytest.mark.parametrize("precision", [abi.DUST_PREC_FP64, abi.DUST_PREC_FP32C])
def test_noalloc_matches_allocating_entry(precision):
    prm = FmmParams(box_length=4.0, origin=(-2.0, -2.0, -2.0), n_octree_levels=5,
                    min_octree_part=5, multipole_degree=4, rankine_rad=0.02,
                    precision=precision)
    c = _case(20000, 700, seed=21)
    stream = torch.cuda.current_stream().cuda_stream
    ref = torch.empty(c["n_pts"] * 3, dtype=torch.float64, device="cuda")
    assert _call(lib().dust_points_uvort_device, prm, c, ref, stream) == abi.DUST_OK
    out = torch.full((c["n_pts"] * 3,), np.nan, dtype=torch.float64, device="cuda")
    for _ in range(2):
        out.fill_(np.nan)
        st = _call(lib().dust_points_uvort_device_noalloc, prm, c, out, stream)
        assert st == abi.DUST_OK, lib().dust_last_error().decode()
        torch.cuda.synchronize()
        assert rel(out.cpu().numpy(), ref.cpu().numpy()) < TOL


def test_noalloc_refuses_oversize():
    prm = FmmParams(box_length=4.0, origin=(-2.0, -2.0, -2.0), n_octree_levels=5,
                    min_octree_part=5, multipole_degree=4, rankine_rad=0.02,
                    precision=abi.DUST_PREC_FP32C)
    n = (4 << 20) // 56 + 1000  # more particles than the scratch holds in FP32C
    c = _case(n, 16, seed=3)
    out = torch.zeros(c["n_pts"] * 3, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    st = _call(lib().dust_points_uvort_device_noalloc, prm, c, out, stream)
    assert st == abi.DUST_ERR_CAPACITY
    assert "no-alloc scratch" in lib().dust_last_error().decode()
    # the same size in FP64 needs scratch only for the two end vortices
    prm64 = prm.replace(precision=abi.DUST_PREC_FP64)
    ref = torch.empty_like(out)
    assert _call(lib().dust_points_uvort_device, prm64, c, ref, stream) == abi.DUST_OK
    assert _call(lib().dust_points_uvort_device_noalloc, prm64, c, out, stream) == abi.DUST_OK
    torch.cuda.synchronize()
    assert rel(out.cpu().numpy(), ref.cpu().numpy()) < TOL


def test_noalloc_allocates_no_device_memory():
    """After one warm-up call, a call at a new, larger size that still fits
    the scratch leaves the device's free memory exactly as it was."""
    prm = FmmParams(box_length=4.0, origin=(-2.0, -2.0, -2.0), n_octree_levels=5,
                    min_octree_part=5, multipole_degree=4, rankine_rad=0.02,
                    precision=abi.DUST_PREC_FP32C)
    stream = torch.cuda.current_stream().cuda_stream
    small = _case(5000, 100, seed=5)
    big = _case(60000, 300, seed=6)  # about 3.4 MB of the 4 MiB scratch in FP32C
    out_s = torch.empty(small["n_pts"] * 3, dtype=torch.float64, device="cuda")
    out_b = torch.empty(big["n_pts"] * 3, dtype=torch.float64, device="cuda")
    assert _call(lib().dust_points_uvort_device_noalloc, prm, small, out_s, stream) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    st = _call(lib().dust_points_uvort_device_noalloc, prm, big, out_b, stream)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert st == abi.DUST_OK, lib().dust_last_error().decode()
    assert free1 == free0


def test_noalloc_rejects_null_arrays():
    prm = FmmParams(box_length=4.0, origin=(-2.0, -2.0, -2.0), rankine_rad=0.02)
    c = _case(1000, 10, seed=7)
    out = torch.empty(c["n_pts"] * 3, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    null = C.POINTER(C.c_double)()
    lines = abi.Lines(2, _p(c["lver"]), _p(c["lmag"]))
    bad_lines = abi.Lines(2, null, _p(c["lmag"]))
    ps = prm.struct()
    for fn in (lib().dust_points_uvort_device_noalloc, lib().dust_points_uvort_device):
        # particles missing
        assert fn(C.byref(ps), c["n_pts"], _p(c["pts"]), c["n"], null, _p(c["dir"]),
                  _p(c["mag"]), _p(c["rv"]), C.byref(lines), _p(out),
                  C.c_void_p(stream)) == abi.DUST_ERR_BAD_ARG
        # output missing
        assert fn(C.byref(ps), c["n_pts"], _p(c["pts"]), c["n"], _p(c["cen"]), _p(c["dir"]),
                  _p(c["mag"]), _p(c["rv"]), C.byref(lines), null,
                  C.c_void_p(stream)) == abi.DUST_ERR_BAD_ARG
        # end-vortex vertices missing
        assert fn(C.byref(ps), c["n_pts"], _p(c["pts"]), c["n"], _p(c["cen"]), _p(c["dir"]),
                  _p(c["mag"]), _p(c["rv"]), C.byref(bad_lines), _p(out),
                  C.c_void_p(stream)) == abi.DUST_ERR_BAD_ARG
