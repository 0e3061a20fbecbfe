"""Parity pinned to the reference's own output.

tests/golden/ref_sym_static_{v,p}.npz come from the reference's regression
fixtures tests/sym_test/static/{v,p}/Output/ref_res_0011.h5 (generated by
tests/golden/make_reference_fixtures.py, which rebuilds the body geometry
from the case's parametric input and checks it against the saved wake start
points).  Each holds the wake that the reference's step-11 linear system was
assembled against (panel wake, end vortices, 360 particles) and that
system's solution, Components/Comp001/Solution/Vort.  Re-solving the step
from that state must give the reference's doublet intensities:

* v: 200 vortex-lattice panels -- uvort by the particles and end vortices
  at the panel centres (get_vort_vel_vortlatt, mod_vortlatt.f90:676-693),
  Neumann rows with the implicit first wake row and the explicit second row
  (build_row_static_vortlatt / add_wake_vortlatt, mod_vortlatt.f90:201-322);
* p: 400 surface panels (source + doublet) -- get_vort_vel_surfpan
  (mod_surfpan.f90:962-977), Dirichlet rows with the source terms and the
  two-sided implicit trailing-edge row (build_row_static_surfpan /
  add_wake_surfpan, mod_surfpan.f90:448-535).

Tolerance: 1e-8 relative L2, the reference's own regression tolerance
(.gitlab-ci.yml:54); the oracle and the GPU reach about 1e-12.
"""
import os

import numpy as np
import pytest

import oracle as O
from dust_b200 import abi
from dust_b200.params import FmmParams

HERE = os.path.dirname(os.path.abspath(__file__))
TOL_REF = 1e-8


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def load(name="sym_static_v"):
    d = np.load(os.path.join(HERE, "golden", "ref_%s.npz" % name))
    ver = d["ver"]
    n = len(ver)
    prm = FmmParams(u_inf=tuple(d["u_inf"]), rankine_rad=float(d["rankine_rad"]),
                    cutoff_rad=float(d["cutoff_rad"]),
                    far_field_ratio_doublet=float(d["far_field_ratio_doublet"]))
    kind = abi.DUST_ELEM_VORTLATT if str(d["eltype"]) == "v" else abi.DUST_ELEM_SURFPAN
    body = abi.PanelSet(ver, n_ver=d["nver"], kind=np.full(n, kind))
    alpha = d["part_alpha"]
    mag = np.linalg.norm(alpha, axis=1)
    dir_ = alpha / np.where(mag > 0, mag, 1.0)[:, None]
    parts = (np.ascontiguousarray(d["part_cen"]), np.ascontiguousarray(dir_), mag,
             np.ascontiguousarray(d["part_rv"]))
    ev = abi.LineSet(d["end_ver"], d["end_mag"])
    wake = abi.PanelSet(d["wake_ver"], kind=np.full(len(d["wake_ver"]), abi.DUST_ELEM_VORTLATT),
                        mag=d["wake_mag"])
    impl = np.ascontiguousarray(d["impl_ind"])
    return prm, body, parts, ev, wake, impl, d["vort_ref"]


CASES = [("sym_static_v", 200), ("sym_static_p", 400)]


@pytest.mark.parametrize("name,n", CASES)
def test_fixture_is_consistent(name, n):
    d = np.load(os.path.join(HERE, "golden", "ref_%s.npz" % name))
    assert d["te_match"] < 1e-12
    assert len(d["ver"]) == len(d["vort_ref"]) == n
    assert len(d["impl_ind"]) == 40 and len(d["part_cen"]) == 360


@pytest.mark.parametrize("name,n", CASES)
def test_oracle_reproduces_reference_solution(name, n):
    prm, body, (cen, dir_, mag, rv), ev, wake, impl, ref = load(name)
    n = body.n
    centres = body.ver.mean(axis=1)
    body.uvort = O.points_uvort(prm, centres, cen, dir_, mag, rv, ev)
    w = (wake, len(impl), impl)
    _, _, res = O.linsys_run(prm, n, n, body, body, w, w)
    assert rel(res, ref) < TOL_REF
    # the particles matter: without their induced velocity the result is off
    body.uvort = np.zeros((n, 3))
    _, _, res0 = O.linsys_run(prm, n, n, body, body, w, w)
    assert rel(res0, ref) > 1e-2


@pytest.mark.gpu
@pytest.mark.parametrize("name,n", CASES)
@pytest.mark.parametrize("mode", [abi.DUST_SOLVE_LU64, abi.DUST_SOLVE_MIXED])
def test_gpu_reproduces_reference_solution(name, n, mode):
    from dust_b200 import linsys, octree
    prm, body, (cen, dir_, mag, rv), ev, wake, impl, ref = load(name)
    n = body.n
    cg, _, _ = octree.panels_geometry(body)
    body.uvort = octree.points_uvort(prm, cg, cen, dir_, mag, rv, ev)
    ls = linsys.initialize_linsys(prm, n, n, body, wake, len(impl), impl)
    ls.assemble_linsys(body, wake, len(impl), impl)
    res, rep = ls.solve_linsys(mode)
    assert rep["fell_back"] == 0
    assert rel(res, ref) < TOL_REF


def test_fixtures_regenerate_identically(tmp_path):
    """Where the reference tree is mounted, regenerating the fixtures from
    its HDF5 files gives the committed arrays bit for bit."""
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_reference_fixtures as M
    if not os.path.isdir(os.path.join(M.DEFAULT_ROOT, "tests", "sym_test")):
        pytest.skip("reference tree not mounted")
    M.main(M.DEFAULT_ROOT, str(tmp_path))
    for name, _ in CASES:
        a = np.load(os.path.join(HERE, "golden", "ref_%s.npz" % name))
        b = np.load(os.path.join(str(tmp_path), "ref_%s.npz" % name))
        for k in a.files:
            assert np.array_equal(a[k], b[k]), (name, k)
