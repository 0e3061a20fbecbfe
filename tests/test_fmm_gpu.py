"""GPU parity of the FMM path (C-ABI) against the CPU oracle.

Tolerance: 1e-10 relative (L2 over all particles) for the FP64 path, the
bound the target states for induced velocities.  The oracle follows the
reference's loop orders, so the remaining difference is rounding order.
"""
import numpy as np
import pytest

import oracle as O
from dust_b200 import abi, octree, synth
from dust_b200.params import FmmParams

pytestmark = pytest.mark.gpu

TOL64 = 1e-10


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def ring(n, seed, core=0.02):
    nr = int(n * 10 / 11)
    cen, dir_, mag = synth.ring_particles(nr, n - nr, seed=seed)
    return cen, dir_, mag, np.full(n, core)


def prm_ring(**kw):
    base = dict(box_length=4.0, origin=(-2.0, -2.0, -2.0), n_octree_levels=5,
                min_octree_part=5, multipole_degree=4, rankine_rad=0.02)
    base.update(kw)
    return FmmParams(**base)


@pytest.mark.parametrize("p,levels,min_part", [(4, 5, 5), (2, 4, 1), (6, 5, 8), (0, 3, 3),
                                               (4, 6, 20)])
def test_fmm_matches_oracle(p, levels, min_part):
    cen, dir_, mag, rv = ring(3000, seed=p + levels)
    prm = prm_ring(multipole_degree=p, n_octree_levels=levels, min_octree_part=min_part)
    ov, os_, orr, cnt = O.fmm_apply(prm, cen, dir_, mag, rv)
    oc = octree.initialize_octree(prm)
    v, s, r = oc.apply_multipole(cen, dir_, mag, rv)
    st = oc.stats()
    assert st["n_leaves"] == cnt[0]
    assert st["n_active_cells"] == cnt[1]
    assert rel(v, ov) < TOL64
    assert rel(s, os_) < TOL64
    assert rel(r, orr) < TOL64


@pytest.mark.parametrize("flags", [(1, 1, 1, 0), (1, 0, 1, 0), (0, 0, 1, 0), (1, 1, 0, 0),
                                   (0, 0, 0, 0), (1, 1, 1, 1)])
def test_fmm_model_switches(flags):
    vs, df, vd, tv = flags
    cen, dir_, mag, rv = ring(2000, seed=3)
    rv = rv * (1.0 + 0.5 * np.random.default_rng(1).random(len(rv)))  # per-particle cores
    prm = prm_ring(vortstretch=vs, divergence_filtering=df, diffusion=vd,
                   turbulent_viscosity=tv, nu_inf=1e-3)
    ov, os_, orr, _ = O.fmm_apply(prm, cen, dir_, mag, rv)
    v, s, r = octree.initialize_octree(prm).apply_multipole(cen, dir_, mag, rv)
    assert rel(v, ov) < TOL64
    if vs or vd:
        assert rel(s, os_) < TOL64
    if vs and df:
        assert rel(r, orr) < TOL64


def test_fmm_multibox_and_wind():
    # n_box > 1: level-1 interaction lists span the whole level-1 grid
    rng = np.random.default_rng(7)
    n = 2500
    cen = rng.uniform(0.01, 2.99, (n, 3)) * np.array([1.0, 2.0 / 3.0, 1.0 / 3.0])
    dir_ = rng.standard_normal((n, 3))
    dir_ /= np.linalg.norm(dir_, axis=1)[:, None]
    mag = rng.uniform(0.5e-3, 1.5e-3, n)
    rv = np.full(n, 0.05)
    prm = FmmParams(box_length=1.0, n_box=(3, 2, 1), origin=(0, 0, 0), n_octree_levels=4,
                    min_octree_part=4, multipole_degree=4, rankine_rad=0.05,
                    u_inf=(1.0, 0.0, 0.1))
    ov, os_, orr, cnt = O.fmm_apply(prm, cen, dir_, mag, rv)
    v, s, r = octree.initialize_octree(prm).apply_multipole(cen, dir_, mag, rv)
    assert rel(v, ov) < TOL64
    assert rel(s, os_) < TOL64


def test_fmm_tree_flags_match():
    cen, dir_, mag, rv = ring(1500, seed=11)
    prm = prm_ring(n_octree_levels=5, min_octree_part=6)
    O.fmm_apply(prm, cen, dir_, mag, rv)
    fl = O.last_tree_flags(prm)
    oc = octree.initialize_octree(prm)
    oc.apply_multipole(cen, dir_, mag, rv)
    st = oc.stats()
    assert st["n_leaves"] == int(np.sum(fl & 1))
    assert st["n_active_cells"] == int(np.sum((fl & 4) > 0))


def test_fmm_with_elements():
    wing, te = synth.flat_wing(span=2.0, chord=0.5, n_span=8, n_chord=4, alpha_deg=5.0)
    rng = np.random.default_rng(5)
    wing.mag = rng.standard_normal(wing.n)
    wing.kind[::3] = abi.DUST_ELEM_SURFPAN
    wing.ub = rng.standard_normal((wing.n, 3)) * 0.1
    wing.uvort = rng.standard_normal((wing.n, 3)) * 0.1
    wake = wing.subset(te)
    wake.ver = wake.ver + np.array([0.6, 0.0, 0.0])
    wake.mag = rng.standard_normal(wake.n)
    wake.kind[:] = abi.DUST_ELEM_VORTLATT
    ev = abi.LineSet(np.array([[[1.1, -1.0, 0.0], [2.0, -1.0, 0.0]],
                               [[1.1, 1.0, 0.0], [2.0, 1.0, 0.0]]]), np.array([0.3, -0.3]))
    els = abi.elements_struct(wing, wake, ev)
    n = 1200
    cen = rng.uniform(-1.5, 1.5, (n, 3)) * np.array([1.0, 1.0, 0.3]) + np.array([1.5, 0, 0])
    dir_ = rng.standard_normal((n, 3))
    dir_ /= np.linalg.norm(dir_, axis=1)[:, None]
    mag = rng.uniform(1e-3, 2e-3, n)
    rv = np.full(n, 0.1)
    prm = FmmParams(box_length=4.0, origin=(-0.5, -2.0, -2.0), n_octree_levels=4,
                    min_octree_part=5, multipole_degree=4, rankine_rad=0.1,
                    u_inf=(1.0, 0.0, 0.05))
    ov, os_, orr, _ = O.fmm_apply(prm, cen, dir_, mag, rv, els)
    v, s, r = octree.initialize_octree(prm).apply_multipole(cen, dir_, mag, rv, els)
    assert rel(v, ov) < TOL64
    assert rel(s, os_) < TOL64
    # element velocity alone at arbitrary points
    pts = rng.uniform(-1, 2, (300, 3))
    ev_o = O.elements_vel(prm, pts, els)
    ev_g = octree.elements_vel(prm, pts, els)
    assert rel(ev_g, ev_o) < TOL64


def test_direct_and_uvort_match_oracle():
    cen, dir_, mag, rv = ring(1500, seed=2)
    prm = prm_ring()
    dv, ds, dr = O.direct_particles(prm, cen, dir_, mag, rv)
    gv, gs, gr = octree.direct_particles(prm, cen, dir_, mag, rv)
    assert rel(gv, dv) < TOL64 and rel(gs, ds) < TOL64 and rel(gr, dr) < TOL64
    pts = np.random.default_rng(0).uniform(-1.5, 1.5, (200, 3))
    ev = abi.LineSet(np.array([[[0.0, 0.0, 0.0], [0.5, 0.5, 0.0]]]), np.array([0.7]))
    uo = O.points_uvort(prm, pts, cen, dir_, mag, rv, ev)
    ug = octree.points_uvort(prm, pts, cen, dir_, mag, rv, ev)
    assert rel(ug, uo) < TOL64


def test_fmm_converges_to_direct_sum():
    cen, dir_, mag, rv = ring(6000, seed=9)
    dv, ds, _ = octree.direct_particles(prm_ring(), cen, dir_, mag, rv)
    errs = []
    for p in (2, 4, 6):
        v, s, _ = octree.initialize_octree(prm_ring(multipole_degree=p)).apply_multipole(
            cen, dir_, mag, rv)
        errs.append(rel(v, dv))
    assert errs[1] < errs[0] and errs[2] < errs[1]
    assert errs[2] < 3e-4


def test_edge_cases():
    prm = prm_ring()
    oc = octree.initialize_octree(prm)
    # empty
    v, s, r = oc.apply_multipole(np.zeros((0, 3)), np.zeros((0, 3)), np.zeros(0), np.zeros(0))
    assert v.shape == (0, 3)
    # single particle: no self-induction
    v, s, r = oc.apply_multipole(np.array([[0.1, 0.2, 0.3]]), np.array([[0, 0, 1.0]]),
                                 np.array([1e-3]), np.array([0.02]))
    assert np.all(v == 0.0) and np.all(r == 0.0)
    # a particle outside the box is an error, as in sort_particles
    with pytest.raises(Exception) as ei:
        oc.apply_multipole(np.array([[5.0, 0.0, 0.0]]), np.array([[0, 0, 1.0]]),
                           np.array([1e-3]), np.array([0.02]))
    assert "status 2" in str(ei.value)
    # the handle stays usable after the error
    cen, dir_, mag, rv = ring(500, seed=1)
    ov, _, _, _ = O.fmm_apply(prm, cen, dir_, mag, rv)
    v, _, _ = oc.apply_multipole(cen, dir_, mag, rv)
    assert rel(v, ov) < TOL64
    # all particles in one finest cell (ragged: one huge leaf)
    c = np.full((300, 3), 0.01) + np.random.default_rng(0).uniform(0, 1e-3, (300, 3))
    d = np.tile([0.0, 1.0, 0.0], (300, 1))
    m = np.full(300, 1e-3)
    ov, os_, _, _ = O.fmm_apply(prm, c, d, m, np.full(300, 0.02))
    v, s, _ = oc.apply_multipole(c, d, m, np.full(300, 0.02))
    assert rel(v, ov) < TOL64 and rel(s, os_) < TOL64


TOL32 = 1e-6  # FP32 arithmetic with compensated accumulation, vs the FP64 oracle


def _elements_case(rng):
    wing, te = synth.flat_wing(span=2.0, chord=0.5, n_span=8, n_chord=4, alpha_deg=5.0)
    wing.mag = rng.standard_normal(wing.n)
    wing.kind[::3] = abi.DUST_ELEM_SURFPAN
    wing.ub = rng.standard_normal((wing.n, 3)) * 0.1
    wing.uvort = rng.standard_normal((wing.n, 3)) * 0.1
    wake = wing.subset(te)
    wake.ver = wake.ver + np.array([0.6, 0.0, 0.0])
    wake.mag = rng.standard_normal(wake.n)
    wake.kind[:] = abi.DUST_ELEM_VORTLATT
    ev = abi.LineSet(np.array([[[1.1, -1.0, 0.0], [2.0, -1.0, 0.0]],
                               [[1.1, 1.0, 0.0], [2.0, 1.0, 0.0]]]), np.array([0.3, -0.3]))
    return abi.elements_struct(wing, wake, ev)


@pytest.mark.parametrize("prec", [abi.DUST_PREC_FP64, abi.DUST_PREC_FP32C])
def test_elements_far_field_path(prec):
    """Particles far from small panels take the far-field fast path; the
    result must equal the reference's tangent-frame formulas."""
    rng = np.random.default_rng(8)
    els = _elements_case(rng)
    n = 3000
    cen = rng.uniform(-8.0, 8.0, (n, 3))
    dir_ = rng.standard_normal((n, 3))
    dir_ /= np.linalg.norm(dir_, axis=1)[:, None]
    mag = rng.uniform(1e-4, 2e-4, n)
    rv = np.full(n, 0.1)
    prm = FmmParams(box_length=16.0, origin=(-8.0, -8.0, -8.0), n_octree_levels=4,
                    min_octree_part=5, multipole_degree=4, rankine_rad=0.1,
                    u_inf=(0.0, 0.0, 0.0), precision=prec)
    ov, _, _, _ = O.fmm_apply(prm, cen, dir_, mag, rv, els)
    v, _, _ = octree.initialize_octree(prm).apply_multipole(cen, dir_, mag, rv, els)
    tol = TOL64 if prec == abi.DUST_PREC_FP64 else TOL32
    assert rel(v, ov) < tol


def test_fp32c_uvort_and_elements():
    rng = np.random.default_rng(5)
    els = _elements_case(rng)
    cen, dir_, mag, rv = ring(4000, seed=4)
    prm = prm_ring(precision=abi.DUST_PREC_FP32C, rankine_rad=0.1, u_inf=(1.0, 0.0, 0.0))
    ov, _, _, _ = O.fmm_apply(prm, cen, dir_, mag, rv, els)
    v, _, _ = octree.initialize_octree(prm).apply_multipole(cen, dir_, mag, rv, els)
    assert rel(v, ov) < TOL32
    pts = rng.uniform(-1.5, 1.5, (500, 3))
    ev = abi.LineSet(np.array([[[0.0, 0.0, 0.0], [0.5, 0.5, 0.0]]]), np.array([0.7]))
    uo = O.points_uvort(prm, pts, cen, dir_, mag, rv, ev)
    ug = octree.points_uvort(prm, pts, cen, dir_, mag, rv, ev)
    assert rel(ug, uo) < TOL32


@pytest.mark.parametrize("p", [2, 4, 6])
def test_fmm_fp32c_matches_oracle(p):
    cen, dir_, mag, rv = ring(4000, seed=12)
    prm = prm_ring(multipole_degree=p, n_octree_levels=5, min_octree_part=5,
                   precision=abi.DUST_PREC_FP32C)
    ov, os_, orr, _ = O.fmm_apply(prm, cen, dir_, mag, rv)
    v, s, r = octree.initialize_octree(prm).apply_multipole(cen, dir_, mag, rv)
    assert rel(v, ov) < TOL32 and rel(s, os_) < TOL32 and rel(r, orr) < TOL32


def test_fmm_degree8_matches_oracle():
    cen, dir_, mag, rv = ring(2500, seed=13)
    prm = prm_ring(multipole_degree=8, n_octree_levels=5, min_octree_part=5)
    ov, os_, orr, _ = O.fmm_apply(prm, cen, dir_, mag, rv)
    v, s, r = octree.initialize_octree(prm).apply_multipole(cen, dir_, mag, rv)
    assert rel(v, ov) < TOL64 and rel(s, os_) < TOL64 and rel(r, orr) < TOL64


@pytest.mark.parametrize("prec", [abi.DUST_PREC_FP64, abi.DUST_PREC_FP32C])
def test_fmm_points_uvort_matches_oracle(prec):
    """apply_multipole_panels: the panels' uvort through the particles' FMM
    (leaf local expansion + near-field particles) plus the end vortices,
    against the oracle's restatement; the split evaluation (prepare, points,
    finish) gives the particles the outputs of dust_fmm_apply."""
    cen, dir_, mag, rv = ring(4000, seed=14)
    pts = np.random.default_rng(3).uniform(-1.6, 1.6, (500, 3))
    ev = abi.LineSet(np.array([[[0.0, 0.0, 0.0], [0.5, 0.5, 0.0]]]), np.array([0.7]))
    prm = prm_ring(precision=prec)
    ref = O.fmm_points_uvort(prm.replace(precision=abi.DUST_PREC_FP64), pts, cen, dir_, mag,
                             rv, ev)
    oc = octree.initialize_octree(prm)
    oc.prepare(cen, dir_, mag, rv, pts)
    u = oc.points_uvort(ev)
    tol = TOL64 if prec == abi.DUST_PREC_FP64 else TOL32
    assert rel(u, ref) < tol
    v1, s1, r1 = oc.finish()
    v0, s0, r0 = octree.initialize_octree(prm).apply_multipole(cen, dir_, mag, rv)
    # the same sums; the extra targets (empty leaves holding points) change
    # only the M2L batching, so the rounding (FP64) or the FP32 partial sums
    # of the tensor-core M2L (FP32C) may differ
    tsplit = 1e-13 if prec == abi.DUST_PREC_FP64 else TOL32
    assert rel(v1, v0) < tsplit and rel(s1, s0) < tsplit and rel(r1, r0) < tsplit
    # the FMM result approximates the direct sum to the FMM's accuracy
    direct = O.points_uvort(prm, pts, cen, dir_, mag, rv, ev)
    assert rel(u, direct) < 5e-3


def test_fmm_points_uvort_errors():
    prm = prm_ring()
    oc = octree.initialize_octree(prm)
    with pytest.raises(Exception) as ei:
        oc.points_uvort()
    assert "status 6" in str(ei.value)  # no prepared tree
    cen, dir_, mag, rv = ring(500, seed=1)
    with pytest.raises(Exception) as ei:
        oc.prepare(cen, dir_, mag, rv, np.array([[5.0, 0.0, 0.0]]))
    assert "status 2" in str(ei.value)  # a point outside the octree box
    with pytest.raises(Exception) as ei:
        oc.points_uvort()
    assert "status 6" in str(ei.value)  # the failed prepare left no tree
    oc.prepare(cen, dir_, mag, rv, np.array([[0.1, 0.2, 0.3]]))  # the handle stays usable
    u = oc.points_uvort()
    assert u.shape == (1, 3) and np.all(np.isfinite(u))
