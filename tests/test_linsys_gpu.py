"""GPU parity of AIC assembly and the LU solves against the CPU oracle.

Tolerances: assembled coefficients and solved doublet strengths 1e-10
relative (L2) for the FP64 path; the mixed path is refined to a normwise
backward error of 1e-12 and must then agree with FP64 to 1e-9.
"""
import numpy as np
import pytest

import oracle as O
from dust_b200 import abi, linsys, synth
from dust_b200.params import FmmParams

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def wing_case(n_span=12, n_chord=5):
    wing, te = synth.flat_wing(span=4.0, chord=1.0, n_span=n_span, n_chord=n_chord,
                               alpha_deg=5.0)
    wake, ind = synth.te_wake(wing, te, (0.3, 0.0, 0.02))
    far, _ = synth.te_wake(wing, te, (1.0, 0.0, 0.05))
    far.ver = far.ver + np.array([0.3, 0.0, 0.02])
    far.mag = np.linspace(-0.1, 0.1, far.n)
    return wing, synth.concat_panels(wake, far), wake.n, ind


def body_rotor_case():
    """Static surface-panel fuselage + moving vortex-lattice rotor."""
    body = synth.cylinder(n_target=300, length=2.0, radius=0.25)
    rot, te = synth.rotor_blades(n_blades=2, radius=0.8, root=0.2, chord=0.1, n_span=8,
                                 n_chord=3, center=(0, 0, 0.5))
    els = synth.concat_panels(body, rot)
    rng = np.random.default_rng(3)
    els.uvort = rng.standard_normal((els.n, 3)) * 0.05
    ub = np.zeros((els.n, 3))
    cen = rot.ver.mean(axis=1)
    ub[body.n:] = np.cross([0, 0, 20.0], cen)  # rotor body velocity
    els.ub = ub
    wake, ind = synth.te_wake(rot, te, (0.0, 0.0, -0.05))
    ind[:, 0] += body.n
    return els, body.n, wake, wake.n, ind


@pytest.mark.parametrize("nst_frac", [1.0, 0.5, 0.0])
def test_linsys_wing_matches_oracle(nst_frac):
    prm = FmmParams(u_inf=(1.0, 0.0, 0.0), rankine_rad=0.1)
    wing, wk, n_impl, ind = wing_case()
    rng = np.random.default_rng(1)
    wing.uvort = rng.standard_normal((wing.n, 3)) * 0.05
    n = wing.n
    nst = int(n * nst_frac)
    Ao, bo, ro = O.linsys_run(prm, n, nst, wing, wing, (wk, n_impl, ind), (wk, n_impl, ind))
    ls = linsys.initialize_linsys(prm, n, nst, wing, wk, n_impl, ind)
    ls.assemble_linsys(wing, wk, n_impl, ind)
    Ag, bg = ls.get_system()
    assert rel(Ag, Ao) < 1e-10
    assert rel(bg, bo) < 1e-10
    res, rep = ls.solve_linsys(abi.DUST_SOLVE_LU64)
    assert rel(res, ro) < 1e-10


def test_linsys_body_rotor_matches_oracle():
    prm = FmmParams(u_inf=(0.5, 0.0, -0.2), rankine_rad=0.1)
    els, nst, wake, n_impl, ind = body_rotor_case()
    n = els.n
    Ao, bo, ro = O.linsys_run(prm, n, nst, els, els, (wake, n_impl, ind), (wake, n_impl, ind))
    ls = linsys.initialize_linsys(prm, n, nst, els, wake, n_impl, ind)
    ls.assemble_linsys(els, wake, n_impl, ind)
    Ag, bg = ls.get_system()
    assert rel(Ag, Ao) < 1e-10
    assert rel(bg, bo) < 1e-10
    res, _ = ls.solve_linsys(abi.DUST_SOLVE_LU64)
    assert rel(res, ro) < 1e-10
    # a second step on the same handle (moving rows rebuilt, static LU reused)
    els.uvort = els.uvort * 0.5
    Ao2, bo2, ro2 = O.linsys_run(prm, n, nst, els, els, (wake, n_impl, ind),
                                 (wake, n_impl, ind))
    ls.assemble_linsys(els, wake, n_impl, ind)
    res2, _ = ls.solve_linsys(abi.DUST_SOLVE_LU64)
    assert rel(res2, ro2) < 1e-10
    # mixed precision on the same system
    ls.assemble_linsys(els, wake, n_impl, ind)
    res3, rep3 = ls.solve_linsys(abi.DUST_SOLVE_MIXED)
    assert rep3["mode_used"] == abi.DUST_SOLVE_MIXED and rep3["fell_back"] == 0
    assert rep3["residual"] <= 1e-14
    assert rel(res3, ro2) < 1e-9
    # mixed twice in a row, then plain again: the handle's LU stays usable
    ls.assemble_linsys(els, wake, n_impl, ind)
    res4, rep4 = ls.solve_linsys(abi.DUST_SOLVE_MIXED)
    assert rep4["fell_back"] == 0 and rel(res4, ro2) < 1e-9
    ls.assemble_linsys(els, wake, n_impl, ind)
    res5, _ = ls.solve_linsys(abi.DUST_SOLVE_LU64)
    assert rel(res5, ro2) < 1e-10


@pytest.mark.parametrize("nst_frac", [1.0, 0.7, 0.0])
def test_linsys_mixed_schur_matches_oracle(nst_frac):
    prm = FmmParams(u_inf=(1.0, 0.0, 0.0), rankine_rad=0.1)
    wing, wk, n_impl, ind = wing_case(n_span=20, n_chord=8)
    rng = np.random.default_rng(5)
    wing.uvort = rng.standard_normal((wing.n, 3)) * 0.05
    n = wing.n
    nst = int(n * nst_frac)
    _, _, ro = O.linsys_run(prm, n, nst, wing, wing, (wk, n_impl, ind), (wk, n_impl, ind))
    ls = linsys.initialize_linsys(prm, n, nst, wing, wk, n_impl, ind)
    for _ in range(2):
        ls.assemble_linsys(wing, wk, n_impl, ind)
        res, rep = ls.solve_linsys(abi.DUST_SOLVE_MIXED)
        assert rep["mode_used"] == abi.DUST_SOLVE_MIXED and rep["fell_back"] == 0
        assert rep["residual"] <= 1e-14
        assert rel(res, ro) < 1e-10


@pytest.mark.parametrize("n,nrhs", [(1, 1), (63, 1), (64, 3), (200, 2), (1000, 4)])
def test_dense_lu64_matches_numpy(n, nrhs):
    rng = np.random.default_rng(n)
    A = rng.standard_normal((n, n)) + n ** 0.5 * np.eye(n)
    B = rng.standard_normal((n, nrhs))
    X, rep = linsys.dense_solve(A, B, abi.DUST_SOLVE_LU64)
    assert rel(X, np.linalg.solve(A, B)) < 1e-10


@pytest.mark.parametrize("n", [300, 2500, 4000, 7000])
def test_dense_lu64_pivoting(n):
    """Random matrices without a dominant diagonal: every column pivots.
    Panels of up to 2048 rows run on one CTA (n = 300 and the last panels
    of the others), taller FP64 ones on a cluster of 8 CTAs (2500) or 16
    (4000), and on the grid-wide kernel when they do not fit a cluster's
    shared memory (7000)."""
    rng = np.random.default_rng(n + 1)
    A = rng.standard_normal((n, n))
    B = rng.standard_normal((n, 2))
    X, rep = linsys.dense_solve(A, B, abi.DUST_SOLVE_LU64)
    assert rep["pivoted"] == 1
    assert rel(X, np.linalg.solve(A, B)) < 1e-9


def _col_dominant(n, seed):
    """Columns dominated by the diagonal: elimination keeps that property, so
    every multiplier stays below 1 and dgetrf interchanges no row."""
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((n, n))
    np.fill_diagonal(A, 0.0)
    A *= 0.95 / np.maximum(np.abs(A).sum(axis=0, keepdims=True), 1e-300)
    A += np.eye(n) * np.where(rng.random(n) < 0.5, -1.0, 1.0)
    return A


@pytest.mark.parametrize("n,nrhs", [(1, 1), (64, 2), (300, 3), (2500, 2)])
def test_dense_unpivoted_certified(n, nrhs):
    """Column-dominant systems take the unpivoted blocked LU, whose multipliers
    (all |l| < 1) certify that partial pivoting makes the same (no) row
    interchanges; the solution is LAPACK's."""
    import scipy.linalg as sl
    A = _col_dominant(n, n + 11)
    B = np.random.default_rng(n).standard_normal((n, nrhs))
    lu, piv = sl.lu_factor(A)
    assert np.array_equal(piv, np.arange(n))  # LAPACK interchanges nothing
    for mode in (abi.DUST_SOLVE_LU64, abi.DUST_SOLVE_MIXED):
        X, rep = linsys.dense_solve(A, B, mode, tol=1e-13)
        assert rep["pivoted"] == 0
        assert rel(X, sl.lu_solve((lu, piv), B)) < 1e-11


@pytest.mark.parametrize("n", [500, 1920])
def test_dense_mixed_pivoting(n):
    rng = np.random.default_rng(n + 2)
    A = rng.standard_normal((n, n))
    B = rng.standard_normal((n, 3))
    X, rep = linsys.dense_solve(A, B, abi.DUST_SOLVE_MIXED, tol=1e-12)
    assert rep["fell_back"] == 0 and rep["residual"] <= 1e-12 and rep["pivoted"] == 1
    assert rel(X, np.linalg.solve(A, B)) < 1e-9


def test_dense_mixed_refines_to_fp64():
    rng = np.random.default_rng(5)
    n = 700
    A = rng.standard_normal((n, n)) + 2 * n ** 0.5 * np.eye(n)
    B = rng.standard_normal((n, 5))
    X, rep = linsys.dense_solve(A, B, abi.DUST_SOLVE_MIXED, tol=1e-12)
    assert rep["residual"] <= 1e-12
    assert rel(X, np.linalg.solve(A, B)) < 1e-10


def test_dense_singular_reported():
    A = np.ones((5, 5))
    with pytest.raises(Exception) as ei:
        linsys.dense_solve(A, np.ones(5), abi.DUST_SOLVE_LU64)
    assert "status 3" in str(ei.value)


def test_ellipsoid_dirichlet_parity():
    body = synth.ellipsoid(n_target=1500, axes=(4.0, 1.0, 0.5), seed=2)
    prm = FmmParams(u_inf=(1.0, 0.1, 0.0))
    n = body.n
    empty = abi.empty_panels()
    Ao, bo, ro = O.linsys_run(prm, n, 0, body, body, (empty, 0, None), (empty, 0, None))
    ls = linsys.initialize_linsys(prm, n, 0, body)
    ls.assemble_linsys(body)
    Ag, bg = ls.get_system()
    assert rel(Ag, Ao) < 1e-10 and rel(bg, bo) < 1e-10
    res, _ = ls.solve_linsys(abi.DUST_SOLVE_LU64)
    assert rel(res, ro) < 1e-10
    assert np.max(np.abs(Ag.sum(axis=1) - 4 * np.pi)) < 0.05 * 4 * np.pi
