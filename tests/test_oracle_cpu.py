"""CPU checks of the oracle against known answers and LAPACK (no GPU).

The reference has no unit-level golden vectors for this path; these tests
pin the oracle by (a) LAPACK itself (the reference's third-party solver,
reached here through scipy), (b) analytic identities of the influence
kernels, (c) FMM -> direct-sum convergence.
"""
import numpy as np
import pytest
import scipy.linalg as sla
from scipy.linalg import lapack

import oracle as O
from dust_b200 import abi, synth
from dust_b200.params import FmmParams


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_oracle_getrf_matches_lapack():
    rng = np.random.default_rng(0)
    for n in (1, 7, 64, 150):
        A = rng.standard_normal((n, n))
        A[0, :] *= 1e-3  # force pivoting
        LU, piv, info = O.dgetrf(A)
        lu_l, piv_l, info_l = lapack.dgetrf(A)
        assert info == info_l == 0
        assert np.array_equal(piv, piv_l + 1)  # scipy returns 0-based
        assert np.max(np.abs(LU - lu_l)) < 1e-12 * max(1.0, np.max(np.abs(lu_l)))


def test_oracle_getrf_singular_info():
    A = np.array([[1.0, 2.0], [2.0, 4.0]])
    _, _, info = O.dgetrf(A)
    _, _, info_l = lapack.dgetrf(A)
    assert info == info_l == 2


def _wing_case(n_span=8, n_chord=4):
    wing, te = synth.flat_wing(span=4.0, chord=1.0, n_span=n_span, n_chord=n_chord,
                               alpha_deg=5.0)
    wake, ind = synth.te_wake(wing, te, (0.3, 0.0, 0.02))
    far, _ = synth.te_wake(wing, te, (1.0, 0.0, 0.05))
    far.ver = far.ver + np.array([0.3, 0.0, 0.02])
    far.mag = np.linspace(-0.1, 0.1, far.n)
    wk = synth.concat_panels(wake, far)
    return wing, wk, wake.n, ind


def test_linsys_schur_sequence_equals_full_lu():
    """solve_linsys' static/moving block LU (dlaswp, dtrsm x2, dgemm, dgetrf,
    dgetrs) gives the solution of the full system."""
    prm = FmmParams(u_inf=(1.0, 0.0, 0.0), rankine_rad=0.1)
    wing, wk, n_impl, ind = _wing_case()
    rng = np.random.default_rng(1)
    wing.uvort = rng.standard_normal((wing.n, 3)) * 0.05
    n = wing.n
    nst = n // 2
    _, _, res_blk = O.linsys_run(prm, n, nst, wing, wing, (wk, n_impl, ind), (wk, n_impl, ind))
    A0, b0, res0 = O.linsys_run(prm, n, 0, wing, wing, (wk, n_impl, ind), (wk, n_impl, ind))
    assert rel(res0, np.linalg.solve(A0, b0)) < 1e-12
    assert rel(res_blk, res0) < 1e-10


def test_closed_body_row_sums_are_4pi():
    """Dirichlet rows of a closed surface: sum_j A(i,j) = 4 pi (solid angle
    of the whole body seen from its surface, self term 2 pi)."""
    body = synth.ellipsoid(n_target=400, axes=(2.0, 1.0, 0.7), seed=3)
    prm = FmmParams(u_inf=(1.0, 0.0, 0.0))
    n = body.n
    A, b, res = O.linsys_run(prm, n, 0, body, body, (abi.empty_panels(), 0, None),
                             (abi.empty_panels(), 0, None))
    rs = A.sum(axis=1)
    assert np.max(np.abs(rs - 4 * np.pi)) < 0.05 * 4 * np.pi
    assert abs(np.mean(rs) - 4 * np.pi) < 0.01 * 4 * np.pi


def test_source_potential_far_near_consistency():
    """The near-field source formula approaches the far-field A/r as the
    point leaves the 10*edge threshold."""
    pan = abi.PanelSet(np.array([[[0, 0, 0], [0.1, 0, 0], [0.1, 0.1, 0], [0, 0.1, 0]]]),
                       kind=np.array([abi.DUST_ELEM_SURFPAN]))
    prm = FmmParams()
    pos = np.array([0.05, 0.05, 0.99])  # just inside 10 * edge
    dou = O.potential_doublet(prm, pan, 0, pos)
    near = O.potential_source(prm, pan, 0, dou, pos)
    far = 0.01 / np.linalg.norm(pos - np.array([0.05, 0.05, 0.0]))
    assert abs(near - far) / far < 1e-3


def test_fmm_oracle_converges_and_factorial_wrap():
    cen, dir_, mag = synth.ring_particles(1800, 200, seed=1)
    rv = np.full(len(mag), 0.02)
    base = dict(box_length=4.0, origin=(-2, -2, -2), n_octree_levels=4, min_octree_part=5,
                rankine_rad=0.02)
    dv, _, _ = O.direct_particles(FmmParams(**base), cen, dir_, mag, rv)
    errs = {}
    for p in (2, 4, 8):
        v, _, _, _ = O.fmm_apply(FmmParams(multipole_degree=p, **base), cen, dir_, mag, rv)
        errs[p] = rel(v, dv)
    assert errs[2] > errs[4] > errs[8]
    # the reference's 32-bit factorials wrap for degree >= 13 (p >= 7)
    O.set_factorial_wrap(1)
    try:
        vw, _, _, _ = O.fmm_apply(FmmParams(multipole_degree=8, **base), cen, dir_, mag, rv)
        v4w, _, _, _ = O.fmm_apply(FmmParams(multipole_degree=4, **base), cen, dir_, mag, rv)
    finally:
        O.set_factorial_wrap(0)
    v4, _, _, _ = O.fmm_apply(FmmParams(multipole_degree=4, **base), cen, dir_, mag, rv)
    assert np.array_equal(v4w, v4)  # no wrap below degree 13
    assert rel(vw, dv) > 3 * errs[8]


def test_oracle_fmm_out_of_box():
    with pytest.raises(RuntimeError):
        O.fmm_apply(FmmParams(box_length=1.0), np.array([[2.0, 0.5, 0.5]]),
                    np.array([[0, 0, 1.0]]), np.array([1.0]), np.array([0.1]))


def test_vortex_particle_pair_analytic():
    """Two particles: the regularised Biot-Savart velocity and the stretching
    term of the reference's kernel (rho^2 = r^2 + sigma_q^2 with the SOURCE
    particle's core, c = -rho^-3, d = 3 rho^-5), written out by hand."""
    rng = np.random.default_rng(7)
    cen = rng.uniform(-0.3, 0.3, (2, 3))
    dir_ = rng.standard_normal((2, 3))
    dir_ /= np.linalg.norm(dir_, axis=1)[:, None]
    mag = np.array([0.7, 1.3])
    rv = np.array([0.05, 0.11])
    prm = FmmParams(box_length=2.0, origin=(-1.0, -1.0, -1.0), vortstretch=True,
                    divergence_filtering=False, diffusion=False)
    vel, st, _ = O.direct_particles(prm, cen, dir_, mag, rv)
    al = mag[:, None] * dir_
    for p, q in ((0, 1), (1, 0)):
        r = cen[p] - cen[q]
        rho2 = r @ r + rv[q] ** 2
        c, d = -rho2 ** -1.5, 3.0 * rho2 ** -2.5
        u = c * np.cross(r, al[q]) / (4 * np.pi)
        v = np.cross(al[p], al[q])
        s = -(c * v + d * r * (r @ v)) / (4 * np.pi)
        assert rel(vel[p], u) < 1e-12
        assert rel(st[p], s) < 1e-12


def test_vortex_segment_analytic():
    """A straight vortex segment (end vortex) at a point beside it: the
    Biot-Savart law Gamma / (4 pi h) (cos t1 - cos t2) about the segment."""
    L, gam = 0.8, 1.7
    lines = abi.LineSet(np.array([[[0.0, 0.0, 0.0], [L, 0.0, 0.0]]]), np.array([gam]))
    prm = FmmParams()
    for a, h in ((0.3, 0.2), (-0.4, 0.5), (1.1, 0.35)):
        pos = np.array([[a, h, 0.0]])
        v = O.elements_vel(prm, pos, abi.elements_struct(end_vort=lines))[0]
        r1, r2 = np.hypot(a, h), np.hypot(L - a, h)
        mag_v = gam / (4 * np.pi * h) * (a / r1 + (L - a) / r2)
        assert rel(v, np.array([0.0, 0.0, mag_v])) < 1e-12


@pytest.mark.parametrize("kind", [abi.DUST_ELEM_VORTLATT, abi.DUST_ELEM_SURFPAN])
def test_panel_velocity_far_near_consistency(kind):
    """Just inside and just outside the far-field radius (10 x max edge) the
    exact doublet/source formulas and the point dipole/source agree to the
    expansion error (edge / r)^2."""
    pan = abi.PanelSet(np.array([[[0, 0, 0], [0.1, 0, 0], [0.1, 0.1, 0], [0, 0.1, 0]]]),
                       kind=np.array([kind]))
    prm = FmmParams()
    cen = np.array([0.05, 0.05, 0.0])
    d = np.array([0.3, -0.2, 0.93])
    d /= np.linalg.norm(d)
    inside, outside = cen + 0.999 * d, cen + 1.001 * d
    vd_in, vd_out = O.velocity_doublet(prm, pan, 0, inside), O.velocity_doublet(prm, pan, 0, outside)
    assert rel(vd_in, vd_out) < 2e-2
    if kind == abi.DUST_ELEM_SURFPAN:
        vs_in, vs_out = O.velocity_source(prm, pan, 0, inside), O.velocity_source(prm, pan, 0, outside)
        assert rel(vs_in, vs_out) < 2e-2


def _wake_case(n, seed, box=1.0):
    rng = np.random.default_rng(seed)
    cen = rng.uniform(-box, box, (n, 3))
    dir_ = rng.standard_normal((n, 3))
    dir_ /= np.linalg.norm(dir_, axis=1)[:, None]
    mag = rng.uniform(0.1, 1.0, n)
    vel = rng.standard_normal((n, 3)) * 2.0
    st = rng.standard_normal((n, 3))
    rot = rng.standard_normal((n, 3))
    free = (rng.random(n) < 0.1).astype(np.int32)
    # one particle whose alpha is exactly zero (no strength): dir kept
    mag[1] = 0.0
    st[1] = 0.0
    vel[1] = 0.0
    free[1] = 0
    return cen, dir_, mag, vel, st, rot, free


def _numpy_update(u, cen, dir_, mag, vel, st, rot, free):
    """Independent vectorised restatement of mod_wake.f90:1309-1355."""
    cen, dir_, st, free = cen.copy(), dir_.copy(), st.copy(), free.copy()
    nd = float(u.ndt_update_wake)
    live = free == 0
    p = cen + vel * u.dt * nd
    inb = np.all(p >= np.array(u.box_min), axis=1) & np.all(p <= np.array(u.box_max), axis=1)
    gone = live & ~inb
    move = live & inb
    free[gone] = 1
    cen[move] = p[move]
    if u.vortstretch or u.diffusion:
        m = mag[:, None]
        if u.divergence_filtering:
            nr = np.sqrt((rot[:, 0] * rot[:, 0] + rot[:, 1] * rot[:, 1]) + rot[:, 2] * rot[:, 2])
            newst = st - (u.filt_eta / nd) * (dir_ * m - rot * m / nr[:, None])
            st[move] = newst[move]
        a = dir_ * m + st * u.dt * nd
        an = np.sqrt((a[:, 0] * a[:, 0] + a[:, 1] * a[:, 1]) + a[:, 2] * a[:, 2])
        ok = move & (an != 0.0)
        dir_[ok] = a[ok] / an[ok, None]
    return cen, dir_, st, free, int(gone.sum())


@pytest.mark.parametrize("vs,vd,df,ndt", [(1, 1, 1, 1), (1, 0, 0, 2), (0, 0, 1, 1),
                                          (0, 1, 1, 3)])
def test_oracle_particles_update_matches_numpy(vs, vd, df, ndt):
    """The oracle's complete_wake particle loop equals an independent numpy
    statement of the same expressions bit for bit (same rounding order, no
    fused multiply-adds), including particles leaving the box, free slots and
    a zero alpha."""
    cen, dir_, mag, vel, st, rot, free = _wake_case(5000, seed=vs + 2 * vd + 4 * df + 8 * ndt)
    u = abi.update_params(0.07, (-1.0, -1.05, -0.9), (1.0, 1.1, 0.95), ndt_update_wake=ndt,
                          vortstretch=vs, diffusion=vd, divergence_filtering=df, filt_eta=0.3)
    got = O.particles_update(u, cen, dir_, mag, vel, st, rot, free)
    ref = _numpy_update(u, cen, dir_, mag, vel, st, rot, free)
    for g, r in zip(got[:4], ref[:4]):
        assert np.array_equal(g, r)
    assert got[4] == ref[4] > 0
    assert np.array_equal(got[1][1], dir_[1]) or not (vs or vd)


def _segment_4pi(v0, v1, p):
    """4 pi x the velocity of a unit-circulation straight segment v0 -> v1 at
    p (Biot-Savart, no core)."""
    e = v1 - v0
    L = np.linalg.norm(e)
    e = e / L
    a = p - v0
    ai = a @ e
    h = np.linalg.norm(a - ai * e)
    r1, r2 = np.linalg.norm(p - v0), np.linalg.norm(p - v1)
    mag = (ai / r1 + (L - ai) / r2) / h
    return mag * np.cross(e, a) / np.linalg.norm(np.cross(e, a))


def test_doublet_velocity_equals_vortex_ring():
    """A constant-strength doublet panel induces the velocity of the vortex
    ring along its edges: inside the far-field radius the oracle's
    velocity_calc_doublet equals the sum of the four straight-segment laws
    (points away from the edges' cores)."""
    rng = np.random.default_rng(11)
    ver = np.array([[0.0, 0.0, 0.0], [0.3, 0.02, 0.01], [0.32, 0.25, -0.02], [0.01, 0.22, 0.0]])
    pan = abi.PanelSet(ver[None], kind=np.array([abi.DUST_ELEM_VORTLATT]))
    prm = FmmParams()
    for _ in range(20):
        pos = ver.mean(axis=0) + rng.uniform(-0.8, 0.8, 3)
        if np.linalg.norm(pos - ver.mean(axis=0)) > 2.5:
            continue
        v = O.velocity_doublet(prm, pan, 0, pos)
        ring = sum(_segment_4pi(ver[i], ver[(i + 1) % 4], pos) for i in range(4))
        assert rel(v, ring) < 1e-12


def _solid_angle_tri(a, b, c):
    """Van Oosterom-Strackee solid angle of triangle (a, b, c) seen from the
    origin."""
    na, nb, nc = np.linalg.norm(a), np.linalg.norm(b), np.linalg.norm(c)
    num = a @ np.cross(b, c)
    den = na * nb * nc + (a @ b) * nc + (a @ c) * nb + (b @ c) * na
    return 2.0 * np.arctan2(num, den)


def test_doublet_potential_is_solid_angle():
    """potential_calc_doublet inside the far-field radius is the solid angle
    the panel subtends (an independent formula: Van Oosterom-Strackee on the
    two triangles of the planar quad), with the reference's sign."""
    rng = np.random.default_rng(12)
    ver = np.array([[0.0, 0.0, 0.0], [0.3, 0.0, 0.0], [0.35, 0.25, 0.0], [0.02, 0.22, 0.0]])
    pan = abi.PanelSet(ver[None], kind=np.array([abi.DUST_ELEM_SURFPAN]))
    prm = FmmParams()
    signs = set()
    for _ in range(20):
        pos = ver.mean(axis=0) + rng.uniform(-0.8, 0.8, 3)
        pos[2] = np.sign(pos[2]) * max(abs(pos[2]), 0.05)
        rel_v = ver - pos
        om = _solid_angle_tri(rel_v[0], rel_v[1], rel_v[2]) + \
            _solid_angle_tri(rel_v[0], rel_v[2], rel_v[3])
        dou = O.potential_doublet(prm, pan, 0, pos)
        assert min(abs(dou - om), abs(dou + om)) < 1e-12
        signs.add(np.sign(dou * om))
    assert len(signs) == 1  # one fixed sign convention


def test_source_potential_equals_quadrature():
    """potential_calc_sou_surfpan inside the far-field radius is the integral
    of 1/r over the flat panel (Hess-Smith closed form): checked against
    Gauss-Legendre quadrature on the bilinear map of the quad."""
    ver = np.array([[0.0, 0.0, 0.0], [0.3, 0.0, 0.0], [0.35, 0.25, 0.0], [0.02, 0.22, 0.0]])
    pan = abi.PanelSet(ver[None], kind=np.array([abi.DUST_ELEM_SURFPAN]))
    prm = FmmParams()
    x, w = np.polynomial.legendre.leggauss(60)
    s, t = (x + 1) / 2, w / 2
    S, T = np.meshgrid(s, s, indexing="ij")
    W = np.outer(t, t)
    # bilinear map q(s, t) and its Jacobian |q_s x q_t|
    q = ((1 - S) * (1 - T))[..., None] * ver[0] + (S * (1 - T))[..., None] * ver[1] + \
        (S * T)[..., None] * ver[2] + ((1 - S) * T)[..., None] * ver[3]
    qs = (1 - T)[..., None] * (ver[1] - ver[0]) + T[..., None] * (ver[2] - ver[3])
    qt = (1 - S)[..., None] * (ver[3] - ver[0]) + S[..., None] * (ver[2] - ver[1])
    jac = np.linalg.norm(np.cross(qs, qt), axis=-1)
    rng = np.random.default_rng(13)
    for _ in range(10):
        pos = ver.mean(axis=0) + rng.uniform(-0.5, 0.5, 3)
        pos[2] = np.sign(pos[2]) * max(abs(pos[2]), 0.15)
        quad = np.sum(W * jac / np.linalg.norm(q - pos, axis=-1))
        dou = O.potential_doublet(prm, pan, 0, pos)
        sou = O.potential_source(prm, pan, 0, dou, pos)
        assert abs(sou - quad) < 1e-9 * abs(quad)


def test_panel_velocities_are_potential_gradients():
    """Inside the far-field radius the doublet and source velocities are the
    gradients of the corresponding potentials (central differences, one sign
    convention each)."""
    ver = np.array([[0.0, 0.0, 0.0], [0.3, 0.0, 0.0], [0.35, 0.25, 0.0], [0.02, 0.22, 0.0]])
    pan = abi.PanelSet(ver[None], kind=np.array([abi.DUST_ELEM_SURFPAN]))
    prm = FmmParams()
    rng = np.random.default_rng(14)
    h = 1e-5
    sd, ss = set(), set()
    for _ in range(10):
        pos = ver.mean(axis=0) + rng.uniform(-0.5, 0.5, 3)
        pos[2] = np.sign(pos[2]) * max(abs(pos[2]), 0.1)
        gd, gs = np.zeros(3), np.zeros(3)
        for k in range(3):
            e = np.zeros(3)
            e[k] = h
            dp, dm = O.potential_doublet(prm, pan, 0, pos + e), O.potential_doublet(prm, pan, 0, pos - e)
            gd[k] = (dp - dm) / (2 * h)
            gs[k] = (O.potential_source(prm, pan, 0, dp, pos + e) -
                     O.potential_source(prm, pan, 0, dm, pos - e)) / (2 * h)
        vd, vs = O.velocity_doublet(prm, pan, 0, pos), O.velocity_source(prm, pan, 0, pos)
        for v, g, signs in ((vd, gd, sd), (vs, gs, ss)):
            sg = 1.0 if np.linalg.norm(v - g) < np.linalg.norm(v + g) else -1.0
            assert rel(v, sg * g) < 1e-6
            signs.add(sg)
    assert len(sd) == 1 and len(ss) == 1


def test_vortex_particle_pair_curl_and_diffusion():
    """The divergence-filter curl (-2 c alpha_q + d r x (r x alpha_q)) and the
    PSE diffusion term ((vol alpha_q - vol alpha_p) / sigma^2 eta(r, sigma)
    (nu), eta = 105 / (8 pi) / ((r / sigma)^2 + 1)^(9/2) / sigma^3, both with
    the source particle's core) of two particles, written out by hand."""
    rng = np.random.default_rng(9)
    cen = rng.uniform(-0.3, 0.3, (2, 3))
    dir_ = rng.standard_normal((2, 3))
    dir_ /= np.linalg.norm(dir_, axis=1)[:, None]
    mag = np.array([0.9, 0.4])
    rv = np.array([0.07, 0.13])
    nu = 2.5e-3
    prm = FmmParams(box_length=2.0, origin=(-1.0, -1.0, -1.0), vortstretch=True,
                    divergence_filtering=True, diffusion=True, nu_inf=nu)
    vel, st, ro = O.direct_particles(prm, cen, dir_, mag, rv)
    al = mag[:, None] * dir_
    for p, q in ((0, 1), (1, 0)):
        r = cen[p] - cen[q]
        rn = np.linalg.norm(r)
        rho2 = rn * rn + rv[q] ** 2
        c, d = -rho2 ** -1.5, 3.0 * rho2 ** -2.5
        v = np.cross(al[p], al[q])
        s = -(c * v + d * r * (r @ v)) / (4 * np.pi)
        rot = (-2.0 * c * al[q] + d * np.cross(r, np.cross(r, al[q]))) / (4 * np.pi)
        vol = 4.0 / 3.0 * np.pi * rv[q] ** 3
        eta = 105.0 / (8.0 * np.pi) / ((rn / rv[q]) ** 2 + 1) ** 4.5 / rv[q] ** 3
        diff = (vol * al[q] - vol * al[p]) / rv[q] ** 2 * eta
        assert rel(ro[p], rot) < 1e-12
        assert rel(st[p], s + diff * nu) < 1e-12


def test_oracle_row_sample_equals_full_assembly():
    """or_linsys_rows (the row sample the configuration-size tests compare
    against) builds exactly the rows of the full all-moving assembly."""
    from dust_b200 import synth
    rng = np.random.default_rng(0)
    prm = FmmParams(u_inf=(1.0, 0.2, 0.0))
    body = synth.ellipsoid(n_target=600, seed=3)
    body.uvort = rng.standard_normal((body.n, 3)) * 0.1
    body.ub = rng.standard_normal((body.n, 3)) * 0.1
    e = abi.empty_panels()
    A, b, _ = O.linsys_run(prm, body.n, 0, body, body, (e, 0, None), (e, 0, None))
    rows = np.array([0, 5, 17, body.n - 1])
    Ar, br = O.linsys_rows(prm, body, rows)
    assert np.array_equal(Ar, A[rows]) and np.array_equal(br, b[rows])
    wing, te = synth.flat_wing(span=4.0, chord=1.0, n_span=12, n_chord=5, alpha_deg=5.0)
    wake, ind = synth.te_wake(wing, te, (0.3, 0.0, 0.02))
    wing.uvort = rng.standard_normal((wing.n, 3)) * 0.05
    A, b, _ = O.linsys_run(prm, wing.n, 0, wing, wing, (wake, wake.n, ind), (wake, wake.n, ind))
    rows = np.arange(0, wing.n, 7)
    Ar, br = O.linsys_rows(prm, wing, rows, (wake, wake.n, ind))
    assert np.array_equal(Ar, A[rows]) and np.array_equal(br, b[rows])


def test_oracle_fmm_panel_uvort_converges_to_direct_sum():
    """apply_multipole_panels (leaf local expansion + near-field particles)
    approaches the direct particle sum as the multipole degree grows; the
    end vortices enter both by direct sum."""
    cen, dir_, mag = synth.ring_particles(3600, 400, seed=2)
    rv = np.full(len(mag), 0.02)
    pts = np.random.default_rng(0).uniform(-1.6, 1.6, (300, 3))
    ev = abi.LineSet(np.array([[[0.0, 0.0, 0.0], [0.5, 0.5, 0.0]]]), np.array([0.7]))
    base = dict(box_length=4.0, origin=(-2.0, -2.0, -2.0), n_octree_levels=5,
                min_octree_part=5, rankine_rad=0.02)
    ref = O.points_uvort(FmmParams(**base), pts, cen, dir_, mag, rv, ev)
    errs = [rel(O.fmm_points_uvort(FmmParams(multipole_degree=p, **base), pts, cen, dir_, mag,
                                   rv, ev), ref) for p in (2, 4, 6)]
    assert errs[2] < errs[1] < errs[0] and errs[2] < 5e-4
