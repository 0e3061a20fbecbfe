"""Seeded synthetic inputs with the shapes of the benchmark cases.

No public dataset exists for this path; every case is generated from a seed
(numpy PCG64):

* ``ring_particles``  -- vortex ring (radius 1, Gaussian cross-section) plus
  uniform background in [-2, 2]^3, tangential circulation vectors with
  Gaussian magnitude (mean 1e-3, sd 1e-4).
* ``flat_wing``       -- flat rectangular vortex-lattice wing.
* ``ellipsoid``       -- closed ellipsoid of quadrilateral surface panels.
* ``rotor``           -- vortex-lattice rotor blades with linear twist.
* ``cylinder``        -- closed cylindrical fuselage of surface panels.
"""
import numpy as np

from . import abi


def ring_particles(n_ring, n_bg, seed=0, R=1.0, sigma=0.1, mean=1e-3, sd=1e-4,
                   half=2.0):
    """Particles of a vortex ring + uniform background.

    Returns cen (n,3), dir (n,3) unit, mag (n,)."""
    rng = np.random.default_rng(seed)
    phi = rng.uniform(0.0, 2.0 * np.pi, n_ring)
    rad = R + sigma * rng.standard_normal(n_ring)
    z = sigma * rng.standard_normal(n_ring)
    cen_r = np.stack([rad * np.cos(phi), rad * np.sin(phi), z], axis=1)
    # keep every particle strictly inside the box
    cen_r = np.clip(cen_r, -half * 0.999, half * 0.999)
    cen_b = rng.uniform(-half * 0.999, half * 0.999, (n_bg, 3))
    cen = np.concatenate([cen_r, cen_b], axis=0)
    ph = np.arctan2(cen[:, 1], cen[:, 0])
    dir_ = np.stack([-np.sin(ph), np.cos(ph), np.zeros_like(ph)], axis=1)
    mag = np.abs(mean + sd * rng.standard_normal(n_ring + n_bg))
    return cen, dir_, mag


def choose_levels(cen, box_length, n_box, origin, max_leaf=64, max_levels=12):
    """Smallest number of octree levels whose finest cells hold at most
    ``max_leaf`` particles (the reference's leaf rule keeps the finest level
    fixed, so a bound on the leaf size is a bound on the finest-cell count)."""
    cen = np.asarray(cen)
    for ll in range(1, max_levels + 1):
        cs = box_length / 2 ** (ll - 1)
        idx = np.ceil((cen - np.asarray(origin)) / cs).astype(np.int64) - 1
        ncl = np.asarray(n_box) * 2 ** (ll - 1)
        lin = idx[:, 0] + ncl[0] * (idx[:, 1] + ncl[1] * idx[:, 2])
        if np.bincount(lin).max() <= max_leaf:
            return ll
    return max_levels


def _quad_grid(P):
    """Quads from a structured grid of points P[i, j, 3] (i: chord, j: span).
    Vertex order (i,j), (i+1,j), (i+1,j+1), (i,j+1)."""
    a, b = P.shape[0] - 1, P.shape[1] - 1
    q = np.stack([P[:-1, :-1], P[1:, :-1], P[1:, 1:], P[:-1, 1:]], axis=2)
    return q.reshape(a * b, 4, 3)


def flat_wing(span=10.0, chord=1.0, n_span=40, n_chord=10, alpha_deg=0.0):
    """Flat rectangular vortex-lattice wing in the x-y plane (x chordwise,
    y spanwise), pitched by alpha about the y axis.  Returns a PanelSet and
    the trailing-edge panel indices (chordwise-last row)."""
    x = np.linspace(0.0, chord, n_chord + 1)
    y = np.linspace(-span / 2, span / 2, n_span + 1)
    X, Y = np.meshgrid(x, y, indexing="ij")
    P = np.stack([X, Y, np.zeros_like(X)], axis=2)
    a = np.deg2rad(alpha_deg)
    R = np.array([[np.cos(a), 0, np.sin(a)], [0, 1, 0], [-np.sin(a), 0, np.cos(a)]])
    P = P @ R.T
    ver = _quad_grid(P)
    n = ver.shape[0]
    te = np.arange((n_chord - 1) * n_span, n_chord * n_span)
    return abi.PanelSet(ver, kind=np.full(n, abi.DUST_ELEM_VORTLATT)), te


def ellipsoid(n_target=16384, axes=(4.0, 1.0, 0.5), seed=0):
    """Closed ellipsoid of quadrilateral surface panels (outward normals),
    n_u x n_v ~ n_target panels, with a seeded random rigid rotation.
    The poles are closed by triangles folded into quads with a repeated
    vertex avoided: the grid is built in a parameter range that excludes the
    poles and the two polar caps are closed by triangle fans."""
    rng = np.random.default_rng(seed)
    n_v = int(round(np.sqrt(n_target / 2.0)))
    # even azimuthal count: with an odd one, a cap triangle's centroid lies on
    # the extension of the opposite fan edge, where the solid-angle formula of
    # potential_calc_doublet divides by zero
    n_u = (n_target // n_v) // 2 * 2
    # quads: n_u (azimuth) x (n_v - 2) latitude bands; caps: 2 * n_u triangles
    n_lat = n_v
    th = np.linspace(0.0, np.pi, n_lat + 1)  # polar angle
    ph = np.linspace(0.0, 2.0 * np.pi, n_u + 1)
    ax = np.asarray(axes, dtype=np.float64)
    TH, PH = np.meshgrid(th[1:-1], ph, indexing="ij")
    ring = np.stack([ax[0] * np.cos(TH), ax[1] * np.sin(TH) * np.cos(PH),
                     ax[2] * np.sin(TH) * np.sin(PH)], axis=2)
    quads = []
    for i in range(ring.shape[0] - 1):
        for j in range(n_u):
            quads.append([ring[i, j], ring[i + 1, j], ring[i + 1, j + 1], ring[i, j + 1]])
    quads = np.asarray(quads)
    north = np.array([ax[0], 0.0, 0.0])
    south = np.array([-ax[0], 0.0, 0.0])
    tris = []
    for j in range(n_u):
        tris.append([north, ring[0, j], ring[0, j + 1], np.zeros(3)])
        tris.append([south, ring[-1, j + 1], ring[-1, j], np.zeros(3)])
    tris = np.asarray(tris)
    ver = np.concatenate([quads, tris], axis=0)
    nver = np.concatenate([np.full(len(quads), 4), np.full(len(tris), 3)])
    # orientation: outward normal
    A = rng.standard_normal((3, 3))
    Q, Rr = np.linalg.qr(A)
    Q = Q @ np.diag(np.sign(np.diag(Rr)))
    if np.linalg.det(Q) < 0:
        Q[:, 0] = -Q[:, 0]
    ver = ver @ Q.T
    n = ver.shape[0]
    ps = abi.PanelSet(ver, n_ver=nver, kind=np.full(n, abi.DUST_ELEM_SURFPAN))
    # flip any panel whose normal points inward
    return _orient_outward(ps)


def _panel_cn(ver, nver):
    cen = np.where(nver[:, None] == 4, ver.mean(axis=1), ver[:, :3].mean(axis=1))
    n4 = np.cross(ver[:, 2] - ver[:, 0], ver[:, 3] - ver[:, 1])
    n3 = np.cross(ver[:, 2] - ver[:, 1], ver[:, 0] - ver[:, 1])
    nor = np.where(nver[:, None] == 4, n4, n3)
    return cen, nor


def _orient_outward(ps):
    cen, nor = _panel_cn(ps.ver, ps.n_ver)
    c0 = cen.mean(axis=0)
    flip = np.einsum("ij,ij->i", nor, cen - c0) < 0
    v = ps.ver.copy()
    for i in np.nonzero(flip)[0]:
        if ps.n_ver[i] == 4:
            v[i] = v[i][[0, 3, 2, 1]]
        else:
            v[i, :3] = v[i, [0, 2, 1]]
    ps.ver = np.ascontiguousarray(v)
    return ps


def rotor_blades(n_blades=3, radius=1.0, root=0.2, chord=0.1, n_span=40, n_chord=8,
                 twist_deg=-8.0, pitch_deg=8.0, phase=0.0, center=(0.0, 0.0, 0.0),
                 spin=1):
    """Vortex-lattice blades of a rotor in the x-y plane, rotating about z.
    Linear twist from root to tip.  Returns (PanelSet, trailing-edge panel
    indices)."""
    vers, tes = [], []
    base = 0
    for b in range(n_blades):
        psi = phase + spin * 2.0 * np.pi * b / n_blades
        r = np.linspace(root, radius, n_span + 1)
        th = np.deg2rad(pitch_deg + twist_deg * (r - root) / (radius - root))
        s = np.linspace(-0.25, 0.75, n_chord + 1) * chord  # chordwise coordinate
        S, Rg = np.meshgrid(s, r, indexing="ij")
        TH = np.broadcast_to(th, S.shape)
        # blade frame: span along x, chord along -spin*y (leading edge ahead)
        xb = Rg
        yb = -spin * S * np.cos(TH)
        zb = -S * np.sin(TH)
        c, sn = np.cos(psi), np.sin(psi)
        P = np.stack([c * xb - sn * yb, sn * xb + c * yb, zb], axis=2) + np.asarray(center)
        q = _quad_grid(P)
        vers.append(q)
        tes.append(base + np.arange((n_chord - 1) * n_span, n_chord * n_span))
        base += q.shape[0]
    ver = np.concatenate(vers, axis=0)
    return abi.PanelSet(ver, kind=np.full(ver.shape[0], abi.DUST_ELEM_VORTLATT)), \
        np.concatenate(tes)


def cylinder(n_target=6000, length=4.0, radius=0.3, center=(0.0, 0.0, -0.6)):
    """Closed cylinder along x of surface panels with triangle-fan end caps."""
    n_th = max(8, int(round(np.sqrt(n_target * 2 * np.pi * radius / length))))
    n_th += n_th % 2  # even: see ellipsoid()
    n_x = max(2, (n_target - 2 * n_th) // n_th)
    x = np.linspace(-length / 2, length / 2, n_x + 1)
    th = np.linspace(0.0, 2 * np.pi, n_th + 1)
    X, TH = np.meshgrid(x, th, indexing="ij")
    P = np.stack([X, radius * np.cos(TH), radius * np.sin(TH)], axis=2) + np.asarray(center)
    quads = _quad_grid(P)
    c0 = np.asarray(center)
    tris = []
    for j in range(n_th):
        tris.append([c0 + [-length / 2, 0, 0], P[0, j + 1], P[0, j], np.zeros(3)])
        tris.append([c0 + [length / 2, 0, 0], P[-1, j], P[-1, j + 1], np.zeros(3)])
    ver = np.concatenate([quads, np.asarray(tris)], axis=0)
    nver = np.concatenate([np.full(len(quads), 4), np.full(len(tris), 3)])
    ps = abi.PanelSet(ver, n_ver=nver, kind=np.full(ver.shape[0], abi.DUST_ELEM_SURFPAN))
    return _orient_outward(ps)


def te_wake(panels, te_idx, offset, second=None, mag=None):
    """One row of wake panels behind trailing-edge panels: the trailing edge
    of panel i is the edge ver[1] -> ver[2] (chordwise-last vertices of the
    structured grids above), extended by ``offset``.  Returns the wake
    PanelSet and the 1-based generating-element pairs (second element 0 when
    ``second`` is None, as for vortex-lattice trailing edges)."""
    te_idx = np.asarray(te_idx)
    v = panels.ver[te_idx]
    off = np.asarray(offset, dtype=np.float64)
    w = np.stack([v[:, 1], v[:, 1] + off, v[:, 2] + off, v[:, 2]], axis=1)
    n = len(te_idx)
    ps = abi.PanelSet(w, kind=np.full(n, abi.DUST_ELEM_VORTLATT),
                      mag=np.zeros(n) if mag is None else mag)
    ind = np.zeros((n, 2), dtype=np.int32)
    ind[:, 0] = te_idx + 1
    if second is not None:
        ind[:, 1] = np.asarray(second) + 1
    return ps, ind


def concat_panels(*sets):
    g = lambda name: None if all(getattr(s, name) is None for s in sets) else np.concatenate(
        [getattr(s, name) if getattr(s, name) is not None else
         np.zeros((s.n, 3) if name in ("ub", "uvort") else s.n) for s in sets])
    return abi.PanelSet(np.concatenate([s.ver for s in sets]),
                        np.concatenate([s.n_ver for s in sets]),
                        np.concatenate([s.kind for s in sets]), g("mag"), g("ub"), g("uvort"))
