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


def ellipsoid(n_target=16384, axes=(4.0, 1.0, 0.5), seed=0, n_u=None, n_lat=None):
    """Closed ellipsoid of quadrilateral surface panels (outward normals),
    n_u x n_v ~ n_target panels (exactly n_u x n_lat when both are given),
    with a seeded random rigid rotation.
    The poles are closed by triangles folded into quads with a repeated
    vertex avoided: the grid is built in a parameter range that excludes the
    poles and the two polar caps are closed by triangle fans."""
    rng = np.random.default_rng(seed)
    if n_u is None or n_lat is None:
        n_v = int(round(np.sqrt(n_target / 2.0)))
        # even azimuthal count: with an odd one, a cap triangle's centroid lies
        # on the extension of the opposite fan edge, where the solid-angle
        # formula of potential_calc_doublet divides by zero
        n_u = (n_target // n_v) // 2 * 2
        n_lat = n_v
    assert n_u % 2 == 0, "the azimuthal count must be even"
    # quads: n_u (azimuth) x (n_lat - 2) latitude bands; caps: 2 * n_u triangles
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


def rotor_fuselage(n_fus=6000, n_blades=4, n_span=30, n_chord=8, phase=0.0, omega=40.0,
                   inflow=(0.0, 0.0, 0.0)):
    """Moving-body case of the learned preconditioner: a rotor (radius 1,
    linear twist -8 deg, `n_blades` blades of n_span x n_chord vortex-lattice
    panels) at azimuth `phase` above a closed cylindrical fuselage of about
    n_fus surface panels.  Returns (elems, nstatic) with the fuselage (static)
    first; the rotor panels carry their body velocity omega x r (+ inflow
    subtracted as a relative wind is the caller's u_inf)."""
    body = cylinder(n_target=n_fus, length=4.0, radius=0.3, center=(0.0, 0.0, -0.6))
    rot, _ = rotor_blades(n_blades=n_blades, radius=1.0, root=0.2, chord=0.1, n_span=n_span,
                          n_chord=n_chord, twist_deg=-8.0, phase=phase, center=(0.0, 0.0, 0.0))
    els = concat_panels(body, rot)
    ub = np.zeros((els.n, 3))
    cen = rot.ver.mean(axis=1)
    ub[body.n:] = np.cross([0.0, 0.0, omega], cen) - np.asarray(inflow)
    els.ub = ub
    return els, body.n


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


def naca_wing(span=6.0, chord=1.0, n_span=98, n_around=120, thick=0.12, alpha_deg=5.0,
              center=(0.0, 0.0, 0.0)):
    """Closed NACA 00xx wing of surface panels: n_span x n_around quads
    (cosine chordwise spacing, sharp trailing edge) plus triangle-fan tip caps
    (2 * n_around triangles).  Returns (PanelSet, te_upper, te_lower, dy):
    the upper/lower trailing-edge panel indices and stripe widths."""
    nh = n_around // 2
    beta = np.linspace(0.0, np.pi, nh + 1)
    xc = 0.5 * (1.0 - np.cos(beta))  # 0 (LE) .. 1 (TE)
    yt = 5 * thick * (0.2969 * np.sqrt(xc) - 0.1260 * xc - 0.3516 * xc ** 2 +
                      0.2843 * xc ** 3 - 0.1036 * xc ** 4)
    # closed loop TE -> upper -> LE -> lower -> TE (n_around + 1 points)
    xs = np.concatenate([xc[::-1], xc[1:]]) * chord
    zs = np.concatenate([yt[::-1], -yt[1:]]) * chord
    y = np.linspace(-span / 2, span / 2, n_span + 1)
    X = np.broadcast_to(xs[:, None], (len(xs), len(y)))
    Z = np.broadcast_to(zs[:, None], (len(xs), len(y)))
    Y = np.broadcast_to(y[None, :], (len(xs), len(y)))
    P = np.stack([X, Y, Z], axis=2)
    a = np.deg2rad(alpha_deg)
    R = np.array([[np.cos(a), 0, np.sin(a)], [0, 1, 0], [-np.sin(a), 0, np.cos(a)]])
    P = P @ R.T + np.asarray(center)
    # quads (i around, j span); around runs TE->upper->LE->lower so with
    # vertex order (i,j),(i,j+1),(i+1,j+1),(i+1,j) the normals point outward
    q = np.stack([P[:-1, :-1], P[:-1, 1:], P[1:, 1:], P[1:, :-1]], axis=2)
    quads = q.reshape(-1, 4, 3)
    # tip caps: fans around the section centroid at each tip
    tris = []
    for jj, sgn in ((0, -1), (len(y) - 1, 1)):
        c = P[:-1, jj].mean(axis=0)
        for i in range(n_around):
            a0, a1 = P[i, jj], P[i + 1, jj]
            t = [c, a1, a0] if sgn < 0 else [c, a0, a1]
            tris.append(t + [np.zeros(3)])
    tris = np.asarray(tris)
    ver = np.concatenate([quads, tris], axis=0)
    nver = np.concatenate([np.full(len(quads), 4), np.full(len(tris), 3)])
    ps = abi.PanelSet(ver, n_ver=nver, kind=np.full(len(ver), abi.DUST_ELEM_SURFPAN))
    # panel (i, j) index = i * n_span + j; TE upper: i = 0, TE lower: i = n_around-1
    te_up = np.arange(0, n_span)
    te_lo = (n_around - 1) * n_span + np.arange(0, n_span)
    dy = np.diff(y)
    return ps, te_up, te_lo, dy


def _rotz(v, ang):
    c, s = np.cos(ang), np.sin(ang)
    out = v.copy()
    out[..., 0] = c * v[..., 0] - s * v[..., 1]
    out[..., 1] = s * v[..., 0] + c * v[..., 1]
    return out


class FullStepCase:
    """Two counter-rotating 3-blade vortex-lattice rotors (radius 1, 40 x 8
    panels per blade) above the tips of a 12,000-panel surface-panel wing,
    with a particle wake (rotor helices + wing sheet) of ``n_particles``.
    Element order: wing (static) first, then the rotors (moving)."""

    def __init__(self, n_particles=2_000_000, seed=0, n_span_blade=40, n_chord_blade=8,
                 wing_span=98, wing_around=120, omega=60.0, u_inf=(5.0, 0.0, 0.0)):
        rng = np.random.default_rng(seed)
        self.u_inf = np.asarray(u_inf, dtype=np.float64)
        self.omega = omega
        self.dt = 2 * np.pi / omega / 72.0
        wing, te_up, te_lo, dy = naca_wing(n_span=wing_span, n_around=wing_around)
        self.wing = wing
        self.centers = [np.array([0.3, -3.2, 1.0]), np.array([0.3, 3.2, 1.0])]
        self.spins = [1, -1]
        rotors, rtes = [], []
        base = wing.n
        for c, sp in zip(self.centers, self.spins):
            r, te = rotor_blades(n_blades=3, radius=1.0, root=0.15, chord=0.08,
                                 n_span=n_span_blade, n_chord=n_chord_blade, center=c,
                                 spin=sp)
            rotors.append(r)
            rtes.append(te + base)
            base += r.n
        self.nstatic = wing.n
        self.rotor_ver0 = np.concatenate([r.ver for r in rotors])
        self.elems = concat_panels(wing, *rotors)
        self.rank = self.elems.n
        self.rotor_slices = [slice(wing.n, wing.n + rotors[0].n),
                             slice(wing.n + rotors[0].n, self.rank)]
        # implicit wake row: wing TE (upper, lower pair) and blade TEs
        off_w = self.u_inf * self.dt * 0.3 / max(np.linalg.norm(self.u_inf), 1e-9) * 5.0
        ww, wind = te_wake(wing, te_up, off_w, second=te_lo)
        self.wing_te = (te_up, te_lo, dy)
        self.rotor_te = rtes
        wr = []
        winds = [wind]
        for k, te in enumerate(rtes):
            v = self.elems.ver[te]
            r = v.mean(axis=1) - self.centers[k]
            tang = np.cross([0, 0, self.spins[k] * self.omega], r)
            offs = -tang * self.dt * 0.3
            w = np.stack([v[:, 1], v[:, 1] + offs, v[:, 2] + offs, v[:, 2]], axis=1)
            wr.append(abi.PanelSet(w, kind=np.full(len(te), abi.DUST_ELEM_VORTLATT)))
            ind = np.zeros((len(te), 2), dtype=np.int32)
            ind[:, 0] = te + 1
            winds.append(ind)
        self.wake = concat_panels(ww, *wr)
        self.wake.mag = np.zeros(self.wake.n)
        self.n_impl = self.wake.n
        self.impl_ind = np.ascontiguousarray(np.concatenate(winds).astype(np.int32))
        # end vortices: downstream edges of the implicit wake panels
        self.end_vort = abi.LineSet(np.stack([self.wake.ver[:, 1], self.wake.ver[:, 2]], axis=1),
                                    rng.standard_normal(self.wake.n) * 0.05)
        self._particles(n_particles, rng)
        self.set_angle(0.0)

    def _particles(self, n, rng):
        n_w = n // 5
        n_r = (n - n_w) // 2
        cen, dirs = [], []
        for k, (c, sp) in enumerate(zip(self.centers, self.spins)):
            m = n_r if k == 0 else n - n_w - n_r
            age = rng.uniform(0.0, 1.5, m)
            r = np.where(rng.random(m) < 0.5, 0.92 + 0.03 * rng.standard_normal(m),
                         rng.uniform(0.2, 0.95, m))
            blade = rng.integers(0, 3, m)
            psi = sp * (2 * np.pi * blade / 3 - self.omega * age)
            contr = 1.0 - 0.25 * np.minimum(age, 1.0)
            x = c[0] + r * contr * np.cos(psi) + self.u_inf[0] * age
            y = c[1] + r * contr * np.sin(psi)
            z = c[2] - 2.5 * age + 0.01 * rng.standard_normal(m)
            cen.append(np.stack([x, y, z], axis=1))
            d = np.stack([-np.sin(psi) * sp, np.cos(psi) * sp, np.zeros(m)], axis=1)
            dirs.append(d)
        age = rng.uniform(0.0, 1.5, n_w)
        yy = rng.uniform(-3.0, 3.0, n_w)
        xw = 1.0 + self.u_inf[0] * age
        zw = 0.02 * rng.standard_normal(n_w) - 0.1 * age
        cen.append(np.stack([xw, yy, zw], axis=1))
        dirs.append(np.tile([0.0, 1.0, 0.0], (n_w, 1)) * np.sign(yy)[:, None])
        self.cen = np.ascontiguousarray(np.concatenate(cen))
        d = np.concatenate(dirs)
        self.dir = np.ascontiguousarray(d / np.linalg.norm(d, axis=1)[:, None])
        self.mag = np.abs(1e-3 + 2e-4 * rng.standard_normal(n))
        self.r_vortex = np.full(n, 0.04)
        lo = self.cen.min(axis=0) - 0.5
        hi = self.cen.max(axis=0) + 0.5
        lo = np.minimum(lo, self.elems.ver.reshape(-1, 3).min(axis=0) - 0.5)
        hi = np.maximum(hi, self.elems.ver.reshape(-1, 3).max(axis=0) + 0.5)
        self.box_length = 2.0
        self.n_box = tuple(int(np.ceil((hi[d] - lo[d]) / self.box_length)) for d in range(3))
        self.origin = tuple(lo)

    def set_angle(self, ang):
        """Rotate the rotors to azimuth ``ang`` and refresh the body velocity."""
        v = self.rotor_ver0.copy().reshape(-1, 4, 3)
        ub = np.zeros((self.rank, 3))
        base = self.nstatic
        for k, (c, sp) in enumerate(zip(self.centers, self.spins)):
            sl = self.rotor_slices[k]
            nk = sl.stop - sl.start
            vk = v[sl.start - base:sl.stop - base] - c
            vk = _rotz(vk, sp * ang) + c
            v[sl.start - base:sl.stop - base] = vk
            cen = vk.mean(axis=1)
            ub[sl] = np.cross([0, 0, sp * self.omega], cen - c)
        ver = self.elems.ver.copy()
        ver[base:] = v
        self.elems.ver = np.ascontiguousarray(ver)
        self.elems.ub = ub
        if self.elems.uvort is None:
            self.elems.uvort = np.zeros((self.rank, 3))

    def fmm_params(self, degree=4, min_part=8, max_leaf=64):
        from .params import FmmParams
        ll = choose_levels(self.cen, self.box_length, self.n_box, self.origin, max_leaf)
        return FmmParams(box_length=self.box_length, n_box=self.n_box, origin=self.origin,
                         n_octree_levels=ll, min_octree_part=min_part,
                         multipole_degree=degree, rankine_rad=0.1, cutoff_rad=0.001,
                         u_inf=tuple(self.u_inf))

    def loads(self, res, uvort=None, rho=1.225):
        """Integrated loads from the doublet strengths: wing lift from the
        trailing-edge doublet jump (rho |U| sum (mu_up - mu_lo) dy) and rotor
        thrust by Kutta-Joukowski on the bound vortices with the panel-centre
        relative velocity u_inf - ub + uvort (restating
        compute_dforce_jukowski_vortlatt, src/aeroel/mod_vortlatt.f90:502-545,
        without the unsteady term); ``uvort`` (rank, 3) is the step's
        wake-induced velocity at the panel centres (default: the case's)."""
        uv = self.elems.uvort if uvort is None else uvort
        te_up, te_lo, dy = self.wing_te
        lift = rho * np.linalg.norm(self.u_inf) * np.sum((res[te_up] - res[te_lo]) * dy)
        out = [lift]
        ver = self.elems.ver
        for k, sl in enumerate(self.rotor_slices):
            idx = np.arange(sl.start, sl.stop)
            nch = 8
            g = res[idx]
            # upstream element of each chordwise stripe (previous chord row)
            nsb = (sl.stop - sl.start) // 3 // nch
            gb = g.reshape(3, nch, nsb)
            gup = np.concatenate([np.zeros((3, 1, nsb)), gb[:, :-1, :]], axis=1).reshape(-1)
            e1 = (ver[idx, 3] - ver[idx, 0])  # spanwise (bound-vortex) edge
            urel = self.u_inf - self.elems.ub[idx] + uv[idx]
            f = rho * np.cross(urel, e1) * (g - gup)[:, None]
            out.append(f.sum(axis=0)[2])
        return np.asarray(out)


class RingCase:
    """Standalone wake FMM workload: ``n_ring`` particles on a vortex ring
    (radius 1, Gaussian cross-section 0.1) plus ``n_bg`` uniform background
    particles in [-2, 2]^3, tangential circulation vectors of Gaussian
    magnitude (mean 1e-3, sd 1e-4), core radius 0.02 (1M + 100k at the named
    size).  The octree box is [-2, 2]^3 with one level-1 box; the number of
    levels is the smallest that keeps every finest cell at <= ``max_leaf``
    particles."""

    def __init__(self, n_ring=1_000_000, n_bg=100_000, seed=0, core=0.02, max_leaf=64):
        self.cen, self.dir, self.mag = ring_particles(n_ring, n_bg, seed=seed)
        self.n = self.mag.shape[0]
        self.r_vortex = np.full(self.n, core)
        self.core = core
        self.levels = choose_levels(self.cen, 4.0, (1, 1, 1), (-2.0, -2.0, -2.0), max_leaf)

    def fmm_params(self, degree=4, precision=abi.DUST_PREC_FP64, min_part=8):
        from .params import FmmParams
        return FmmParams(box_length=4.0, origin=(-2.0, -2.0, -2.0),
                         n_octree_levels=self.levels, min_octree_part=min_part,
                         multipole_degree=degree, rankine_rad=self.core, precision=precision)

    def truth_order(self, n_tgt, seed=1):
        """A permutation that puts a seeded random subset of ``n_tgt``
        particles first (the direct-sum targets); the FMM result does not
        depend on the particle order."""
        rng = np.random.default_rng(seed)
        sub = rng.choice(self.n, n_tgt, replace=False)
        rest = np.setdiff1d(np.arange(self.n), sub, assume_unique=False)
        return np.concatenate([sub, rest])

    def permuted(self, order):
        c = RingCase.__new__(RingCase)
        c.__dict__.update(self.__dict__)
        c.cen = np.ascontiguousarray(self.cen[order])
        c.dir = np.ascontiguousarray(self.dir[order])
        c.mag = np.ascontiguousarray(self.mag[order])
        c.r_vortex = np.ascontiguousarray(self.r_vortex[order])
        return c


class EllipsoidCase:
    """Mixed-precision dense-solve workload: closed ellipsoid (semi-axes 4, 1,
    0.5) of ``n_target`` surface panels (source + doublet, Dirichlet rows) in
    a seeded random rigid rotation, with ``nrhs`` right-hand sides from
    seeded random unit freestream directions.

    The Dirichlet right-hand side is linear in the freestream u
    (b_i = sum_j sou_ij n_j . (ub_j - u - uvort_j), mod_surfpan.f90:448-481),
    so the three assemblies with a unit body velocity along x, y, z (u = 0)
    give the columns G = [b_x b_y b_z] and the right-hand side of a
    freestream u is -G u."""

    def __init__(self, n_target=16384, nrhs=64, seed=0):
        # n_u x n_lat = n_target panels when n_target is 2 * a square
        # (16,384 = 128 x 128: 16,128 quads and 256 cap triangles)
        side = int(round(np.sqrt(n_target)))
        kw = dict(n_u=side, n_lat=side) if side * side == n_target and side % 2 == 0 else {}
        self.body = ellipsoid(n_target=n_target, axes=(4.0, 1.0, 0.5), seed=seed, **kw)
        self.n = self.body.n
        rng = np.random.default_rng(seed + 1000)
        U = rng.standard_normal((3, nrhs))
        self.U = U / np.linalg.norm(U, axis=0)[None, :]
        self.nrhs = nrhs

    def fmm_params(self):
        from .params import FmmParams
        return FmmParams(u_inf=(0.0, 0.0, 0.0))

    def unit_ub(self, d):
        ub = np.zeros((self.n, 3))
        ub[:, d] = 1.0
        return ub


class RotorFuselageCase:
    """Learned-preconditioner workload: a 4-blade vortex-lattice rotor
    (radius 1, 30 x 8 panels per blade, linear twist -8 deg) above a closed
    cylindrical fuselage of about 6,000 surface panels (static), about 7k
    unknowns.  ``system(seed)`` draws one time step of a plain-method run:
    rotor azimuth uniform in one blade passage, rpm within +-20 % of the
    nominal, inflow of 2 m/s at an angle within +-30 deg of the rotor axis.
    The freestream enters as a body velocity (ub = omega x r - inflow for the
    rotor, -inflow for the fuselage) with u_inf = 0, so one linear-system
    handle (static fuselage LU built once) serves every draw."""

    def __init__(self, n_fus=6000, n_blades=4, n_span=30, n_chord=8, omega=40.0):
        self.n_fus, self.n_blades, self.n_span, self.n_chord = n_fus, n_blades, n_span, n_chord
        self.omega0 = omega
        els, nst = rotor_fuselage(n_fus=n_fus, n_blades=n_blades, n_span=n_span,
                                  n_chord=n_chord, phase=0.0, omega=omega)
        self.nstatic = nst
        self.rank = els.n

    def system(self, seed):
        rng = np.random.default_rng(seed)
        phase = rng.uniform(0.0, 2.0 * np.pi / self.n_blades)
        omega = self.omega0 * rng.uniform(0.8, 1.2)
        ang = np.deg2rad(rng.uniform(-30.0, 30.0))
        az = rng.uniform(0.0, 2.0 * np.pi)
        inflow = 2.0 * np.array([np.sin(ang) * np.cos(az), np.sin(ang) * np.sin(az),
                                 -np.cos(ang)])
        els, nst = rotor_fuselage(n_fus=self.n_fus, n_blades=self.n_blades,
                                  n_span=self.n_span, n_chord=self.n_chord, phase=phase,
                                  omega=omega, inflow=inflow)
        ub = els.ub.copy()
        ub[:nst] = -inflow
        els.ub = ub
        els.uvort = np.zeros((els.n, 3))
        return els

    def fmm_params(self):
        from .params import FmmParams
        return FmmParams(u_inf=(0.0, 0.0, 0.0), rankine_rad=0.1)


class WingWakeCase:
    """Flat rectangular vortex-lattice wing (span 10, chord 1, 40 x 10
    panels: 400 unknowns, all static) at 5 degrees of incidence in a 1 m/s
    stream, with the reference's panel wake (n_wake_panels rows behind the
    trailing edge) shedding one particle per stripe per step once it is
    full (classical complete_wake branch).  Trailing-edge topology as the
    pre-processor builds it for a structured strip (build_te_parametric,
    src/geo/mod_build_geo.f90:2244-2310): stripe i spans trailing-edge
    points (i + 1, i), neighbours i +- 1 with orientation 1, generating
    element = the strip's last chordwise panel; t_te the chordwise unit
    vector of the trailing panels' side edges; first-row scaling 0.3
    (implicit_panel_scale).  Particle core 0.1 chord for every particle
    (vortex_rad = rankine_rad = 0.1, k_vortex_rad = 0)."""

    def __init__(self, span=10.0, chord=1.0, n_span=40, n_chord=10, alpha_deg=5.0, dt=0.05,
                 n_wake_panels=4, n_wake_particles=None, steps=200, u_inf=(1.0, 0.0, 0.0),
                 box_min=(-1.0, -8.0, -8.0), box_max=(15.0, 8.0, 8.0)):
        x = np.linspace(0.0, chord, n_chord + 1)
        y = np.linspace(-span / 2, span / 2, n_span + 1)
        X, Y = np.meshgrid(x, y, indexing="ij")
        P = np.stack([X, Y, np.zeros_like(X)], axis=2)
        a = np.deg2rad(alpha_deg)
        R = np.array([[np.cos(a), 0, np.sin(a)], [0, 1, 0], [-np.sin(a), 0, np.cos(a)]])
        P = P @ R.T
        ver = _quad_grid(P)  # panel (i, j) at index i * n_span + j
        self.body = abi.PanelSet(ver, kind=np.full(len(ver), abi.DUST_ELEM_VORTLATT))
        self.rank = self.nstatic = len(ver)
        ns = n_span
        i = np.arange(1, ns + 1)
        self.ii = np.stack([i + 1, i], axis=1).astype(np.int32)
        self.neigh = np.stack([i + 1, i - 1], axis=1).astype(np.int32)
        self.neigh[-1, 0] = 0
        self.neigh[0, 1] = 0
        self.neigh_o = np.ones((ns, 2), dtype=np.int32)
        self.neigh_o[-1, 0] = 0
        self.neigh_o[0, 1] = 0
        self.gen = np.zeros((ns, 2), dtype=np.int32)
        self.gen[:, 0] = (n_chord - 1) * n_span + np.arange(ns) + 1
        self.te_pts = np.ascontiguousarray(P[n_chord])
        t = P[n_chord] - P[n_chord - 1]
        self.te_dir = np.ascontiguousarray(t / np.linalg.norm(t, axis=1)[:, None])
        self.te_scaling = np.full(ns + 1, 0.3)
        self.u_inf = np.asarray(u_inf, dtype=np.float64)
        self.dt = float(dt)
        self.steps = int(steps)
        self.n_wake_panels = int(n_wake_panels)
        self.box_min = np.asarray(box_min, dtype=np.float64)
        self.box_max = np.asarray(box_max, dtype=np.float64)
        self.n_slots = int(n_wake_particles or ns * (steps + 1))
        self.vortex_rad = 0.1

    def wake_params(self):
        return abi.wake_params(len(self.ii), len(self.te_pts), self.n_wake_panels, self.dt,
                               self.box_min, self.box_max, self.u_inf,
                               vortex_rad=self.vortex_rad, k_vortex_rad=0.0)

    def fmm_params(self, levels=6, degree=4, precision=abi.DUST_PREC_FP64):
        from .params import FmmParams
        side = float(np.max(self.box_max - self.box_min))
        return FmmParams(box_length=side, n_box=(1, 1, 1), origin=tuple(self.box_min),
                         n_octree_levels=levels, min_octree_part=5, multipole_degree=degree,
                         rankine_rad=self.vortex_rad, cutoff_rad=0.001, vortstretch=True,
                         diffusion=True, nu_inf=1.8e-5 / 1.225,
                         u_inf=tuple(float(v) for v in self.u_inf), precision=precision)

    def update_params(self):
        return abi.update_params(self.dt, self.box_min, self.box_max, 1, True, True, False, 0.0)
