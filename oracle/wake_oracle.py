"""The reference's panel wake and its particle shedding, restated in numpy
(test infrastructure only: tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg use it as the checker; the product never does).

Follows src/aeroel/mod_wake.f90:
  initialize_wake   :468-512   first two rows of points, len = 1
  load_wake         :597-778   state from a result file
  update_wake       :881-892   first-row intensities from the solution
                    :894-939   velocities at the wake points, rows moved,
                                points_end of a full wake
                    :1128-1176 length, end_pan_idou, intensities shifted
  complete_wake     :1247-1292 first two rows from the trailing edge
                    :1358-2010 shedding (the classical and refine_wake
                                branch, :1797-2010; interpolate_wake and
                                join_te are not restated)
                    :2091-2103 end vortices of a full wake
compute_vel_from_all (:2109-2150) is the caller's ``vel_fn``.

Every expression keeps the reference's operand order (norm2 as the square
root of the sum of squares); arrays are 0-based, the topology (ii, neigh,
neigh_o, gen) 1-based as the reference stores it.
"""
import numpy as np


def _norm(v):
    return np.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])


def _cross(a, b):
    return np.array([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2],
                     a[0] * b[1] - a[1] * b[0]])


class PanelWake:
    """t_wake's panel part.  ``prm``: abi.WakeParams (or an object with the
    same fields); ii, neigh, neigh_o, gen: (n_stripes, 2) ints, 1-based."""

    def __init__(self, prm, ii, neigh, neigh_o, gen, te_pts, te_dir, te_scaling, te_vel=None):
        self.p = prm
        self.ns, self.npt, self.nmax = int(prm.n_stripes), int(prm.n_points), int(prm.n_wake_panels)
        self.ii = np.asarray(ii, dtype=np.int64).reshape(self.ns, 2)
        self.neigh = np.asarray(neigh, dtype=np.int64).reshape(self.ns, 2)
        self.neigh_o = np.asarray(neigh_o, dtype=np.int64).reshape(self.ns, 2)
        self.gen = np.asarray(gen, dtype=np.int64).reshape(self.ns, 2)
        self.pts = np.zeros((self.nmax + 1, self.npt, 3))
        self.pvel = np.zeros((self.nmax + 1, self.npt, 3))
        self.idou = np.zeros((self.nmax, self.ns))
        self.last = np.zeros(self.ns)
        self.endi = np.zeros(self.ns)
        self.pend = np.zeros((self.npt, 3))
        self.len = 1
        self.full = False
        self.attached = False  # end vortices attached (:2091-2103, load_wake :766-777)
        self._te_rows(te_pts, te_dir, te_scaling, te_vel, normalised_below_min=False)

    # ------------------------------------------------------------ rows 1-2
    def _te_rows(self, te_pts, te_dir, te_scaling, te_vel, normalised_below_min):
        """initialize_wake :484-512 (unnormalised below min_vel_at_te) /
        complete_wake :1258-1282 (normalised)."""
        p = self.p
        te_pts = np.asarray(te_pts, dtype=np.float64).reshape(self.npt, 3)
        te_dir = np.asarray(te_dir, dtype=np.float64).reshape(self.npt, 3)
        sc = np.asarray(te_scaling, dtype=np.float64).reshape(self.npt)
        tv = (np.zeros((self.npt, 3)) if te_vel is None
              else np.asarray(te_vel, dtype=np.float64).reshape(self.npt, 3))
        wind = np.array([p.u_inf[0], p.u_inf[1], p.u_inf[2]], dtype=np.float64)
        dt, nd = float(p.dt), float(p.ndt_update_wake)
        self.pts[0] = te_pts
        for ip in range(self.npt):
            dist = te_dir[ip]
            w = _norm(wind - tv[ip])
            if w > p.min_vel_at_te:
                self.pts[1, ip] = self.pts[0, ip] + dist * sc[ip] * w * dt * nd / _norm(dist)
            elif normalised_below_min:
                self.pts[1, ip] = (self.pts[0, ip] + dist * sc[ip] * p.min_vel_at_te * dt * nd
                                   / _norm(dist))
            else:
                self.pts[1, ip] = self.pts[0, ip] + dist * sc[ip] * p.min_vel_at_te * dt * nd

    # ------------------------------------------------------------ load_wake
    def set_state(self, length, points, point_vel, idou, last):
        """load_wake :620-633, :764 (len = rows of idou, full when it
        reaches n_wake_panels) and :730 (last_pan_idou)."""
        self.len = int(length)
        self.pts[:self.len + 1] = np.asarray(points).reshape(self.len + 1, self.npt, 3)
        self.pvel[:self.len + 1] = (0.0 if point_vel is None
                                    else np.asarray(point_vel).reshape(self.len + 1, self.npt, 3))
        self.idou[:self.len] = np.asarray(idou).reshape(self.len, self.ns)
        self.last[:] = np.asarray(last).reshape(self.ns)
        self.full = self.len == self.nmax
        self.attached = self.full

    # ------------------------------------------------------------ elements
    def panels(self):
        """Wake panels of rows 1..len in pan_p order: (len*ns, 4, 3) vertices
        (p1, p2 of the row, p2, p1 of the next, :1285-1289) and intensities."""
        ver = np.zeros((self.len * self.ns, 4, 3))
        for r in range(self.len):
            for iw in range(self.ns):
                p1, p2 = self.ii[iw] - 1
                ver[r * self.ns + iw] = [self.pts[r, p1], self.pts[r, p2],
                                         self.pts[r + 1, p2], self.pts[r + 1, p1]]
        return ver, self.idou[:self.len].reshape(-1).copy()

    def end_vortices(self):
        """End vortices of a full wake (:2091-2103): (ns, 2, 3), mag =
        last_pan_idou; empty until complete_wake of a full wake has attached
        them (before that their mag pointers are not associated and
        compute_vel_vortline gives 0, src/aeroel/mod_vortline.f90:138)."""
        if not self.attached:
            return np.zeros((0, 2, 3)), np.zeros(0)
        ver = np.zeros((self.ns, 2, 3))
        for iw in range(self.ns):
            p1, p2 = self.ii[iw] - 1
            ver[iw] = [self.pts[self.len, p1], self.pts[self.len, p2]]
        return ver, self.last.copy()

    # ------------------------------------------------------------ update_wake
    def set_first_row(self, res):
        """:884-892: mag(gen 1) - mag(gen 2) (gen 2 = 0: mag(gen 1))."""
        res = np.asarray(res, dtype=np.float64)
        for iw in range(self.ns):
            g1, g2 = self.gen[iw]
            self.idou[0, iw] = res[g1 - 1] - res[g2 - 1] if g2 > 0 else res[g1 - 1]

    def update(self, vel_fn):
        """:894-939 and :1128-1176.  vel_fn(points (m, 3)) -> velocities
        (compute_vel_from_all + wind) of the wake points, all evaluated on
        the state before any row moves."""
        p = self.p
        dt, nd = float(p.dt), float(p.ndt_update_wake)
        if self.len == self.nmax:
            self.full = True  # :882
        point_old = self.pts.copy()
        np_ = self.len + 1 + (0 if self.full else 1)
        rows = list(range(3, np_ + 1))  # ipan, 1-based
        src = [point_old[ipan - 2] for ipan in rows]
        if self.full:
            src.append(point_old[self.len])
        if src:
            v = vel_fn(np.concatenate(src, axis=0)).reshape(len(src), self.npt, 3)
        for k, ipan in enumerate(rows):
            self.pvel[ipan - 1] = v[k]
            for iw in range(self.npt):
                if ipan != 3:
                    self.pts[ipan - 1, iw] = point_old[ipan - 2, iw] + v[k, iw] * dt * nd
                else:
                    self.pts[ipan - 1, iw] = point_old[ipan - 2, iw] + v[k, iw] * dt
        if self.full:
            ve = v[len(rows)]
            for iw in range(self.npt):
                self.pend[iw] = point_old[self.len, iw] + ve[iw] * dt * nd
        # :1132-1176
        if not self.full:
            self.len += 1
        self.endi[:] = self.idou[self.len - 1]
        for ipan in range(self.len, 1, -1):
            self.idou[ipan - 1] = self.idou[ipan - 2]

    # ----------------------------------------------------------- complete_wake
    def complete_rows(self, te_pts, te_dir, te_scaling, te_vel=None):
        """:1247-1292."""
        self._te_rows(te_pts, te_dir, te_scaling, te_vel, normalised_below_min=True)

    def shed(self, cen, dir_, mag, rv, vel, free):
        """:1358-2010 (classical / refine_wake branch): in place on the slot
        arrays (cen, dir, vel (n, 3); mag, rv (n,); free (n,) 0/1).  Returns
        the number of particles shed; raises on a slot shortage (:1985).
        Attaches the end vortices of a full wake."""
        if not self.full:
            return 0
        self.attached = True
        p = self.p
        nm = self.nmax
        lo = np.array([p.box_min[0], p.box_min[1], p.box_min[2]])
        hi = np.array([p.box_max[0], p.box_max[1], p.box_max[2]])
        nslot = len(mag)
        k = 0
        shed = 0

        def take(pos, m, pv, area, n_sub):
            nonlocal k, shed
            ip = k
            while ip < nslot and not free[ip]:
                ip += 1
            if ip >= nslot:
                raise RuntimeError("Exceeding the maximum number of wake particles")
            free[ip] = 0
            k = ip + 1
            shed += 1
            nrm = _norm(pv)
            mag[ip] = nrm / float(n_sub) if n_sub else nrm
            dir_[ip] = pv / nrm if nrm > 1.0e-13 else pv
            cen[ip] = pos
            rv[ip] = (p.k_vortex_rad * np.sqrt(2.0 * area) if p.k_vortex_rad >= 1e-10
                      else p.vortex_rad)
            if vel is not None:
                vel[ip] = 0.5 * (self.pvel[nm, p1] + self.pvel[nm, p2])

        for iw in range(self.ns):
            p1, p2 = self.ii[iw] - 1
            partvec = np.zeros(3)
            # left side :1804-1819
            d = self.pts[nm, p1] - self.pend[p1]
            chord_side_len = _norm(d)
            if self.neigh[iw, 0] > 0:
                ave = self.endi[iw] - float(self.neigh_o[iw, 0]) * self.endi[self.neigh[iw, 0] - 1]
                ave = ave / 2.0
            else:
                ave = self.endi[iw]
            partvec = partvec + d * ave
            # right side :1822-1835
            d = -self.pts[nm, p2] + self.pend[p2]
            if self.neigh[iw, 1] > 0:
                ave = self.endi[iw] - float(self.neigh_o[iw, 1]) * self.endi[self.neigh[iw, 1] - 1]
                ave = ave / 2.0
            else:
                ave = self.endi[iw]
            partvec = partvec + d * ave
            # end side :1838-1842
            d = self.pend[p1] - self.pend[p2]
            span_side_len = _norm(d)
            ave = self.endi[iw] - self.last[iw]
            self.last[iw] = self.endi[iw]
            partvec = partvec + d * ave
            if p.refine_wake:  # :1844-1923
                kr = float(p.k_refine)
                if chord_side_len >= span_side_len:
                    mx, mn = chord_side_len, span_side_len
                    n_chord = int(np.ceil(mx / (mn / kr)))
                    n_span = int(p.k_refine)
                    step_chord, step_span = mx / float(n_chord), mn / float(n_span)
                else:
                    mx, mn = span_side_len, chord_side_len
                    n_chord = int(p.k_refine)
                    n_span = int(np.ceil(mx / (mn / kr)))
                    step_chord, step_span = mn / float(n_chord), mx / float(n_span)
                for ic in range(1, n_chord + 1):
                    for is_ in range(1, n_span + 1):
                        pos = (self.pts[nm, p1]
                               + (float(ic) - 0.5) / float(n_chord) * (self.pend[p1] - self.pts[nm, p1])
                               + (float(is_) - 0.5) / float(n_span) * (self.pts[nm, p2] - self.pts[nm, p1]))
                        area = step_chord * step_span
                        if np.all(pos >= lo) and np.all(pos <= hi):
                            take(pos, None, partvec, area, n_span * n_chord)
            else:  # :1925-1992
                pos = (self.pend[p1] + self.pend[p2] + self.pts[nm, p1] + self.pts[nm, p2]) / 4.0
                area = _norm(_cross(self.pend[p1] - self.pts[nm, p2],
                                    self.pend[p2] - self.pts[nm, p2]))
                if np.all(pos >= lo) and np.all(pos <= hi):
                    take(pos, None, partvec, area, 0)
        return shed


def vel_from_all(O, fprm, pts, body, wake_ver, wake_mag, end_ver, end_mag, cen, dir_, mag, rv):
    """compute_vel_from_all + wind (mod_wake.f90:2109-2169) with the C
    oracle: body panels (abi.PanelSet with mag), wake panels (vortex rings),
    end vortices and the particles, then u_inf."""
    from dust_b200 import abi
    wk = abi.PanelSet(wake_ver, mag=wake_mag) if len(wake_ver) else abi.empty_panels()
    ev = abi.LineSet(end_ver, end_mag) if len(end_ver) else abi.empty_lines()
    v = O.elements_vel(fprm, pts, abi.elements_struct(body, wk, ev))
    if len(mag):
        v = v + O.points_uvort(fprm, pts, cen, dir_, mag, rv)
    return v


class OracleWakeRun:
    """The time loop of a static body with a panel wake on the CPU oracle,
    in the reference's order (src/dust.f90:510-1160): prepare_wake (live
    particles in slot order), uvort at the body centres (particles + end
    vortices), assemble_linsys + solve_linsys (the block LU of the oracle,
    static system), update_wake (first wake row, particle velocities by the
    FMM with the body, wake panels and end vortices, wake points by
    compute_vel_from_all), complete_wake (particles moved, optional
    penetration avoidance, wake rows, shedding).  ``case`` as
    dust_b200.synth.WingWakeCase, ``fprm`` an FmmParams."""

    def __init__(self, O, case, fprm, pa=None):
        from dust_b200 import abi
        self.O, self.abi, self.case, self.fprm, self.pa = O, abi, case, fprm, pa
        c = case
        self.w = PanelWake(c.wake_params(), c.ii, c.neigh, c.neigh_o, c.gen, c.te_pts, c.te_dir,
                           c.te_scaling)
        ns = c.n_slots
        self.cen, self.dir, self.vel = np.zeros((ns, 3)), np.zeros((ns, 3)), np.zeros((ns, 3))
        self.str, self.rot = np.zeros((ns, 3)), np.zeros((ns, 3))
        self.mag, self.rv = np.zeros(ns), np.zeros(ns)
        self.free = np.ones(ns, dtype=np.int32)
        self.upd = c.update_params()
        wv, wm = self.w.panels()
        self.init_wake = abi.PanelSet(wv, kind=np.full(len(wv), abi.DUST_ELEM_VORTLATT), mag=wm)
        self.centres = c.body.ver.mean(axis=1)
        self.res = None

    def step(self):
        O, abi, c, w = self.O, self.abi, self.case, self.w
        live = np.nonzero(self.free == 0)[0]
        lc, ld, lm, lr = self.cen[live], self.dir[live], self.mag[live], self.rv[live]
        ev, em = w.end_vortices()
        evs = abi.LineSet(ev, em) if len(em) else None
        body = abi.PanelSet(c.body.ver, c.body.n_ver, c.body.kind)
        body.uvort = (O.points_uvort(self.fprm, self.centres, lc, ld, lm, lr, evs) if len(live)
                      else O.points_uvort(self.fprm, self.centres, np.zeros((0, 3)),
                                          np.zeros((0, 3)), np.zeros(0), np.zeros(0), evs))
        wv, wm = w.panels()
        wnow = abi.PanelSet(wv, kind=np.full(len(wv), abi.DUST_ELEM_VORTLATT), mag=wm)
        n = c.rank
        _, _, res = O.linsys_run(self.fprm, n, c.nstatic, body, body,
                                 (self.init_wake, len(c.ii), c.gen), (wnow, len(c.ii), c.gen))
        self.res = res
        w.set_first_row(res)
        body.mag = res
        wv, wm = w.panels()
        ev, em = w.end_vortices()
        if len(live):
            wk = abi.PanelSet(wv, kind=np.full(len(wv), abi.DUST_ELEM_VORTLATT), mag=wm)
            els = abi.elements_struct(body, wk, abi.LineSet(ev, em) if len(em) else None)
            v, s, r, _ = O.fmm_apply(self.fprm, lc, ld, lm, lr, els)
            self.vel[live], self.str[live], self.rot[live] = v, s, r
        w.update(lambda pts: vel_from_all(O, self.fprm, pts, body, wv, wm, ev, em, lc, ld, lm, lr))
        if len(live):
            if self.pa is not None:
                (self.cen, self.dir, self.vel, self.str, self.free, _) = O.particles_update_pa(
                    self.upd, self.pa, body, self.cen, self.dir, self.mag, self.rv, self.vel,
                    self.str, self.rot, self.free)
            else:
                (self.cen, self.dir, self.str, self.free, _) = O.particles_update(
                    self.upd, self.cen, self.dir, self.mag, self.vel, self.str, self.rot,
                    self.free)
        w.complete_rows(c.te_pts, c.te_dir, c.te_scaling)
        return w.shed(self.cen, self.dir, self.mag, self.rv, self.vel, self.free)

    def particles(self):
        live = np.nonzero(self.free == 0)[0]
        return self.cen[live], self.dir[live] * self.mag[live][:, None], self.rv[live]
