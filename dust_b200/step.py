"""One aerodynamic timestep of the hot path, in the reference's order.

The reference's time loop (src/dust.f90:510-1160) runs, per step:
prepare_wake (sort_particles + calculate_multipole, mod_wake.f90:797-801),
assemble_linsys (uvort by direct sum over particles + end vortices, rows,
wake terms; dust.f90:620), solve_linsys (dust.f90:647-649) and
update_wake -> apply_multipole (mod_wake.f90:1115-1118).  ``Stepper`` runs
the same sequence on the GPU through the C ABI:

  1. uvort at every implicit element centre  (dust_points_uvort[_device])
  2. dust_linsys_assemble[_device]
  2b. the pressure integral equation of the surface panels, when there are
     any (dust_pressure_assemble[_device] every step, _solve from the second
     step: dust.f90:621, 641-643)
  3. dust_linsys_solve[_device]              (doublet intensities)
  4. wake bookkeeping: implicit wake panel mag = mag(ind1) - mag(ind2)
     (update_wake, mod_wake.f90:881-889)
  5. dust_fmm_apply[_device]                 (particle velocity, stretching,
                                              div-filter curl: tree build,
                                              multipoles, L2P, P2P, elements)
  6. dust_particles_update[_device]          (complete_wake's particle loop:
                                              explicit Euler move, box culling,
                                              direction renewal; mod_wake.f90:
                                              1309-1355), when ``advect``

Two drivers: ``HostStepper`` takes host (pinned) arrays and lets the library
copy them every step (end-to-end); ``DeviceStepper`` keeps everything in HBM
(torch tensors as plumbing) and calls the *_device entry points.
"""
import ctypes as C

import numpy as np

from . import abi
from ._lib import check, lib
from .linsys import Linsys, Pressure
from .octree import Octree


def update_params_for(case, params):
    """The particles' Euler step of the case: dt, a particle box that holds
    the whole octree box (no particle is freed by the move), the model
    switches of the FMM; divergence filtering off, as the reference runs it
    (sim_param%use_divfilt is never assigned, mod_sim_param.f90:450-451)."""
    lo = np.asarray(params.origin, dtype=np.float64)
    hi = lo + np.asarray(params.n_box, dtype=np.float64) * params.box_length
    return abi.update_params(case.dt, lo, hi, 1, params.vortstretch, params.diffusion, False,
                             0.0)


class HostStepper:
    def __init__(self, case, params, mode=abi.DUST_SOLVE_LU64, out=None, advect=False,
                 fmm_uvort=False, uvort_params=None, pressure=True):
        """``out``: optional (vel, stretch, rotu) host arrays the particle
        outputs are written to every step (e.g. page-locked buffers);
        ``advect``: move the particles at the end of each step;
        ``fmm_uvort``: uvort through the particles' FMM (prepare, points,
        finish: the particles are uploaded once per step) instead of the
        direct sum; ``uvort_params``: parameters of the direct uvort sum when
        they differ from the FMM's (e.g. an FP64 uvort beside an FP32C FMM)."""
        self.fmm_uvort = fmm_uvort
        self.case = case
        self.params = params
        self.uvort_params = uvort_params if uvort_params is not None else params
        self.mode = mode
        self.out = out
        self.advect = advect
        self.upd = update_params_for(case, params)
        c = case
        self.free = np.zeros(c.mag.shape[0], dtype=np.int32)
        self.ls = Linsys(params, c.rank, c.nstatic, c.elems, c.wake, c.n_impl, c.impl_ind)
        self.pr = (Pressure(self.ls) if pressure and np.any(c.elems.kind == abi.DUST_ELEM_SURFPAN)
                   else None)
        self.vel_prev = np.zeros((c.mag.shape[0], 3))
        self.steps_done = 0
        self.oc = Octree(params)
        self.ind = c.impl_ind.astype(np.int64) - 1

    def step(self):
        """Returns (res, vel, stretch, rotu) as host arrays."""
        c, p = self.case, self.params
        cen_el = c.elems.ver.mean(axis=1)  # overwritten below for triangles
        nv = c.elems.n_ver
        tri = nv == 3
        if tri.any():
            cen_el[tri] = c.elems.ver[tri, :3].mean(axis=1)
        ps = self.uvort_params.struct()
        evs = c.end_vort.struct()
        uv = np.empty((c.rank, 3))
        cen_el = np.ascontiguousarray(cen_el)
        pterm = None
        if self.fmm_uvort:
            self.oc.prepare(c.cen, c.dir, c.mag, c.r_vortex, cen_el)
            uv = self.oc.points_uvort(c.end_vort)
        elif self.pr is not None:
            # the pressure equation's particle term in the same pass as uvort,
            # with the particles' velocities of the previous update
            pterm = np.empty(c.rank)
            check(lib().dust_points_uvort_pressure(
                C.byref(ps), c.rank, abi.dptr(cen_el), c.mag.shape[0], abi.dptr(c.cen),
                abi.dptr(c.dir), abi.dptr(c.mag), abi.dptr(c.r_vortex), abi.dptr(self.vel_prev),
                C.byref(evs), abi.dptr(uv), abi.dptr(pterm)), "dust_points_uvort_pressure")
        else:
            check(lib().dust_points_uvort(C.byref(ps), c.rank, abi.dptr(cen_el),
                                          c.mag.shape[0], abi.dptr(c.cen), abi.dptr(c.dir),
                                          abi.dptr(c.mag), abi.dptr(c.r_vortex), C.byref(evs),
                                          abi.dptr(uv)), "dust_points_uvort")
        c.elems.uvort = uv
        self.ls.assemble_linsys(c.elems, c.wake, c.n_impl, c.impl_ind)
        if self.pr is not None:
            # assemble_pressure_sys every step, solve_pressure_sys from the
            # second (dust.f90:621, 641-643); the body is at rest in the
            # frame of its Bernoulli sources, the particles' velocities are
            # those of the previous update
            if pterm is not None:
                self.pr.assemble_terms(None, pterm)
            else:
                self.pr.assemble(None, (c.cen, c.dir, c.mag, c.r_vortex), self.vel_prev)
            if self.steps_done > 0:
                self.res_pres = self.pr.solve()
        res, rep = self.ls.solve_linsys(self.mode)
        self.last_report = rep
        c.elems.mag = res
        m2 = np.where(self.ind[:, 1] >= 0, res[np.maximum(self.ind[:, 1], 0)], 0.0)
        c.wake.mag = res[self.ind[:, 0]] - m2
        els = abi.elements_struct(c.elems, c.wake, c.end_vort)
        if self.fmm_uvort:
            vel, st, ro = self.oc.finish(els, out=self.out)
        else:
            vel, st, ro = self.oc.apply_multipole(c.cen, c.dir, c.mag, c.r_vortex, els,
                                                  out=self.out)
        self.vel_prev = vel
        self.steps_done += 1
        if self.advect:
            nf = C.c_int(0)
            check(lib().dust_particles_update(C.byref(self.upd), c.mag.shape[0], abi.dptr(c.cen),
                                              abi.dptr(c.dir), abi.dptr(c.mag), abi.dptr(vel),
                                              abi.dptr(st), abi.dptr(ro),
                                              self.free.ctypes.data_as(C.POINTER(C.c_int)),
                                              C.byref(nf)), "dust_particles_update")
        return res, vel, st, ro


class DeviceStepper:
    """All per-step inputs resident in HBM; library calls on device pointers."""

    def __init__(self, case, params, mode=abi.DUST_SOLVE_LU64, device="cuda", advect=False,
                 fmm_uvort=False, uvort_params=None, pressure=True):
        import torch
        self.torch = torch
        self.case = case
        self.params = params
        self._ups = (uvort_params if uvort_params is not None else params).struct()
        self.mode = mode
        self.advect = advect
        self.fmm_uvort = fmm_uvort
        self.upd = update_params_for(case, params)
        c = case
        dev = torch.device(device)
        T = lambda a, dt=torch.float64: torch.as_tensor(np.ascontiguousarray(a), dtype=dt,
                                                        device=dev)
        self.cen = T(c.cen)
        self.dir = T(c.dir)
        self.mag = T(c.mag)
        self.rv = T(c.r_vortex)
        self.n = c.mag.shape[0]
        self.ever = T(c.elems.ver)
        self.env = T(c.elems.n_ver, torch.int32)
        self.ekind = T(c.elems.kind, torch.int32)
        self.eub = T(c.elems.ub)
        self.euv = torch.zeros((c.rank, 3), dtype=torch.float64, device=dev)
        self.emag = torch.zeros(c.rank, dtype=torch.float64, device=dev)
        self.ecen = torch.zeros((c.rank, 3), dtype=torch.float64, device=dev)
        self.wver = T(c.wake.ver)
        self.wnv = T(c.wake.n_ver, torch.int32)
        self.wkind = T(c.wake.kind, torch.int32)
        self.wmag = torch.zeros(c.wake.n, dtype=torch.float64, device=dev)
        self.impl = T(c.impl_ind, torch.int32)
        ind = c.impl_ind.astype(np.int64) - 1
        self.i1 = T(ind[:, 0], torch.int64)
        self.i2 = T(np.maximum(ind[:, 1], 0), torch.int64)
        self.has2 = T((ind[:, 1] >= 0).astype(np.float64))
        self.lver = T(c.end_vort.ver)
        self.lmag = T(c.end_vort.mag)
        self.vel = torch.zeros((self.n, 3), dtype=torch.float64, device=dev)
        self.str = torch.empty((self.n, 3), dtype=torch.float64, device=dev)
        self.rot = torch.empty((self.n, 3), dtype=torch.float64, device=dev)
        self.res = torch.empty(c.rank, dtype=torch.float64, device=dev)
        self.free = torch.zeros(self.n, dtype=torch.int32, device=dev)
        self.n_freed = torch.zeros(1, dtype=torch.int32, device=dev)
        self.ls = Linsys(params, c.rank, c.nstatic, c.elems, c.wake, c.n_impl, c.impl_ind)
        # the pressure integral equation of the surface panels
        # (mod_pressure_equation.f90), assembled every step, solved from the
        # second (dust.f90:621, 641-643)
        self.pr = (Pressure(self.ls) if pressure and np.any(c.elems.kind == abi.DUST_ELEM_SURFPAN)
                   else None)
        if self.pr is not None:
            self.res_pres = torch.zeros(self.pr.n_sp, dtype=torch.float64, device=dev)
            self.pterm = torch.zeros(c.rank, dtype=torch.float64, device=dev)
        # with a direct uvort the pressure equation's particle term is
        # evaluated in the same pass (dust_points_uvort_pressure_device, in
        # the uvort's precision)
        self.fused_pterm = self.pr is not None and not fmm_uvort
        self.steps_done = 0
        self.oc = Octree(params)
        self._ps = params.struct()
        self.phase_events = False
        self.events = []

    def _mark(self):
        if self.phase_events:
            e = self.torch.cuda.Event(enable_timing=True)
            e.record()
            self.events.append(e)

    @staticmethod
    def _p(t, ctype=C.c_double):
        return C.cast(C.c_void_p(t.data_ptr()), C.POINTER(ctype))

    def step(self):
        torch = self.torch
        c = self.case
        P = self._p
        stream = torch.cuda.current_stream().cuda_stream
        self.events = []
        self._mark()
        el = abi.Panels(c.rank, P(self.env, C.c_int), P(self.ekind, C.c_int), P(self.ever),
                        P(self.emag), P(self.eub), P(self.euv))
        check(lib().dust_panels_centres_device(C.byref(el), P(self.ecen), C.c_void_p(stream)),
              "dust_panels_centres_device")
        lines = abi.Lines(c.end_vort.n, P(self.lver), P(self.lmag))
        if self.fmm_uvort:
            # prepare_wake: the particles enter the tree once per step
            check(lib().dust_fmm_prepare_device(self.oc._h, self.n, P(self.cen), P(self.dir),
                                                P(self.mag), P(self.rv), c.rank, P(self.ecen),
                                                C.c_void_p(stream)), "dust_fmm_prepare_device")
            check(lib().dust_fmm_points_uvort_device(self.oc._h, C.byref(lines), P(self.euv),
                                                     C.c_void_p(stream)),
                  "dust_fmm_points_uvort_device")
        elif self.fused_pterm:
            # the particles' velocities of the previous update go into the
            # pressure term
            check(lib().dust_points_uvort_pressure_device(
                C.byref(self._ups), c.rank, P(self.ecen), self.n, P(self.cen), P(self.dir),
                P(self.mag), P(self.rv), P(self.vel), C.byref(lines), P(self.euv),
                P(self.pterm), C.c_void_p(stream)), "dust_points_uvort_pressure_device")
        else:
            check(lib().dust_points_uvort_device(C.byref(self._ups), c.rank, P(self.ecen),
                                                 self.n, P(self.cen), P(self.dir), P(self.mag),
                                                 P(self.rv), C.byref(lines), P(self.euv),
                                                 C.c_void_p(stream)), "dust_points_uvort_device")
        self._mark()
        torch.cuda.current_stream().synchronize()
        wk = abi.WakeRows(abi.Panels(c.wake.n, P(self.wnv, C.c_int), P(self.wkind, C.c_int),
                                     P(self.wver), P(self.wmag), abi._dp(), abi._dp()),
                          c.n_impl, P(self.impl, C.c_int))
        check(lib().dust_linsys_assemble_device(self.ls._h, C.byref(el), C.byref(wk)),
              "dust_linsys_assemble_device")
        if self.phase_events:
            self.ls.sync()
        self._mark()
        if self.pr is not None:
            # the particles' velocities of the previous update (the body is at
            # rest in the frame of its Bernoulli sources)
            if self.fused_pterm:
                self.pr.assemble_terms_device(None, self.pterm, stream=stream)
            else:
                self.pr.assemble_device(None, (self.cen, self.dir, self.mag, self.rv), self.vel,
                                        stream=stream)
            if self.steps_done > 0:
                self.pr.solve_device(self.res_pres, stream)
        self._mark()
        rep = abi.SolveReport()
        check(lib().dust_linsys_solve_device(self.ls._h, int(self.mode), P(self.res),
                                             C.byref(rep)), "dust_linsys_solve_device")
        self.last_report = {k: getattr(rep, k) for k, _ in abi.SolveReport._fields_}
        self._mark()
        # element strengths and implicit wake panels (update_wake :881-889)
        self.emag.copy_(self.res)
        self.wmag.copy_(self.res[self.i1] - self.res[self.i2] * self.has2)
        body = abi.Panels(c.rank, P(self.env, C.c_int), P(self.ekind, C.c_int), P(self.ever),
                          P(self.emag), P(self.eub), P(self.euv))
        wake = abi.Panels(c.wake.n, P(self.wnv, C.c_int), P(self.wkind, C.c_int),
                          P(self.wver), P(self.wmag), abi._dp(), abi._dp())
        els = abi.Elements(body, wake, lines)
        if self.fmm_uvort:
            check(lib().dust_fmm_finish_device(self.oc._h, C.byref(els), P(self.vel),
                                               P(self.str), P(self.rot), C.c_void_p(stream), 0),
                  "dust_fmm_finish_device")
        else:
            check(lib().dust_fmm_apply_device(self.oc._h, self.n, P(self.cen), P(self.dir),
                                              P(self.mag), P(self.rv), C.byref(els), P(self.vel),
                                              P(self.str), P(self.rot), C.c_void_p(stream), 0),
                  "dust_fmm_apply_device")
        self._mark()
        self.steps_done += 1
        if self.advect:
            check(lib().dust_particles_update_device(
                C.byref(self.upd), self.n, P(self.cen), P(self.dir), P(self.mag), P(self.vel),
                P(self.str), P(self.rot), P(self.free, C.c_int), P(self.n_freed, C.c_int),
                C.c_void_p(stream)), "dust_particles_update_device")
        self._mark()
        return self.res


class WakeStepper:
    """The reference's time loop for static bodies with panel wakes, device
    resident (src/dust.f90:510-1160 with update_wake / complete_wake of
    src/aeroel/mod_wake.f90).  Per step:

      1. prepare_wake: the live particles in slot order (dust_particles_live_device)
      2. uvort at the body centres from the particles and the end vortices
      3. assemble_linsys with the wake's rows (implicit first row + explicit
         rows), solve_linsys (static LU of initialize_linsys reused)
      4. update_wake: first wake row from the solution; particle velocity,
         stretching, diffusion by the FMM with body, wake panels and end
         vortices (scattered to the slots); wake points moved
      5. complete_wake: particles moved (penetration avoidance when ``pa``),
         wake rows from the trailing edge, shedding, end vortices

    ``case``: synth.WingWakeCase (body, trailing-edge topology, parameters);
    ``fprm``: FmmParams of the FMM and of the direct sums."""

    def __init__(self, case, fprm, mode=abi.DUST_SOLVE_LU64, pa=None, device="cuda"):
        import torch
        from . import wake as WK
        self.torch, self.WK = torch, WK
        self.case, self.fprm, self.mode, self.pa = case, fprm, mode, pa
        dev = torch.device(device)
        self.dev = dev
        T = lambda a, dt=torch.float64: torch.as_tensor(np.ascontiguousarray(a), dtype=dt,
                                                        device=dev)
        c = case
        self.wake = WK.PanelWake(c.wake_params(), c.ii, c.neigh, c.neigh_o, c.gen, c.te_pts,
                                 c.te_dir, c.te_scaling)
        self.te_pts, self.te_dir, self.te_sc = T(c.te_pts), T(c.te_dir), T(c.te_scaling)
        self.ever, self.env = T(c.body.ver), T(c.body.n_ver, torch.int32)
        self.ekind = T(c.body.kind, torch.int32)
        self.n = c.rank
        self.euv = torch.zeros((self.n, 3), dtype=torch.float64, device=dev)
        self.ecen = torch.zeros((self.n, 3), dtype=torch.float64, device=dev)
        self.res = torch.zeros(self.n, dtype=torch.float64, device=dev)
        ns = c.n_slots
        Z = lambda *s: torch.zeros(s, dtype=torch.float64, device=dev)
        self.S = dict(cen=Z(ns, 3), dir=Z(ns, 3), mag=Z(ns), rv=Z(ns), vel=Z(ns, 3),
                      str=Z(ns, 3), rot=Z(ns, 3))
        self.free = torch.ones(ns, dtype=torch.int32, device=dev)
        self.L = dict(cen=Z(ns, 3), dir=Z(ns, 3), mag=Z(ns), rv=Z(ns), vel=Z(ns, 3),
                      str=Z(ns, 3), rot=Z(ns, 3))
        self.idx = torch.zeros(ns, dtype=torch.int32, device=dev)
        self.n_freed = torch.zeros(1, dtype=torch.int32, device=dev)
        self.upd = c.update_params()
        self._ps = fprm.struct()
        # initialize_linsys: static rows with the first (implicit) wake row
        wp, ev, ni, ip = self.wake.elements()
        self._init_wake = self._host_wake_rows()
        self.ls = Linsys(fprm, c.rank, c.nstatic, c.body, self._init_wake[0], ni, c.gen)
        self.oc = Octree(fprm)
        # every library call of the step is queued on this stream (a NULL
        # stream would send the FMM to the octree's own stream)
        self.stream = torch.cuda.Stream()
        self.phase_events = False  # CUDA events between the phases of a step
        self.events = []
        self.n_live = 0
        self.shed_total = 0
        self.steps_done = 0

    def _host_wake_rows(self):
        L, pts, _, idou, _ = self.wake.get_state()
        c = self.case
        ver = np.zeros((L * len(c.ii), 4, 3))
        for r in range(L):
            for iw, (p1, p2) in enumerate(c.ii - 1):
                ver[r * len(c.ii) + iw] = [pts[r, p1], pts[r, p2], pts[r + 1, p2], pts[r + 1, p1]]
        return (abi.PanelSet(ver, kind=np.full(len(ver), abi.DUST_ELEM_VORTLATT),
                             mag=idou.reshape(-1)),)

    @staticmethod
    def _p(t, ctype=C.c_double):
        return C.cast(C.c_void_p(t.data_ptr()), C.POINTER(ctype))

    def body_struct(self, with_mag=True):
        P = self._p
        return abi.Panels(self.n, P(self.env, C.c_int), P(self.ekind, C.c_int), P(self.ever),
                          P(self.res) if with_mag else abi._dp(), abi._dp(), P(self.euv))

    def step(self):
        torch = self.torch
        torch.cuda.current_stream().synchronize()
        with torch.cuda.stream(self.stream):
            self._step()
        self.stream.synchronize()
        return self.res

    PHASES = ("live", "uvort", "assemble_solve", "fmm", "wake_update", "particles",
              "wake_complete")

    def _mark(self):
        if self.phase_events:
            e = self.torch.cuda.Event(enable_timing=True)
            e.record(self.stream)
            self.events.append(e)

    def phase_ms(self):
        """Milliseconds of each phase of the last step (phase_events on)."""
        ev = self.events
        return {k: ev[i].elapsed_time(ev[i + 1]) for i, k in enumerate(self.PHASES)
                if i + 1 < len(ev)}

    def _step(self):
        torch, WK, P = self.torch, self.WK, self._p
        S, L = self.S, self.L
        stream = self.stream.cuda_stream
        self.events = []
        self._mark()
        # 1. prepare_wake
        nl = WK.live_particles_device(self.free, S["cen"], S["dir"], S["mag"], S["rv"],
                                      L["cen"], L["dir"], L["mag"], L["rv"], self.idx, stream)
        self.n_live = nl
        self._mark()
        # 2. uvort at the body centres
        body = self.body_struct()
        check(lib().dust_panels_centres_device(C.byref(body), P(self.ecen), C.c_void_p(stream)),
              "dust_panels_centres_device")
        wp, ev, ni, ip = self.wake.elements()
        check(lib().dust_points_uvort_device(C.byref(self._ps), self.n, P(self.ecen), nl,
                                             P(L["cen"]), P(L["dir"]), P(L["mag"]), P(L["rv"]),
                                             C.byref(ev), P(self.euv), C.c_void_p(stream)),
              "dust_points_uvort_device")
        self.stream.synchronize()
        self._mark()
        # 3. assemble + solve
        wk = abi.WakeRows(wp, ni, ip)
        check(lib().dust_linsys_assemble_device(self.ls._h, C.byref(body), C.byref(wk)),
              "dust_linsys_assemble_device")
        rep = abi.SolveReport()
        check(lib().dust_linsys_solve_device(self.ls._h, int(self.mode), P(self.res),
                                             C.byref(rep)), "dust_linsys_solve_device")
        self.last_report = {k: getattr(rep, k) for k, _ in abi.SolveReport._fields_}
        self._mark()
        # 4. update_wake
        self.wake.set_first_row(self.res, stream)
        wp, ev, ni, ip = self.wake.elements()
        if nl > 0:
            els = abi.Elements(body, wp, ev)
            check(lib().dust_fmm_apply_device(self.oc._h, nl, P(L["cen"]), P(L["dir"]),
                                              P(L["mag"]), P(L["rv"]), C.byref(els),
                                              P(L["vel"]), P(L["str"]), P(L["rot"]),
                                              C.c_void_p(stream), 0), "dust_fmm_apply_device")
            WK.scatter_particles_device(nl, self.idx, L["vel"], L["str"], L["rot"], S["vel"],
                                        S["str"], S["rot"], stream)
        self._mark()
        self.wake.update(self._ps, body, L["cen"], L["dir"], L["mag"], L["rv"], n=nl,
                         stream=stream)
        self._mark()
        # 5. complete_wake
        if nl > 0:
            if self.pa is not None:
                WK.complete_wake_particles_pa_device(self.upd, self.pa, body, S["cen"], S["dir"],
                                                     S["mag"], S["rv"], S["vel"], S["str"],
                                                     S["rot"], self.free, self.n_freed, stream)
            else:
                check(lib().dust_particles_update_device(
                    C.byref(self.upd), int(self.free.shape[0]), P(S["cen"]), P(S["dir"]),
                    P(S["mag"]), P(S["vel"]), P(S["str"]), P(S["rot"]), P(self.free, C.c_int),
                    P(self.n_freed, C.c_int), C.c_void_p(stream)), "dust_particles_update_device")
        self._mark()
        shed = self.wake.complete(self.te_pts, self.te_dir, self.te_sc, None, S["cen"],
                                  S["dir"], S["mag"], S["rv"], S["vel"], self.free, stream)
        self._mark()
        self.shed_total += shed
        self.steps_done += 1

    def particles(self):
        """Live particles in slot order (host): cen, alpha = dir mag, r_vortex."""
        live = self.torch.nonzero(self.free == 0).flatten()
        S = self.S
        return (S["cen"][live].cpu().numpy(),
                (S["dir"][live] * S["mag"][live][:, None]).cpu().numpy(),
                S["rv"][live].cpu().numpy())

    def close(self):
        self.wake.close()
        self.oc.close()
