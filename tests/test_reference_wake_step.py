"""The wake's time advance pinned to the reference's own output.

tests/golden/ref_sym_static_nl_v_steps_10_11.npz comes from the reference's
regression fixtures tests/sym_test/static/nl_v/Output/ref_res_00{10,11}.h5
(tests/golden/make_reference_fixtures.py).  Output step 10 holds the state
that step 10's update_wake and complete_wake start from (saved after the
solve, src/dust.f90:648, 1017): 200 vortex-lattice panels with their solved
intensities, one row of wake panels on 40 stripes, the end vortices, 360
particles.  Step 11 holds the particles after the advance: the 360 moved
ones and the 40 that the full panel wake shed.  The case runs with fmm = F,
vortex stretching, vortex diffusion and penetration avoidance on.

One step from the step-10 state, in the reference's order:
  update_wake (src/aeroel/mod_wake.f90:860-1214): first wake row from the
    solution; particle velocities, stretching and diffusion by direct sums
    over all elements and particles (:1016-1077, compute_vel_from_all
    :2109-2150); velocities of the last wake row's points -> points_end;
  complete_wake (:1222-2105): first two wake rows from the trailing edge;
    penetration avoidance (avoid_collision, :2350-2534), Euler move and
    direction update of every particle; one particle shed per stripe from
    the last wake row into the lowest free slots; end vortices.

The CPU oracle (C + oracle/wake_oracle.py) reproduces the saved step-11
particles to about 1e-16 (moved) and 1e-14 (shed; the new wake row is built
from the trailing edge, which matches the saved one to 2e-13).  The GPU path
runs the same step through the C ABI: the particle sums through the FMM with
one octree level (one leaf: the all-pairs direct sum of fmm = F), the rest
through dust_wake_* and dust_particles_update_pa_device.  Tolerance: 1e-8
relative L2, the reference's regression tolerance (.gitlab-ci.yml:54).
"""
import os

import numpy as np
import pytest

import oracle as O
import wake_oracle as W
from dust_b200 import abi
from dust_b200.params import FmmParams

HERE = os.path.dirname(os.path.abspath(__file__))
NAME = "ref_sym_static_nl_v_steps_10_11.npz"
TOL_REF = 1e-8


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def load():
    return dict(np.load(os.path.join(HERE, "golden", NAME)))


def params(d):
    ns, npt = len(d["ii"]), len(d["te_pts"])
    wp = abi.wake_params(ns, npt, int(d["n_wake_panels"]), float(d["dt"]), d["box_min"],
                         d["box_max"], d["u_inf"], vortex_rad=float(d["vortex_rad"]),
                         k_vortex_rad=float(d["k_vortex_rad"]),
                         min_vel_at_te=float(d["min_vel_at_te"]))
    fp = FmmParams(rankine_rad=float(d["rankine_rad"]), cutoff_rad=float(d["cutoff_rad"]),
                   far_field_ratio_doublet=float(d["far_field_ratio_doublet"]),
                   vortstretch=bool(d["vortstretch"]), diffusion=bool(d["diffusion"]),
                   nu_inf=float(d["nu_inf"]), u_inf=tuple(float(x) for x in d["u_inf"]))
    u = abi.update_params(float(d["dt"]), d["box_min"], d["box_max"], 1,
                          bool(d["vortstretch"]), bool(d["diffusion"]), False, 0.0)
    pa = abi.pa_params(float(d["u_ref"]), float(d["pa_check_radius"]),
                       float(d["pa_element_radius"]))
    return wp, fp, u, pa


def particles10(d):
    a = d["part_alpha10"]
    m = np.sqrt((a * a).sum(axis=1))
    return d["part_cen10"].copy(), a / m[:, None], m, d["part_rv10"].copy()


def check_against_step11(d, cen, alpha, rv, last, wake_pts, n10):
    # moved particles, shed particles, their cores, the stripes' last
    # intensities and the panel wake
    assert len(cen) == len(d["part_cen11"])
    errs = {
        "moved_cen": rel(cen[:n10], d["part_cen11"][:n10]),
        "moved_alpha": rel(alpha[:n10], d["part_alpha11"][:n10]),
        "shed_cen": rel(cen[n10:], d["part_cen11"][n10:]),
        "shed_alpha": rel(alpha[n10:], d["part_alpha11"][n10:]),
        "shed_rv": rel(rv[n10:], d["part_rv11"][n10:]),
        "last": rel(last, d["last11"]),
        "wake_pts": rel(wake_pts, d["wake_pts11"]),
    }
    assert all(e < TOL_REF for e in errs.values()), errs
    return errs


def oracle_step(d):
    wp, fp, u, pa = params(d)
    ns, npt = len(d["ii"]), len(d["te_pts"])
    sc = np.full(npt, float(d["te_scaling"]))
    w = W.PanelWake(wp, d["ii"], d["neigh"], d["neigh_o"], d["gen"], d["te_pts"], d["te_dir"], sc)
    L = d["wake_vort10"].shape[0]
    w.set_state(L, d["wake_pts10"], d["wake_vel10"], d["wake_vort10"], d["last10"])
    res = d["vort10"]
    body = abi.PanelSet(d["ver"], n_ver=d["nver"], mag=res)
    cen, dr, m, rv = particles10(d)
    n = len(m)
    # update_wake
    w.set_first_row(res)
    wv, wm = w.panels()
    ev, em = w.end_vortices()
    vel_fn = lambda pts: W.vel_from_all(O, fp, pts, body, wv, wm, ev, em, cen, dr, m, rv)
    pv = vel_fn(cen)
    _, st, ro = O.direct_particles(fp, cen, dr, m, rv)
    w.update(vel_fn)
    # complete_wake
    w.complete_rows(d["te_pts"], d["te_dir"], sc)
    ns_ = int(d["n_wake_particles"])
    C_, D_, V_, S_, R_ = (np.zeros((ns_, 3)) for _ in range(5))
    M_, RV_ = np.zeros(ns_), np.zeros(ns_)
    F_ = np.ones(ns_, dtype=np.int32)
    C_[:n], D_[:n], V_[:n], S_[:n], R_[:n], M_[:n], RV_[:n], F_[:n] = cen, dr, pv, st, ro, m, rv, 0
    assert d["penetration_avoidance"]
    C_, D_, V_, S_, F_, nf = O.particles_update_pa(u, pa, body, C_, D_, M_, RV_, V_, S_, R_, F_)
    shed = w.shed(C_, D_, M_, RV_, V_, F_)
    live = np.nonzero(F_ == 0)[0]
    return (C_[live], D_[live] * M_[live][:, None], RV_[live], w.last.copy(),
            w.pts[:L + 1].copy(), n, nf, shed)


def test_fixture_pair_is_consistent():
    d = load()
    assert d["te_match"] < 1e-12
    assert len(d["part_cen10"]) == 360 and len(d["part_cen11"]) == 400
    assert abs(d["time11"] - d["time10"] - d["dt"]) < 1e-12
    assert d["n_wake_panels"] == 1
    assert bool(d["vortstretch"]) and bool(d["diffusion"]) and bool(d["penetration_avoidance"])


def test_oracle_wake_step_matches_reference():
    d = load()
    cen, alpha, rv, last, wpts, n10, nfreed, shed = oracle_step(d)
    assert nfreed == 0 and shed == 40
    errs = check_against_step11(d, cen, alpha, rv, last, wpts, n10)
    assert errs["moved_cen"] < 1e-14 and errs["moved_alpha"] < 1e-14, errs


@pytest.mark.gpu
def test_gpu_wake_step_matches_reference():
    import ctypes as C
    import torch
    from dust_b200 import wake as WK
    from dust_b200._lib import check, lib
    from dust_b200.octree import Octree
    d = load()
    wp, fp, u, pa = params(d)
    dev = torch.device("cuda")
    T = lambda a, dt=torch.float64: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=dev)
    npt = len(d["te_pts"])
    sc = np.full(npt, float(d["te_scaling"]))
    w = WK.PanelWake(wp, d["ii"], d["neigh"], d["neigh_o"], d["gen"], d["te_pts"], d["te_dir"], sc)
    L = d["wake_vort10"].shape[0]
    w.set_state(L, d["wake_pts10"], d["wake_vel10"], d["wake_vort10"], d["last10"])
    cen, dr, m, rv = particles10(d)
    n = len(m)
    ns_ = int(d["n_wake_particles"])
    # particle slots as the reference's wake_parts: the first n live
    S = dict(cen=torch.zeros((ns_, 3), dtype=torch.float64, device=dev),
             dir=torch.zeros((ns_, 3), dtype=torch.float64, device=dev),
             mag=torch.zeros(ns_, dtype=torch.float64, device=dev),
             rv=torch.zeros(ns_, dtype=torch.float64, device=dev),
             vel=torch.zeros((ns_, 3), dtype=torch.float64, device=dev),
             str=torch.zeros((ns_, 3), dtype=torch.float64, device=dev),
             rot=torch.zeros((ns_, 3), dtype=torch.float64, device=dev),
             free=torch.ones(ns_, dtype=torch.int32, device=dev))
    S["cen"][:n], S["dir"][:n], S["mag"][:n], S["rv"][:n] = T(cen), T(dr), T(m), T(rv)
    S["free"][:n] = 0
    # prepare_wake: the live list
    lc, ld = torch.empty((ns_, 3), dtype=torch.float64, device=dev), torch.empty(
        (ns_, 3), dtype=torch.float64, device=dev)
    lm, lr = torch.empty(ns_, dtype=torch.float64, device=dev), torch.empty(
        ns_, dtype=torch.float64, device=dev)
    idx = torch.empty(ns_, dtype=torch.int32, device=dev)
    nl = WK.live_particles_device(S["free"], S["cen"], S["dir"], S["mag"], S["rv"], lc, ld, lm,
                                  lr, idx)
    assert nl == n
    res = T(d["vort10"])
    ver, nver = T(d["ver"]), T(d["nver"], torch.int32)
    body = abi.Panels(len(d["ver"]), WK._ip(nver), abi._ip(), WK._dp(ver), WK._dp(res),
                      abi._dp(), abi._dp())
    # update_wake: first row, particle velocities (one octree level: the
    # all-pairs direct sum), wake points
    w.set_first_row(res)
    wpan, ev, _, _ = w.elements()
    lo = np.asarray(d["box_min"], dtype=np.float64)
    side = float(np.max(np.asarray(d["box_max"]) - lo)) + 1.0
    fmm = fp.replace(box_length=side, n_box=(1, 1, 1), origin=tuple(lo - 0.5),
                     n_octree_levels=1, min_octree_part=1, multipole_degree=2)
    oc = Octree(fmm)
    lvel, lstr, lrot = (torch.empty((nl, 3), dtype=torch.float64, device=dev) for _ in range(3))
    els = abi.Elements(body, wpan, ev)
    oc.apply_multipole_device(lc[:nl], ld[:nl], lm[:nl], lr[:nl], lvel, lstr, lrot,
                              elements=(els, None))
    WK.scatter_particles_device(nl, idx, lvel, lstr, lrot, S["vel"], S["str"], S["rot"])
    w.update(fp.struct(), body, lc, ld, lm, lr, n=nl)
    # complete_wake
    nf = torch.zeros(1, dtype=torch.int32, device=dev)
    WK.complete_wake_particles_pa_device(u, pa, body, S["cen"], S["dir"], S["mag"], S["rv"],
                                         S["vel"], S["str"], S["rot"], S["free"], nf)
    te_pts, te_dir, te_sc = T(d["te_pts"]), T(d["te_dir"]), T(sc)
    shed = w.complete(te_pts, te_dir, te_sc, None, S["cen"], S["dir"], S["mag"], S["rv"],
                      S["vel"], S["free"])
    torch.cuda.synchronize()
    assert int(nf.item()) == 0 and shed == 40
    live = torch.nonzero(S["free"] == 0).flatten()
    c11 = S["cen"][live].cpu().numpy()
    a11 = (S["dir"][live] * S["mag"][live][:, None]).cpu().numpy()
    r11 = S["rv"][live].cpu().numpy()
    Lw, pts, _, _, last = w.get_state()
    errs = check_against_step11(d, c11, a11, r11, last, pts, n)
    # and the same step on the CPU oracle
    oc_, oa, orv, olast, _, _, _, _ = oracle_step(d)
    assert rel(c11, oc_) < 1e-13 and rel(a11, oa) < 1e-12 and rel(r11, orv) < 1e-13, errs
    oc.close()
    w.close()
