"""The pressure integral equation (src/linsys/mod_pressure_equation.f90):
the CPU oracle's restatement checked against independent evaluations, and
the GPU path through the C ABI against the oracle.

Case: a static surface-panel ellipsoid, a moving one (displaced between
initialize_linsys and the step, with body velocities), a moving
vortex-lattice wing with a row of implicit wake panels and explicit wake
panels, end vortices, 3,000 particles with velocities, random Bernoulli
sources.  A_pres is the surface panels' block of the influence matrix
before the wake correction (static block from the initial geometry),
b_pres the Bernoulli source terms plus the rotational terms of the
particles, end vortices and wake panels; the solve is the block LU
sequence of solve_linsys on A_pres.
"""
import numpy as np
import pytest

import oracle as O
from dust_b200 import abi, synth
from dust_b200.params import FmmParams


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def case(seed=0, n_part=3000):
    rng = np.random.default_rng(seed)
    ea = synth.ellipsoid(n_target=240, axes=(1.5, 0.6, 0.4), seed=1)
    eb = synth.ellipsoid(n_target=120, axes=(0.6, 0.3, 0.3), seed=2)
    eb = abi.PanelSet(eb.ver + np.array([0.0, 2.0, 0.3]), eb.n_ver, eb.kind)
    wing, te = synth.flat_wing(span=2.0, chord=0.5, n_span=8, n_chord=3, alpha_deg=4.0)
    wing = abi.PanelSet(wing.ver + np.array([0.0, -2.0, 0.2]), wing.n_ver, wing.kind)
    init = synth.concat_panels(ea, eb, wing)
    nst = ea.n
    mv = np.zeros((init.n, 3))
    mv[nst:] = np.array([0.03, -0.01, 0.02])
    ver_step = init.ver.copy()
    ver_step[nst:] += mv[nst:, None, :]
    ub = np.zeros((init.n, 3))
    ub[nst:] = rng.normal(0, 0.5, (init.n - nst, 3))
    step = abi.PanelSet(ver_step, init.n_ver, init.kind, ub=ub)
    w1, ind = synth.te_wake(step, te + ea.n + eb.n, (0.2, 0.0, 0.01))
    w2, _ = synth.te_wake(step, te + ea.n + eb.n, (0.45, 0.0, 0.03))
    wake = synth.concat_panels(w1, w2)
    wake.mag = rng.normal(0, 0.1, wake.n)
    wake_vv = rng.normal(0, 1.0, (wake.n, 4, 3))
    ev = rng.normal(0, 1.0, (5, 2, 3)) + np.array([3.0, 0.0, 0.0])
    lines = abi.LineSet(ev, rng.normal(0, 0.1, 5))
    end_vv = rng.normal(0, 1.0, (5, 2, 3))
    cen = rng.uniform(-3, 3, (n_part, 3))
    dir_ = rng.normal(size=(n_part, 3))
    dir_ /= np.linalg.norm(dir_, axis=1)[:, None]
    mag = rng.uniform(1e-3, 1e-2, n_part)
    rv = rng.uniform(0.05, 0.1, n_part)
    vel = rng.normal(0, 1.0, (n_part, 3))
    nsp = ea.n + eb.n
    bern = rng.normal(0, 1.0, nsp)
    prm = FmmParams(u_inf=(1.0, 0.0, 0.0), box_length=8.0, origin=(-4.0, -4.0, -4.0))
    return dict(prm=prm, init=init, step=step, nst=nst, wake=wake, ind=ind, wake_vv=wake_vv,
                lines=lines, end_vv=end_vv, parts=(cen, dir_, mag, rv), vel=vel, bern=bern,
                nsp=nsp)


def test_oracle_pressure_terms_and_solve():
    c = case()
    A, b, res = O.pressure_run(c["prm"], c["init"].n, c["nst"], c["init"], c["step"], c["bern"],
                               c["parts"], c["vel"], c["wake"], c["wake_vv"], c["lines"],
                               c["end_vv"])
    nsp, nst = c["nsp"], c["nst"]
    assert A.shape == (nsp, nsp)
    # the rotational particle term written out independently
    zero = np.zeros_like(c["bern"])
    _, b_part, _ = O.pressure_run(c["prm"], c["init"].n, nst, c["init"], c["step"], zero,
                                  c["parts"], c["vel"])
    cen, dir_, mag, rv = c["parts"]
    sp_cen, _, _ = O.panel_geometry(c["step"])
    w = np.cross(dir_, c["vel"]) * mag[:, None]
    d = cen[None, :, :] - sp_cen[:nsp, None, :]
    rr = np.sqrt((d * d).sum(axis=2) + rv[None, :] ** 2)
    ref = ((d * w[None]).sum(axis=2) / rr ** 3).sum(axis=1)
    assert rel(b_part, ref) < 1e-12
    # A_pres = the surface panels' block of the system's influence matrix
    # before the wake correction (the assembled system without a wake)
    empty = (abi.empty_panels(), 0, None)
    A_full, _, _ = O.linsys_run(c["prm"], c["init"].n, 0, c["step"], c["step"], empty, empty)
    Af = A_full[:nsp, :nsp]
    # moving rows and the static rows' moving columns come from the step
    assert rel(A[nst:, :], Af[nst:, :]) < 1e-13
    assert rel(A[:nst, nst:], Af[:nst, nst:]) < 1e-13
    # the solution solves A_pres x = b_pres with the static block of the
    # initial geometry
    A_init, _, _ = O.linsys_run(c["prm"], c["init"].n, 0, c["init"], c["init"], empty, empty)
    Ap = Af.copy()
    Ap[:nst, :nst] = A_init[:nst, :nst]
    assert rel(Ap @ res, b) < 1e-11


@pytest.mark.gpu
def test_gpu_pressure_matches_oracle():
    import torch
    from dust_b200 import linsys
    c = case()
    n, nst, nsp = c["init"].n, c["nst"], c["nsp"]
    w = (c["wake"], len(c["ind"]), c["ind"])
    ls = linsys.Linsys(c["prm"], n, nst, c["init"], *w)
    pr = linsys.Pressure(ls)
    assert (pr.n_sp, pr.nstatic_sp) == (nsp, nst)
    ls.assemble_linsys(c["step"], *w)
    dev = torch.device("cuda")
    T = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    parts = tuple(T(a) for a in c["parts"])
    wv, wnv, wm = T(c["wake"].ver), torch.as_tensor(c["wake"].n_ver, dtype=torch.int32,
                                                   device=dev), T(c["wake"].mag)
    wp = abi.Panels(c["wake"].n, abi._ip(), abi._ip(), abi._dp(), abi._dp(), abi._dp(), abi._dp())
    import ctypes as C
    ip = lambda t: C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_int))
    dp = lambda t: C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_double))
    wp.n_ver, wp.ver, wp.mag = ip(wnv), dp(wv), dp(wm)
    lv, lm = T(c["lines"].ver), T(c["lines"].mag)
    lp = abi.Lines(c["lines"].n, dp(lv), dp(lm))
    wvv, evv, bern = T(c["wake_vv"]), T(c["end_vv"]), T(c["bern"])
    pr.assemble_device(bern, parts, T(c["vel"]), wp, wvv, lp, evv)
    Ag, bg = pr.get_system()
    res = torch.zeros(nsp, dtype=torch.float64, device=dev)
    pr.solve_device(res)
    A, b, ref = O.pressure_run(c["prm"], n, nst, c["init"], c["step"], c["bern"], c["parts"],
                               c["vel"], c["wake"], c["wake_vv"], c["lines"], c["end_vv"])
    assert rel(bg, b) < 1e-12
    assert rel(Ag[nst:, :], A[nst:, :]) < 1e-12 and rel(Ag[:nst, nst:], A[:nst, nst:]) < 1e-12
    assert rel(res.cpu().numpy(), ref) < 1e-10
    pr.close()
    ls.close()
    # DUST_PREC_FP32C: the particle sum in packed FP32 on tile-relative
    # coordinates, FP64 across tiles
    p32 = c["prm"].replace(precision=abi.DUST_PREC_FP32C)
    ls32 = linsys.Linsys(p32, n, nst, c["init"], *w)
    pr32 = linsys.Pressure(ls32)
    ls32.assemble_linsys(c["step"], *w)
    pr32.assemble_device(bern, parts, T(c["vel"]), wp, wvv, lp, evv)
    _, b32 = pr32.get_system()
    res32 = torch.zeros(nsp, dtype=torch.float64, device=dev)
    pr32.solve_device(res32)
    assert rel(b32, b) < 1e-6 and rel(res32.cpu().numpy(), ref) < 1e-6
    pr32.close()
    ls32.close()
    # the particle term evaluated in the uvort pass at every element centre
    from dust_b200._lib import check, lib
    cen_el, _, _ = O.panel_geometry(c["step"])
    pts = T(cen_el)
    uv, uv2, pt = (torch.zeros((n, 3), dtype=torch.float64, device=dev),
                   torch.zeros((n, 3), dtype=torch.float64, device=dev),
                   torch.zeros(n, dtype=torch.float64, device=dev))
    ps = c["prm"].struct()
    check(lib().dust_points_uvort_pressure_device(C.byref(ps), n, dp(pts), parts[2].shape[0],
                                                  dp(parts[0]), dp(parts[1]), dp(parts[2]),
                                                  dp(parts[3]), dp(T(c["vel"])), C.byref(lp),
                                                  dp(uv), dp(pt), None), "uvort+pressure")
    check(lib().dust_points_uvort_device(C.byref(ps), n, dp(pts), parts[2].shape[0],
                                         dp(parts[0]), dp(parts[1]), dp(parts[2]), dp(parts[3]),
                                         C.byref(lp), dp(uv2), None), "uvort")
    torch.cuda.synchronize()
    assert rel(uv.cpu().numpy(), uv2.cpu().numpy()) < 1e-13
    ref_pt = O.pressure_particles(cen_el, *c["parts"], c["vel"])
    assert rel(pt.cpu().numpy(), ref_pt) < 1e-12
    # the same fused pass in DUST_PREC_FP32C (Morton-sorted packed FP32
    # pairs): uvort against the FP32C uvort-only pass and the FP64 sum, the
    # particle term against the oracle
    ps32 = p32.struct()
    uv32, uv32b, pt32 = (torch.zeros((n, 3), dtype=torch.float64, device=dev),
                         torch.zeros((n, 3), dtype=torch.float64, device=dev),
                         torch.zeros(n, dtype=torch.float64, device=dev))
    check(lib().dust_points_uvort_pressure_device(C.byref(ps32), n, dp(pts), parts[2].shape[0],
                                                  dp(parts[0]), dp(parts[1]), dp(parts[2]),
                                                  dp(parts[3]), dp(T(c["vel"])), C.byref(lp),
                                                  dp(uv32), dp(pt32), None), "uvort+pressure f32")
    check(lib().dust_points_uvort_device(C.byref(ps32), n, dp(pts), parts[2].shape[0],
                                         dp(parts[0]), dp(parts[1]), dp(parts[2]), dp(parts[3]),
                                         C.byref(lp), dp(uv32b), None), "uvort f32")
    torch.cuda.synchronize()
    assert rel(uv32.cpu().numpy(), uv32b.cpu().numpy()) < 1e-13
    assert rel(uv32.cpu().numpy(), uv2.cpu().numpy()) < 1e-6
    assert rel(pt32.cpu().numpy(), ref_pt) < 1e-6
    ls2 = linsys.Linsys(c["prm"], n, nst, c["init"], *w)
    pr2 = linsys.Pressure(ls2)
    ls2.assemble_linsys(c["step"], *w)
    pr2.assemble_terms_device(bern, pt, wp, wvv, lp, evv)
    _, bt = pr2.get_system()
    assert rel(bt, b) < 1e-12
    # the host-array form of the fused pass: the same kernels (the chunks'
    # partial sums meet in atomic FP64 adds, so equal up to their order);
    # its term through the host-array assembly (no wake rows, end vortices or
    # Bernoulli sources there) against the device assembly of the same inputs
    hp = [np.ascontiguousarray(a) for a in c["parts"]]
    uvh, pth = np.empty((n, 3)), np.empty(n)
    evs = c["lines"].struct()
    check(lib().dust_points_uvort_pressure(C.byref(ps), n, abi.dptr(np.ascontiguousarray(cen_el)),
                                           hp[2].shape[0], *(abi.dptr(a) for a in hp),
                                           abi.dptr(np.ascontiguousarray(c["vel"])),
                                           C.byref(evs), abi.dptr(uvh), abi.dptr(pth)),
          "uvort+pressure host")
    assert rel(uvh, uv.cpu().numpy()) < 1e-13 and rel(pth, pt.cpu().numpy()) < 1e-13
    pr2.assemble_terms_device(None, T(pth))
    _, bd = pr2.get_system()
    pr2.assemble_terms(None, pth)
    _, bh = pr2.get_system()
    assert np.array_equal(bh, bd)
    pr2.close()
    ls2.close()
