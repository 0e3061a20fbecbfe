"""Panel wake, shedding and penetration avoidance on the GPU against the CPU
oracle (C + oracle/wake_oracle.py, which the reference's own step 10 -> 11
fixture pins, tests/test_reference_wake_step.py).

* avoid_collision (src/aeroel/mod_wake.f90:2350-2534) inside the particle
  update: surface panels and vortex rings, particles aimed at the bodies so
  that the corrections act; the same FP64 operations in the same order, so
  the results are compared bit for bit.
* the live-particle list and the scatter back to the slots;
* the time loop of a vortex-lattice wing with a three-row panel wake
  (update_wake / complete_wake, shedding from the full wake, end vortices,
  the FMM with body, wake panels and end vortices) for 12 steps, GPU vs
  oracle: solution, wake state and particles at 1e-10 relative;
* refine_wake sub-particles and the slot-shortage error.
"""
import numpy as np
import pytest

import oracle as O
import wake_oracle as W
from dust_b200 import abi, synth

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def _tensors(dev, **arrs):
    import torch
    out = {}
    for k, a in arrs.items():
        dt = torch.int32 if np.asarray(a).dtype.kind in "iu" else torch.float64
        out[k] = torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=dev)
    return out


def _pa_case(kind, n=4000, seed=3):
    """Particles within a chord of a body, moving towards it."""
    rng = np.random.default_rng(seed)
    if kind == abi.DUST_ELEM_VORTLATT:
        body, _ = synth.flat_wing(span=4.0, chord=1.0, n_span=16, n_chord=6, alpha_deg=4.0)
        cen = np.column_stack([rng.uniform(-0.2, 1.2, n), rng.uniform(-2.2, 2.2, n),
                               rng.uniform(-0.3, 0.3, n)])
        vel = np.column_stack([rng.normal(1.0, 0.3, n), rng.normal(0, 0.2, n),
                               -np.sign(cen[:, 2]) * rng.uniform(0.5, 4.0, n)])
    else:
        body = synth.ellipsoid(n_target=600, axes=(2.0, 1.0, 0.5), seed=1)
        d = rng.normal(size=(n, 3))
        d /= np.linalg.norm(d, axis=1)[:, None]
        cen = d * np.array([2.0, 1.0, 0.5]) * rng.uniform(1.01, 1.3, n)[:, None]
        vel = -cen * rng.uniform(2.0, 12.0, n)[:, None] + rng.normal(0, 0.3, (n, 3))
    ub = rng.normal(0, 0.05, (body.n, 3))
    body = abi.PanelSet(body.ver, body.n_ver, body.kind, ub=ub)
    dir_ = rng.normal(size=(n, 3))
    dir_ /= np.linalg.norm(dir_, axis=1)[:, None]
    mag = rng.uniform(1e-3, 2e-3, n)
    rv = rng.uniform(0.02, 0.08, n)
    st = rng.normal(0, 1e-3, (n, 3))
    free = np.zeros(n, dtype=np.int32)
    free[::97] = 1
    return body, cen, dir_, mag, rv, vel, st, free


@pytest.mark.parametrize("kind", [abi.DUST_ELEM_VORTLATT, abi.DUST_ELEM_SURFPAN])
def test_penetration_avoidance_matches_oracle(kind):
    import torch
    from dust_b200 import wake as WK
    body, cen, dir_, mag, rv, vel, st, free = _pa_case(kind)
    u = abi.update_params(0.05, (-50, -50, -50), (50, 50, 50), 1, True, True, False, 0.0)
    pa = abi.pa_params(u_ref=10.0)
    rot = np.zeros_like(cen)
    oc, od, ov, os_, of, onf = O.particles_update_pa(u, pa, body, cen, dir_, mag, rv, vel, st,
                                                     rot, free)
    changed = np.any(ov != vel, axis=1)
    assert changed.mean() > 0.05, "the corrections must act on a share of the particles"
    dev = torch.device("cuda")
    t = _tensors(dev, cen=cen, dir=dir_, mag=mag, rv=rv, vel=vel, st=st, rot=rot, free=free,
                 ver=body.ver, nv=body.n_ver, kind=body.kind, ub=body.ub)
    nf = torch.zeros(1, dtype=torch.int32, device=dev)
    bs = abi.Panels(body.n, WK._ip(t["nv"]), WK._ip(t["kind"]), WK._dp(t["ver"]), abi._dp(),
                    WK._dp(t["ub"]), abi._dp())
    WK.complete_wake_particles_pa_device(u, pa, bs, t["cen"], t["dir"], t["mag"], t["rv"],
                                         t["vel"], t["st"], t["rot"], t["free"], nf)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(t["vel"].cpu().numpy(), ov)
    np.testing.assert_array_equal(t["cen"].cpu().numpy(), oc)
    np.testing.assert_array_equal(t["dir"].cpu().numpy(), od)
    assert int(nf.item()) == onf


def test_live_list_and_scatter():
    import torch
    from dust_b200 import wake as WK
    rng = np.random.default_rng(0)
    n = 100_003
    free = (rng.uniform(size=n) < 0.3).astype(np.int32)
    cen, dir_ = rng.normal(size=(n, 3)), rng.normal(size=(n, 3))
    mag, rv = rng.uniform(size=n), rng.uniform(size=n)
    dev = torch.device("cuda")
    t = _tensors(dev, free=free, cen=cen, dir=dir_, mag=mag, rv=rv)
    E = lambda *s: torch.zeros(s, dtype=torch.float64, device=dev)
    lc, ld, lm, lr = E(n, 3), E(n, 3), E(n), E(n)
    idx = torch.zeros(n, dtype=torch.int32, device=dev)
    nl = WK.live_particles_device(t["free"], t["cen"], t["dir"], t["mag"], t["rv"], lc, ld, lm,
                                  lr, idx)
    live = np.nonzero(free == 0)[0]
    assert nl == len(live)
    np.testing.assert_array_equal(idx[:nl].cpu().numpy(), live)
    np.testing.assert_array_equal(lc[:nl].cpu().numpy(), cen[live])
    np.testing.assert_array_equal(lr[:nl].cpu().numpy(), rv[live])
    out = E(n, 3)
    WK.scatter_particles_device(nl, idx, lc, None, None, out, None, None)
    torch.cuda.synchronize()
    o = out.cpu().numpy()
    np.testing.assert_array_equal(o[live], cen[live])
    assert not np.any(o[free == 1])


@pytest.mark.parametrize("pa", [False, True])
def test_wing_wake_loop_matches_oracle(pa):
    from dust_b200.step import WakeStepper
    case = synth.WingWakeCase(n_span=10, n_chord=4, n_wake_panels=3, steps=12)
    fp = case.fmm_params(levels=5)
    pap = abi.pa_params(u_ref=1.0) if pa else None
    gpu = WakeStepper(case, fp, pa=pap)
    cpu = W.OracleWakeRun(O, case, fp, pa=pap)
    for s in range(12):
        r = gpu.step().cpu().numpy()
        shed = cpu.step()
        assert rel(r, cpu.res) < 1e-10, (s, rel(r, cpu.res))
        assert gpu.n_live == int(np.sum(cpu.free == 0)) - shed or s == 0
    L, pts, pv, idou, last = gpu.wake.get_state()
    assert L == cpu.w.len == 3
    assert rel(pts, cpu.w.pts[:L + 1]) < 1e-10
    assert rel(idou, cpu.w.idou[:L]) < 1e-10 and rel(last, cpu.w.last) < 1e-10
    gc, ga, gr = gpu.particles()
    oc, oa, orv = cpu.particles()
    assert len(gc) == len(oc) == 10 * 10 == gpu.shed_total
    assert rel(gc, oc) < 1e-10 and rel(ga, oa) < 1e-10
    np.testing.assert_array_equal(gr, orv)
    gpu.close()


def test_refined_shedding_and_slot_shortage():
    from dust_b200._lib import DustError
    from dust_b200.step import WakeStepper
    # 6 stripes of span 1/3 behind a wing with dt 0.2: 4 sub-particles each
    case = synth.WingWakeCase(span=2.0, n_span=6, n_chord=3, n_wake_panels=1, dt=0.2, steps=6,
                              n_wake_particles=400)
    wp = case.wake_params()
    wp.refine_wake, wp.k_refine = 1, 2
    case.wake_params = lambda: wp
    fp = case.fmm_params(levels=4)
    gpu = WakeStepper(case, fp)
    cpu = W.OracleWakeRun(O, case, fp)
    for s in range(4):
        gpu.step()
        cpu.step()
    gc, ga, gr = gpu.particles()
    oc, oa, orv = cpu.particles()
    assert len(gc) == len(oc) and len(gc) > 4 * 6 * 2
    assert rel(gc, oc) < 1e-10 and rel(ga, oa) < 1e-10 and rel(gr, orv) < 1e-12
    gpu.close()
    # a slot array too small for the next shedding
    small = synth.WingWakeCase(n_span=6, n_chord=3, n_wake_panels=1, steps=3,
                               n_wake_particles=8)
    g2 = WakeStepper(small, small.fmm_params(levels=4))
    with pytest.raises(DustError) as e:
        for _ in range(3):
            g2.step()
    assert e.value.status == abi.DUST_ERR_CAPACITY
    g2.close()
