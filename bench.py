#!/usr/bin/env python
"""Benchmark: one aerodynamic timestep of DUST's hot path on B200.

Workload (the full-step case): two counter-rotating 3-blade vortex-lattice
rotors (radius 1, 40 x 8 panels per blade, 1,920 moving unknowns) over a
12,000-panel surface-panel wing (static), 338 implicit wake panels and end
vortices, and a particle wake of 2,000,000 particles; FMM degree 4, leaves
<= 64 particles.  Synthetic, seeded (dust_b200.synth.FullStepCase); no
public dataset exists for this path.

A step = uvort at the 13,920 collocation points (direct sum over particles
and end vortices) + AIC assembly + solve + FMM evaluation of the particle
velocities/stretching (tree, multipoles, L2P, P2P, element sums).

Arms:
  default            this library; ``value`` = device-resident step time of
                     the fastest solve mode, ``e2e`` = host-API step time
                     with pinned host buffers (copies inside the timed region)
  --impl reference   the reference's algorithm on the host cores (the C/OpenMP
                     oracle; the Fortran reference cannot be built here),
                     timed on a bounded sample and scaled to one step

One process per GPU under torchrun; the path does not shard (replicas only):
every rank runs its own replica, timing is the max over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ms/timestep (2M particles, 12k panels) vs plain FP64 GPU at ≤1e-6 load error"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--particles", type=int, default=2_000_000)
    ap.add_argument("--degree", type=int, default=4)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--quick", action="store_true", help="small case (smoke)")
    ap.add_argument("--no-learned", action="store_true",
                    help="skip the learned-preconditioner mode (and its training)")
    ap.add_argument("--train-iters", type=int, default=400)
    ap.add_argument("--profile-step", action="store_true",
                    help="run warm-up + one step only (for ncu launch lists)")
    return ap.parse_args()


class Clocks:
    """Samples nvidia-smi during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) > 8:
                for k, nm in enumerate(names):
                    if r[5 + k].lower().startswith("active"):
                        reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.rows)}


def dist_init(args):
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        # gloo without a GPU: only the reference arm (host cores) runs there
        cuda = torch.cuda.is_available()
        if cuda:
            torch.cuda.set_device(local)
        dist.init_process_group("nccl" if cuda else "gloo",
                                timeout=datetime.timedelta(seconds=600))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return rank, ws, local


def max_over_ranks(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def workload(case, degree):
    """The benchmark's workload description (both arms)."""
    nmv = case.rank - case.nstatic
    return ("full step: 2x3-blade VLM rotors (%s moving unknowns) + %s-panel surface-panel "
            "wing, %d wake panels, %d particles, FMM p=%d, leaves<=64"
            % (format(nmv, ","), format(case.nstatic, ","), case.wake.n, case.mag.shape[0],
               degree))


def make_case(args):
    from dust_b200 import synth
    if args.quick:
        return synth.FullStepCase(n_particles=200_000, wing_span=20, wing_around=40,
                                  n_span_blade=10, n_chord_blade=4)
    return synth.FullStepCase(n_particles=args.particles)


def time_steps(stepper, steps, flush):
    import torch
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    for k in range(steps):
        flush.zero_()  # 256 MB write between steps: L2 (126 MB) holds nothing of the last
        torch.cuda.synchronize()
        ev[k][0].record()
        stepper.step()
        ev[k][1].record()
        torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in ev]


def cpu_baseline(case, params, budget_s=20.0):
    """The oracle (C restatement of the reference, OpenMP on all host cores)
    on a bounded sample of one step, scaled to a full step."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from dust_b200 import abi
    rng = np.random.default_rng(0)
    n = case.mag.shape[0]
    cen_el = case.elems.ver.mean(axis=1)
    tri = case.elems.n_ver == 3
    cen_el[tri] = case.elems.ver[tri, :3].mean(axis=1)
    parts = {}
    # (1) uvort: sample of collocation points, all particles
    ns = 24
    idx = rng.choice(case.rank, ns, replace=False)
    t = time.perf_counter()
    O.points_uvort(params, cen_el[idx], case.cen, case.dir, case.mag, case.r_vortex,
                   case.end_vort)
    parts["uvort"] = (time.perf_counter() - t) * case.rank / ns
    # (2) element -> particle sums: sample of particles, all elements
    npart = 400
    pid = rng.choice(n, npart, replace=False)
    els = abi.elements_struct(case.elems, case.wake, case.end_vort)
    t = time.perf_counter()
    O.elements_vel(params, case.cen[pid], els)
    parts["elements"] = (time.perf_counter() - t) * n / npart
    # (3) FMM tree + multipoles + near field on a 1/20 particle subsample
    sub = rng.choice(n, n // 20, replace=False)
    t = time.perf_counter()
    O.fmm_apply(params, case.cen[sub], case.dir[sub], case.mag[sub], case.r_vortex[sub])
    parts["fmm"] = (time.perf_counter() - t) * 20
    # (4) assembly + Schur LU per step: a reduced system, scaled by flop count
    m = min(1200, case.nstatic)
    nmv_s = min(160, case.rank - case.nstatic)
    sl = np.arange(m)
    sub_el = case.elems.subset(np.concatenate([sl, np.arange(case.nstatic,
                                                             case.nstatic + nmv_s)]))
    nst_s = m
    t = time.perf_counter()
    O.linsys_run(params, sub_el.n, nst_s, sub_el, sub_el, (abi.empty_panels(), 0, None),
                 (abi.empty_panels(), 0, None))
    t_small = time.perf_counter() - t
    # per-step flops: trsm x2 (nst^2 nmv each) + gemm (2 nmv^2 nst) + getrf(nmv)
    def step_flops(nst, nmv):
        return 2 * nst * nst * nmv + 2 * nmv * nmv * nst + 2 / 3 * nmv ** 3
    # the sample also paid its static LU (2/3 nst^3); scale by total flops
    fl_small = 2 / 3 * nst_s ** 3 + step_flops(nst_s, nmv_s)
    parts["linsys"] = t_small * step_flops(case.nstatic, case.rank - case.nstatic) / fl_small
    total_ms = 1e3 * sum(parts.values())
    return total_ms, {k: round(v * 1e3, 1) for k, v in parts.items()}


def run_reference(args, rank, ws):
    """--impl reference: the reference's algorithm on the host cores."""
    if rank != 0:
        return
    from dust_b200 import synth
    case = synth.FullStepCase(n_particles=args.particles) if not args.quick else make_case(args)
    params = case.fmm_params(degree=args.degree)
    vals = []
    # each step is a bounded sample (about 20 s of host work); at most 2
    for _ in range(max(1, min(args.steps, 2))):
        ms, parts = cpu_baseline(case, params)
        vals.append(ms)
    cores = os.cpu_count()
    v = float(np.median(vals))
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 1), "unit": "ms",
            "n_gpus": args.gpus, "steps": len(vals), "warmup": 0, "ms_per_step": round(v, 1),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic (seeded FullStepCase)",
            "config": {"workload": workload(case, args.degree), "mode": "reference (FP64 CPU)",
                       "levels": params.n_octree_levels,
                       "parallelism": "rank 0 only" if ws > 1 else "host cores"},
            "cpu_baseline": {"value": round(v, 1), "unit": "ms", "cores": cores, "kind": "port",
                             "sample": "per-phase samples scaled to one step: " +
                             json.dumps(parts)},
            "e2e": {"value": round(v, 1), "unit": "ms", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank, ws, local = dist_init(args)
    if args.impl == "reference":
        run_reference(args, rank, ws)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    import torch
    from dust_b200 import abi, step
    # all work on one explicit stream: the library treats a NULL stream as
    # "the handle's own stream", so torch's legacy default stream (handle 0)
    # must not be used for timing
    torch.cuda.set_stream(torch.cuda.Stream())
    case = make_case(args)
    params = case.fmm_params(degree=args.degree)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    modes = [("plain", abi.DUST_SOLVE_LU64), ("mixed", abi.DUST_SOLVE_MIXED)]
    learned = None
    if not args.no_learned:
        # the learned preconditioner trains (untimed) on the plain solutions
        # of the same geometry at rotor azimuths other than the benchmarked one
        from dust_b200 import precond
        period = 2 * np.pi / 3
        angles = (np.arange(12) + 0.5) * period / 12
        pc, info = precond.train_for_case(case, params, angles, iters=args.train_iters)
        learned = {"precond": pc, "info": info}
        modes.append(("learned", abi.DUST_SOLVE_GMRES_NN))
    results = {}
    steppers = {}
    for name, mode in modes:
        prm = params if name == "plain" else params.replace(precision=abi.DUST_PREC_FP32C)
        st = step.DeviceStepper(case, prm, mode)
        if name == "learned":
            learned["precond"].attach(st.ls)
        steppers[name] = st
        for _ in range(max(args.warmup, 1 if args.profile_step else 3)):
            st.step()
        torch.cuda.synchronize()
        if args.profile_step:
            continue
        barrier(ws)
        with Clocks(local) as clk:
            times = time_steps(st, args.steps, flush)
        barrier(ws)
        ms = max_over_ranks(float(np.mean(times)), ws)
        res = st.res.cpu().numpy()
        results[name] = {"ms": ms, "times": times, "loads": case.loads(res),
                         "report": st.last_report, "clocks": clk.summary(), "res": res,
                         "fmm": [t.cpu().numpy() for t in (st.vel, st.str, st.rot)]}
    if args.profile_step:
        return
    # phase breakdown (plain and mixed share the FMM): one timed step with events
    ph = {k: phase_breakdown(steppers[k], case, params) for k in steppers}
    lp = results["plain"]["loads"]
    load_err = {k: float(np.max(np.abs(results[k]["loads"] - lp) / np.maximum(np.abs(lp), 1e-30)))
                for k in results}
    # particle outputs of the step (velocity without the wind, stretching,
    # div-filter curl) against the FP64 step: relative L2 norms
    uinf = np.asarray(params.u_inf)
    def fmm_err(k):
        a, b = results[k]["fmm"], results["plain"]["fmm"]
        rel = lambda x, y: float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))
        return {"vel_induced": rel(a[0] - uinf, b[0] - uinf), "stretch": rel(a[1], b[1]),
                "rot": rel(a[2], b[2])}
    fmm_errs = {k: fmm_err(k) for k in results}
    # the headline mode: the fastest whose loads are within 1e-6 of FP64
    best = min((k for k in results if load_err[k] <= 1e-6), key=lambda k: results[k]["ms"])
    # end to end through the host API (pinned buffers)
    e2e = None
    if not args.no_e2e:
        prm_best = params if best == "plain" else params.replace(precision=abi.DUST_PREC_FP32C)
        e2e = run_e2e(case, prm_best, dict(modes)[best], args, ws,
                      learned["precond"] if best == "learned" else None)
    cpu = None
    if not args.no_cpu and rank == 0 and ws == 1:
        ms_cpu, parts = cpu_baseline(case, params)
        cpu = {"value": round(ms_cpu, 1), "unit": "ms", "cores": os.cpu_count(), "kind": "port",
               "sample": "oracle per-phase samples scaled to one step: " + json.dumps(parts)}
    launches = count_launches(steppers[best])
    rf = roofline(ph, case, params, best)
    if rank == 0:
        r = results[best]
        line = {
            "metric": METRIC, "value": round(r["ms"] / ws, 3), "unit": "ms", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(r["ms"], 3),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if best == "plain" else "f32/tf32 with f64 refinement",
            "data": "synthetic (seeded FullStepCase)",
            "config": {"workload": workload(case, args.degree),
                       "mode": best, "levels": params.n_octree_levels,
                       "l2": "256 MB flush between timed steps; A is 1.55 GB",
                       "parallelism": "replicas" if ws > 1 else "single GPU"},
            "plain_fp64_ms": round(results["plain"]["ms"], 3),
            "speedup_vs_plain_fp64": round(results["plain"]["ms"] / r["ms"], 3),
            "load_error_vs_fp64": load_err[best],
            "modes": {k: {"ms": round(v["ms"], 3), "load_error_vs_fp64": load_err[k],
                          "particle_error_vs_fp64": fmm_errs[k], "solve": v["report"]}
                      for k, v in results.items()},
            "learned_training": learned["info"] if learned else None,
            "phases_ms": ph,
            "clocks": r["clocks"],
            "roofline": rf,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def phase_breakdown(st, case, params):
    """Per-phase device times of one step (CUDA events at the phase
    boundaries of DeviceStepper.step; the library records its own FMM phase
    events on the same stream)."""
    import torch
    st.oc.set_timing(True)
    st.phase_events = True
    torch.cuda.synchronize()
    st.step()
    torch.cuda.synchronize()
    s = st.oc.stats()
    ev = st.events
    st.oc.set_timing(False)
    st.phase_events = False
    t = lambda a, b: round(ev[a].elapsed_time(ev[b]), 3)
    return {"total": t(0, 4), "uvort": t(0, 1), "assemble": t(1, 2), "solve": t(2, 3),
            "fmm_total": t(3, 4), "fmm_tree": round(s["ms_tree"], 3),
            "fmm_upward": round(s["ms_upward"], 3), "fmm_m2l": round(s["ms_m2l"], 3),
            "fmm_p2p": round(s["ms_p2p"], 3), "fmm_elements": round(s["ms_elems"], 3),
            "n_leaves": s["n_leaves"], "n_active_cells": s["n_active_cells"],
            "n_m2l_pairs": s["n_m2l_pairs"], "n_p2p_pairs": s["n_p2p_pairs"],
            "n_elem_pairs": s["n_elem_pairs"],
            "k_m2l_tc_ms": round(s["ms_m2l_kernel"], 3), "k_elem_far_ms": round(s["ms_elem_far"], 3)}


# Algorithmic work per unit (FMA = 2 flops), from the kernels' formulas:
#  far element pair (k_elem_far): r (3) + r^2 (5) + rsqrt (1) + 1/r^2 (1)
#    + r.n (5) + 1/r^3 (1) + coefficient (3) + 3 x fma(k3, fma(coef, r, -mu n)) (12)
FLOP_ELEM_PAIR = 31
#  uvort pair (k_uvort_sorted): d (3) + rho^2 (6) + rsqrt (1) + rho^-3 (2) + 6 fma (12)
FLOP_UVORT_PAIR = 24
#  M2L pair at p = 4 with stretching: 56 outputs x 35 inputs x 3 components x
#  2 cross-product terms, one FMA each
FLOP_M2L_PAIR = 56 * 35 * 6 * 2
# DRAM bytes per launch measured by ncu (dram__bytes_read.sum +
# dram__bytes_write.sum) on the 300k-particle case and scaled by the particle
# count to 2M (profiles/traffic_mixed_step_300k.txt)
TRAFFIC_ELEM_FAR_PER_PARTICLE = 381.5


def roofline(ph, case, params, best):
    """Roofline of the dominant kernel of the headline mode, plus the other
    large kernels.  Peaks: MEASURED_PEAKS.json (HBM copy GB/s, cuBLAS bf16
    TFLOP/s); the FP32 SIMT peak is not measured there and is the nominal
    148 SMs x 128 lanes x 2 flops x sm_max_mhz; the TF32 dense peak is half
    the measured bf16 figure (the nominal ratio)."""
    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
    mhz = peaks.get("sm_max_mhz", 1965.0)
    fp32_peak = 148 * 128 * 2 * mhz * 1e6 / 1e12
    src = "of measured" if peaks else "of fallback"
    bf16 = peaks.get("bf16_tflops", 1590.0)
    p = ph.get(best, {})
    n = case.mag.shape[0]
    out = {}
    if p.get("k_elem_far_ms"):
        a = FLOP_ELEM_PAIR * p["n_elem_pairs"] / (p["k_elem_far_ms"] * 1e-3) / 1e12
        tr = None if TRAFFIC_ELEM_FAR_PER_PARTICLE is None else int(TRAFFIC_ELEM_FAR_PER_PARTICLE * n)
        out = {"kernel": "k_elem_far", "bound": "fp32", "achieved": round(a, 2),
               "peak": round(fp32_peak, 1), "unit": "TFLOP/s", "frac": round(a / fp32_peak, 3),
               "traffic": tr, "peak_source": "nominal FP32 SIMT (148 SMs x 128 x 2 x %g MHz)" % mhz,
               "flop_per_pair": FLOP_ELEM_PAIR, "pairs": p["n_elem_pairs"],
               "ms": p["k_elem_far_ms"]}
    others = []
    if p.get("k_m2l_tc_ms"):
        a = FLOP_M2L_PAIR * p["n_m2l_pairs"] / (p["k_m2l_tc_ms"] * 1e-3) / 1e12
        others.append({"kernel": "k_m2l_tc", "bound": "tensor", "achieved": round(a, 2),
                       "peak": round(bf16 / 2, 1), "unit": "TFLOP/s",
                       "frac": round(a / (bf16 / 2), 4), "ms": p["k_m2l_tc_ms"],
                       "peak_source": "TF32 = bf16 %s / 2" % src,
                       "note": "useful FP32-equivalent flops; 3xTF32 issues 3x on the tensor pipe"})
    if p.get("uvort"):
        pairs = case.rank * n
        a = FLOP_UVORT_PAIR * pairs / (p["uvort"] * 1e-3) / 1e12
        others.append({"kernel": "uvort phase (k_uvort_sorted + sort)", "bound": "fp32",
                       "achieved": round(a, 2), "peak": round(fp32_peak, 1), "unit": "TFLOP/s",
                       "frac": round(a / fp32_peak, 3), "ms": p["uvort"]})
    out["others"] = others
    out["peaks_file"] = bool(peaks)
    return out


def count_launches(st):
    """Kernels launched by one step (CUPTI through torch.profiler)."""
    import torch
    try:
        from torch.profiler import ProfilerActivity, profile
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            st.step()
            torch.cuda.synchronize()
        names = [e.name for e in prof.events() if e.device_type == torch.autograd.DeviceType.CUDA
                 and "memcpy" not in e.name.lower() and "memset" not in e.name.lower()]
        return len(names)
    except Exception:
        return None


def run_e2e(case, params, mode, args, ws, pc=None):
    """Same step through the host API with pinned host buffers: every step
    copies particles and panels in and velocities/strengths out."""
    import torch
    from dust_b200 import step
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    case.cen, case.dir, case.mag, case.r_vortex = (pin(case.cen), pin(case.dir),
                                                  pin(case.mag), pin(case.r_vortex))
    n = case.mag.shape[0]
    out = tuple(pin(np.empty((n, 3))) for _ in range(3))  # page-locked outputs
    hs = step.HostStepper(case, params, mode, out=out)
    if pc is not None:
        pc.attach(hs.ls)
    for _ in range(3):
        hs.step()
    torch.cuda.synchronize()
    barrier(ws)
    times = []
    for _ in range(args.steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        res, vel, st_, ro = hs.step()
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = max_over_ranks(float(np.mean(times)), ws)
    h2d = n * 8 * 8 + case.rank * 8 * (12 + 3 + 3 + 1) + case.wake.n * 8 * 13 + case.end_vort.n * 56
    d2h = n * 9 * 8 + case.rank * 8
    return {"value": round(ms, 3), "unit": "ms", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "step_ms": [round(t, 2) for t in times]}


if __name__ == "__main__":
    main()
