#!/usr/bin/env python
"""Benchmark: one aerodynamic timestep of DUST's hot path on B200.

Workload (the full-step case): two counter-rotating 3-blade vortex-lattice
rotors (radius 1, 40 x 8 panels per blade, 1,920 moving unknowns) over a
12,000-panel surface-panel wing (static), 338 implicit wake panels and end
vortices, and a particle wake of 2,000,000 particles; FMM degree 4, leaves
<= 64 particles.  Synthetic, seeded (dust_b200.synth.FullStepCase); no
public dataset exists for this path.

A step = uvort at the 13,920 collocation points (direct sum over particles
and end vortices; --uvort fmm takes it from the particles' FMM instead) +
AIC assembly + solve + FMM evaluation of the particle velocities/stretching
(tree, multipoles, L2P, P2P, element sums) + the particle update of
complete_wake (explicit Euler advection and stretching, so the next step's
tree is built on moved particles; --no-advect leaves them in place).

Arms:
  default            this library; ``value`` = device-resident step time of
                     the fastest solve mode, ``e2e`` = host-API step time
                     with pinned host buffers (copies inside the timed region)
  --impl reference   the reference's algorithm on the host cores (the C/OpenMP
                     oracle + LAPACK/BLAS; the Fortran reference cannot be
                     built here): one whole step timed in full, after the
                     untimed initialize_linsys

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
    ap.add_argument("--workload", default="full",
                    choices=["full", "fmm", "dense", "learned", "wing"],
                    help="full: the full-step line (with the fmm and dense workloads as "
                         "sub-objects); fmm / dense: that workload's own line")
    ap.add_argument("--dense-panels", type=int, default=16384,
                    help="panels of the dense-solve workload's ellipsoid (smaller for "
                         "profiling captures)")
    ap.add_argument("--no-workloads", action="store_true",
                    help="full step only, without the fmm / dense sub-objects")
    ap.add_argument("--degrees", default="4,6,8", help="FMM degrees of the fmm workload")
    ap.add_argument("--uvort", default="direct", choices=["fmm", "direct"],
                    help="panels' uvort by the direct sum (the reference's get_vort_vel) or "
                         "through the particles' FMM (apply_multipole_panels; then the plain "
                         "FP64 step with the direct sum is timed as well)")
    ap.add_argument("--no-advect", action="store_true",
                    help="leave the particles in place (no complete_wake particle update)")
    ap.add_argument("--modes", default="",
                    help="comma-separated subset of the step modes to run (plain always "
                         "runs: it is the reference of the load errors); default all")
    ap.add_argument("--accuracy-steps", type=int, default=20,
                    help="advected steps over which every mode's loads are compared with "
                         "the plain FP64 run (warm-up + timed + untimed steps)")
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
        return synth.FullStepCase(n_particles=min(200_000, args.particles), wing_span=20,
                                  wing_around=40, n_span_blade=10, n_chord_blade=4)
    return synth.FullStepCase(n_particles=args.particles)


def time_steps(stepper, steps, flush, after=None):
    """CUDA-event time of each step; ``after()`` runs between steps, outside
    the timed events (e.g. reading the step's loads)."""
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
        if after is not None:
            after()
    return [a.elapsed_time(b) for a, b in ev]


def host_cores():
    """Physical host cores (the CPU baseline's thread count)."""
    try:
        import psutil
        n = psutil.cpu_count(logical=False)
        if n:
            return int(n)
    except Exception:
        pass
    return os.cpu_count() or 1


def cpu_baseline(case, params, m2l_pairs, fmm_stride=32, uvort_stride=64):
    """The reference's step on the host cores (the oracle's C loops with
    OpenMP and LAPACK/BLAS through scipy, oracle/cpu_step.py) on a bounded
    sample of the full-step workload, scaled to one step phase by phase by
    the exact ratio of work:

    * uvort: every `uvort_stride`-th collocation point (all particles and end
      vortices), scaled by the point count;
    * assembly: 8 moving rows over all columns through the oracle's row
      builder, scaled by the entries a step rebuilds
      (nstatic x nmoving + nmoving x rank);
    * solve: the reference's LAPACK sequence (dlaswp, dtrsm x 2, dgemm,
      dgetrf, dlaswp, dgetrs) on blocks of the full sizes, timed in full
      (its time does not depend on the values);
    * FMM: tree, P2M, M2M and L2L in full; M2L for every `fmm_stride`-th
      target cell scaled by the M2L pair count; L2P + P2P + element sums for
      every `fmm_stride`-th leaf scaled by the particle count."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import cpu_step
    import oracle as O
    from dust_b200 import abi
    cores = host_cores()
    cpu_step.set_threads(cores)
    n = case.mag.shape[0]
    parts = {}
    cen_el = np.where(case.elems.n_ver[:, None] == 4, case.elems.ver.mean(axis=1),
                      case.elems.ver[:, :3].mean(axis=1))
    # (1) uvort
    pts = np.ascontiguousarray(cen_el[::uvort_stride])
    t = time.perf_counter()
    O.points_uvort(params, pts, case.cen, case.dir, case.mag, case.r_vortex, case.end_vort)
    parts["uvort"] = (time.perf_counter() - t) * case.rank / len(pts)
    # (2) assembly: moving rows
    nst, rank = case.nstatic, case.rank
    nmv = rank - nst
    rows = np.arange(nst, rank, max(1, nmv // 8))[:8]
    t = time.perf_counter()
    O.linsys_rows(params, case.elems, rows, (case.wake, case.n_impl, case.impl_ind))
    per_entry = (time.perf_counter() - t) / (len(rows) * rank)
    parts["assemble"] = per_entry * (nst * nmv + nmv * rank)
    # (3) solve: LAPACK sequence at the full sizes on a well-conditioned
    # stand-in (an LU of the static block as the reference keeps it)
    rng = np.random.default_rng(0)
    A = np.asfortranarray(rng.standard_normal((rank, rank)) * (1.0 / rank))
    A[np.arange(rank), np.arange(rank)] += 1.0
    P = np.arange(rank, dtype=np.int32)
    t = time.perf_counter()
    cpu_step.solve_linsys_lapack(A, P, nst, np.ones(rank))
    parts["solve"] = time.perf_counter() - t
    del A
    # (3b) the pressure equation of the surface panels: the particles'
    # rotational term at every uvort_stride-th surface panel (scaled by the
    # panel count) and the LAPACK dgetrs on a system of the full size
    sp = np.nonzero(case.elems.kind == abi.DUST_ELEM_SURFPAN)[0]
    if len(sp):
        pts = np.ascontiguousarray(cen_el[sp][::uvort_stride])
        vel0 = np.zeros_like(case.cen)
        vel0[:, 0] = 1.0
        t = time.perf_counter()
        O.pressure_particles(pts, case.cen, case.dir, case.mag, case.r_vortex, vel0)
        parts["pressure"] = (time.perf_counter() - t) * len(sp) / len(pts)
        from scipy.linalg import lapack
        Ap = np.asfortranarray(rng.standard_normal((len(sp), len(sp))) * (1.0 / len(sp)))
        Ap[np.arange(len(sp)), np.arange(len(sp))] += 1.0
        Pp = np.arange(1, len(sp) + 1, dtype=np.int32)
        t = time.perf_counter()
        lapack.dgetrs(Ap, Pp - 1, np.ones(len(sp)))
        parts["pressure"] += time.perf_counter() - t
        del Ap
    # (4) FMM with the element sums
    els = abi.elements_struct(case.elems, case.wake, case.end_vort)
    O.set_sample_stride(fmm_stride)
    try:
        O.fmm_apply(params, case.cen, case.dir, case.mag, case.r_vortex, els)
        (t_tree, t_up, t_m2l, t_app), (m2l_s, npart_s) = O.last_fmm_times()
    finally:
        O.set_sample_stride(1)
    parts["fmm"] = (t_tree + t_up + t_m2l * m2l_pairs / max(m2l_s, 1)
                    + t_app * n / max(npart_s, 1))
    total_ms = 1e3 * sum(parts.values())
    sample = ("bounded sample scaled to one step per phase by the exact work ratio: uvort at "
              "1/%d of the collocation points (the pressure equation's particle term at the "
              "same share of the surface panels, plus its dgetrs in full); assembly from 8 "
              "moving rows (per entry); "
              "LAPACK solve in full; FMM tree/P2M/M2M/L2L in full, M2L at 1/%d of the target "
              "cells (by pair count), L2P+P2P+elements at 1/%d of the leaves (by particle "
              "count); phase s: %s" % (uvort_stride, fmm_stride, fmm_stride,
                                       json.dumps({k: round(v, 2) for k, v in parts.items()})))
    return total_ms, cores, sample


def run_reference(args, rank, ws):
    """--impl reference: whole steps of the reference's algorithm on the host
    cores (the oracle's C loops with OpenMP + LAPACK/BLAS, oracle/cpu_step.py),
    timed in full.  initialize_linsys (static rows + static LU) runs once
    before the timed steps.  A step of the full-size workload takes minutes
    on the host, so the arm runs one whole step (``steps`` reports the steps
    that ran)."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import cpu_step
    case = make_case(args)
    params = case.fmm_params(degree=args.degree)
    cores = host_cores()
    cpu_step.set_threads(cores)
    t0 = time.perf_counter()
    cs = cpu_step.CpuStep(case, params)
    t_init = time.perf_counter() - t0
    nsteps = 1 if not args.quick else max(1, min(args.steps, 2))
    times, phases = [], []
    for _ in range(nsteps):
        t0 = time.perf_counter()
        ph = cs.step()
        times.append((time.perf_counter() - t0) * 1e3)
        phases.append({k: round(v * 1e3, 1) for k, v in ph.items()})
    v = float(np.mean(times))
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 1), "unit": "ms",
            "n_gpus": args.gpus, "steps": nsteps, "warmup": 0, "ms_per_step": round(v, 1),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded FullStepCase)",
            "config": config_of(case, args, params),
            "mode": "reference algorithm on the host cores (FP64)",
            "phases_ms": phases, "init_s": round(t_init, 1),
            "cpu_baseline": {"value": round(v, 1), "unit": "ms", "cores": cores,
                             "kind": "port",
                             "sample": "%d whole step(s) (uvort, assembly, solve, the "
                                       "pressure equation, FMM with the element sums, the "
                                       "particle update), timed in full, after "
                                       "initialize_linsys and the static LUs (%.1f s, "
                                       "untimed); oracle C loops (OpenMP, %d threads) + "
                                       "OpenBLAS LAPACK/BLAS" % (nsteps, t_init, cores)},
            "e2e": {"value": round(v, 1), "unit": "ms", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def config_of(case, args, params):
    """The workload description both arms print (identical dicts)."""
    return {"workload": workload(case, args.degree), "levels": params.n_octree_levels,
            "l2": "256 MB flush between timed steps; A is %.2f GB"
                  % (case.rank * case.rank * 8 / 1e9),
            "parallelism": "single GPU or host; replicas under torchrun"}


def main():
    args = parse()
    rank, ws, local = dist_init(args)
    if args.impl == "reference":
        run_reference(args, rank, ws)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.workload != "full":
        line = workload_line(args, ws, args.workload)
        if rank == 0:
            print(json.dumps(line), flush=True)
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
    # mixed: FP32C FMM and uvort, mixed solve; mixed_f64uvort: the same with
    # the direct uvort sum in FP64
    modes = [("plain", abi.DUST_SOLVE_LU64), ("mixed", abi.DUST_SOLVE_MIXED),
             ("mixed_f64uvort", abi.DUST_SOLVE_MIXED)]
    learned = None
    if not args.no_learned and (not args.modes or "learned" in args.modes.split(",")):
        # the learned preconditioner trains (untimed) on the plain solutions
        # of the same geometry at rotor azimuths other than the benchmarked one
        from dust_b200 import precond
        period = 2 * np.pi / 3
        angles = (np.arange(12) + 0.5) * period / 12
        pc, info = precond.train_for_case(case, params, angles, iters=args.train_iters)
        learned = {"precond": pc, "info": info}
        modes.append(("learned", abi.DUST_SOLVE_GMRES_NN))
    fmm_uv = args.uvort == "fmm"
    if fmm_uv:
        # the reference's own uvort (direct sum) in the plain step, for comparison
        modes.append(("plain_direct_uvort", abi.DUST_SOLVE_LU64))
    if not args.no_advect and not args.profile_step:
        # FP64's own sensitivity: the plain step from particle positions
        # moved by 1e-12 (seeded), advected like the others
        modes.append(("plain_perturbed", abi.DUST_SOLVE_LU64))
    if args.modes:
        # (a profiling run, --profile-step, needs no reference mode)
        keep = set(args.modes.split(",")) | (set() if args.profile_step else {"plain"})
        modes = [m for m in modes if m[0] in keep]
    results = {}
    steppers = {}
    by_step = {}
    first_out = {}
    n_acc = max(args.accuracy_steps, max(args.warmup, 3) + args.steps)
    for name, mode in modes:
        prm = params if name.startswith("plain") else params.replace(precision=abi.DUST_PREC_FP32C)
        st = step.DeviceStepper(case, prm, mode, advect=not args.no_advect,
                                fmm_uvort=fmm_uv and name != "plain_direct_uvort",
                                uvort_params=params if name == "mixed_f64uvort" else None)
        if name == "learned":
            learned["precond"].attach(st.ls)
        if name == "plain_perturbed":
            g = torch.Generator(device="cpu").manual_seed(7)
            st.cen += (1e-12 * torch.randn(st.cen.shape, generator=g,
                                           dtype=torch.float64)).to(st.cen.device)
        steppers[name] = st
        by_step[name] = []
        # loads after every advected step (read between steps, untimed): how
        # the modes drift apart
        record = (lambda: by_step[name].append(
            case.loads(st.res.cpu().numpy(), st.euv.cpu().numpy()))) \
            if not args.profile_step else (lambda: None)
        for w in range(max(args.warmup, 1 if args.profile_step else 3)):
            st.step()
            record()
            if w == 0 and not args.profile_step:
                # the first step's particle outputs: every mode evaluates the
                # same initial wake, so their difference is the method's own
                # (no trajectory divergence yet)
                first_out[name] = [t.cpu().numpy() for t in (st.vel, st.str, st.rot)]
        torch.cuda.synchronize()
        if args.profile_step:
            continue
        barrier(ws)
        with Clocks(local) as clk:
            times = time_steps(st, args.steps, flush, after=record)
        barrier(ws)
        ms = max_over_ranks(float(np.mean(times)), ws)
        res = st.res.cpu().numpy()
        results[name] = {"ms": ms, "times": times,
                         "loads": case.loads(res, st.euv.cpu().numpy()),
                         "report": st.last_report, "clocks": clk.summary(), "res": res,
                         "fmm": [t.cpu().numpy() for t in (st.vel, st.str, st.rot)],
                         "cen": st.cen.cpu().numpy(), "n_freed": int(st.free.sum()),
                         "res_pres": st.res_pres.cpu().numpy() if st.pr is not None else None}
        # further untimed steps up to the accuracy horizon (phase breakdown and
        # launch counts below run one more step each)
        while not args.no_advect and len(by_step[name]) < n_acc:
            st.step()
            record()
    if args.profile_step:
        return
    # phase breakdown (plain and mixed share the FMM): one timed step with events
    ph = {k: phase_breakdown(steppers[k], case, params) for k in steppers}
    lp = results["plain"]["loads"]
    # Each load's error is taken relative to that load's largest magnitude
    # over the FP64 run's advected steps: the wing lift changes sign during
    # the run (|lift| falls to 0.7 % of its peak at one step), and an error
    # relative to a value that passes through zero measures nothing about the
    # method (FP64 itself, perturbed by 1e-12, shows a tenfold spike there).
    # The error relative to each step's own value is kept beside it.
    plain_steps = np.asarray(by_step.get("plain") or [lp])
    scale = np.maximum(np.max(np.abs(plain_steps), axis=0), 1e-30)
    lerr = lambda a, b: float(np.max(np.abs(a - b) / scale))
    lerr_pt = lambda a, b: float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-30)))
    load_err = {k: lerr(results[k]["loads"], lp) for k in results}
    load_err_by_step = {k: [lerr(a, b) for a, b in zip(by_step[k], by_step["plain"])]
                        for k in by_step}
    load_err_max = {k: max(v) if v else 0.0 for k, v in load_err_by_step.items()}
    load_err_pt_by_step = {k: [lerr_pt(a, b) for a, b in zip(by_step[k], by_step["plain"])]
                           for k in by_step}
    load_err_pt_max = {k: max(v) if v else 0.0 for k, v in load_err_pt_by_step.items()}
    # particle outputs of the step (velocity without the wind, stretching,
    # div-filter curl) against the FP64 step: relative L2 norms
    uinf = np.asarray(params.u_inf)
    def fmm_err(k):
        a, b = results[k]["fmm"], results["plain"]["fmm"]
        rel = lambda x, y: float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))
        return {"vel_induced": rel(a[0] - uinf, b[0] - uinf), "stretch": rel(a[1], b[1]),
                "rot": rel(a[2], b[2])}
    fmm_errs = {k: fmm_err(k) for k in results}
    for k in results:
        if k in first_out and "plain" in first_out:
            a, b = first_out[k], first_out["plain"]
            rel = lambda x, y: float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))
            fmm_errs[k]["first_step"] = {"vel_induced": rel(a[0] - uinf, b[0] - uinf),
                                         "stretch": rel(a[1], b[1]), "rot": rel(a[2], b[2])}
    # the pressure equation's solution (surface panels) against the FP64 step
    for k in results:
        a, b = results[k]["res_pres"], results["plain"]["res_pres"]
        fmm_errs[k]["pressure_solution"] = (
            float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
            if a is not None and b is not None else None)
    # the particles after all advected steps against the FP64 run's
    cp = results["plain"]["cen"]
    for k in results:
        fmm_errs[k]["position_max_abs"] = float(np.max(np.abs(results[k]["cen"] - cp)))
    # the headline mode: the fastest whose loads stay within 1e-6 of FP64 (the
    # plain step of the same algorithm) after every one of the advected steps,
    # or within twice FP64's own drift from a 1e-12 perturbation at that step
    # where that is larger
    floor = load_err.get("plain_perturbed", 0.0)
    floor_by_step = load_err_by_step.get("plain_perturbed", [])
    def within(k):
        steps_ok = all(e <= max(1e-6, 2.0 * f)
                       for e, f in zip(load_err_by_step[k], floor_by_step or
                                       [0.0] * len(load_err_by_step[k])))
        return steps_ok and load_err[k] <= max(1e-6, 2.0 * floor)
    best = min((k for k in results if within(k) and k not in ("plain_direct_uvort",
                                                              "plain_perturbed")),
               key=lambda k: results[k]["ms"])
    # end to end through the host API (pinned buffers)
    e2e = None
    if not args.no_e2e:
        prm_best = params if best == "plain" else params.replace(precision=abi.DUST_PREC_FP32C)
        e2e = run_e2e(case, prm_best, dict(modes)[best], args, ws,
                      learned["precond"] if best == "learned" else None, fmm_uv,
                      uvort_params=params if best == "mixed_f64uvort" else None)
    cpu = None
    if not args.no_cpu and rank == 0 and ws == 1:
        ms_cpu, cores, sample = cpu_baseline(case, params, ph[best]["n_m2l_pairs"])
        cpu = {"value": round(ms_cpu, 1), "unit": "ms", "cores": cores, "kind": "port",
               "sample": sample}
    launches = count_launches(steppers[best])
    rf = roofline(ph, case, params, best)
    subs = None
    if not args.no_workloads and not args.quick:
        # the other named workloads at their full sizes, 5 timed calls each
        # after 3 warm-ups (time per call, not per step)
        subs = {"fmm": run_fmm_workload(5, 3, flush=flush),
                "dense": run_dense_workload(5, 3, flush=flush),
                "learned": run_learned_workload(n_train=500, n_test=6, train_iters=2000,
                                                flush=flush),
                "wing": run_wing_workload(n_steps=200, cpu=not args.no_cpu)}
    if rank == 0:
        r = results[best]
        line = {
            "metric": METRIC, "value": round(r["ms"] / ws, 3), "unit": "ms", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(r["ms"], 3),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if best == "plain" else "f32 (uvort f64)/tf32 with f64 refinement"
                     if best == "mixed_f64uvort" else "f32/tf32 with f64 refinement",
            "data": "synthetic (seeded FullStepCase)",
            "config": config_of(case, args, params),
            "mode": best,
            "uvort": "FMM (apply_multipole_panels) in plain and mixed" if fmm_uv
                     else "direct sum",
            "plain_fp64_ms": round(results["plain"]["ms"], 3),
            "speedup_vs_plain_fp64": round(results["plain"]["ms"] / r["ms"], 3),
            "load_error_vs_fp64": load_err[best],
            "steps_advected": 0 if args.no_advect else n_acc,
            "load_error_by_step": load_err_by_step,
            "load_error_max_over_steps": load_err_max,
            "load_error_pointwise_by_step": load_err_pt_by_step,
            "load_error_pointwise_max_over_steps": load_err_pt_max,
            "loads_by_step": {k: [[float(x) for x in l] for l in v] for k, v in by_step.items()},
            "load_scale": [float(x) for x in scale],
            "fp64_sensitivity_floor": floor,
            "headline_rule": "fastest mode whose loads are within max(1e-6, 2 x the FP64 "
                             "sensitivity floor at that step) of the plain FP64 run after "
                             "every one of the %d advected steps, each load's error "
                             "relative to that load's largest magnitude over the FP64 run "
                             "(load_scale; the pointwise relative error is kept in "
                             "load_error_pointwise_*)" % n_acc,
            "load_error_note": "loads (wing lift, two rotor thrusts); every mode advects its "
                               "own particles from the same initial wake for %d steps (warm-up, "
                               "timed and untimed), so the FMM error of each step reaches the "
                               "loads of the next; load_error_vs_fp64 is after the last timed "
                               "step" % n_acc,
            "modes": {k: {"ms": round(v["ms"], 3), "load_error_vs_fp64": load_err[k],
                          "load_error_max_over_steps": load_err_max.get(k),
                          "load_error_pointwise_max_over_steps": load_err_pt_max.get(k),
                          "particle_error_vs_fp64": fmm_errs[k], "solve": v["report"]}
                      for k, v in results.items()},
            "learned_training": learned["info"] if learned else None,
            "phases_ms": ph,
            "clocks": r["clocks"],
            "roofline": rf,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "workloads": subs,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def _peaks():
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peaks = json.load(open(pk)) if os.path.exists(pk) else {}
    mhz = peaks.get("sm_max_mhz", 1965.0)
    return {
        "hbm_gbs": peaks.get("hbm_gbs", 6650.0),
        "bf16": peaks.get("bf16_tflops", 1590.0),
        "fp32": 148 * 128 * 2 * mhz * 1e6 / 1e12,
        "fp64": 148 * 64 * 2 * mhz * 1e6 / 1e12,
        "src": "of measured" if peaks else "of fallback",
        "mhz": mhz,
    }


def _event_times(fn, reps, flush):
    """CUDA-event times (ms) of `reps` calls of fn on the current stream, with
    a 256 MB write between calls (L2 holds nothing of the previous one)."""
    import torch
    out = []
    for _ in range(reps):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        out.append(e0.elapsed_time(e1))
    return out


def nmon(p):
    return (p + 1) * (p + 2) * (p + 3) // 6


# P2P flops per particle pair with stretching, divergence-filter curl and PSE
# diffusion on (the reference defaults): 27 + 30 + 18 + 20
FLOP_P2P_PAIR = 95


def run_fmm_workload(reps, warm, degrees=(4, 6, 8), n_truth=32768, flush=None):
    """Standalone wake FMM: 1M ring + 100k background particles, velocity,
    stretching, div-filter curl and PSE diffusion in FP64 and FP32C at each
    degree; errors against the FP64 direct sum at a seeded 32k-particle
    subset (all 1.1M sources); M2L roofline in HBM GB/s (source a, target b
    read and write, stretching c: 27 n_mon(p) words per pair) and P2P in
    FLOP/s (95 per pair)."""
    import torch
    from dust_b200 import octree as OCT
    from dust_b200 import synth
    pk = _peaks()
    case = synth.RingCase()
    case = case.permuted(case.truth_order(n_truth))
    n = case.n
    dev = torch.device("cuda")
    T = lambda a: torch.as_tensor(a, device=dev)
    cen, dir_, mag, rv = T(case.cen), T(case.dir), T(case.mag), T(case.r_vortex)
    vel, st, ro = (torch.empty((n, 3), dtype=torch.float64, device=dev) for _ in range(3))
    if flush is None:
        flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    t0 = time.perf_counter()
    tv, ts, _ = OCT.direct_particles(case.fmm_params(4), case.cen, case.dir, case.mag,
                                     case.r_vortex, n_tgt=n_truth)
    t_direct = time.perf_counter() - t0
    rel = lambda a, b: float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
    stream = torch.cuda.current_stream().cuda_stream
    out = {}
    for p in degrees:
        full64 = None
        for name, prec in (("fp64", 0), ("fp32c", 1)):
            prm = case.fmm_params(p, prec)
            oc = OCT.Octree(prm)
            call = lambda: oc.apply_multipole_device(cen, dir_, mag, rv, vel, st, ro,
                                                     stream=stream, sync=False)
            for _ in range(warm):
                call()
            torch.cuda.synchronize()
            times = _event_times(call, reps, flush)
            oc.set_timing(True)
            call()
            torch.cuda.synchronize()
            sx = oc.stats()
            oc.set_timing(False)
            v, s_ = vel.cpu().numpy(), st.cpu().numpy()
            r = {"ms": round(float(np.mean(times)), 3), "ms_min": round(min(times), 3),
                 "error_vs_direct_fp64": {"vel": rel(v[:n_truth], tv),
                                          "stretch": rel(s_[:n_truth], ts)},
                 "phases_ms": {k: round(sx[k], 3) for k in
                               ("ms_tree", "ms_upward", "ms_m2l", "ms_p2p", "ms_total",
                                "ms_m2l_kernel")},
                 "n_leaves": sx["n_leaves"], "n_m2l_pairs": sx["n_m2l_pairs"],
                 "n_p2p_pairs": sx["n_p2p_pairs"]}
            if full64 is None:
                full64 = (v.copy(), s_.copy())
            else:
                r["error_vs_fmm_fp64"] = {"vel": rel(v, full64[0]),
                                          "stretch": rel(s_, full64[1])}
            w = 8 if prec == 0 else 4
            m2l_ms = sx["ms_m2l"]
            byts = 27 * nmon(p) * w * sx["n_m2l_pairs"]
            flo = 12 * nmon(p + 1) * nmon(p) * sx["n_m2l_pairs"]
            p2p_peak = pk["fp64"] if prec == 0 else pk["fp32"]
            p2p_ach = FLOP_P2P_PAIR * sx["n_p2p_pairs"] / (sx["ms_p2p"] * 1e-3) / 1e12
            r["roofline"] = {
                "m2l": {"bound": "hbm", "achieved": round(byts / (m2l_ms * 1e-3) / 1e9, 1),
                        "peak": pk["hbm_gbs"], "unit": "GB/s",
                        "frac": round(byts / (m2l_ms * 1e-3) / 1e9 / pk["hbm_gbs"], 3),
                        "tflops": round(flo / (m2l_ms * 1e-3) / 1e12, 2),
                        "algorithmic_bytes": int(byts), "ms": round(m2l_ms, 3),
                        "peak_source": "HBM copy " + pk["src"]},
                "p2p": {"bound": "fp64" if prec == 0 else "fp32", "achieved": round(p2p_ach, 2),
                        "peak": round(p2p_peak, 1), "unit": "TFLOP/s",
                        "frac": round(p2p_ach / p2p_peak, 3), "flop_per_pair": FLOP_P2P_PAIR,
                        "ms": round(sx["ms_p2p"], 3),
                        "peak_source": "nominal %s SIMT (148 SMs x %d lanes x 2 x %g MHz)"
                                       % ("FP64" if prec == 0 else "FP32",
                                          64 if prec == 0 else 128, pk["mhz"])}}
            out["p%d_%s" % (p, name)] = r
            oc.close()
    return {"workload": "standalone wake FMM: 1,000,000 ring + 100,000 background particles, "
                        "core 0.02, %d levels (leaves <= 64), vel + stretching + div-filter "
                        "curl + PSE" % case.levels,
            "unit": "ms per FMM evaluation", "reps": reps, "warmup": warm,
            "truth": "FP64 direct sum (GPU) at %d seeded targets over all %d sources, %.1f s"
                     % (n_truth, n, t_direct),
            "l2": "256 MB flush between timed calls", "results": out}


def run_dense_workload(reps, warm, n_target=16384, nrhs=64, flush=None):
    """Mixed-precision dense solve: 16,384-panel ellipsoid, Dirichlet AIC, 64
    right-hand sides; plain FP64 LU against the FP32 LU with tensor-core
    (tcgen05 TF32) trailing updates + FP64 refinement to 1e-12."""
    import torch
    from dust_b200 import abi, linsys, synth
    pk = _peaks()
    case = synth.EllipsoidCase(n_target=n_target, nrhs=nrhs)
    n = case.n
    prm = case.fmm_params()
    body = case.body
    body.uvort = np.zeros((n, 3))
    ls = linsys.Linsys(prm, n, 0, body)
    G = np.empty((n, 3))
    t_asm = []
    for d in range(3):
        body.ub = case.unit_ub(d)
        t0 = time.perf_counter()
        ls.assemble_linsys(body)
        ls.sync()
        t_asm.append((time.perf_counter() - t0) * 1e3)
        A, b = ls.get_system()
        G[:, d] = b
    ls.close()
    B = -G @ case.U
    dev = torch.device("cuda")
    Ad = torch.as_tensor(np.ascontiguousarray(A.T), device=dev)  # column-major A
    del A
    Bd = torch.as_tensor(np.ascontiguousarray(B.T), device=dev)
    X64 = torch.empty_like(Bd)
    X32 = torch.empty_like(Bd)
    if flush is None:
        flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    res = {}
    for name, mode, X in (("lu64", abi.DUST_SOLVE_LU64, X64), ("mixed", abi.DUST_SOLVE_MIXED, X32)):
        reps_ = []
        call = lambda: reps_.append(linsys.dense_solve_device(Ad, Bd, X, mode, 1e-12, stream))
        for _ in range(warm):
            call()
        times = _event_times(call, reps, flush)
        rep = reps_[-1]
        res[name] = {"ms": round(float(np.mean(times)), 3), "ms_min": round(min(times), 3),
                     "report": rep}
    # backward errors ||B - A X||_inf / (||A||_inf ||X||_inf) per column (FP64 on the GPU)
    Anorm = float(Ad.abs().sum(dim=0).max())  # rows of A are columns of Ad
    def berr(X):
        R = Bd - X @ Ad  # (nrhs, n): row c = (A x_c)^T
        return float((R.abs().amax(dim=1) / (Anorm * X.abs().amax(dim=1))).max())
    for name, X in (("lu64", X64), ("mixed", X32)):
        res[name]["backward_error"] = berr(X)
    res["mixed"]["rel_error_vs_lu64"] = float(torch.linalg.norm(X32 - X64) / torch.linalg.norm(X64))
    flops_lu = 2.0 / 3.0 * n ** 3
    flops_tot = flops_lu + 2.0 * n * n * nrhs
    tf32 = pk["bf16"] / 2
    f = res["mixed"]["report"]["ms_factor"]
    res["mixed"]["roofline"] = {
        "bound": "tensor", "achieved": round(flops_lu / (f * 1e-3) / 1e12, 1), "peak": tf32,
        "unit": "TFLOP/s", "frac": round(flops_lu / (f * 1e-3) / 1e12 / tf32, 3),
        "what": "FP32 LU (TF32 tcgen05 trailing updates), (2/3) n^3 over ms_factor",
        "peak_source": "TF32 = bf16 %s / 2" % pk["src"]}
    f64 = res["lu64"]["report"]["ms_factor"]
    res["lu64"]["roofline"] = {
        "bound": "fp64", "achieved": round(flops_lu / (f64 * 1e-3) / 1e12, 2),
        "peak": round(pk["fp64"], 1), "unit": "TFLOP/s",
        "frac": round(flops_lu / (f64 * 1e-3) / 1e12 / pk["fp64"], 3),
        "peak_source": "nominal FP64 (148 SMs x 64 x 2 x %g MHz)" % pk["mhz"]}
    del Ad
    torch.cuda.empty_cache()
    return {"workload": "dense solve: closed ellipsoid (4, 1, 0.5) of %d surface panels "
                        "(%d quads + %d cap triangles), Dirichlet AIC, %d freestream RHS"
                        % (n, int(np.sum(body.n_ver == 4)), int(np.sum(body.n_ver == 3)), nrhs),
            "unit": "ms per solve (factor + all RHS)", "reps": reps, "warmup": warm,
            "assembly_ms_wall": [round(t, 2) for t in t_asm],
            "flops_factor": flops_lu, "flops_total": flops_tot,
            "speedup_mixed_vs_lu64": round(res["lu64"]["ms"] / res["mixed"]["ms"], 3),
            "l2": "256 MB flush between timed calls; A is %.2f GB" % (n * n * 8 / 1e9),
            "results": res}


def run_learned_workload(n_train=500, n_test=8, train_iters=2000, flush=None):
    """Learned preconditioner on the moving-body system: rotor over a
    fuselage (about 7k unknowns, 960 moving), systems drawn from plain-method
    steps with seeded rpm (+-20 %), azimuth and inflow angle.  The network is
    trained on n_train systems the plain LU solved; on n_test held-out draws
    the plain per-step solve (LU64: static LU reused, Schur update of the
    moving block) is timed against the learned-preconditioned GMRES
    (iterations, fallback, error against LU)."""
    import torch
    from dust_b200 import abi, linsys, precond, synth
    case = synth.RotorFuselageCase()
    prm = case.fmm_params()
    t0 = time.perf_counter()
    els0 = case.system(10 ** 6)
    ls = linsys.Linsys(prm, case.rank, case.nstatic, els0)
    pc = precond.Precond(precond._centres(els0), k=8, seed=0)
    for q in range(n_train):
        els = case.system(q)
        ls.assemble_linsys(els)
        x, _ = ls.solve_linsys(abi.DUST_SOLVE_LU64)
        ls.assemble_linsys(els)
        pc.add_sample(ls, x, seed=q)
    t_data = time.perf_counter() - t0
    t0 = time.perf_counter()
    l0 = float(np.mean([pc.loss_grad(i, with_grad=False)[0] for i in range(min(64, n_train))]))
    l1 = pc.train(train_iters, 2e-3)
    t_train = time.perf_counter() - t0
    untrained = precond.Precond(precond._centres(els0), k=8, seed=0)
    stream = torch.cuda.current_stream()
    rows = []
    for q in range(n_test):
        els = case.system(10 ** 6 + q)
        rec = {}
        for name, mode, p in (("lu64", abi.DUST_SOLVE_LU64, None),
                              ("gmres_untrained", abi.DUST_SOLVE_GMRES_NN, untrained),
                              ("gmres_nn", abi.DUST_SOLVE_GMRES_NN, pc)):
            if p is not None:
                p.attach(ls)
            ls.assemble_linsys(els)
            ls.sync()
            if flush is not None:
                flush.zero_()
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            x, rep = ls.solve_linsys(mode)
            ms = (time.perf_counter() - t1) * 1e3
            rec[name] = {"ms": ms, "x": x, "rep": rep}
            if p is not None:
                precond.Precond.detach(ls)
        xl = rec["lu64"]["x"]
        rows.append({k: {"ms": round(v["ms"], 3), "iterations": int(v["rep"]["iterations"]),
                         "fell_back": int(v["rep"]["fell_back"]),
                         "rel_error_vs_lu64": float(np.linalg.norm(v["x"] - xl)
                                                    / np.linalg.norm(xl))}
                     for k, v in rec.items()})
    ls.close()
    summ = {}
    for k in ("lu64", "gmres_untrained", "gmres_nn"):
        r = [row[k] for row in rows[1:]]  # the first draw warms the handles up
        summ[k] = {"ms_mean": round(float(np.mean([x["ms"] for x in r])), 3),
                   "iterations_mean": round(float(np.mean([x["iterations"] for x in r])), 2),
                   "fallbacks": int(sum(x["fell_back"] for x in r)),
                   "max_rel_error_vs_lu64": max(x["rel_error_vs_lu64"] for x in r)}
    return {"workload": "learned preconditioner: 4-blade rotor (30 x 8 VLM per blade, 960 "
                        "moving unknowns) over a %d-panel fuselage, %d unknowns"
                        % (case.nstatic, case.rank),
            "unit": "ms per solve (host wall clock around the synchronous solve call)",
            "train": {"systems": n_train, "adam_iters": train_iters, "loss_untrained": l0,
                      "loss_trained": l1, "s_data": round(t_data, 1),
                      "s_train": round(t_train, 1)},
            "test_draws": n_test - 1, "results": summ}


def run_wing_workload(n_steps=200, n_wake_panels=1, levels=6, cpu=True):
    """Plain method, small: flat rectangular vortex-lattice wing (span 10,
    chord 1, 40 x 10 panels, 400 unknowns, LU factored once) at 5 degrees in
    a 1 m/s stream, dt 0.05, n_steps steps of the reference's time loop with
    its panel wake (n_wake_panels rows) shedding one particle per stripe per
    step (40 per step once the wake is full), particle core 0.1 chord, FMM
    p = 4 with leaves <= 64.  Every step runs on the GPU through the C ABI
    (WakeStepper: live list, uvort, assembly, solve, update_wake with the
    FMM, complete_wake with shedding); the same loop runs on the CPU oracle
    for the solution's agreement and the CPU time."""
    import torch
    from dust_b200 import synth
    from dust_b200.step import WakeStepper
    case = synth.WingWakeCase(steps=n_steps, n_wake_panels=n_wake_panels)
    fp = case.fmm_params(levels=levels)
    gpu = WakeStepper(case, fp)
    ms, res, phases = [], [], []
    for s in range(n_steps):
        gpu.phase_events = s >= n_steps - 20
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        gpu.step()
        e1.record()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
        res.append(gpu.res.cpu().numpy())
        if gpu.phase_events:
            phases.append(gpu.phase_ms())
    gc, ga, gr = gpu.particles()
    gpu.close()
    out = {"workload": "VLM wing 40 x 10 (400 unknowns), panel wake of %d row(s), %d steps of "
                       "dt 0.05 with trailing-edge shedding to %d particles, core 0.1, FMM p = 4, "
                       "%d levels" % (n_wake_panels, n_steps, len(gc), levels),
           "unit": "ms per timestep (CUDA events around each whole step, its host "
                   "synchronisations included)",
           "steps": n_steps, "particles_final": int(len(gc)),
           "ms_per_step_mean": round(float(np.mean(ms)), 4),
           "ms_per_step_last20": round(float(np.mean(ms[-20:])), 4),
           "ms_total": round(float(np.sum(ms)), 2),
           "phases_ms_last20": {k: round(float(np.mean([p[k] for p in phases])), 4)
                                for k in phases[0]} if phases else None}
    if cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import cpu_step
        import oracle as O
        import wake_oracle as W
        cpu_step.set_threads(host_cores())
        run = W.OracleWakeRun(O, case, fp)
        t0 = time.perf_counter()
        errs = []
        for s in range(n_steps):
            run.step()
            errs.append(float(np.linalg.norm(res[s] - run.res) / np.linalg.norm(run.res)))
        t_cpu = time.perf_counter() - t0
        oc, oa, orv = run.particles()
        out["cpu_baseline"] = {"value": round(t_cpu / n_steps * 1e3, 3), "unit": "ms per timestep",
                               "cores": host_cores(), "kind": "port",
                               "sample": "the whole %d-step loop on the oracle (C restatement "
                                         "with OpenMP; the oracle re-assembles and re-factors "
                                         "the 400-unknown system every step)" % n_steps}
        out["solution_rel_error_vs_oracle_max_over_steps"] = max(errs)
        out["solution_rel_error_vs_oracle_last"] = errs[-1]
        out["particles_equal_count"] = bool(len(oc) == len(gc))
        if len(oc) == len(gc) and len(gc):
            out["particle_position_max_abs_diff"] = float(np.abs(oc - gc).max())
    return out


def workload_line(args, ws, name):
    """--workload fmm / dense: that workload as the bench line."""
    import torch
    torch.cuda.set_stream(torch.cuda.Stream())
    warm = max(args.warmup, 3)
    if name == "fmm":
        degs = tuple(int(x) for x in args.degrees.split(","))
        with Clocks(0) as clk:
            w = run_fmm_workload(args.steps, warm, degs)
        best = w["results"]["p%d_fp32c" % degs[0]]
        plain = w["results"]["p%d_fp64" % degs[0]]
        metric = "ms per FMM evaluation (1.1M ring particles, p=%d, FP32C vs FP64)" % degs[0]
        rf = dict(best["roofline"]["m2l"])
        rf["kernel"] = "M2L phase"
        rf["traffic"] = None
        rf["others"] = [dict(best["roofline"]["p2p"], kernel="P2P phase")]
        dtype = "f32/tf32 (FP32C)"
    elif name == "wing":
        with Clocks(0) as clk:
            w = run_wing_workload(n_steps=200, cpu=not args.no_cpu)
        w["l2"] = "not flushed: the whole state (400 panels, <= 8,000 particles) is cache resident"
        best = {"ms": w["ms_per_step_mean"]}
        plain = {"ms": w["ms_per_step_mean"]}
        metric = "ms per timestep (VLM wing 40 x 10, wake shedding, 200 steps, FP64)"
        rf = {"kernel": "whole step", "bound": "latency", "achieved": None, "peak": None,
              "unit": "GB/s", "frac": None, "traffic": None,
              "note": "a few hundred unknowns and <= 8,000 particles: launch- and "
                      "synchronisation-bound; no roofline claimed"}
        dtype = "f64"
    elif name == "learned":
        with Clocks(0) as clk:
            w = run_learned_workload(n_train=2000, n_test=max(args.steps, 3) + 1,
                                     train_iters=6000)
        best = dict(w["results"]["gmres_nn"], ms=w["results"]["gmres_nn"]["ms_mean"])
        plain = dict(w["results"]["lu64"], ms=w["results"]["lu64"]["ms_mean"])
        metric = "ms per moving-body solve (~7k unknowns), learned GMRES vs per-step LU"
        rf = {"kernel": "GMRES_NN solve", "bound": "hbm", "achieved": None, "peak": None,
              "unit": "GB/s", "frac": None, "traffic": None,
              "note": "latency-bound iterative solve; no roofline claimed"}
        dtype = "f64 GMRES with f32 preconditioner"
    else:
        with Clocks(0) as clk:
            w = run_dense_workload(args.steps, warm, n_target=args.dense_panels)
        best = w["results"]["mixed"]
        plain = w["results"]["lu64"]
        metric = "ms per dense solve (%s-panel ellipsoid, 64 RHS), MIXED vs LU64" % format(
            args.dense_panels, ",")
        rf = dict(best["roofline"])
        rf["kernel"] = "FP32 LU with tcgen05 TF32 trailing updates"
        rf["traffic"] = None
        dtype = "f32/tf32 with f64 refinement"
    ms = max_over_ranks(best["ms"], ws)
    line = {"metric": metric, "value": round(ms, 3), "unit": "ms", "n_gpus": ws,
            "steps": args.steps, "warmup": warm, "ms_per_step": round(ms, 3),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": dtype,
            "data": "synthetic (seeded)", "config": {"workload": w["workload"],
                                                     "l2": w["l2"]},
            "plain_fp64_ms": plain["ms"], "detail": w, "roofline": rf,
            "clocks": clk.summary(), "cpu_baseline": w.get("cpu_baseline"), "e2e": None}
    return line


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
    first = "fmm_prepare_and_uvort" if st.fmm_uvort else "uvort"
    return {"total": t(0, 6), first: t(0, 1), "assemble": t(1, 2), "pressure": t(2, 3),
            "solve": t(3, 4), "fmm_total": t(4, 5), "particles_update": t(5, 6),
            "fmm_tree": round(s["ms_tree"], 3),
            "fmm_upward": round(s["ms_upward"], 3), "fmm_m2l": round(s["ms_m2l"], 3),
            "fmm_p2p": round(s["ms_p2p"], 3), "fmm_elements": round(s["ms_elems"], 3),
            "n_leaves": s["n_leaves"], "n_active_cells": s["n_active_cells"],
            "n_m2l_pairs": s["n_m2l_pairs"], "n_p2p_pairs": s["n_p2p_pairs"],
            "n_elem_pairs": s["n_elem_pairs"],
            "k_m2l_batch_ms": round(s["ms_m2l_kernel"], 3),
            "k_elem_far_ms": round(s["ms_elem_far"], 3)}


# Algorithmic work per unit (FMA = 2 flops), from the kernels' formulas:
#  far element pair (k_elem_far): r (3) + r^2 (5) + rsqrt (1) + 1/r^2 (1)
#    + r.n (5) + 1/r^3 (1) + coefficient (3) + 3 x fma(k3, fma(coef, r, -mu n)) (12)
FLOP_ELEM_PAIR = 31
#  uvort pair (k_uvort / k_uvort_sorted): d (3) + rho^2 (6) + rsqrt (1) + rho^-3 (2)
#  + c d (3) + c d x alpha accumulated (6 fma, 12)
FLOP_UVORT_PAIR = 27
#  with the pressure equation's particle term in the same pass (k_uvort_pres /
#  k_uvort_pres_sorted; difference and rho^-3 shared): d . (-w) (5) + times
#  rho^-3 (1) + accumulation (1)
FLOP_UVORT_PRES_PAIR = FLOP_UVORT_PAIR + 7
#  M2L pair at p = 4 with stretching, in the scalar form the kernel evaluates:
#  L_c(j) = sum_n Shat(j+n) a_c(n) for the 83 indices 1 <= |j| <= 6, the 35
#  source monomials and 3 components, one FMA each (the cross-product form
#  it replaces takes 56 x 35 x 6 FMAs)
FLOP_M2L_PAIR = 83 * 35 * 3 * 2
#  M2L pair, algorithmic bytes at p = 4 (35 monomials, w bytes a word): source
#  a (3 x 35 w) + target b read and write (2 x 3 x 35 w) + stretching c read
#  and write (2 x 9 x 35 w)
BYTES_M2L_PAIR_WORDS = 3 * 35 + 2 * 3 * 35 + 2 * 9 * 35
#  P2P pair with stretching, div-filter rotu and PSE diffusion: 27 + 30 + 18 + 20
FLOP_P2P_PAIR = 95
# DRAM bytes per launch measured by ncu (dram__bytes_read.sum +
# dram__bytes_write.sum) on the 300k-particle case and scaled by the particle
# count to 2M (profiles/k_elem_far_300k.txt)
TRAFFIC_ELEM_FAR_PER_PARTICLE = 381.5
# DRAM bytes per launch per particle of the 300k-particle full step (ncu,
# profiles/k_uvort_300k.txt, k_m2l_batch_f32_300k.txt, k_p2p_w_f32_300k.txt),
# scaled by the particle count to the benchmark's size
TRAFFIC_UVORT_PER_PARTICLE = 19.88e6 / 3.0e5
TRAFFIC_M2L_F32_PER_PARTICLE = (138.53e6 + 53.36e6) / 3.0e5
TRAFFIC_P2P_F32_PER_PARTICLE = (119.11e6 + 21.72e6) / 3.0e5
# FMA-pipe activity of the FP32C kernels in the same captures
# (sm__pipe_fma_cycles_active, profiles/*_300k.txt)
FMA_PIPE_NCU = {"k_m2l_batch": 0.376, "k_p2p_w": 0.305, "k_uvort_pres_sorted": 0.807,
                "k_elem_far": 0.67}


def roofline(ph, case, params, best):
    """Roofline of the dominant kernel of the headline mode (``best``), with
    the step's other large kernels in ``others``.  Peaks: MEASURED_PEAKS.json
    (HBM copy GB/s); the FP32 and FP64 SIMT peaks are not measured there and
    are the nominal 148 SMs x 128 (FP32) or 64 (FP64) lanes x 2 flops x
    sm_max_mhz."""
    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
    mhz = peaks.get("sm_max_mhz", 1965.0)
    fp32_peak = 148 * 128 * 2 * mhz * 1e6 / 1e12
    fp64_peak = fp32_peak / 2
    hbm = peaks.get("hbm_gbs", 6650.0)
    hbm_src = "of measured" if "hbm_gbs" in peaks else "of fallback"
    p = ph.get(best, {})
    # FMM kernels are FP64 in the plain modes; the direct uvort sum also in
    # mixed_f64uvort
    f64 = best.startswith("plain")
    uv64 = f64 or best == "mixed_f64uvort"
    w = 8 if f64 else 4
    simt = fp64_peak if f64 else fp32_peak
    name_of = lambda d: "nominal %s SIMT (148 SMs x %d x 2 x %g MHz)" % (
        "FP64" if d else "FP32", 64 if d else 128, mhz)
    simt_name = name_of(f64)
    n = case.mag.shape[0]
    ks = []
    if p.get("k_elem_far_ms"):
        a = FLOP_ELEM_PAIR * p["n_elem_pairs"] / (p["k_elem_far_ms"] * 1e-3) / 1e12
        tr = None if TRAFFIC_ELEM_FAR_PER_PARTICLE is None else int(TRAFFIC_ELEM_FAR_PER_PARTICLE * n)
        ks.append({"kernel": "k_elem_far", "bound": "fp32", "achieved": round(a, 2),
                   "peak": round(fp32_peak, 1), "unit": "TFLOP/s", "frac": round(a / fp32_peak, 3),
                   "traffic": tr, "peak_source": simt_name, "flop_per_pair": FLOP_ELEM_PAIR,
                   "fma_pipe_active_ncu": FMA_PIPE_NCU["k_elem_far"],
                   "pairs": p["n_elem_pairs"], "ms": p["k_elem_far_ms"]})
    elif p.get("fmm_elements"):
        a = FLOP_ELEM_PAIR * p["n_elem_pairs"] / (p["fmm_elements"] * 1e-3) / 1e12
        ks.append({"kernel": "k_elem_out (elements, end vortices, outputs)",
                   "bound": "fp64" if f64 else "fp32", "achieved": round(a, 2),
                   "peak": round(simt, 1), "unit": "TFLOP/s", "frac": round(a / simt, 3),
                   "traffic": None, "peak_source": simt_name, "flop_per_pair": FLOP_ELEM_PAIR,
                   "pairs": p["n_elem_pairs"], "ms": p["fmm_elements"]})
    if p.get("k_m2l_batch_ms"):
        t = p["k_m2l_batch_ms"] * 1e-3
        gbs = BYTES_M2L_PAIR_WORDS * w * p["n_m2l_pairs"] / t / 1e9
        fl = FLOP_M2L_PAIR * p["n_m2l_pairs"] / t / 1e12
        ks.append({"kernel": "k_m2l_batch", "bound": "hbm", "achieved": round(gbs, 1),
                   "peak": round(hbm, 1), "unit": "GB/s", "frac": round(gbs / hbm, 3),
                   "traffic": None if f64 else int(TRAFFIC_M2L_F32_PER_PARTICLE * n),
                   "peak_source": "HBM copy %s" % hbm_src,
                   "bytes_per_pair": BYTES_M2L_PAIR_WORDS * w, "pairs": p["n_m2l_pairs"],
                   "ms": p["k_m2l_batch_ms"],
                   "flops": {"achieved": round(fl, 2), "peak": round(simt, 1),
                             "unit": "TFLOP/s", "frac": round(fl / simt, 3),
                             "flop_per_pair": FLOP_M2L_PAIR, "peak_source": simt_name,
                             "fma_pipe_active_ncu": None if f64 else
                             FMA_PIPE_NCU["k_m2l_batch"]}})
    if p.get("fmm_p2p"):
        a = FLOP_P2P_PAIR * p["n_p2p_pairs"] / (p["fmm_p2p"] * 1e-3) / 1e12
        ks.append({"kernel": "k_p2p_w (L2P + P2P)", "bound": "fp64" if f64 else "fp32",
                   "achieved": round(a, 2), "peak": round(simt, 1), "unit": "TFLOP/s",
                   "frac": round(a / simt, 3),
                   "traffic": None if f64 else int(TRAFFIC_P2P_F32_PER_PARTICLE * n),
                   "peak_source": simt_name,
                   "fma_pipe_active_ncu": None if f64 else FMA_PIPE_NCU["k_p2p_w"],
                   "flop_per_pair": FLOP_P2P_PAIR, "pairs": p["n_p2p_pairs"], "ms": p["fmm_p2p"]})
    if p.get("uvort"):
        pairs = case.rank * n
        # with the pressure equation the step's uvort pass carries its
        # particle term (dust_points_uvort_pressure_device)
        fused = bool(p.get("pressure"))
        fpp = FLOP_UVORT_PRES_PAIR if fused else FLOP_UVORT_PAIR
        a = fpp * pairs / (p["uvort"] * 1e-3) / 1e12
        pk_uv = fp64_peak if uv64 else fp32_peak
        kname = ("k_uvort_pres" if fused else "k_uvort") if uv64 else \
            ("k_uvort_pres_sorted + sort" if fused else "k_uvort_sorted + sort")
        ks.append({"kernel": "uvort phase (%s)" % kname,
                   "bound": "fp64" if uv64 else "fp32", "achieved": round(a, 2),
                   "peak": round(pk_uv, 1), "unit": "TFLOP/s", "frac": round(a / pk_uv, 3),
                   "traffic": int(TRAFFIC_UVORT_PER_PARTICLE * n) if uv64 else None,
                   "peak_source": name_of(uv64),
                   "fp64_pipe_active_ncu": 0.723 if uv64 else None,
                   "fma_pipe_active_ncu": None if uv64 or not fused else
                   FMA_PIPE_NCU["k_uvort_pres_sorted"],
                   "flop_per_pair": fpp, "pairs": pairs, "ms": p["uvort"]})
    if not ks:
        return {"others": [], "peaks_file": bool(peaks)}
    ks.sort(key=lambda k: -k["ms"])
    out = dict(ks[0])
    out["others"] = ks[1:]
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


def e2e_bytes(case, n, advect, fmm_uvort=False):
    """Bytes the host entry points copy per step (each call copies its own
    inputs and outputs): dust_points_uvort (points, particles, end vortices ->
    uvort), dust_linsys_assemble (panels, wake rows), dust_linsys_solve (->
    strengths), dust_fmm_apply (particles, panels, wake panels, end vortices
    -> vel, stretch, rotu) and, when advecting, dust_particles_update
    (cen, dir, mag, vel, stretch, rotu, free flags -> cen, dir, stretch, free
    flags, count); with surface panels, uvort through
    dust_points_uvort_pressure (also the particles' velocities -> the
    pressure equation's particle term), dust_pressure_assemble_terms (that
    term) and dust_pressure_solve (-> solution); with the FMM uvort,
    dust_pressure_assemble (particles and their velocities) instead."""
    d, i = 8, 4
    nr, nw, nl = case.rank, case.wake.n, case.end_vort.n
    panels = nr * (12 * d + 2 * i + 7 * d)        # ver, n_ver, kind, mag, ub, uvort
    wakep = nw * (12 * d + 2 * i + d)             # ver, n_ver, kind, mag
    lines = nl * 7 * d
    parts = n * 8 * d                             # cen, dir, mag, r_vortex
    if fmm_uvort:
        # dust_fmm_prepare (particles once), dust_fmm_points_uvort (points,
        # end vortices), dust_fmm_finish (panels, wake panels, end vortices)
        h2d = parts + nr * 3 * d + lines
        h2d += panels + wakep + nw * 2 * i        # assemble (+ implicit indices)
        h2d += panels + wakep + lines             # FMM finish
    else:
        h2d = (nr * 3 * d + parts + lines)        # uvort
        h2d += panels + wakep + nw * 2 * i        # assemble (+ implicit indices)
        h2d += parts + panels + wakep + lines     # FMM
    d2h = nr * 3 * d + nr * d + n * 9 * d         # uvort, strengths, vel/stretch/rotu
    from dust_b200 import abi
    nsp = int(np.sum(case.elems.kind == abi.DUST_ELEM_SURFPAN))
    if nsp and fmm_uvort:
        # dust_pressure_assemble (particles with their velocities), and from
        # the second step dust_pressure_solve (-> the surface panels' solution)
        h2d += parts + n * 3 * d
        d2h += nsp * d
    elif nsp:
        # the particles' velocities into dust_points_uvort_pressure (-> its
        # term at every element), that term into dust_pressure_assemble_terms,
        # dust_pressure_solve (-> the surface panels' solution)
        h2d += n * 3 * d + nr * d
        d2h += nr * d + nsp * d
    if advect:
        h2d += n * (16 * d + i)
        d2h += n * (9 * d + i) + i
    return h2d, d2h


def run_e2e(case, params, mode, args, ws, pc=None, fmm_uvort=False, uvort_params=None):
    """Same step through the host API with pinned host buffers: every step
    copies particles and panels in and velocities/strengths out."""
    import torch
    from dust_b200 import step
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    case.cen, case.dir, case.mag, case.r_vortex = (pin(case.cen), pin(case.dir),
                                                  pin(case.mag), pin(case.r_vortex))
    n = case.mag.shape[0]
    out = tuple(pin(np.empty((n, 3))) for _ in range(3))  # page-locked outputs
    hs = step.HostStepper(case, params, mode, out=out, advect=not args.no_advect,
                          fmm_uvort=fmm_uvort, uvort_params=uvort_params)
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
    h2d, d2h = e2e_bytes(case, n, not args.no_advect, fmm_uvort)
    return {"value": round(ms, 3), "unit": "ms", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "step_ms": [round(t, 2) for t in times]}


if __name__ == "__main__":
    main()
