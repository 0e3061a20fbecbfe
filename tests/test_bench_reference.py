"""The reference arm of bench.py (the oracle's CPU restatement of the
reference, timed on the host cores) prints one JSON line in the benchmark
contract; run here on the small case."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--quick", "--particles", "20000", "--steps", "1", "--warmup", "0"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "ms" and d["higher_is_better"] is False
    assert d["value"] > 0 and d["ms_per_step"] == d["value"]
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    # whole steps timed in full: the reported time fits the run
    assert d["steps"] >= 1 and "whole step" in d["cpu_baseline"]["sample"]
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "ms", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert "particles" in d["config"]["workload"]


def test_reference_arm_two_ranks():
    """Under torchrun only rank 0 runs the reference arm and prints; the other
    rank exits 0 without work (gloo here, no GPU needed)."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", "29617",
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--quick", "--particles", "20000",
           "--steps", "1", "--warmup", "0", "--gpus", "2"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0


def test_roofline_fields():
    """The roofline object of the bench line from a phase breakdown: the
    headline mode's dominant kernel (here the FP32C element far field),
    achieved = algorithmic flops (or bytes) / kernel time, frac = achieved /
    peak, traffic scaled by the particles; M2L in GB/s with its flop rate."""
    sys.path.insert(0, ROOT)
    import bench
    from dust_b200 import synth
    case = synth.FullStepCase(n_particles=10_000)
    params = case.fmm_params()
    ph = {"mixed": {"k_elem_far_ms": 2.0, "n_elem_pairs": 10_000 * 14_596,
                    "k_m2l_batch_ms": 1.0, "n_m2l_pairs": 1000, "uvort": 1.5,
                    "fmm_p2p": 0.5, "n_p2p_pairs": 4000}}
    rf = bench.roofline(ph, case, params, "mixed")
    for k in ("bound", "achieved", "peak", "unit", "frac", "traffic"):
        assert k in rf
    ach = bench.FLOP_ELEM_PAIR * 10_000 * 14_596 / 2e-3 / 1e12
    assert rf["kernel"] == "k_elem_far"
    assert abs(rf["achieved"] - ach) <= 0.01 and abs(rf["frac"] - ach / rf["peak"]) <= 1e-3
    assert rf["unit"] == "TFLOP/s" and rf["traffic"] > 0
    names = [o["kernel"] for o in rf["others"]]
    assert names[0].startswith("uvort") and "k_m2l_batch" in names
    m2l = rf["others"][names.index("k_m2l_batch")]
    assert m2l["unit"] == "GB/s" and m2l["bound"] == "hbm"
    gbs = bench.BYTES_M2L_PAIR_WORDS * 4 * 1000 / 1e-3 / 1e9
    assert abs(m2l["achieved"] - gbs) <= 0.1 and m2l["flops"]["unit"] == "TFLOP/s"
