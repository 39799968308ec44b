"""The reference arm of bench.py runs on the CPU alone and prints the one
JSON line of the bench contract (impl, metric, value, unit, config,
cpu_baseline, e2e), on the same metric and workload names as the GPU arm."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_the_contract_line():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1",
                          "--ref-budget", "0.3"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["unit"] == "matvec/s" and d["value"] > 0
    assert d["config"]["workload"] and d["cpu_baseline"]["kind"] in ("port", "reference")
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0


def test_reference_arm_on_a_three_body_workload_says_unavailable():
    # the CPU restatements time two-body bundles only: the reference arm of a
    # three-body workload prints its `unavailable` line and exits 0
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "pf4p3n3b"], cwd=ROOT,
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    d = json.loads([ln for ln in out.stdout.splitlines() if ln.startswith("{")][0])
    assert d["impl"] == "reference" and "unavailable" in d


def test_alg_bytes_counts_three_body_updates_and_tables():
    sys.path.insert(0, ROOT)
    import bench
    from bigstickpublick_b200 import model
    T = model.build_tables3(model.sd_model(3, 2, seed=3, jz2=1), w2=1.0, w3=0.2, seed=1)
    import oracle
    ops3 = oracle.count_ops3(T)
    spe = int(oracle.count_ops(T)[0])
    stats = {"n_ops_pp": 0, "n_ops_nn": 0, "n_ops_pn": 0, "n_ops_spe": spe,
             "n_ops_ppp": ops3[0], "n_ops_nnn": ops3[1], "n_ops_ppn": ops3[2], "n_ops_pnn": ops3[3]}
    b, nops = bench.alg_bytes(stats, T, 1, 4)
    assert nops == spe + sum(ops3)
    assert b > nops * 12
