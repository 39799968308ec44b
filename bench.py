#!/usr/bin/env python
"""Benchmark: BIGSTICK M-scheme applyH on B200.

Default workload: sd shell, 6 protons + 6 neutrons, 2Jz = 0 (M-scheme dim
93,710), seeded synthetic isospin interaction (63 TBMEs ~ N(0,1) MeV, seed 2,
SPEs -3.9/-3.2/+2.1 MeV), FP32 applyH (fp32 matrix elements, fp32 vectors,
fp32 accumulation).  One step = one applyH over one vector.

Timing: W warm-up matvecs, then exactly K timed matvecs; before every timed
matvec the L2 is flushed by writing a 256 MiB buffer, and the matvec kernel
itself is timed with CUDA events on its stream; barrier + synchronize on both
sides; max over ranks.  `e2e` calls the C ABI with pinned host buffers, so
the host->device copy of the input and the device->host copy of the output
are inside each timed step.

`--impl reference` times the reference's CPU algorithm for this path on the
host cores: the reference is Fortran and no Fortran compiler exists in this
image, so it runs the oracle's C restatement of applyHbundled_g with its
OpenMP partition (kind "port").

Multi-GPU: the matvec does not shard across GPUs in this build; --gpus N runs
N independent replicas (one per rank) and reports the aggregate rate.
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

METRIC = "applyH matvec/s & HBM-roofline %, mixed vs FP64 GPU at ≤1e-6 rel eigval err"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0}
WORKLOADS = {
    # name: (shell, np, nn, jz2, seed)
    "sd6p6n": ("sd", 6, 6, 0, 2),
    "sd2p2n": ("sd", 2, 2, 0, 1),
    "pf4p4n": ("pf", 4, 4, 0, 3),
}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


def make_tables(name):
    from bigstickpublick_b200 import model
    shell, np_, nn, jz2, seed = WORKLOADS[name]
    m = model.sd_model(np_, nn, seed=seed, jz2=jz2) if shell == "sd" else model.pf_model(np_, nn, seed=seed, jz2=jz2)
    return model.build_tables(m)


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sms, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sms.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sms)) if sms else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sms)}


def alg_bytes(stats, tables, nb, s):
    """B_alg = N_ops*nb*(s_in + 2 s_out) + J_bytes + dim*nb*(s_in + s_out).
    J_bytes = 21 B per stored jump + pstart/nstart (8 B each) + hmat (4 B each)."""
    nops = stats["n_ops_pp"] + stats["n_ops_nn"] + stats["n_ops_pn"] + stats["n_ops_spe"]
    S = tables.s
    jumps = S["np1b"] + S["nn1b"] + S["np2b"] + S["nn2b"]
    jb = 21 * jumps + 8 * (S["nsd_p"] + S["nsd_n"]) + 4 * (S["nmatpp"] + S["nmatnn"] + S["nmatpn"])
    return nops * nb * 3 * s + jb + tables.dim * nb * 2 * s, nops


def reduce_max(x, dist, device=None):
    """Max over ranks of a per-rank time (the slowest replica sets the pace)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(steps, world, max_seconds):
    """Whole-job rate: every rank runs `steps` matvecs on its own replica."""
    return world * steps / max_seconds


def table_checksum(tables):
    """Digest of every table array: replicas must run identical workloads."""
    import hashlib
    h = hashlib.sha256()
    for k in sorted(tables.a):
        h.update(k.encode())
        h.update(np.ascontiguousarray(tables.a[k]).tobytes())
    return h.hexdigest()


def cpu_baseline(tables, nb, prec, budget_s=10.0, nthreads=None):
    import oracle
    dt = np.float32 if prec == 4 else np.float64
    rng = np.random.default_rng(0)
    vin = rng.standard_normal(tables.dim * nb).astype(dt)
    out = np.zeros_like(vin)
    nthreads = nthreads or os.cpu_count()
    oracle.applyh_omp(tables, vin, nb=nb, nthreads=nthreads, out=out)  # warm-up
    n, t0 = 0, time.perf_counter()
    while True:
        out[:] = 0
        oracle.applyh_omp(tables, vin, nb=nb, nthreads=nthreads, out=out)
        n += 1
        el = time.perf_counter() - t0
        if el > budget_s or n >= 2000:
            break
    return n / el, nthreads, n, el


def traffic_from_profile(workload, nb, prec):
    p = os.path.join(ROOT, "profiles", "applyh_traffic.json")
    if not os.path.exists(p):
        return None
    try:
        d = json.load(open(p))
        return d.get(f"{workload}:nb{nb}:p{prec}")
    except Exception:
        return None


def lanczos_leg(H, tables, args):
    """The eigenvalue side of the metric: FP64 vs mixed (FP32 applyH, FP64
    Lanczos) on the same workload and pivot, lowest 10 states, fixed
    iteration count; relative eigenvalue error of mixed vs FP64 and the
    iterations per second of each.  For the pf 4p4n workload also the block
    (nb = 8) mixed run with thick restart keeping 20 vectors."""
    import torch
    rng = np.random.default_rng(11)
    piv = rng.standard_normal(tables.dim)
    out = {}
    niter = args.lanczos_iters
    runs = {}
    # untimed warm-up solves: the first use of a kernel loads its code
    for prec in (8, 4):
        H.lanczos(nkeep=2, niter=6, matvec_prec=prec, fixed_iter=True, pivot=piv)
    for name, prec in (("fp64", 8), ("mixed", 4)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ev, _, rep = H.lanczos(nkeep=10, niter=niter, matvec_prec=prec, fixed_iter=True, pivot=piv)
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        runs[name] = (ev, rep, el)
        # rates on the solver's own device clock (CUDA events around the whole
        # solve, host-driven steps included); the Python wall time beside it
        tot = rep["t_total_ms"] / 1e3
        out[name] = {"iterations": rep["total_iterations"], "its_per_s": rep["total_iterations"] / tot,
                     "solve_s": tot, "wall_s": el, "t_matvec_ms": rep["t_matvec_ms"], "t_reorth_ms": rep["t_reorth_ms"],
                     "t_eig_ms": rep["t_eig_ms"], "lowest": [float(x) for x in ev[:3]]}
    e64, e32 = runs["fp64"][0], runs["mixed"][0]
    out["mixed_vs_fp64_max_rel_eig_err"] = float(np.max(np.abs(e32 - e64) / np.abs(e64)))
    out["speedup_its_per_s"] = out["mixed"]["its_per_s"] / out["fp64"]["its_per_s"]
    out["config"] = f"{niter} iterations, lowest 10, fixed iteration count, seeded generic pivot"
    if args.block_leg:
        nb = 8
        pivb = rng.standard_normal(tables.dim * nb)
        H.lanczos(nkeep=2, niter=3, nb=nb, matvec_prec=4, fixed_iter=True, pivot=pivb)  # untimed warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        evb, _, repb = H.lanczos(nkeep=10, niter=args.block_iters, nb=nb, nthick_add=10, max_restarts=args.block_restarts,
                                 matvec_prec=4, converge_tol=1e-9, pivot=pivb)
        torch.cuda.synchronize()
        elb = time.perf_counter() - t0
        totb = repb["t_total_ms"] / 1e3
        out["block_mixed"] = {"nb": nb, "keep": 20, "iterations": repb["total_iterations"], "restarts": repb["restarts"],
                              "vector_matvecs_per_s": repb["total_iterations"] * nb / totb, "solve_s": totb, "wall_s": elb,
                              "max_rel_eig_err_vs_fp64": float(np.max(np.abs(evb - e64) / np.abs(e64))),
                              "converged": repb["converged"], "t_matvec_ms": repb["t_matvec_ms"],
                              "t_reorth_ms": repb["t_reorth_ms"], "t_eig_ms": repb["t_eig_ms"]}
        out["block_vs_fp64_vector_matvec_rate"] = out["block_mixed"]["vector_matvecs_per_s"] / out["fp64"]["its_per_s"]
        out["fp64"]["vector_matvecs_per_s"] = out["fp64"]["its_per_s"]
    return out


def density_leg(H, tables, args, k=10, reps=5):
    """One-body transition densities of every pair of k states (bsg_density1b):
    device time of its kernels (CUDA events inside the call) and the call's
    wall time with host vectors in and host densities out; and a one-body
    operator applied to the k vectors (bsg_apply1b, device time).  The work does not
    depend on the vector values, so k seeded normalized vectors stand in for
    eigenvectors."""
    X = np.random.default_rng(5).standard_normal((tables.dim, k))
    X /= np.linalg.norm(X, axis=0)
    X = np.asfortranarray(X)
    H.density1b(X)  # untimed: first use loads the kernels
    dev, wall = [], []
    for _ in range(reps):
        t0 = time.perf_counter()
        H.density1b(X)
        wall.append(time.perf_counter() - t0)
        dev.append(H.stats()["density_ms"])
    st = H.stats()
    rows = st["density_rows"]
    kms = float(np.median(dev))
    # the spin-like one-body operator (isoscalar, J = 1) on the same k vectors
    nqp = int(tables.s["nhsps_pl"] + tables.s["nhsps_pr"])
    nqn = int(tables.s["nhsps_nl"] + tables.s["nhsps_nr"])
    rng = np.random.default_rng(6)
    P, N = rng.standard_normal((nqp, nqp)), rng.standard_normal((nqn, nqn))
    H.apply1b(P, N, X)
    ams = []
    for _ in range(reps):
        H.apply1b(P, N, X)
        ams.append(H.stats()["apply1b_ms"])
    return {"states": k, "pairs": k * k, "rows": rows, "kernel_ms": kms, "e2e_ms": float(np.median(wall)) * 1e3,
            "launches": st["density_launches"],
            "fp64_gflop_per_s": 2.0 * rows * k * k / (kms * 1e-3) / 1e9,
            "gathered_gb_per_s": rows * 2 * k * 8 / (kms * 1e-3) / 1e9,
            "h2d_bytes": tables.dim * k * 8,
            "apply1b_ms": float(np.median(ams)), "apply1b_vectors": k}


def batch_leg(args):
    """Config 4: 256 sd-shell Hamiltonians (seeds 1000..1255, valence Z and N
    uniform in 2..8), one persistent launch per batched matvec, lock-step
    Lanczos with one captured graph per iteration, then the adjoint gradient
    of the lowest 5 eigenvalues of every system with respect to its 63 TBMEs
    and 3 SPEs."""
    import torch
    from bigstickpublick_b200 import model
    from bigstickpublick_b200.engine import Batch
    t0 = time.perf_counter()
    tabs = model.build_tables_many([model.batch_member(s) for s in range(1000, 1000 + args.batch_n)])
    t_build = time.perf_counter() - t0
    t0 = time.perf_counter()
    cache = os.path.join(ROOT, ".tune_cache", "batch_tuning.json") if args.tune_cache else None
    b = Batch(tabs, autotune=True, tune_cache=cache)
    t_create = time.perf_counter() - t0
    dims = [t.dim for t in tabs]
    vin = [torch.randn(d, dtype=torch.float32, device="cuda") for d in dims]
    vout = [torch.empty_like(v) for v in vin]
    for _ in range(3):
        b.applyh(vin, vout)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(20):
        b.applyh(vin, vout)
    e1.record()
    torch.cuda.synchronize()
    mv_ms = e0.elapsed_time(e1) / 20
    ev, vecs, rep = b.lanczos(nkeep=5, niter=args.batch_iters, matvec_prec=8, want_vectors=True)
    t0 = time.perf_counter()
    grads = []
    for s, t in enumerate(tabs):
        g = b.system(s).grad(vecs[s])
        grads.append([model.chain_rule(t, {k: v[i] for k, v in g.items()}) for i in range(5)])
    t_grad = time.perf_counter() - t0
    b.close()
    return {"systems": len(tabs), "dims_min": min(dims), "dims_max": max(dims), "dims_sum": int(sum(dims)),
            "tuning": b.tuning, "build_s": t_build, "create_s": t_create,
            "batched_matvec_ms": mv_ms, "system_matvecs_per_s": len(tabs) / (mv_ms / 1e3),
            "lanczos_iters": args.batch_iters, "lanczos_graph_ms": rep["t_matvec_ms"],
            "lanczos_eig_ms": rep["t_eig_ms"], "grad_s_all_systems_5_states": t_grad,
            "ground_states_first4": [float(x) for x in ev[:4, 0]]}


def large_leg(args):
    """Config 5: pf shell 6p6n, 2Jz = 0 (M-scheme dim 109,954,620), seeded
    synthetic pf interaction; FP32 applyH rate, thick-restart mixed-precision
    Lanczos for the lowest 5 states (FP64 history and reorthogonalization),
    adjoint gradient of the ground state w.r.t. all 195 TBMEs and 4 SPEs,
    everything resident in device memory."""
    import torch
    from bigstickpublick_b200 import model
    from bigstickpublick_b200.engine import Hamiltonian
    t0 = time.perf_counter()
    T = model.build_tables(model.pf_model(6, 6, seed=5))
    t_build = time.perf_counter() - t0
    t0 = time.perf_counter()
    H = Hamiltonian(T)
    t_create = time.perf_counter() - t0
    st = H.stats()
    x = torch.randn(T.dim, dtype=torch.float32, device="cuda")
    y = torch.empty_like(x)
    H.applyh(x, y)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(3):
        H.applyh(x, y)
    e1.record()
    torch.cuda.synchronize()
    mv_s = e0.elapsed_time(e1) / 3 / 1e3
    balg, nops = alg_bytes(st, T, 1, 4)
    peaks, _ = load_peaks()
    del x, y
    t0 = time.perf_counter()
    ev, vecs, rep = H.lanczos(nkeep=5, niter=args.large_iters, nthick_add=15, max_restarts=args.large_restarts,
                              matvec_prec=4, converge_tol=args.large_tol, want_vectors=True)
    t_lz = time.perf_counter() - t0
    t0 = time.perf_counter()
    g = H.grad(vecs[:, :1])
    gtb, gspe = model.chain_rule(T, {k: v[0] for k, v in g.items()})
    t_grad = time.perf_counter() - t0
    spec = T.extra["spec"]
    euler = float(np.array([t[6] for t in spec.tbme]) @ gtb + np.array(spec.spe) @ gspe)
    free, total = torch.cuda.mem_get_info()
    H.close()
    return {"dim": T.dim, "ops_per_matvec": nops, "build_s": t_build, "create_s": t_create,
            "matvec_fp32_s": mv_s, "matvec_alg_GBps": balg / mv_s / 1e9,
            "matvec_roofline_frac": balg / mv_s / 1e9 / peaks["hbm_gbs"],
            "lanczos": {"evals": [float(v) for v in ev], "restarts": rep["restarts"],
                        "total_iterations": rep["total_iterations"], "converged": rep["converged"],
                        "wall_s": t_lz, "t_matvec_ms": rep["t_matvec_ms"], "t_reorth_ms": rep["t_reorth_ms"],
                        "t_eig_ms": rep["t_eig_ms"], "converge_tol": args.large_tol,
                        "basis": f"{args.large_iters} vectors, thick restart keeping 20"},
            "grad_ground_state_s": t_grad, "euler_identity_rel_err": abs(euler - ev[0]) / abs(ev[0]),
            "grad_tbme_norm": float(np.linalg.norm(gtb)), "grad_spe": [float(v) for v in gspe],
            "device_mem_total_GB": total / 1e9}


def workload_config(args, tables, world):
    """The `config` object of both arms' JSON lines."""
    return {"workload": args.workload, "dim": tables.dim, "nb": args.nb,
            "interaction": "seeded synthetic isospin TBMEs N(0,1) MeV",
            "l2": "flushed (256 MiB write) before every timed matvec; kernel timed alone",
            "parallelism": f"replicas x{world}"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    tables = make_tables(args.workload)
    per_step = []
    n_total = 0
    t_total = 0.0
    nthreads = os.cpu_count()
    for _ in range(args.warmup):
        cpu_baseline(tables, args.nb, args.prec, budget_s=0.0, nthreads=nthreads)
    for _ in range(args.steps):
        rate, cores, n, el = cpu_baseline(tables, args.nb, args.prec, budget_s=args.ref_budget, nthreads=nthreads)
        per_step.append(rate)
        n_total += n
        t_total += el
    value = n_total / t_total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "matvec/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_total / max(1, n_total),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if args.prec == 4 else "f64", "data": "synthetic",
        "config": workload_config(args, tables, int(os.environ.get("WORLD_SIZE", "1"))),
        "cpu_baseline": {"value": value, "unit": "matvec/s", "cores": nthreads, "kind": "port",
                         "sample": f"{n_total} matvecs over {t_total:.1f} s (reference is Fortran; "
                                   "no Fortran compiler in the image)"},
        "e2e": {"value": value, "unit": "matvec/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="sd6p6n", choices=sorted(WORKLOADS))
    ap.add_argument("--nb", type=int, default=1)
    ap.add_argument("--prec", type=int, default=4, choices=[4, 8])
    ap.add_argument("--ref-budget", type=float, default=3.0)
    ap.add_argument("--cpu-budget", type=float, default=10.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-lanczos", action="store_true")
    ap.add_argument("--no-density", action="store_true")
    ap.add_argument("--lanczos-iters", type=int, default=300)
    ap.add_argument("--block-leg", action="store_true")
    ap.add_argument("--block-iters", type=int, default=20)
    ap.add_argument("--block-restarts", type=int, default=30)
    ap.add_argument("--batch-leg", action="store_true")
    ap.add_argument("--batch-n", type=int, default=256)
    ap.add_argument("--batch-iters", type=int, default=150)
    ap.add_argument("--tune-cache", action="store_true")
    ap.add_argument("--large-leg", action="store_true")
    ap.add_argument("--large-iters", type=int, default=60)
    ap.add_argument("--large-restarts", type=int, default=20)
    ap.add_argument("--large-tol", type=float, default=1e-4)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    if args.impl == "reference":
        return run_reference(args)

    import torch
    from bigstickpublick_b200.engine import Hamiltonian

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    tables = make_tables(args.workload)
    H = Hamiltonian(tables, device=local)
    st = H.stats()
    nb, prec = args.nb, args.prec
    dt = torch.float32 if prec == 4 else torch.float64
    s_bytes = 4 if prec == 4 else 8
    g = torch.Generator(device="cuda").manual_seed(1234)
    shape = (tables.dim,) if nb == 1 else (tables.dim, nb)
    vin = torch.randn(shape, dtype=dt, device="cuda", generator=g)
    vout = torch.empty_like(vin)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB > L2
    stream = torch.cuda.current_stream()

    for _ in range(args.warmup):
        H.applyh(vin, vout)
    barrier()

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier()
    for k in range(args.steps):
        flush.fill_(float(k))
        evs[k][0].record(stream)
        H.applyh(vin, vout)
        evs[k][1].record(stream)
    barrier()
    kern_ms = [a.elapsed_time(b) for a, b in evs]
    # warm-L2 rate (vectors resident in L2, the steady state inside Lanczos)
    w0, w1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0.record(stream)
    for _ in range(args.steps):
        H.applyh(vin, vout)
    w1.record(stream)
    barrier()
    warm_ms = w0.elapsed_time(w1) / args.steps
    clocks = sampler.stop()

    total_ms = reduce_max(float(sum(kern_ms)), dist, device="cuda")
    value = replica_rate(args.steps, world, total_ms / 1e3)

    # ---- end to end through the C ABI with pinned host buffers
    hin = torch.empty(shape, dtype=dt, pin_memory=True)
    hin.copy_(vin.cpu())
    hout = torch.empty(shape, dtype=dt, pin_memory=True)
    hin_np, hout_np = hin.numpy(), hout.numpy()
    for _ in range(2):
        H.applyh(hin_np, hout_np)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        H.applyh(hin_np, hout_np)  # H2D copy, kernel, D2H copy, synchronize
    e2e_s = reduce_max(time.perf_counter() - t0, dist, device="cuda")
    e2e = replica_rate(args.steps, world, e2e_s)
    vbytes = tables.dim * nb * s_bytes

    peaks, peak_kind = load_peaks()
    balg, nops = alg_bytes(st, tables, nb, s_bytes)
    mean_s = total_ms / 1e3 / args.steps
    achieved = balg / mean_s / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "matvec/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32" if prec == 4 else "f64", "data": "synthetic",
        "config": workload_config(args, tables, world),
        "e2e": {"value": e2e, "unit": "matvec/s", "h2d_bytes_per_step": vbytes, "d2h_bytes_per_step": vbytes},
        "gpu_launches": args.steps * st["kernel_launches_per_matvec"],
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "traffic": traffic_from_profile(args.workload, nb, prec),
                     "peak_kind": peak_kind, "alg_bytes_per_launch": balg, "ops_per_matvec": nops},
        "clocks": clocks,
        "warm_l2_matvec_per_s": world / (warm_ms / 1e3),
    }
    if rank == 0 and not args.no_lanczos:
        line["lanczos"] = lanczos_leg(H, tables, args)
    if rank == 0 and not args.no_density:
        line["density"] = density_leg(H, tables, args)
    if rank == 0 and args.batch_leg:
        line["batch"] = batch_leg(args)
    if rank == 0 and args.large_leg:
        line["large"] = large_leg(args)
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, cores, n, el = cpu_baseline(tables, nb, prec, budget_s=args.cpu_budget)
        line["cpu_baseline"] = {"value": rate, "unit": "matvec/s", "cores": cores, "kind": "port",
                                "sample": f"{n} full matvecs of the same workload in {el:.1f} s, "
                                          "oracle C restatement of applyHbundled_g with OpenMP"}
    if rank == 0:
        print(json.dumps(line))
    del H
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
