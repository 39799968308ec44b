#!/usr/bin/env python
"""Benchmark: BIGSTICK M-scheme applyH on B200.

Default workload (the largest single-GPU configuration): pf shell
(0f7/2, 1p3/2, 0f5/2, 1p1/2), 6 protons + 6 neutrons, 2Jz = 0 (M-scheme dim
109,954,620), seeded synthetic isospin interaction (195 TBMEs ~ N(0,1) MeV
and 4 SPEs, seed 5), FP32 applyH (fp32 matrix elements, fp32 vectors, fp32
accumulation).  One step = one applyH over one vector (152,771,809,712
inner-loop updates).

Timing: W warm-up matvecs, then exactly K timed matvecs; the vectors (0.44 GB
each) are larger than the 126 MB L2 and a 256 MiB buffer is also written
before every timed matvec; the matvec kernel is timed with CUDA events on its
stream; barrier + synchronize on both sides; max over ranks.  `e2e` calls the
C ABI with pinned host buffers, so the host->device copy of the input and the
device->host copy of the output are inside each timed step.

Legs beside the headline (rank 0): Lanczos on sd 6p6n (FP64 against mixed),
time to a 1e-6 solution on pf 4p4n (FP64 scalar against mixed scalar and
mixed block nb = 8), the 256-system batch with its gradients, the pf 6p6n
thick-restart solve (mixed against FP64 on the same schedule) with the
ground-state gradient, one-body densities, and a three-body Hamiltonian
(pf 4p4n, PPP/PPN/PNN/NNN bundles); each reports its eigenvalue and
wavefunction-overlap error against FP64 where it solves.

`--impl reference` times the reference's CPU algorithm for this path on the
host cores: the reference is Fortran and no Fortran compiler exists in this
image, so it runs the oracle's C restatement of applyHbundled_omp with its
owner-computes OpenMP partition (kind "port"), each step a bounded sample of
the same matvec (a slice of every thread's output rows), scaled to matvec/s
by the exact share of the inner-loop updates it covered.

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
    "sd2p2n": ("sd", 2, 2, 0, 1),
    "sd6p6n": ("sd", 6, 6, 0, 2),
    "pf4p4n": ("pf", 4, 4, 0, 3),
    "pf5p5n": ("pf", 5, 5, 0, 5),
    "pf6p5n": ("pf", 6, 5, 1, 5),
    "pf6p6n": ("pf", 6, 6, 0, 5),
}
# three-body Hamiltonians (PPP / PPN / PNN / NNN bundles): the seeded pf
# interaction in three-body form plus a seeded three-body part of 0.1 MeV
# (model.build_tables3(w2=1, w3=0.1, seed=5)); headline path only (--quick)
WORKLOADS3 = {
    "pf4p3n3b": ("pf", 4, 3, 1, 5),
    "pf4p4n3b": ("pf", 4, 4, 0, 5),
}
DEFAULT_WORKLOAD = "pf6p6n"


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


def make_tables(name):
    from bigstickpublick_b200 import model
    shell, np_, nn, jz2, seed = WORKLOADS[name] if name in WORKLOADS else WORKLOADS3[name]
    m = model.sd_model(np_, nn, seed=seed, jz2=jz2) if shell == "sd" else model.pf_model(np_, nn, seed=seed, jz2=jz2)
    if name in WORKLOADS3:
        return model.build_tables3(m, w2=1.0, w3=0.1, seed=seed)
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
    nops = sum(stats["n_ops_" + k] for k in ("pp", "nn", "pn", "spe", "ppp", "nnn", "ppn", "pnn"))
    S = tables.s
    jumps = S["np1b"] + S["nn1b"] + S["np2b"] + S["nn2b"]
    jb = 21 * jumps + 8 * (S["nsd_p"] + S["nsd_n"]) + 4 * (S["nmatpp"] + S["nmatnn"] + S["nmatpn"])
    if getattr(tables, "threebody", False):
        S3 = tables.s3
        jb += 21 * (S3["np3b"] + S3["nn3b"]) + 4 * (S3["nmatppp"] + S3["nmatnnn"] + S3["nmatppn"] + S3["nmatpnn"])
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


class CpuSampler:
    """The reference arm's matvec on the host cores, in bounded samples.

    applyHbundled_omp gives every OpenMP thread the output rows getLoadDist
    assigns it (src/bapplyhlibOMP.f90:34-868); the oracle restates that
    owner-computes matvec.  A sample runs a slice of every owner range (the
    rows holding the fraction `frac` of that range's inner-loop updates,
    starting at fraction `offset`), so it touches the whole basis the way the
    full matvec does, and the rate is scaled by the exact share of updates it
    covered."""

    def __init__(self, tables, nb=1, prec=4, nthreads=None, seed=0):
        import oracle
        self.oracle = oracle
        self.T = tables
        self.nb, self.prec = nb, prec
        self.nthreads = nthreads or os.cpu_count()
        self.rs, self.ops = oracle.row_ops(tables)
        self.csum = np.cumsum(self.ops)
        self.total = int(self.csum[-1])
        self.ends = np.append(self.rs[1:], tables.dim)
        # one owner range per thread, as getLoadDist assigns them
        self.owners = oracle.owner_ranges(self.rs, self.ops, tables.dim, self.nthreads)
        dt = np.float32 if prec == 4 else np.float64
        self.vin = np.random.default_rng(seed).standard_normal(tables.dim * nb).astype(dt)
        self.out = np.zeros_like(self.vin)

    def ranges(self, frac, offset=0.0):
        """Row ranges of one sample and the updates they hold."""
        out, n = [], 0
        for lo, hi in self.owners:
            i0, i1 = int(np.searchsorted(self.rs, lo)), int(np.searchsorted(self.rs, hi))
            if i1 <= i0:
                continue
            base = int(self.csum[i0 - 1]) if i0 > 0 else 0
            w = int(self.csum[i1 - 1]) - base
            off = (offset % 1.0) * w
            a = min(i1 - 1, int(np.searchsorted(self.csum, base + off, side="right")))
            b = min(i1, max(a + 1, int(np.searchsorted(self.csum, base + off + frac * w, side="left")) + 1))
            out.append((int(self.rs[a]), int(self.ends[b - 1])))
            n += int(self.csum[b - 1]) - (int(self.csum[a - 1]) if a > 0 else 0)
        return np.array(out, dtype=np.int64).reshape(-1, 2), n

    def run(self, frac, offset=0.0):
        """(share of one matvec covered, seconds)."""
        rg, n = self.ranges(frac, offset)
        t0 = time.perf_counter()
        self.oracle.applyh_owner(self.T, self.vin, rg, nb=self.nb, nthreads=self.nthreads, out=self.out)
        return n / self.total, time.perf_counter() - t0

    def calibrate(self, budget_s):
        """The sample fraction that takes about budget_s seconds: the fixed
        cost of a sample (every owner scans its bundles' jump lists, as the
        reference's 'b' bundles do) measured apart from the cost per share."""
        _, t0 = self.run(1e-6)
        f = 1e-3
        share, el = self.run(f)
        while el - t0 < 0.2 and f < 1.0:
            f = min(1.0, f * 8)
            share, el = self.run(f)
        per = max(el - t0, 1e-6) / max(share, 1e-12)
        return float(min(1.0, max(1e-4, (budget_s - t0) / per)))


def cpu_baseline(tables, nb, prec, budget_s=10.0, nthreads=None):
    """matvec/s of the oracle's owner-computes OpenMP matvec on all host
    cores, timed on bounded samples of about budget_s seconds in total."""
    cs = CpuSampler(tables, nb, prec, nthreads)
    frac = cs.calibrate(budget_s / 3)
    shares, secs = 0.0, 0.0
    for k in range(3):
        sh, el = cs.run(frac, offset=0.37 * (k + 1))
        shares += sh
        secs += el
    return shares / secs, cs.nthreads, shares, secs


def traffic_from_profile(workload, nb, prec):
    p = os.path.join(ROOT, "profiles", "applyh_traffic.json")
    if not os.path.exists(p):
        return None
    try:
        d = json.load(open(p))
        return d.get(f"{workload}:nb{nb}:p{prec}")
    except Exception:
        return None


def compare_states(ev, vecs, ev_ref, vecs_ref):
    """max relative eigenvalue error and the smallest |<psi|psi_ref>| over the
    states (vectors dim x k, normalized)."""
    ev, ev_ref = np.asarray(ev), np.asarray(ev_ref)
    k = min(len(ev), len(ev_ref))
    out = {"max_rel_eig_err": float(np.max(np.abs(ev[:k] - ev_ref[:k]) / np.abs(ev_ref[:k])))}
    if vecs is not None and vecs_ref is not None:
        ov = [abs(float(vecs[:, j] @ vecs_ref[:, j])) for j in range(k)]
        out["min_overlap"] = float(min(ov))
        out["overlaps"] = [float(x) for x in ov]
    return out


def _solve(H, **kw):
    import torch
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ev, vecs, rep = H.lanczos(**kw)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    tot = rep["t_total_ms"] / 1e3
    nb = kw.get("nb", 1)
    info = {"iterations": rep["total_iterations"], "restarts": rep["restarts"], "converged": rep["converged"],
            "vector_matvecs": rep["matvecs"] * nb, "solve_s": tot, "wall_s": wall,
            "its_per_s": rep["total_iterations"] / tot, "vector_matvecs_per_s": rep["matvecs"] * nb / tot,
            "t_matvec_ms": rep["t_matvec_ms"], "t_reorth_ms": rep["t_reorth_ms"], "t_eig_ms": rep["t_eig_ms"]}
    return ev, vecs, info


MIXED = dict(matvec_prec=4, lanc_prec=4)   # FP32 applyH, FP32-stored Lanczos vectors, FP64 sums
FP64 = dict(matvec_prec=8, lanc_prec=8)


def lanczos_sd6p6n_leg(args):
    """sd 6p6n, lowest 10 states, 300 iterations (fixed) from one seeded
    pivot: the FP64 path against mixed precision (FP32 applyH, Lanczos
    vectors stored in FP32 as the reference's lanc_prec = 4 stores them,
    every dot product, alpha, beta and the projected eigenproblem in FP64);
    the mixed run's eigenvalue and wavefunction-overlap error against FP64,
    and the iterations per second of each."""
    from bigstickpublick_b200.engine import Hamiltonian
    T = make_tables("sd6p6n")
    H = Hamiltonian(T)
    try:
        piv = np.random.default_rng(11).standard_normal(T.dim)
        for prec in (FP64, MIXED):  # untimed: the first use of a kernel loads its code
            H.lanczos(nkeep=10, niter=20, fixed_iter=True, pivot=piv, **prec)
        out = {}
        res = {}
        for name, prec in (("fp64", FP64), ("mixed", MIXED)):
            # the faster of two identical runs (a run is 60-70 ms, so one
            # stall of the host or the box would decide a single sample)
            runs = [_solve(H, nkeep=10, niter=args.lanczos_iters, fixed_iter=True, pivot=piv, want_vectors=True,
                           **prec) for _ in range(2)]
            ev, vecs, info = min(runs, key=lambda r: r[2]["solve_s"])
            info["solve_s_runs"] = [r[2]["solve_s"] for r in runs]
            res[name] = (ev, vecs)
            info["lowest"] = [float(x) for x in ev[:3]]
            out[name] = info
        out["mixed"].update(compare_states(*res["mixed"], *res["fp64"]))
        out["speedup_its_per_s"] = out["mixed"]["its_per_s"] / out["fp64"]["its_per_s"]
        out["config"] = (f"sd 6p6n, {args.lanczos_iters} iterations (fixed), lowest 10, seeded generic pivot; "
                         "mixed = FP32 applyH + FP32-stored Lanczos vectors with FP64 sums; errors of mixed "
                         "against FP64 from the same pivot; each the faster of two identical runs")
        return out
    finally:
        H.close()


TTS_TOLS = (1e-2, 3e-3, 1e-3, 3e-4, 1e-4, 1e-5)


def time_to_solution_leg(args):
    """pf 4p4n, lowest 10 states to a relative eigenvalue error of 1e-6:
    the plain FP64 path (scalar Lanczos, FP64 applyH and vectors) against
    mixed precision (FP32 applyH, FP32-stored vectors, FP64 sums), scalar
    and block, each with thick restart (keep 20 or 30) and the reference's
    convergence test.  For every method the convergence tolerance is swept
    and the fastest run whose 10 eigenvalues all lie within 1e-6 of a
    tightly converged FP64 solve (from the same pivot) is kept, so each
    method is timed at its own best setting for the same accuracy.  Times
    are the solver's device clock.  Also the one-body density leg on the same
    Hamiltonian."""
    from bigstickpublick_b200.engine import Hamiltonian
    T = make_tables("pf4p4n")
    H = Hamiltonian(T)
    try:
        rng = np.random.default_rng(11)
        piv = rng.standard_normal(T.dim)
        pivs = {nb: np.concatenate([piv[:, None], rng.standard_normal((T.dim, nb - 1))], axis=1).reshape(-1)
                for nb in (2, 4, 8)}
        for prec in (FP64, MIXED):
            H.lanczos(nkeep=2, niter=6, fixed_iter=True, pivot=piv, **prec)
        for nb in (2, 4, 8):
            H.lanczos(nkeep=2, niter=3, nb=nb, fixed_iter=True, pivot=pivs[nb], **MIXED)
        ev_ref, v_ref, info_ref = _solve(H, nkeep=10, niter=150, nthick_add=10, max_restarts=200, converge_tol=1e-9,
                                         pivot=piv, want_vectors=True, **FP64)
        out = {"reference": dict(info_ref, converge_tol=1e-9, lowest=[float(x) for x in ev_ref[:3]])}
        methods = [
            ("fp64", [dict(nkeep=10, niter=n, nthick_add=10, max_restarts=200, pivot=piv, **FP64) for n in (100, 150)]),
            ("mixed", [dict(nkeep=10, niter=n, nthick_add=10, max_restarts=200, pivot=piv, **MIXED) for n in (100, 150)]),
            ("block2_mixed", [dict(nkeep=10, niter=80, nb=2, nthick_add=10, max_restarts=200, pivot=pivs[2], **MIXED)]),
            ("block4_mixed", [dict(nkeep=10, niter=40, nb=4, nthick_add=a, max_restarts=200, pivot=pivs[4], **MIXED)
                              for a in (10, 20)]),
            ("block8_mixed", [dict(nkeep=10, niter=20, nb=8, nthick_add=20, max_restarts=200, pivot=pivs[8], **MIXED)]),
        ]
        for name, cfgs in methods:
            best, tried = None, []
            for kw in cfgs:
                for tol in args.tts_tols:
                    ev, _, info = _solve(H, converge_tol=tol, **kw)
                    err = float(np.max(np.abs(ev - ev_ref) / np.abs(ev_ref)))
                    desc = {"niter": kw["niter"], "nb": kw.get("nb", 1), "keep": kw["nkeep"] + kw["nthick_add"],
                            "tol": tol, "solve_s": info["solve_s"], "max_rel_eig_err": err}
                    tried.append(desc)
                    if err <= 1e-6 and (best is None or info["solve_s"] < best[1]["solve_s"]):
                        best = (kw, dict(info, **desc))
            if best is None:
                out[name] = {"meets_1e-6": False, "tried": tried}
                continue
            kw, info = best
            # the chosen run again with its eigenvectors, for the overlap error
            ev, vecs, _ = _solve(H, converge_tol=info["tol"], want_vectors=True, **kw)
            info.update(compare_states(ev, vecs, ev_ref, v_ref))
            info["meets_1e-6"] = True
            info["tried"] = tried
            out[name] = info
        for name in ("mixed", "block2_mixed", "block4_mixed", "block8_mixed"):
            if out.get(name, {}).get("meets_1e-6") and out["fp64"].get("meets_1e-6"):
                out[name]["speedup_time_to_solution_vs_fp64"] = out["fp64"]["solve_s"] / out[name]["solve_s"]
        out["config"] = ("pf 4p4n, lowest 10 within 1e-6 relative of an FP64 solve converged to 1e-9; per method "
                         f"the fastest of convergence tolerances {list(args.tts_tols)} MeV and the listed bases; "
                         "solver device clock")
        if not args.no_density:
            try:
                out["density"] = density_leg(H, T)
            except Exception as e:  # a failing leg must not cost the headline line
                out["density"] = {"error": repr(e)[:300]}
        return out
    finally:
        H.close()


def density_leg(H, tables, k=10, reps=5):
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
    return {"states": k, "pairs": k * k, "rows": rows, "kernel_ms": kms,
            "e2e_ms": float(np.median(wall)) * 1e3, "launches": st["density_launches"],
            "fp64_gflop_per_s": 2.0 * rows * k * k / (kms * 1e-3) / 1e9,
            "gathered_gb_per_s": rows * 2 * k * 8 / (kms * 1e-3) / 1e9,
            "h2d_bytes": tables.dim * k * 8,
            "apply1b_ms": float(np.median(ams)), "apply1b_vectors": k}


def batch_leg(args):
    """Config 4: 256 sd-shell Hamiltonians (seeds 1000..1255, valence Z and N
    uniform in 2..8), one persistent launch per batched matvec, lock-step
    Lanczos with one captured graph per iteration from a seeded random pivot
    per system (FP64 applyH, and mixed: FP32 applyH, with its eigenvalue and
    overlap error against FP64 over all systems), then the adjoint gradient
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
    if cache:
        b = Batch(tabs, autotune=True, tune_cache=cache)
        t_create, t_tune = time.perf_counter() - t0, 0.0
    else:
        # the contexts, then the autotuner, timed apart
        b = Batch(tabs)
        t_create = time.perf_counter() - t0
        t0 = time.perf_counter()
        b.tuning = b.autotune()
        t_tune = time.perf_counter() - t0
    try:
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
        res = {}
        for name, prec in (("fp64", 8), ("mixed", 4)):
            t0 = time.perf_counter()
            ev, vecs, rep = b.lanczos(nkeep=5, niter=args.batch_iters, matvec_prec=prec, want_vectors=True,
                                      pivot="random", seed=77)
            res[name] = (ev, vecs, rep, time.perf_counter() - t0)
        ev64, v64 = res["fp64"][0], res["fp64"][1]
        evm, vm = res["mixed"][0], res["mixed"][1]
        rel = np.abs(evm - ev64) / np.abs(ev64)
        ovl = np.array([[abs(float(vm[s][:, j] @ v64[s][:, j])) for j in range(5)] for s in range(len(tabs))])
        b.grad([v[:, :1] for v in v64[:2]] + [v[:, :1] for v in v64[2:]])  # untimed: loads the kernels
        t0 = time.perf_counter()
        gb = b.grad(v64)  # all systems and states: one launch
        t_grad_dev = time.perf_counter() - t0
        grad_kernel_ms = b.grad_ms
        for t, g in zip(tabs, gb):
            [model.chain_rule(t, {k: v[i] for k, v in g.items()}) for i in range(5)]
        t_grad = time.perf_counter() - t0
        return {"systems": len(tabs), "dims_min": min(dims), "dims_max": max(dims), "dims_sum": int(sum(dims)),
                "tuning": b.tuning, "build_s": t_build, "create_s": t_create, "autotune_s": t_tune,
                "batched_matvec_ms": mv_ms, "system_matvecs_per_s": len(tabs) / (mv_ms / 1e3),
                "lanczos_iters": args.batch_iters,
                "fp64": {"graph_ms": res["fp64"][2]["t_matvec_ms"], "eig_ms": res["fp64"][2]["t_eig_ms"],
                         "wall_s": res["fp64"][3]},
                "mixed": {"graph_ms": res["mixed"][2]["t_matvec_ms"], "eig_ms": res["mixed"][2]["t_eig_ms"],
                          "wall_s": res["mixed"][3], "max_rel_eig_err": float(rel.max()),
                          "min_overlap": float(ovl.min())},
                "grad_s_all_systems_5_states": t_grad, "grad_call_s": t_grad_dev,
                "grad_kernel_ms": grad_kernel_ms, "grad_launches": 2,
                "ground_states_first4": [float(x) for x in ev64[:4, 0]]}
    finally:
        b.close()


def threebody_leg(args):
    """Three-body Hamiltonian (PPP / PPN / PNN / NNN bundles,
    src/bapplyhlib1.f90:1390-2804): pf 4p4n, 2Jz = 0 (dim 1,963,461), the
    seeded pf interaction (seed 5) in three-body form, W = V2/(A-2), plus a
    seeded three-body part 0.1 MeV * R.  FP32 and FP64 applyH timed alone
    (256 MiB written before each launch); hermiticity <u|Hv> = <v|Hu> in
    FP64; the same interaction with R = 0 against the two-body engine on the
    same basis (equal up to the float rounding of the matrix elements); the
    oracle's restated bundle loops on one thread over a seeded sample of
    bundles as the CPU figure."""
    import torch
    import oracle
    from bigstickpublick_b200 import model
    from bigstickpublick_b200.engine import Hamiltonian
    spec = model.pf_model(4, 4, seed=5, jz2=0)
    t0 = time.perf_counter()
    T = model.build_tables3(spec, w2=1.0, w3=0.1, seed=5)
    t_build = time.perf_counter() - t0
    t0 = time.perf_counter()
    H = Hamiltonian(T)
    t_create = time.perf_counter() - t0
    st = H.stats()
    ops = {k: int(st["n_ops_" + k]) for k in ("spe", "ppp", "nnn", "ppn", "pnn")}
    nops = sum(ops.values())
    peaks, peak_kind = load_peaks()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    out = {"config": "pf 4p4n 2Jz=0, W = V2/(A-2) + 0.1 MeV R (seeded), nb = 1", "dim": T.dim,
           "ops_per_matvec": ops, "build_s": t_build, "create_s": t_create, "launches_per_matvec": 1}
    g = torch.Generator(device="cuda").manual_seed(4321)
    x64 = torch.randn(T.dim, dtype=torch.float64, device="cuda", generator=g)
    S, S3 = T.s, T.s3
    jumps = S["np1b"] + S["nn1b"] + S["np2b"] + S["nn2b"] + S3["np3b"] + S3["nn3b"]
    jb = 21 * jumps + 8 * (S["nsd_p"] + S["nsd_n"]) + 4 * (S3["nmatppp"] + S3["nmatnnn"] + S3["nmatppn"] +
                                                           S3["nmatpnn"])
    for name, dt, sb in (("fp32", torch.float32, 4), ("fp64", torch.float64, 8)):
        x = x64.to(dt)
        y = torch.empty_like(x)
        for _ in range(3):
            H.applyh(x, y)
        reps = 10
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
        for k in range(reps):
            flush.fill_(float(k))
            evs[k][0].record()
            H.applyh(x, y)
            evs[k][1].record()
        torch.cuda.synchronize()
        ms = float(np.mean([a.elapsed_time(b) for a, b in evs]))
        balg = nops * 3 * sb + jb + T.dim * 2 * sb
        out[name] = {"matvec_ms": ms, "matvec_per_s": 1e3 / ms, "gupdates_per_s": nops / ms / 1e6,
                     "alg_GBps": balg / ms / 1e6, "alg_frac_of_hbm": balg / ms / 1e6 / peaks["hbm_gbs"],
                     "peak_kind": peak_kind}
    u64 = torch.randn(T.dim, dtype=torch.float64, device="cuda", generator=g)
    hv, hu = H.applyh(x64), H.applyh(u64)
    a, b = float(torch.dot(u64, hv)), float(torch.dot(x64, hu))
    out["hermiticity_rel"] = abs(a - b) / abs(a)
    H.close()
    del H, hv, hu, flush
    # the two-body interaction in three-body form against the two-body engine
    H0 = Hamiltonian(model.build_tables3(spec, w2=1.0, w3=0.0, seed=5))
    H2 = Hamiltonian(model.build_tables(spec))
    y0, y2 = H0.applyh(x64), H2.applyh(x64)
    out["three_vs_two_body_rel"] = float(torch.linalg.vector_norm(y0 - y2) / torch.linalg.vector_norm(y2))
    H0.close()
    H2.close()
    # CPU: the oracle's bundle loops, one thread, a seeded sample of bundles
    a_ = T.a
    size = (a_["pxend"] - a_["pxstart"] + 1) * (a_["nxend"] - a_["nxstart"] + 1)
    order = np.random.default_rng(5).permutation(len(size))
    pick, acc = [], 0
    for ib in order:
        if a_["optype"][ib] == 1:
            continue
        pick.append(int(ib))
        acc += int(size[ib])
        if acc >= 4e8:
            break
    xin = x64.cpu().numpy().astype(np.float32)
    t0 = time.perf_counter()
    oracle.applyh3_bundles(T, xin, pick)
    secs = time.perf_counter() - t0
    out["cpu_oracle_1thread"] = {"matvec_per_s": acc / secs / nops, "sample_updates": acc,
                                 "sample_share": acc / nops, "seconds": secs}
    out["speedup_fp32_vs_cpu_1thread"] = out["fp32"]["matvec_per_s"] / out["cpu_oracle_1thread"]["matvec_per_s"]
    return out


def large_leg(H, T, args):
    """Config 5 (the headline workload): thick-restart Lanczos for the lowest
    5 states, keep 20, mixed (FP32 applyH, FP32-stored Lanczos vectors, FP64
    sums) and FP64 on the same fixed schedule from the same
    seeded pivot, so that their difference is the precision alone; each
    state's FP64 residual |H psi - E psi| / |E|; the adjoint gradient of the
    ground state w.r.t. all 195 TBMEs and 4 SPEs with the Euler identity
    E = sum V dE/dV + sum e dE/de; everything resident in device memory."""
    import torch
    from bigstickpublick_b200 import model
    piv = np.random.default_rng(11).standard_normal(T.dim)
    kw = dict(nkeep=5, niter=args.large_iters, nthick_add=15, max_restarts=args.large_restarts, fixed_iter=True,
              pivot=piv, want_vectors=True)
    res, out = {}, {}
    for name, prec in (("mixed", MIXED), ("fp64", FP64)):
        ev, vecs, info = _solve(H, **prec, **kw)
        # FP64 residuals of the returned Ritz pairs
        r = []
        for j in range(len(ev)):
            x = torch.from_numpy(np.ascontiguousarray(vecs[:, j])).cuda()
            y = H.applyh(x)
            r.append(float(torch.linalg.vector_norm(y - ev[j] * x).item() / abs(ev[j])))
            del x, y
        info["evals"] = [float(v) for v in ev]
        info["rel_residuals"] = r
        res[name] = (ev, vecs)
        out[name] = info
    out["mixed"].update(compare_states(*res["mixed"], *res["fp64"]))
    t0 = time.perf_counter()
    g = H.grad(res["fp64"][1][:, :1])
    gtb, gspe = model.chain_rule(T, {k: v[0] for k, v in g.items()})
    t_grad = time.perf_counter() - t0
    spec = T.extra["spec"]
    e0 = res["fp64"][0][0]
    euler = float(np.array([t[6] for t in spec.tbme]) @ gtb + np.array(spec.spe) @ gspe)
    free, total = torch.cuda.mem_get_info()
    out.update({"config": f"pf 6p6n, lowest 5, {args.large_iters}-vector basis, keep 20, {args.large_restarts} "
                          "restarts (fixed schedule), seeded generic pivot",
                "grad_ground_state_s": t_grad, "euler_identity_rel_err": abs(euler - e0) / abs(e0),
                "grad_tbme_norm": float(np.linalg.norm(gtb)), "grad_spe": [float(v) for v in gspe],
                "device_mem_total_GB": total / 1e9})
    return out


def workload_config(args, tables, world):
    """The `config` object of both arms' JSON lines."""
    return {"workload": args.workload, "dim": tables.dim, "nb": args.nb,
            "interaction": "seeded synthetic isospin TBMEs N(0,1) MeV" + (
                ", in three-body form W = V2/(A-2) + 0.1 MeV R (seeded)" if args.workload in WORKLOADS3 else ""),
            "l2": "vectors larger than L2, and a 256 MiB write before every timed matvec; kernel timed alone",
            "parallelism": f"replicas x{world}"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    tables = make_tables(args.workload)
    cs = CpuSampler(tables, args.nb, args.prec)
    frac = cs.calibrate(args.ref_budget)
    for k in range(args.warmup):
        cs.run(min(frac, 1e-3), offset=0.11 * k)
    shares, secs, per = 0.0, 0.0, []
    for k in range(args.steps):
        sh, el = cs.run(frac, offset=(0.618 * k) % 1.0)
        shares += sh
        secs += el
        per.append(el)
    value = shares / secs
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "matvec/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / max(1, args.steps),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if args.prec == 4 else "f64", "data": "synthetic",
        "config": workload_config(args, tables, int(os.environ.get("WORLD_SIZE", "1"))),
        "matvec_share_per_step": shares / max(1, args.steps),
        "cpu_baseline": {"value": value, "unit": "matvec/s", "cores": cs.nthreads, "kind": "port",
                         "sample": f"{args.steps} steps, each {100 * shares / max(1, args.steps):.2f}% of one "
                                   f"matvec (a slice of every owner's rows), {secs:.1f} s in all; oracle C "
                                   "restatement of applyHbundled_omp's owner-computes OpenMP partition (the "
                                   "reference is Fortran; no Fortran compiler in the image)"},
        "e2e": {"value": value, "unit": "matvec/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def _leg(line, key, fn, *a):
    """Run one leg; a failing leg is recorded and does not cost the line."""
    try:
        line[key] = fn(*a)
    except Exception as e:
        line[key] = {"error": repr(e)[:500]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS) + sorted(WORKLOADS3))
    ap.add_argument("--nb", type=int, default=1)
    ap.add_argument("--prec", type=int, default=4, choices=[4, 8])
    ap.add_argument("--ref-budget", type=float, default=4.0, help="seconds of CPU work per reference step")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--quick", action="store_true", help="headline line only (no legs)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-lanczos", action="store_true")
    ap.add_argument("--no-density", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-large", action="store_true")
    ap.add_argument("--no-tts", action="store_true")
    ap.add_argument("--no-three", action="store_true")
    ap.add_argument("--density", action="store_true",
                    help="also run the one-body density leg on the headline workload (with --quick)")
    ap.add_argument("--lanczos-iters", type=int, default=300)
    ap.add_argument("--tts-tols", type=float, nargs="+", default=list(TTS_TOLS))
    ap.add_argument("--batch-n", type=int, default=256)
    ap.add_argument("--batch-iters", type=int, default=150)
    ap.add_argument("--tune-cache", action="store_true")
    ap.add_argument("--large-iters", type=int, default=50)
    ap.add_argument("--large-restarts", type=int, default=3)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.quick:
        args.no_cpu = args.no_lanczos = args.no_density = args.no_batch = args.no_large = args.no_tts = True
        args.no_three = True

    if args.workload in WORKLOADS3:
        # the CPU restatements time the two-body bundles only
        args.no_cpu = True
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "three-body workloads have no OpenMP CPU port; "
                              "the threebody leg times the oracle's three-body loops on one thread"}))
            return 0
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

    t0 = time.perf_counter()
    tables = make_tables(args.workload)
    t_build = time.perf_counter() - t0
    t0 = time.perf_counter()
    H = Hamiltonian(tables, device=local)
    t_create = time.perf_counter() - t0
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
    clocks = sampler.stop()

    total_ms = reduce_max(float(sum(kern_ms)), dist, device="cuda")
    value = replica_rate(args.steps, world, total_ms / 1e3)

    # ---- end to end through the C ABI with pinned host buffers
    hin = torch.empty(shape, dtype=dt, pin_memory=True)
    hin.copy_(vin.cpu())
    hout = torch.empty(shape, dtype=dt, pin_memory=True)
    hin_np, hout_np = hin.numpy(), hout.numpy()
    del vin, vout, flush
    for _ in range(2):
        H.applyh(hin_np, hout_np)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        H.applyh(hin_np, hout_np)  # H2D copy, kernel, D2H copy, synchronize
    e2e_s = reduce_max(time.perf_counter() - t0, dist, device="cuda")
    e2e = replica_rate(args.steps, world, e2e_s)
    vbytes = tables.dim * nb * s_bytes
    del hin, hout, hin_np, hout_np

    peaks, peak_kind = load_peaks()
    balg, nops = alg_bytes(st, tables, nb, s_bytes)
    mean_s = total_ms / 1e3 / args.steps
    achieved = balg / mean_s / 1e9
    traffic = traffic_from_profile(args.workload, nb, prec)
    line = {
        "metric": METRIC, "value": value, "unit": "matvec/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32" if prec == 4 else "f64", "data": "synthetic",
        "config": workload_config(args, tables, world),
        "e2e": {"value": e2e, "unit": "matvec/s", "h2d_bytes_per_step": vbytes, "d2h_bytes_per_step": vbytes},
        "gpu_launches": args.steps * st["kernel_launches_per_matvec"],
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
                     "peak_kind": peak_kind, "alg_bytes_per_launch": balg, "ops_per_matvec": nops,
                     "dram_GBps": (traffic / mean_s / 1e9) if traffic else None,
                     "dram_frac": (traffic / mean_s / 1e9 / peaks["hbm_gbs"]) if traffic else None},
        "clocks": clocks,
        "setup_s": {"tables": t_build, "bsg_create": t_create},
    }
    if rank == 0 and not args.no_large and args.workload == "pf6p6n":
        _leg(line, "large", large_leg, H, tables, args)
    if rank == 0 and args.density:
        _leg(line, "density", density_leg, H, tables)
    H.close()
    del H
    if rank == 0 and not args.no_lanczos:
        _leg(line, "lanczos", lanczos_sd6p6n_leg, args)
    if rank == 0 and not args.no_tts:
        _leg(line, "time_to_solution", time_to_solution_leg, args)
    if rank == 0 and not args.no_batch:
        _leg(line, "batch", batch_leg, args)
    if rank == 0 and not args.no_three:
        _leg(line, "threebody", threebody_leg, args)
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, cores, shares, secs = cpu_baseline(tables, nb, prec, budget_s=args.cpu_budget)
        line["cpu_baseline"] = {"value": rate, "unit": "matvec/s", "cores": cores, "kind": "port",
                                "sample": f"{100 * shares:.2f}% of one matvec of the same workload (slices of "
                                          f"every owner's rows) in {secs:.1f} s, oracle C restatement of "
                                          "applyHbundled_omp's owner-computes OpenMP partition"}
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
