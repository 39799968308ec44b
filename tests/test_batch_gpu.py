"""Batched systems: one persistent launch for many uneven Hamiltonians, the
graph-captured lock-step Lanczos, the autotuner, and the adjoint on batch
members (gradients vs central finite differences)."""
import json
import os

import numpy as np
import pytest

from bigstickpublick_b200 import model
import oracle
from oracle import dense_h

pytestmark = pytest.mark.gpu

SEEDS = [1000, 1003, 1006, 1008, 1009, 1012]   # dims 20564 .. 4206, uneven


@pytest.fixture(scope="module")
def batch():
    from bigstickpublick_b200.engine import Batch
    tabs = [model.build_tables(model.batch_member(s)) for s in SEEDS]
    b = Batch(tabs)
    yield tabs, b
    b.close()


@pytest.mark.parametrize("prec", [8, 4])
def test_batch_applyh_equals_single_system(batch, prec):
    import torch
    from bigstickpublick_b200.engine import Hamiltonian
    tabs, b = batch
    dt = torch.float64 if prec == 8 else torch.float32
    g = torch.Generator(device="cuda").manual_seed(3)
    vin = [torch.randn(t.dim, dtype=dt, device="cuda", generator=g) for t in tabs]
    vout = [torch.empty_like(v) for v in vin]
    b.applyh(vin, vout)
    torch.cuda.synchronize()
    for t, x, y in zip(tabs, vin, vout):
        ref = oracle.applyh(t, x.cpu().numpy())
        err = np.abs(y.cpu().numpy() - ref).max() / np.abs(ref).max()
        assert err < (1e-12 if prec == 8 else 2e-5)
        H = Hamiltonian(t)
        assert torch.equal(H.applyh(x), y), "batched and single-system kernels share the tile body"
        H.close()


def test_batch_lanczos_matches_single_system(batch):
    tabs, b = batch
    ev, vecs, rep = b.lanczos(nkeep=5, niter=150, matvec_prec=8, want_vectors=True)
    for s, t in enumerate(tabs):
        H = b.system(s)
        ref, _, _ = H.lanczos(nkeep=5, niter=150, matvec_prec=8, fixed_iter=True)
        assert np.abs(ev[s] - ref).max() / np.abs(ref).max() < 1e-9, (s, ev[s], ref)
        # Ritz vectors: residual and normalization
        v = vecs[s][:, 0]
        r = oracle.applyh(t, v) - ev[s][0] * v
        assert abs(np.linalg.norm(v) - 1) < 1e-8
        assert np.linalg.norm(r) < 1e-5 * abs(ev[s][0])


def test_autotune_and_cache(batch, tmp_path):
    from bigstickpublick_b200.engine import Batch
    tabs, b = batch
    cache = str(tmp_path / "tune.json")
    b2 = Batch(tabs[:3], autotune=True, tune_cache=cache)
    assert b2.tuning["source"] == "autotune" and b2.tuning["items"] in (1, 2, 4, 8)
    d = json.load(open(cache))
    assert b2.signature() in d
    b3 = Batch(tabs[:3], tune_cache=cache)
    assert b3.tuning["source"] == "cache"
    b2.close()
    b3.close()


def test_batch_member_gradients_vs_fd():
    """Small batch members (sd 2p2n and 2p3n shapes): dE/dV and dE/de of the
    lowest 3 states through the batch's per-system adjoint vs central FD of
    the independent dense double-precision H (h = 1e-4 MeV)."""
    from bigstickpublick_b200.engine import Batch
    specs = []
    for seed in (2001, 2002):
        m = model.batch_member(seed)
        m = model.ModelSpec(m.orbits, 2, 1 + (seed % 2), (2 + 1 + seed % 2) % 2, 1, m.spe, m.tbme)
        specs.append(m)
    tabs = [model.build_tables(m) for m in specs]
    b = Batch(tabs)
    for s, (m, t) in enumerate(zip(specs, tabs)):
        w, Z = np.linalg.eigh(oracle.dense_from_applyh(t))
        g = b.system(s).grad(Z[:, :3])
        h = 1e-4
        for k in range(3):
            gtb, gspe = model.chain_rule(t, {key: v[k] for key, v in g.items()})
            for i in (0, 7, 19, 41, 62):
                tp = [list(x) for x in m.tbme]
                tm = [list(x) for x in m.tbme]
                tp[i][6] += h
                tm[i][6] -= h
                ep = np.linalg.eigvalsh(dense_h.dense_h(m.orbits, m.np_, m.nn, m.jz2, m.spe, [tuple(x) for x in tp])[0])[k]
                em = np.linalg.eigvalsh(dense_h.dense_h(m.orbits, m.np_, m.nn, m.jz2, m.spe, [tuple(x) for x in tm])[0])[k]
                assert abs((ep - em) / (2 * h) - gtb[i]) < 1e-5, (s, k, i)
    b.close()


def test_batch_random_pivot_mixed_against_fp64(batch):
    """From a seeded random pivot per system (no symmetry of the uniform
    pivot restricting the Krylov space), the mixed batch (FP32 applyH) and
    the FP64 batch give the same lowest 5 eigenvalues to 1e-6 relative and
    eigenvector overlaps above 1 - 1e-5, system by system; the random pivot
    is a pure function of (seed, system), so two runs are bitwise equal."""
    tabs, b = batch
    ev8, v8, _ = b.lanczos(nkeep=5, niter=150, matvec_prec=8, want_vectors=True, pivot="random", seed=77)
    ev4, v4, _ = b.lanczos(nkeep=5, niter=150, matvec_prec=4, want_vectors=True, pivot="random", seed=77)
    ev8b, _, _ = b.lanczos(nkeep=5, niter=150, matvec_prec=8, pivot="random", seed=77)
    assert np.array_equal(ev8, ev8b)
    for s in range(len(tabs)):
        rel = np.abs(ev4[s] - ev8[s]) / np.abs(ev8[s])
        assert rel.max() < 1e-6, (s, rel)
        ov = np.abs(np.sum(v4[s] * v8[s], axis=0))
        assert ov.min() > 1 - 1e-5, (s, ov)
