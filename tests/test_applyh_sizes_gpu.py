"""applyH parity against the oracle at the benchmark sizes, where the long-row
kernels run.

The small systems of test_applyh_gpu.py all have median rows of at most 32
positions, so they only reach the one-position-per-lane tiles.  These cases
reach the tiles that the benchmark workloads use (tile width = the smallest
power of two times 32 covering the median row, capped at 256 positions for
FP32 and 128 for FP64 single vectors):

* sd 6p6n (dim 93,710, median row 109): single vectors in 128-position tiles
  (k_rows_f1<4,...> / k_rows_d1<4,...>), nb = 8 in 64-position tiles
  (k_rows<float|double, 8, 2, ...>);
* pf 4p4n (dim 1,963,461, median row 483): single FP32 vectors in
  256-position tiles at 32 registers (k_rows_f1<8,...>), FP64 in
  128-position tiles (k_rows_d1<4,...>), nb = 8 in k_rows<float, 8, 2, ...>;
* pf 6p6n (dim 109,954,620): k_rows_f1<8,...> / k_rows_d1<4,...> on the full
  vector, compared row by row with the oracle restricted to a few output rows
  (the owner-computes share of applyHbundled_omp, src/bapplyhlibOMP.f90
  :954-1442: one thread's rows, every jump whose output lands there).

The oracle runs the reference's arithmetic: FP32 matrix elements, and
accumulation in the vector precision.  Tolerances are relative to the largest
output: 1e-12 for FP64 (summation order only) and 2e-5 for FP32 (FP32
accumulation over up to about 1,400 terms per output in a different order).
"""
import os

import numpy as np
import pytest

from bigstickpublick_b200 import model
import oracle
from oracle import lanczos as olz

pytestmark = pytest.mark.gpu

NTHR = os.cpu_count()
TOL = {8: 1e-12, 4: 2e-5}


def _tables(shell, np_, nn, seed):
    mk = model.sd_model if shell == "sd" else model.pf_model
    return model.build_tables(mk(np_, nn, seed=seed))


@pytest.fixture(scope="module")
def sd66():
    from bigstickpublick_b200.engine import Hamiltonian
    T = _tables("sd", 6, 6, 2)
    H = Hamiltonian(T)
    yield T, H
    H.close()


@pytest.fixture(scope="module")
def pf44():
    from bigstickpublick_b200.engine import Hamiltonian
    T = _tables("pf", 4, 4, 3)
    H = Hamiltonian(T)
    yield T, H
    H.close()


def _full_parity(T, H, prec, nb, seed):
    dt = np.float64 if prec == 8 else np.float32
    vin = np.random.default_rng(seed).standard_normal(T.dim * nb).astype(dt)
    rs, ops = oracle.row_ops(T)
    ref = oracle.applyh_owner(T, vin, oracle.owner_ranges(rs, ops, T.dim, 4 * NTHR), nb=nb, nthreads=NTHR)
    got = H.applyh(vin if nb == 1 else vin.reshape(T.dim, nb)).reshape(-1)
    err = np.abs(got - ref).max() / np.abs(ref).max()
    return err


@pytest.mark.parametrize("prec,nb", [(4, 1), (8, 1), (4, 8), (8, 8)])
def test_sd6p6n_matches_oracle(sd66, prec, nb):
    T, H = sd66
    err = _full_parity(T, H, prec, nb, seed=100 + nb)
    assert err < TOL[prec], f"sd 6p6n prec={prec} nb={nb}: rel err {err:.3e}"


@pytest.mark.parametrize("prec,nb", [(4, 1), (8, 1), (4, 8)])
def test_pf4p4n_matches_oracle(pf44, prec, nb):
    T, H = pf44
    err = _full_parity(T, H, prec, nb, seed=200 + nb)
    assert err < TOL[prec], f"pf 4p4n prec={prec} nb={nb}: rel err {err:.3e}"


def test_pf4p4n_accumulate_and_repeatable(pf44):
    """vout += H vin on the long-row kernel, and two calls bit for bit equal."""
    import torch
    T, H = pf44
    g = torch.Generator(device="cuda").manual_seed(3)
    x = torch.randn(T.dim, dtype=torch.float32, device="cuda", generator=g)
    y1, y2 = H.applyh(x), H.applyh(x)
    torch.cuda.synchronize()
    assert torch.equal(y1, y2)
    base = torch.randn(T.dim, dtype=torch.float32, device="cuda", generator=g)
    acc = base.clone()
    H.applyh(x, acc, accumulate=True)
    torch.cuda.synchronize()
    assert torch.equal(acc, base + y1)


@pytest.mark.parametrize("prec", [4, 8])
def test_pf6p6n_rows_match_oracle(prec):
    """The largest configuration: the full GPU matvec against the oracle on
    the first row, a middle row, the last row and the row with the most work
    (a few thousand output positions)."""
    from bigstickpublick_b200.engine import Hamiltonian
    import torch
    T = _tables("pf", 6, 6, 5)
    assert T.dim == 109_954_620
    H = Hamiltonian(T)
    try:
        dt = np.float64 if prec == 8 else np.float32
        tdt = torch.float64 if prec == 8 else torch.float32
        vin = np.random.default_rng(7).standard_normal(T.dim).astype(dt)
        x = torch.from_numpy(vin).cuda()
        y = H.applyh(x)
        rs, ops = oracle.row_ops(T)
        ends = np.append(rs[1:], T.dim)
        pick = sorted({0, len(rs) // 2, len(rs) - 1, int(np.argmax(ops))})
        out = np.zeros_like(vin)
        n = 0
        for r in pick:
            oracle.applyh_rows(T, vin, rs[r], ends[r], out=out)
            lo, hi = int(rs[r]), int(ends[r])
            ref = out[lo:hi]
            got = y[lo:hi].to(tdt).cpu().numpy()
            err = np.abs(got - ref).max() / np.abs(ref).max()
            assert err < TOL[prec], f"pf 6p6n row {r} prec={prec}: rel err {err:.3e}"
            n += hi - lo
        assert n >= 1000
    finally:
        H.close()


def test_sd6p6n_fp64_lanczos_matches_oracle(sd66):
    """300 FP64 Lanczos iterations at sd 6p6n, lowest 10, against the oracle's
    lanczos_p restatement from the same pivot, within 1e-10 relative."""
    T, H = sd66
    piv = np.random.default_rng(11).standard_normal(T.dim)
    ev, _, rep = H.lanczos(nkeep=10, niter=300, matvec_prec=8, fixed_iter=True, pivot=piv)
    ref, _, _ = olz.lanczos(T, nkeep=10, niter=300, fixed_iter=True, pivot=piv, nthreads=NTHR)
    rel = np.abs(ev - ref) / np.abs(ref)
    assert rel.max() < 1e-10, rel


def test_sd6p6n_mixed_fp32_history_against_fp64(sd66):
    """sd 6p6n, 300 iterations: FP32 applyH with FP32-stored Lanczos vectors
    (lanc_prec = 4) against the FP64 path from the same pivot: eigenvalues
    within 1e-6 relative and eigenvector overlaps above 1 - 1e-6 for the
    lowest 10 states."""
    T, H = sd66
    piv = np.random.default_rng(11).standard_normal(T.dim)
    ev8, v8, _ = H.lanczos(nkeep=10, niter=300, matvec_prec=8, fixed_iter=True, pivot=piv, want_vectors=True)
    ev4, v4, _ = H.lanczos(nkeep=10, niter=300, matvec_prec=4, lanc_prec=4, fixed_iter=True, pivot=piv,
                           want_vectors=True)
    rel = np.abs(ev4 - ev8) / np.abs(ev8)
    assert rel.max() < 1e-6, rel
    ov = np.abs(np.sum(v4 * v8, axis=0))
    assert ov.min() > 1 - 1e-6, ov
