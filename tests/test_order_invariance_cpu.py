"""The engine's answer does not depend on the table orders (jump order inside
a sector jump, where the builder's order is its own; matrix-element labels and
pair order inside an (M, parity) section): permuted tables give the same
matvec to summation order and the same spectrum (oracle on the CPU; the GPU
engine in test_order_invariance_gpu.py)."""
import numpy as np
import pytest

from bigstickpublick_b200 import model
from bigstickpublick_b200.engine import validate_tables
import oracle
from _perm import permute_jumps, permute_labels

CASES = [lambda: model.sd_model(2, 2, seed=1), lambda: model.sd_model(3, 2, seed=3, jz2=1),
         lambda: model.pf_model(2, 2, seed=5), lambda: model.sd_model(1, 0, seed=12, jz2=1)]


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("how", ["jumps", "labels", "both"])
def test_oracle_matvec_and_spectrum_invariant(case, how):
    T = model.build_tables(CASES[case]())
    rng = np.random.default_rng(100 + case)
    T2 = T
    if how in ("jumps", "both"):
        T2 = permute_jumps(T2, rng)
    if how in ("labels", "both"):
        T2 = permute_labels(T2, rng)
    assert validate_tables(T2)[0] == 0
    if how != "jumps" and T.s["np1b"]:
        assert any(not np.array_equal(T.a[k], T2.a[k]) for k in ("hmatpp", "hmatnn", "hmatpn"))
    v = rng.standard_normal(T.dim)
    y1, y2 = oracle.applyh(T, v), oracle.applyh(T2, v)
    assert np.abs(y1 - y2).max() <= 1e-12 * np.abs(y1).max()
    if T.dim <= 2000:
        e1 = np.linalg.eigvalsh(oracle.dense_from_applyh(T))
        e2 = np.linalg.eigvalsh(oracle.dense_from_applyh(T2))
        assert np.abs(e1 - e2).max() <= 1e-12 * np.abs(e1).max()
