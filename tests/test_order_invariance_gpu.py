"""The GPU engine on reordered tables (jumps permuted inside every sector
jump, hmat labels and pn pair sections renumbered; see _perm.py): the same
matvec to summation order and the same eigenvalues to 1e-12, so the orders
the builder chose where the reference's could not be run do not matter."""
import numpy as np
import pytest

from bigstickpublick_b200 import model
from _perm import permute_jumps, permute_labels

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mk", [lambda: model.sd_model(4, 4, seed=8), lambda: model.pf_model(2, 3, seed=9, jz2=1)])
def test_engine_invariant_under_table_orders(mk):
    from bigstickpublick_b200.engine import Hamiltonian
    T = model.build_tables(mk())
    rng = np.random.default_rng(7)
    T2 = permute_labels(permute_jumps(T, rng), rng)
    H1, H2 = Hamiltonian(T), Hamiltonian(T2)
    try:
        for dt, tol in ((np.float64, 1e-12), (np.float32, 2e-5)):
            v = rng.standard_normal(T.dim).astype(dt)
            y1, y2 = H1.applyh(v), H2.applyh(v)
            assert np.abs(y1 - y2).max() <= tol * np.abs(y1).max(), dt
        piv = rng.standard_normal(T.dim)
        e1, _, _ = H1.lanczos(nkeep=6, niter=300, matvec_prec=8, converge_tol=1e-13, pivot=piv)
        e2, _, _ = H2.lanczos(nkeep=6, niter=300, matvec_prec=8, converge_tol=1e-13, pivot=piv)
        assert np.abs(e1 - e2).max() <= 1e-12 * np.abs(e1).max(), (e1, e2)
    finally:
        H1.close()
        H2.close()
