"""Device Lanczos (lanczos_p / lanczos_block with thick restart) against
exact diagonalization and the oracle's numpy restatement."""
import numpy as np
import pytest

from bigstickpublick_b200 import model
import oracle
from oracle import lanczos as olz

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sd22():
    from bigstickpublick_b200.engine import Hamiltonian
    T = model.build_tables(model.sd_model(2, 2, seed=1))
    H = Hamiltonian(T)
    exact = np.linalg.eigvalsh(oracle.dense_from_applyh(T))
    return T, H, exact


def generic_pivot(n, nb=1, seed=5):
    # no proton-neutron exchange symmetry, unlike the uniform pivot
    return np.random.default_rng(seed).standard_normal(n * nb)


def test_fp64_matches_exact(sd22):
    T, H, exact = sd22
    ev, _, rep = H.lanczos(nkeep=10, niter=300, matvec_prec=8, converge_tol=1e-13,
                           pivot=generic_pivot(T.dim))
    rel = np.abs(ev - exact[:10]) / np.abs(exact[:10])
    assert rel.max() < 1e-10, (rel, rep)


def test_uniform_pivot_ground_state(sd22):
    """The reference's option-0 pivot (uniform 1/sqrt(dim)) is symmetric under
    proton-neutron exchange for N = Z; the ground state lies in its class.
    (Round-off slowly seeds the other class, so only the ground state is a
    well-posed comparison.)"""
    T, H, exact = sd22
    ev, _, rep = H.lanczos(nkeep=1, niter=120, matvec_prec=8, converge_tol=1e-13)
    assert abs(ev[0] - exact[0]) / abs(exact[0]) < 1e-10


def test_fp64_matches_oracle_lanczos(sd22):
    T, H, exact = sd22
    piv = generic_pivot(T.dim)
    ev, _, rep = H.lanczos(nkeep=10, niter=100, matvec_prec=8, fixed_iter=True, pivot=piv)
    ref, _, _ = olz.lanczos(T, nkeep=10, niter=100, fixed_iter=True, pivot=piv)
    assert np.abs(ev - ref).max() / np.abs(ref).max() < 1e-10


def test_mixed_precision_error_bound(sd22):
    T, H, exact = sd22
    ev, _, rep = H.lanczos(nkeep=10, niter=300, matvec_prec=4, converge_tol=1e-10,
                           pivot=generic_pivot(T.dim))
    rel = np.abs(ev - exact[:10]) / np.abs(exact[:10])
    assert rel.max() < 1e-6, rel


def test_eigenvectors(sd22):
    T, H, exact = sd22
    ev, vecs, rep = H.lanczos(nkeep=5, niter=300, matvec_prec=8, want_vectors=True, converge_tol=1e-13,
                              pivot=generic_pivot(T.dim))
    assert vecs.shape == (T.dim, 5)
    for k in range(5):
        v = vecs[:, k]
        r = oracle.applyh(T, v) - ev[k] * v
        assert abs(np.linalg.norm(v) - 1) < 1e-8
        assert np.linalg.norm(r) < 1e-6 * abs(ev[k])


def test_thick_restart_converges(sd22):
    T, H, exact = sd22
    ev, _, rep = H.lanczos(nkeep=5, niter=40, nthick_add=10, max_restarts=80, matvec_prec=8,
                           converge_tol=1e-9, pivot=generic_pivot(T.dim))
    assert rep["restarts"] >= 1, rep
    rel = np.abs(ev - exact[:5]) / np.abs(exact[:5])
    assert rel.max() < 1e-9, (rel, rep)


@pytest.mark.parametrize("kw", [dict(nkeep=5, niter=200),
                                dict(nkeep=5, niter=30, nthick_add=10, max_restarts=40)])
def test_convergence_stop_matches_oracle(sd22, kw):
    """The convergence test of a step runs beside the next step's applyH;
    the run must still stop at the same step as the reference's order (the
    oracle's stop step is the same for tol within +-2 %, so round-off cannot
    move it)."""
    T, H, exact = sd22
    piv = generic_pivot(T.dim)
    ev, _, rep = H.lanczos(matvec_prec=8, converge_tol=1e-6, pivot=piv, **kw)
    ref, _, orep = olz.lanczos(T, tol=1e-6, pivot=piv, **kw)
    assert rep["converged"] == 1
    assert rep["total_iterations"] == orep["total_iterations"], (rep, orep)
    assert rep["restarts"] == orep["restarts"]
    assert rep["iterations"] == orep["iterations"]
    assert np.abs(ev - ref).max() < 1e-9 * np.abs(ref).max()


def test_thick_restart_matches_oracle(sd22):
    T, H, exact = sd22
    kw = dict(nkeep=5, niter=30, nthick_add=5, max_restarts=3, converge_tol=1e-30)
    piv = generic_pivot(T.dim)
    ev, _, rep = H.lanczos(matvec_prec=8, pivot=piv, **kw)
    ref, _, orep = olz.lanczos(T, tol=1e-30, pivot=piv, **{k: v for k, v in kw.items() if k != "converge_tol"})
    assert rep["restarts"] == orep["restarts"] == 3
    assert np.abs(ev - ref).max() / np.abs(ref).max() < 1e-10, (ev, ref)


@pytest.mark.parametrize("nb", [2, 4, 8])
def test_block_lanczos(sd22, nb):
    T, H, exact = sd22
    ev, vecs, rep = H.lanczos(nkeep=8, niter={2: 150, 4: 100, 8: 60}[nb], nb=nb, matvec_prec=8, want_vectors=True,
                              converge_tol=1e-10)
    rel = np.abs(ev - exact[:8]) / np.abs(exact[:8])
    assert rel.max() < 1e-9, (nb, rel, rep)


def test_block_thick_restart(sd22):
    T, H, exact = sd22
    ev, _, rep = H.lanczos(nkeep=6, niter=12, nb=4, nthick_add=6, max_restarts=60, matvec_prec=4,
                           converge_tol=1e-8)
    assert rep["restarts"] >= 1
    rel = np.abs(ev - exact[:6]) / np.abs(exact[:6])
    assert rel.max() < 1e-6, (rel, rep)


BLOCK_RUNS = {
    # nb: (plain run, thick-restart run); stop steps verified stable for tol
    # within +-2 % in the oracle, so round-off cannot move them
    2: (dict(nkeep=6, niter=150), dict(nkeep=5, niter=20, nthick_add=7, max_restarts=40)),
    4: (dict(nkeep=6, niter=80), dict(nkeep=5, niter=10, nthick_add=7, max_restarts=40)),
    8: (dict(nkeep=6, niter=40), dict(nkeep=5, niter=8, nthick_add=11, max_restarts=40)),
}


@pytest.mark.parametrize("thick", [False, True])
@pytest.mark.parametrize("nb", [2, 4, 8])
def test_block_matches_oracle(sd22, nb, thick):
    """Block Lanczos (and block thick restart) against the oracle's
    lanczos_block restatement from the same pivot block: the same stop step
    and restart count under the reference's convergence test (tol 1e-3), and
    the same eigenvalues."""
    T, H, exact = sd22
    piv = generic_pivot(T.dim, nb)
    kw = BLOCK_RUNS[nb][1 if thick else 0]
    ev, _, rep = H.lanczos(nb=nb, matvec_prec=8, converge_tol=1e-3, pivot=piv, **kw)
    ref, _, orep = olz.lanczos_block(T, nb, tol=1e-3, pivot=piv, **kw)
    assert orep["converged"] == 1 and rep["converged"] == 1
    assert rep["total_iterations"] == orep["total_iterations"], (rep, orep)
    assert rep["restarts"] == orep["restarts"], (rep, orep)
    if thick:
        assert rep["restarts"] >= 1
    assert np.abs(ev - ref).max() / np.abs(ref).max() < 1e-10, (ev, ref)


@pytest.mark.parametrize("nb", [4, 8])
def test_block_fixed_schedule_matches_oracle(sd22, nb):
    """A fixed schedule with three block thick restarts: the eigenvalues after
    the same steps agree with the oracle's to 1e-10."""
    T, H, exact = sd22
    piv = generic_pivot(T.dim, nb, seed=9)
    kw = dict(nkeep=5, niter=6, nthick_add=11, max_restarts=3)
    ev, _, rep = H.lanczos(nb=nb, matvec_prec=8, converge_tol=1e-30, pivot=piv, **kw)
    ref, _, orep = olz.lanczos_block(T, nb, tol=1e-30, pivot=piv, **kw)
    assert rep["restarts"] == orep["restarts"] == 3
    assert rep["total_iterations"] == orep["total_iterations"]
    assert np.abs(ev - ref).max() / np.abs(ref).max() < 1e-10, (ev, ref)


@pytest.mark.parametrize("matvec_prec", [8, 4])
def test_fp32_history_error_bound(sd22, matvec_prec):
    """Lanczos vectors stored in FP32 (the reference's shipped lanc_prec = 4),
    dots and updates accumulated in FP64: eigenvalues within 1e-6 relative of
    exact diagonalization, with the FP64 or the FP32 applyH."""
    T, H, exact = sd22
    ev, vecs, rep = H.lanczos(nkeep=10, niter=300, matvec_prec=matvec_prec, lanc_prec=4, converge_tol=1e-10,
                              pivot=generic_pivot(T.dim), want_vectors=True)
    rel = np.abs(ev - exact[:10]) / np.abs(exact[:10])
    assert rel.max() < 1e-6, rel
    for k in range(3):
        v = vecs[:, k]
        assert abs(np.linalg.norm(v) - 1) < 1e-5
        assert np.linalg.norm(oracle.applyh(T, v) - ev[k] * v) < 1e-4 * abs(ev[k])


@pytest.mark.parametrize("nb", [1, 4])
def test_fp32_history_thick_restart(sd22, nb):
    """FP32 history through thick restarts (basis rotation stored in FP32)."""
    T, H, exact = sd22
    kw = dict(nkeep=5, niter=40 if nb == 1 else 10, nthick_add=7, max_restarts=60)
    ev, _, rep = H.lanczos(nb=nb, matvec_prec=4, lanc_prec=4, converge_tol=1e-8, pivot=generic_pivot(T.dim, nb),
                           **kw)
    assert rep["restarts"] >= 1
    rel = np.abs(ev - exact[:5]) / np.abs(exact[:5])
    assert rel.max() < 1e-6, (rel, rep)
