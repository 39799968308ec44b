"""bsg_apply1b on the GPU against the oracle's restatement of
applyP1Bopbundled_g / applyN1Bopbundled_g (src/bdenslib3.f90:319-584), and
the ²⁵Mg spin strength function (apply the operator of sdspin.opme to the
ground state, 30 Lanczos steps from the result) against
examples/sd/output/mg25spinstrength1.res."""
import json
import os

import numpy as np
import pytest

from bigstickpublick_b200 import densities as D
from bigstickpublick_b200 import model
from oracle import density1b as od

from test_strength_cpu import GOLD, _mg25_spec, strength_checks

pytestmark = pytest.mark.gpu


def _H(T):
    from bigstickpublick_b200.engine import Hamiltonian
    return Hamiltonian(T)


@pytest.mark.parametrize("np_,nn,jz,shell,k", [(2, 2, 0, "sd", 1), (3, 2, 1, "sd", 3), (0, 3, 3, "sd", 2),
                                               (2, 1, 1, "pf", 1), (6, 6, 0, "sd", 2)])
def test_apply1b_matches_oracle(np_, nn, jz, shell, k):
    m = model.sd_model(np_, nn, seed=4, jz2=jz) if shell == "sd" else model.pf_model(np_, nn, seed=4, jz2=jz)
    T = model.build_tables(m)
    rng = np.random.default_rng(5)
    nqp = T.s["nhsps_pl"] + T.s["nhsps_pr"]
    nqn = T.s["nhsps_nl"] + T.s["nhsps_nr"]
    P, N = rng.standard_normal((nqp, nqp)), rng.standard_normal((nqn, nqn))
    X = rng.standard_normal((T.dim, k))
    H = _H(T)
    Y = H.apply1b(P, N, X)
    ref = od.apply1b_bundled(T, P, N, X)
    assert np.abs(Y - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())
    assert np.array_equal(Y, H.apply1b(P, N, X))
    # one species only
    Yp = H.apply1b(P, None, X)
    assert np.abs(Yp - od.apply1b_bundled(T, P, None, X)).max() <= 1e-12 * max(1.0, np.abs(Yp).max())
    # <f|O|i> against the GPU densities
    md = H.density1b(X)
    rhs = np.einsum("fpcd,cd->fp", md["p"], P) + np.einsum("fpcd,cd->fp", md["n"], N)
    assert np.abs(X.T @ Y - rhs).max() <= 1e-11 * max(1.0, np.abs(rhs).max())
    H.close()


def test_mg25_spin_strength_function():
    T = model.build_tables(_mg25_spec())
    H = _H(T)
    ev, vecs, rep = H.lanczos(nkeep=1, niter=300, matvec_prec=8, want_vectors=True, converge_tol=1e-13)
    P, N = D.onebody_operator(T, D.read_opme(GOLD["spin_operator"]["text"]))
    piv = H.apply1b(P, N, vecs[:, 0])
    E, S, total = D.strength_function(H, piv, niter=30)
    H.close()
    assert len(E) == 30
    strength_checks(E, S, total, GOLD["spin_strength"])


def test_apply1b_backward_bundles_equal_forward():
    from test_density_gpu import _split_with_backward, _with_density
    T = model.build_tables(model.sd_model(4, 3, seed=4, jz2=1))
    rng = np.random.default_rng(8)
    nqp = T.s["nhsps_pl"] + T.s["nhsps_pr"]
    nqn = T.s["nhsps_nl"] + T.s["nhsps_nr"]
    P, N = rng.standard_normal((nqp, nqp)), rng.standard_normal((nqn, nqn))
    X = rng.standard_normal((T.dim, 2))
    H = _H(T)
    ref = H.apply1b(P, N, X)
    dt, keep = _with_density(T, _split_with_backward(T))
    got = H.apply1b(P, N, X, density_tables=dt)
    assert np.abs(got - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())
    assert np.abs(got - od.apply1b_bundled(keep, P, N, X)).max() <= 1e-12 * max(1.0, np.abs(ref).max())
    H.close()
