"""One-body operators and strength functions on the CPU: the .opme reader and
the M = 0 operator of decouple1bodyop (bigstickpublick_b200.densities), the
oracle's restatement of applyP1Bopbundled_g / applyN1Bopbundled_g against
second quantization, and the whole strength chain of the reference's example
(input.mg25apply1b + input.mg25strength) against
examples/sd/output/mg25spinstrength1.res."""
import json
import os

import numpy as np
import pytest

from bigstickpublick_b200 import densities as D
from bigstickpublick_b200 import model
import oracle
from oracle import density1b as od
from oracle import lanczos as ol

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "mg25.json")))


def test_read_opme_and_operator_selection_rules():
    op = D.read_opme(GOLD["spin_operator"]["text"])
    assert op.kind == "iso" and op.jop == 1 and op.top == 0
    assert op.orbits == [(0, 2, 3), (0, 2, 5), (1, 0, 1)]
    assert op.iso[(1, 2)] == pytest.approx(4.38178) and op.iso[(3, 3)] == pytest.approx(3.46410)
    T = model.build_tables(model.sd_model(2, 2, seed=4, jz2=0))
    P, N = D.onebody_operator(T, op)
    m2 = T.extra["sp_m2_p"]
    # M = 0 operator: nothing between different m
    for c in range(P.shape[0]):
        for d in range(P.shape[1]):
            if m2[c] != m2[d]:
                assert P[c, d] == 0.0 and N[c, d] == 0.0
    # isoscalar: protons and neutrons carry the same elements
    assert np.abs(P - N).max() < 1e-15
    bad = D.read_opme(GOLD["spin_operator"]["text"].replace("  3    1    0  0.5", "  3    0    0  0.5"))
    with pytest.raises(ValueError):
        D.onebody_operator(T, bad)


def test_read_opme_pn_formats():
    pns = "pns\n 3\n 1 0 2 1.5\n 2 0 2 2.5\n 3 1 0 0.5\n 1\n 1 2 1.0 2.0\n"
    op = D.read_opme(pns)
    assert op.kind == "pns" and op.prot[(1, 2)] == 1.0 and op.neut[(1, 2)] == 2.0
    xpn = "xpn\n 3\n 1 4 0 2 1.5\n 2 5 0 2 2.5\n 3 6 1 0 0.5\n 1\n 1 2 1.5\n 4 5 2.5\n 1 5 9.0\n"
    op = D.read_opme(xpn)
    assert op.prot == {(1, 2): 1.5} and op.neut == {(1, 2): 2.5}


@pytest.mark.parametrize("np_,nn,jz,shell", [(2, 2, 0, "sd"), (3, 2, 1, "sd"), (0, 3, 3, "sd"), (2, 1, 1, "pf")])
def test_apply1b_oracle_matches_second_quantization_and_densities(np_, nn, jz, shell):
    m = model.sd_model(np_, nn, seed=4, jz2=jz) if shell == "sd" else model.pf_model(np_, nn, seed=4, jz2=jz)
    T = model.build_tables(m)
    rng = np.random.default_rng(3)
    nqp = T.s["nhsps_pl"] + T.s["nhsps_pr"]
    nqn = T.s["nhsps_nl"] + T.s["nhsps_nr"]
    P, N = rng.standard_normal((nqp, nqp)), rng.standard_normal((nqn, nqn))
    X = rng.standard_normal((T.dim, 2))
    Y = od.apply1b_bundled(T, P, N, X)
    assert np.abs(Y - od.apply1b_from_bits(T, P, N, X)).max() < 1e-12 * max(1.0, np.abs(Y).max())
    # <f|O|i> = sum_cd pot(c,d) <f|a+_c a_d|i>
    Dp, Dn = od.bundled(T, X)
    rhs = np.einsum("fpcd,cd->fp", Dp, P) + np.einsum("fpcd,cd->fp", Dn, N)
    assert np.abs(X.T @ Y - rhs).max() < 1e-11 * max(1.0, np.abs(rhs).max())


def strength_checks(E, S, total, gold):
    """What a 30-step strength run can share with the reference's: the total
    |O psi|^2, the converged lowest Ritz pair, and the moments sum S E^m of
    the distribution.  The reference runs Lanczos with FP32 vectors
    (lanc_prec = 4, src/bmodules_main.f90:171); their rounding, amplified over
    30 steps, moves its interior Ritz values by up to 1e-2 MeV (they sit
    between those of 29 and 31 exact steps), while the low moments stay fixed
    to the table's 5 printed decimals."""
    g = np.array(gold["table"])
    assert abs(total / gold["total"] - 1.0) < 1e-6
    assert abs(E[0] - g[0, 0]) < 5e-5 and abs(S[0] - g[0, 1]) < 5e-5
    assert abs(S.sum() - total) < 1e-9 * total
    for m in range(9):
        a = float((S * E ** m).sum())
        b = float((g[:, 1] * g[:, 0] ** m).sum())
        assert abs(a - b) <= 3e-5 * abs(b), (m, a, b)


def _mg25_spec():
    r = GOLD["runs"]["mg25ref"]
    ss, ts = model.ModelSpec.scaling(*r["scaling"])
    orbits = [tuple(o) for o in GOLD["orbits"]]
    return model.ModelSpec(orbits, r["np"], r["nn"], r["jz2"], 1, GOLD["spe"], [tuple(t) for t in GOLD["tbme"]], ss, ts)


def test_mg25_spin_strength_oracle_chain():
    from scipy.sparse.linalg import LinearOperator, eigsh
    T = model.build_tables(_mg25_spec())
    mv = lambda v: oracle.applyh(T, np.ascontiguousarray(v, dtype=np.float64))
    w, Z = eigsh(LinearOperator((T.dim, T.dim), matvec=mv, dtype=np.float64), k=1, which="SA", tol=1e-13,
                 v0=np.ones(T.dim))
    P, N = D.onebody_operator(T, D.read_opme(GOLD["spin_operator"]["text"]))
    piv = od.apply1b_bundled(T, P, N, Z[:, 0])
    total = float(piv @ piv)
    ev, vecs, rep = ol.lanczos(T, nkeep=30, niter=30, fixed_iter=True, want_vectors=True, pivot=piv, matvec=mv)
    S = (vecs.T @ (piv / np.sqrt(total))) ** 2 * total
    strength_checks(ev, S, total, GOLD["spin_strength"])


def test_backward_bundles_equal_forward_in_oracle():
    """The oracle's 'b' branches (densities and operator application) on
    tables where half the jumps come through 'b' bundles equal the all-'f'
    tables: the split is the one the GPU tests use."""
    from test_density_gpu import _split_with_backward
    T = model.build_tables(model.sd_model(3, 2, seed=4, jz2=1))
    d = _split_with_backward(T)
    assert (d["hchar"] == ord("b")).any()
    alt = model.Tables(T.a, T.s, dict(T.extra, density=d))
    rng = np.random.default_rng(2)
    X = rng.standard_normal((T.dim, 3))
    nqp = T.s["nhsps_pl"] + T.s["nhsps_pr"]
    nqn = T.s["nhsps_nl"] + T.s["nhsps_nr"]
    P, N = rng.standard_normal((nqp, nqp)), rng.standard_normal((nqn, nqn))
    for a, b in zip(od.bundled(alt, X), od.bundled(T, X)):
        assert np.abs(a - b).max() < 1e-12 * max(1.0, np.abs(b).max())
    Y, Yref = od.apply1b_bundled(alt, P, N, X), od.apply1b_bundled(T, P, N, X)
    assert np.abs(Y - Yref).max() < 1e-12 * max(1.0, np.abs(Yref).max())


def test_pn_operator_elements_follow_their_species():
    """A 'pns' operator: the proton table comes from the proton column, the
    neutron table from the neutron one, with 1/sqrt(2J+1) and no isospin
    factors (decouple1bodyop's pnoperators branch)."""
    T = model.build_tables(model.sd_model(2, 2, seed=4, jz2=0))
    text = "pns\n 3\n 1 0 2 1.5\n 2 0 2 2.5\n 3 1 0 0.5\n 0\n 2 2 1.0 0.0\n 3 3 0.0 2.0\n"
    P, N = D.onebody_operator(T, D.read_opme(text))
    orb_p, orb_n = T.extra["sp_orb_p"], T.extra["sp_orb_n"]
    # J = 0: diagonal in (orbit, m), (-1)^(j-m) (j m, j -m | 0 0) = 1/sqrt(2j+1)
    for q in range(len(orb_p)):
        if orb_p[q] == 1:
            assert abs(P[q, q] - 1.0 / np.sqrt(6.0)) < 1e-14
        else:
            assert P[q, q] == 0.0
        if orb_n[q] == 2:
            assert abs(N[q, q] - 2.0 / np.sqrt(2.0)) < 1e-14
    assert np.count_nonzero(P - np.diag(np.diag(P))) == 0


def test_read_opme_rejects_unknown_format():
    with pytest.raises(ValueError):
        D.read_opme("foo\n 3\n")
