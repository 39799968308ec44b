"""Adjoint (bsg_grad): dE/dhmat on the GPU against the oracle's restatement of
the two-body-density traversal, dE/dV through the uncoupling chain rule
against central finite differences of an independent double-precision H, the
25Mg SPE gradient against the reference's one-body densities, and the Euler
identity E = sum V dE/dV + sum e dE/de (H is linear in its parameters)."""
import json
import os

import numpy as np
import pytest

from bigstickpublick_b200 import model
import oracle
from oracle import dense_h

pytestmark = pytest.mark.gpu
GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "mg25.json")))


def _H(T):
    from bigstickpublick_b200.engine import Hamiltonian
    return Hamiltonian(T)


@pytest.mark.parametrize("np_,nn,jz,shell", [(2, 2, 0, "sd"), (3, 2, 1, "sd"), (1, 0, 1, "sd"), (2, 2, 0, "pf")])
def test_grad_matches_oracle_density(np_, nn, jz, shell):
    m = model.sd_model(np_, nn, seed=4, jz2=jz) if shell == "sd" else model.pf_model(np_, nn, seed=4, jz2=jz)
    T = model.build_tables(m)
    w, Z = np.linalg.eigh(oracle.dense_from_applyh(T))
    ns = min(3, T.dim)
    H = _H(T)
    g = H.grad(Z[:, :ns])
    for k in range(ns):
        ref = oracle.density(T, Z[:, k])
        for key in ("pp", "nn", "pn") + (("spe_p", "spe_n") if T.s["call_spe"] else ()):
            if ref[key].size == 0:
                continue
            scale = max(1e-30, np.abs(ref[key]).max())
            assert np.abs(g[key][k] - ref[key]).max() / scale < 1e-10, (key, k)
        # Hellmann-Feynman consistency: E = psi^T H psi = sum_label hmat * dE/dhmat
        e = sum(float(np.dot(g[nm][k], T.a["hmat" + nm])) for nm in ("pp", "nn", "pn"))
        if T.s["call_spe"]:
            e += float(np.dot(g["spe_p"][k], T.a["pspe_h"]) + np.dot(g["spe_n"][k], T.a["nspe_h"]))
        assert abs(e - w[k]) < 1e-9 * max(1.0, abs(w[k]))
    H.close()


def test_tbme_and_spe_gradient_vs_central_fd():
    """sd 2p1n, 2Jz=1: dE0/dV_i and dE0/de_a vs (E(+h)-E(-h))/2h, h = 1e-4 MeV,
    on the independent dense H in double precision."""
    spe, tb = model.synthetic_interaction(model.SD_ORBITS, 7, spe=model.SD_SYNTH_SPE)
    spec = model.ModelSpec(model.SD_ORBITS, 2, 1, 1, 1, spe, tb)
    T = model.build_tables(spec)
    w, Z = np.linalg.eigh(oracle.dense_from_applyh(T))
    H = _H(T)
    g = H.grad(Z[:, :1])
    gtb, gspe = model.chain_rule(T, {k: v[0] for k, v in g.items()})
    h = 1e-4

    def e0(spe_, tb_):
        return np.linalg.eigvalsh(dense_h.dense_h(model.SD_ORBITS, 2, 1, 1, spe_, tb_)[0])[0]

    for i in range(len(tb)):
        tp = [list(x) for x in tb]
        tm = [list(x) for x in tb]
        tp[i][6] += h
        tm[i][6] -= h
        fd = (e0(spe, [tuple(x) for x in tp]) - e0(spe, [tuple(x) for x in tm])) / (2 * h)
        assert abs(fd - gtb[i]) < 1e-5, (i, fd, gtb[i])
    for a in range(3):
        sp, sm = list(spe), list(spe)
        sp[a] += h
        sm[a] -= h
        fd = (e0(sp, tb) - e0(sm, tb)) / (2 * h)
        assert abs(fd - gspe[a]) < 1e-5
    H.close()


def test_mg25_spe_gradient_equals_reference_occupations():
    """dE_k/de_a = <n_a>_k, and the reference prints <n_a> through its Jt=0,
    Tt=0 one-body densities: n_a = rho(a,a) sqrt((2j_a+1)/(2J+1))
    (examples/sd/output/mg25ref.res)."""
    r = GOLD["runs"]["mg25ref"]
    ss, ts = model.ModelSpec.scaling(*r["scaling"])
    orbits = [tuple(o) for o in GOLD["orbits"]]
    spec = model.ModelSpec(orbits, r["np"], r["nn"], r["jz2"], 1, GOLD["spe"], [tuple(t) for t in GOLD["tbme"]], ss, ts)
    T = model.build_tables(spec)
    H = _H(T)
    ev, vecs, rep = H.lanczos(nkeep=10, niter=400, matvec_prec=8, want_vectors=True, converge_tol=1e-11)
    gold = np.array([s["E"] for s in r["states"]])
    assert np.abs(ev - gold).max() < 1.5e-5
    g = H.grad(vecs)
    for k in range(10):
        gtb, gspe = model.chain_rule(T, {key: v[k] for key, v in g.items()})
        dens = r["density_jt0"][str(k + 1)]
        occ = np.zeros(3)
        for a, b, rho0, _ in dens["rho"]:
            if a == b:
                occ[a - 1] = rho0 * np.sqrt((orbits[a - 1][2] + 1) / (dens["J2"] + 1))
        assert abs(occ.sum() - 9.0) < 1e-3
        assert np.abs(gspe - ss * occ).max() < 3e-5, (k, gspe, occ)
    H.close()


def test_euler_identity_sd6p6n():
    """E0 = sum_i V_i dE0/dV_i + sum_a e_a dE0/de_a for the 93,710-dim
    benchmark system (size-independent check of the whole adjoint chain)."""
    m = model.sd_model(6, 6, seed=2)
    T = model.build_tables(m)
    H = _H(T)
    piv = np.random.default_rng(3).standard_normal(T.dim)
    ev, vecs, rep = H.lanczos(nkeep=1, niter=300, matvec_prec=8, want_vectors=True, converge_tol=1e-12, pivot=piv)
    g = H.grad(vecs)
    gtb, gspe = model.chain_rule(T, {k: v[0] for k, v in g.items()})
    spec = T.extra["spec"]
    V = np.array([t[6] for t in spec.tbme])
    e = float(V @ gtb + np.array(spec.spe) @ gspe)
    # float32 rounding of the uncoupled matrix elements bounds the agreement
    assert abs(e - ev[0]) < 1e-5 * abs(ev[0]), (e, ev[0])
    H.close()


def test_grad_bitwise_repeatable():
    """Every label's sum is exact 128-bit fixed point: two calls agree bit for
    bit, and one state's gradient does not depend on the other states of the
    call (the work split differs)."""
    T = model.build_tables(model.sd_model(3, 3, seed=6))
    rng = np.random.default_rng(1)
    V = rng.standard_normal((T.dim, 3))
    V /= np.linalg.norm(V, axis=0)
    H = _H(T)
    g1, g2 = H.grad(V), H.grad(V)
    g0 = H.grad(V[:, :1])
    H.close()
    for key in ("pp", "nn", "pn"):
        assert np.array_equal(g1[key], g2[key]), key
        assert np.array_equal(g1[key][:1], g0[key]), key


def test_batch_grad_one_launch_equals_per_system():
    """bsg_batch_grad: all systems and states in one launch, bitwise equal to
    each member's own bsg_grad, and equal to the oracle's density traversal."""
    from bigstickpublick_b200.engine import Batch
    tabs = [model.build_tables(model.batch_member(s)) for s in (1000, 1003, 1006)]
    b = Batch(tabs)
    rng = np.random.default_rng(2)
    vecs = []
    for t in tabs:
        V = rng.standard_normal((t.dim, 2))
        vecs.append(V / np.linalg.norm(V, axis=0))
    gb = b.grad(vecs)
    assert b.grad_ms > 0
    for s, t in enumerate(tabs):
        gs = b.system(s).grad(vecs[s])
        for key in ("pp", "nn", "pn"):
            assert np.array_equal(gb[s][key], gs[key]), (s, key)
        ref = oracle.density(t, vecs[s][:, 1])
        for key in ("pp", "nn", "pn"):
            scale = max(1e-30, np.abs(ref[key]).max())
            assert np.abs(gb[s][key][1] - ref[key]).max() / scale < 1e-10, (s, key)
    b.close()
