"""Three-body applyH on the GPU (bsg_create3) against the oracle's
restatement of the three-body bundle loops (applyhPPPbundled_g,
applyhPPNbundled_g, applyhPNNbundled_g, applyhNNNbundled_g,
src/bapplyhlib1.f90:1390-2804; block forms src/bapplyhblocklib.f90:741-1541).

PPP / NNN run as the PP / NN row contributions, PPN / PNN as PN-form
contributions over the appended triplet tables; these tests cover every
kind (systems with 3+ protons, 3+ neutrons, and both species), FP64 and
FP32, single vectors and blocks, and the Lanczos eigenvalues of the
three-body form of a two-body interaction against the two-body ones."""
import numpy as np
import pytest

import oracle
from bigstickpublick_b200 import model

pytestmark = pytest.mark.gpu

CASES = [
    ("sd 3p0n", lambda: model.sd_model(3, 0, seed=11, jz2=1)),
    ("sd 0p3n", lambda: model.sd_model(0, 3, seed=11, jz2=3)),
    ("sd 2p2n", lambda: model.sd_model(2, 2, seed=1)),
    ("sd 3p2n", lambda: model.sd_model(3, 2, seed=3, jz2=1)),
    ("sd 4p3n", lambda: model.sd_model(4, 3, seed=3, jz2=1)),
    ("pf 3p1n", lambda: model.pf_model(3, 1, seed=3, jz2=2)),
    ("pf 2p3n", lambda: model.pf_model(2, 3, seed=5, jz2=1)),
]


@pytest.fixture(scope="module")
def built():
    from bigstickpublick_b200.engine import Hamiltonian
    out = {}
    for name, mk in CASES:
        T = model.build_tables3(mk(), w2=1.0, w3=0.4, seed=77)
        out[name] = (T, Hamiltonian(T))
    return out


@pytest.mark.parametrize("name", [c[0] for c in CASES])
@pytest.mark.parametrize("prec", [8, 4])
@pytest.mark.parametrize("nb", [1, 2, 3, 8])
def test_threebody_applyh_matches_oracle(built, name, prec, nb):
    T, H = built[name]
    rng = np.random.default_rng(99 + nb)
    dt = np.float64 if prec == 8 else np.float32
    vin = rng.standard_normal((T.dim, nb)).astype(dt)
    if nb == 1:
        vin = vin[:, 0].copy()
    ref = oracle.applyh(T, vin.reshape(-1), nb=nb).reshape(vin.shape)
    got = H.applyh(vin)
    scale = np.abs(ref).max() + 1e-30
    err = np.abs(got - ref).max() / scale
    tol = 1e-12 if prec == 8 else 2e-5
    assert err < tol, f"{name} prec={prec} nb={nb}: rel err {err:.3e}"


def test_threebody_kinds_present(built):
    # the cases cover every three-body kind
    kinds = set()
    for T, H in built.values():
        st = H.stats()
        for k in ("ppp", "nnn", "ppn", "pnn"):
            if st["n_ops_" + k] > 0:
                kinds.add(k)
        assert sum(st["n_ops_" + k] for k in ("ppp", "nnn", "ppn", "pnn")) == sum(oracle.count_ops3(T))
        assert st["n_ops_pp"] == st["n_ops_nn"] == st["n_ops_pn"] == 0
    assert kinds == {"ppp", "nnn", "ppn", "pnn"}


def test_threebody_accumulate_and_repeatable(built):
    T, H = built["sd 4p3n"]
    rng = np.random.default_rng(3)
    vin = rng.standard_normal(T.dim)
    base = rng.standard_normal(T.dim)
    out = base.copy()
    H.applyh(vin, out, accumulate=True)
    ref = base + oracle.applyh(T, vin)
    assert np.abs(out - ref).max() < 1e-12 * (np.abs(ref).max() + 1)
    a, b = H.applyh(vin), H.applyh(vin)
    assert np.array_equal(a, b)


def test_threebody_form_of_two_body_interaction_has_the_two_body_spectrum():
    from bigstickpublick_b200.engine import Hamiltonian
    spec = model.sd_model(3, 3, seed=21)
    H2 = Hamiltonian(model.build_tables(spec))
    H3 = Hamiltonian(model.build_tables3(spec, w2=1.0, w3=0.0, seed=1))
    e2, _, _ = H2.lanczos(nkeep=5, niter=200, matvec_prec=8)
    e3, _, _ = H3.lanczos(nkeep=5, niter=200, matvec_prec=8)
    # the matrix elements are float32 in both forms: agreement to their rounding
    assert np.allclose(e2, e3, atol=2e-5 * np.abs(e2).max()), (e2, e3)


def test_threebody_grad_is_refused(built):
    from bigstickpublick_b200.engine import BsgError
    T, H = built["sd 2p2n"]
    v = np.zeros((T.dim, 1))
    v[0, 0] = 1.0
    with pytest.raises(BsgError) as e:
        H.grad(v)
    assert e.value.status == 8


@pytest.mark.parametrize("tmax", [32, 100])
def test_split_neutron_operators_match_oracle(tmax):
    # neutron operators with more (b,d) pairs than pn_table_max are split into
    # sub-operators; two-body PN and three-body PPN / PNN both
    from bigstickpublick_b200.engine import Hamiltonian
    rng = np.random.default_rng(tmax)
    for T in (model.build_tables(model.pf_model(3, 3, seed=5)),
              model.build_tables3(model.sd_model(3, 3, seed=3), w2=1.0, w3=0.4, seed=8)):
        H = Hamiltonian(T, pn_table_max=tmax)
        for prec, tol in ((8, 1e-12), (4, 2e-5)):
            v = rng.standard_normal(T.dim).astype(np.float64 if prec == 8 else np.float32)
            ref = oracle.applyh(T, v)
            got = H.applyh(v)
            assert np.abs(got - ref).max() / np.abs(ref).max() < tol
        H.close()


def test_threebody_engine_on_reordered_jumps():
    # the engine consumes any jump order inside a sector jump: the same
    # matvec (to summation order) on the three-body tables with every jump
    # range of every bundle permuted
    from _perm import permute_jumps3
    from bigstickpublick_b200.engine import Hamiltonian
    T = model.build_tables3(model.sd_model(4, 3, seed=3, jz2=1), w2=1.0, w3=0.3, seed=4)
    T2 = permute_jumps3(T, np.random.default_rng(5))
    H2 = Hamiltonian(T2)
    v = np.random.default_rng(6).standard_normal(T.dim)
    ref = oracle.applyh(T, v)
    assert np.abs(H2.applyh(v) - ref).max() < 1e-12 * np.abs(ref).max()
    H2.close()


@pytest.mark.parametrize("run", ["mg25ref", "mg25alt"])
def test_mg25_energies_in_three_body_form_match_reference_output(run):
    # the reference's own 25Mg USDB answers (examples/sd/output/mg25ref.res:8-17,
    # mg25alt.res:8-17, 10 states to 5 decimals) through the three-body
    # machinery: the interaction carried entirely by PPP / PPN / PNN / NNN
    # bundles (W = V2/(A-2)), solved by the engine's Lanczos
    import json
    import os
    from bigstickpublick_b200.engine import Hamiltonian
    gold = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "mg25.json")))
    r = gold["runs"][run]
    ss, ts = model.ModelSpec.scaling(*r["scaling"])
    spec = model.ModelSpec([tuple(o) for o in gold["orbits"]], r["np"], r["nn"], r["jz2"], 1, gold["spe"],
                           [tuple(t) for t in gold["tbme"]], ss, ts)
    T3 = model.build_tables3(spec, w2=1.0, w3=0.0, seed=1)
    assert T3.dim == 44133
    H = Hamiltonian(T3)
    ev, _, _ = H.lanczos(nkeep=10, niter=400, matvec_prec=8, converge_tol=1e-12)
    H.close()
    e_gold = np.array([s["E"] for s in r["states"]])
    assert np.abs(ev - e_gold).max() < 1.5e-5, (ev, e_gold)
