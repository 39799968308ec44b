"""Host-side table builder: dimensions, table invariants, determinism and an
independent physics check (dense second-quantization H, coupled 2-body spectra)."""
import numpy as np
import pytest

from bigstickpublick_b200 import model
import oracle
from oracle import dense_h


@pytest.mark.parametrize("np_,nn,jz,dim", [(2, 2, 0, 640), (6, 6, 0, 93710), (4, 5, 1, 44133), (1, 0, 1, 3)])
def test_sd_dimensions(np_, nn, jz, dim):
    T = model.build_tables(model.sd_model(np_, nn, seed=1, jz2=jz))
    assert T.dim == dim


def test_pf_4p4n_dimension():
    T = model.build_tables(model.pf_model(4, 4, seed=3))
    assert T.dim == 1963461


def test_canonical_tbme_counts():
    assert len(model.canonical_tbme_keys(model.SD_ORBITS)) == 63
    assert len(model.canonical_tbme_keys(model.PF_ORBITS)) == 195


def test_synthetic_interaction_is_seeded():
    a = model.synthetic_interaction(model.PF_ORBITS, 3)
    b = model.synthetic_interaction(model.PF_ORBITS, 3)
    c = model.synthetic_interaction(model.PF_ORBITS, 4)
    assert a == b and a != c


def test_build_is_deterministic():
    t1 = model.build_tables(model.sd_model(3, 2, seed=9, jz2=1))
    t2 = model.build_tables(model.sd_model(3, 2, seed=9, jz2=1))
    for k in t1.a:
        assert np.array_equal(t1.a[k], t2.a[k]), k


def test_table_invariants():
    T = model.build_tables(model.sd_model(3, 3, seed=2))
    a, s = T.a, T.s
    ps = a["pstart"]
    assert ps[0] == 0 and np.all(np.diff(ps) > 0)
    assert set(np.unique(a["p1b_phase"])) <= {-1, 1}
    assert a["p2b_op"].min() >= 1 and a["p2b_op"].max() <= s["nmatpp"]
    pvals = set(ps.tolist())
    assert set(a["p1b_isd"].tolist()) <= pvals and set(a["p2b_fsd"].tolist()) <= pvals
    # two-body jumps keep isd >= fsd inside a sector (hermitian half)
    assert np.all(a["p2b_isd"] >= a["p2b_fsd"])
    # PN bundles: protons sorted on fsd, neutrons on isd (sort_bundled_jumps)
    for ib in range(s["nbundles"]):
        if a["optype"][ib] != 4:
            continue
        p0, p1, n0, n1 = a["pxstart"][ib], a["pxend"][ib], a["nxstart"][ib], a["nxend"][ib]
        assert np.all(np.diff(a["p1b_fsd"][p0 - 1:p1]) >= 0)
        assert np.all(np.diff(a["n1b_isd"][n0 - 1:n1]) >= 0)
    # bundle order of draft_opbundles: PP f, NN f, PN f, PN h, PP b, NN b, PN b
    seq = [(int(o), chr(int(h))) for o, h in zip(a["optype"], a["hchar"])]
    kinds = [k for i, k in enumerate(seq) if i == 0 or seq[i - 1] != k]
    assert kinds == [(2, "f"), (3, "f"), (4, "f"), (4, "h"), (2, "b"), (3, "b"), (4, "b")]


@pytest.mark.parametrize("np_,nn,jz", [(1, 1, 0), (2, 0, 0), (2, 2, 0), (1, 2, 1), (0, 3, 3)])
def test_oracle_matvec_equals_independent_dense_h(np_, nn, jz):
    spe, tb = model.synthetic_interaction(model.SD_ORBITS, 7, spe=model.SD_SYNTH_SPE)
    spec = model.ModelSpec(model.SD_ORBITS, np_, nn, jz, 1, spe, tb)
    T = model.build_tables(spec)
    H = oracle.dense_from_applyh(T)
    assert np.array_equal(H, H.T)
    Hd, basis = dense_h.dense_h(model.SD_ORBITS, np_, nn, jz, spe, tb)
    assert len(basis) == T.dim
    ev, evd = np.linalg.eigvalsh(H), np.linalg.eigvalsh(Hd)
    assert np.abs(ev - evd).max() < 1e-6 * max(1.0, np.abs(evd).max())


def test_two_particle_pn_spectrum_equals_coupled_jt_blocks():
    """1p1n at M=0: the M-scheme spectrum is the union over J,T of the coupled
    two-particle matrices (isospin formalism of src/binput_tbme.f90:36-56)."""
    spe, tb = model.synthetic_interaction(model.SD_ORBITS, 21, spe=model.SD_SYNTH_SPE)
    T = model.build_tables(model.ModelSpec(model.SD_ORBITS, 1, 1, 0, 1, spe, tb))
    ev = np.sort(np.linalg.eigvalsh(oracle.dense_from_applyh(T)))
    cs = dense_h.coupled_two_body_spectrum(model.SD_ORBITS, spe, tb, 0) + \
        dense_h.coupled_two_body_spectrum(model.SD_ORBITS, spe, tb, 1)
    ref = np.sort([e for e, J in cs])
    assert np.abs(ev - ref).max() < 1e-5


@pytest.mark.parametrize("np_,nn,jz", [(2, 2, 0), (1, 2, 1), (3, 2, 1)])
def test_jsq_tsq_operator_spectra(np_, nn, jz):
    """The J^2 and T^2 operators built through the uncoupling (model.jsq_spec,
    model.tsq_spec) have spectra J(J+1), T(T+1) with J half-integer for odd A
    and integer for even A, and T between |Tz| and A/2."""
    base = model.sd_model(np_, nn, seed=1, jz2=jz)
    a = np_ + nn
    for mk, lo, hi in ((model.jsq_spec, None, None), (model.tsq_spec, abs(np_ - nn) / 2, a / 2)):
        T = model.build_tables(mk(base))
        M = oracle.dense_from_applyh(T)
        x = model.j_from_jsq(np.linalg.eigvalsh(0.5 * (M + M.T)))
        twice = np.round(2 * x)
        assert np.abs(2 * x - twice).max() < 1e-5
        assert np.all(twice % 2 == a % 2)
        if lo is not None:
            assert x.min() > lo - 1e-6 and x.max() < hi + 1e-6


def test_build_tables_many_equals_serial():
    """Tables built on several host threads at once equal the serial build
    byte for byte (the builder keeps no shared mutable state)."""
    specs = [model.batch_member(s) for s in range(1000, 1012)]
    par = model.build_tables_many(specs, threads=6)
    for sp, t in zip(specs, par):
        ref = model.build_tables(sp)
        assert ref.s == t.s
        for k in ref.a:
            assert np.array_equal(ref.a[k], t.a[k]), k
        for k in ("pp", "nn", "pn"):
            assert np.array_equal(ref.extra["jacobian"][k][0], t.extra["jacobian"][k][0])
