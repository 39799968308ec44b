"""Three-body tables and the oracle's three-body bundle loops, on the CPU.

* A three-body Hamiltonian built from the two-body interaction alone
  (W = V2 / (A - 2) between three-particle states, the conversion of
  src/b3from2bme.f90) is the two-body Hamiltonian on A-particle states: the
  oracle's PPP / PPN / PNN / NNN loops (src/bapplyhlib1.f90:1390-2804) on
  those tables reproduce its two-body loops to float rounding of the
  matrix elements.
* The seeded three-body part R is checked against an independent dense
  second-quantization build, sum over triplets R(T, T') A+_T A_T', from the
  builder's s.p. labels only: no jumps, phases, labels or bundles shared.
* The engine's host-side validator accepts the builder's three-body tables
  and rejects corrupted ones.
"""
import itertools

import numpy as np
import pytest

import oracle
from bigstickpublick_b200 import engine, model

MASK = (1 << 64) - 1

SYSTEMS = [  # orbits, Z, N, 2Jz
    ("sd", 2, 2, 0), ("sd", 3, 1, 0), ("sd", 1, 3, 0), ("sd", 3, 0, 1), ("sd", 0, 3, 3),
    ("sd", 4, 3, 1), ("pf", 2, 2, 0), ("pf", 3, 1, 2),
]


def _spec(orb, z, n, jz2, spe=True):
    s = model.sd_model(z, n, seed=11, jz2=jz2) if orb == "sd" else model.pf_model(z, n, seed=3, jz2=jz2)
    if not spe:
        s.spe = [0.0] * len(s.orbits)
    return s


@pytest.mark.parametrize("orb,z,n,jz2", SYSTEMS)
def test_three_body_from_two_body_is_the_two_body_hamiltonian(orb, z, n, jz2):
    spec = _spec(orb, z, n, jz2)
    T2 = model.build_tables(spec)
    T3 = model.build_tables3(spec, w2=1.0, w3=0.0, seed=5)
    assert T3.threebody and T3.dim == T2.dim
    assert not np.isin(T3.a["optype"], [2, 3, 4]).any()    # no two-body bundles
    rng = np.random.default_rng(7)
    v = rng.standard_normal((T2.dim, 2))
    y2 = oracle.applyh(T2, v.ravel(), nb=2)
    y3 = oracle.applyh(T3, v.ravel(), nb=2)
    scale = np.abs(y2).max()
    assert np.abs(y2 - y3).max() < 2e-7 * scale * 10, np.abs(y2 - y3).max() / scale


def test_three_body_spectrum_matches_independent_dense_two_body():
    # the whole three-body pipeline against the independent dense two-body H
    from oracle import dense_h
    spec = _spec("sd", 2, 1, 1)
    T3 = model.build_tables3(spec, w2=1.0, w3=0.0, seed=5)
    H3 = oracle.dense_from_applyh(T3)
    Hd = dense_h.dense_h(spec.orbits, spec.np_, spec.nn, spec.jz2, spec.spe, spec.tbme)[0]
    e3 = np.linalg.eigvalsh(0.5 * (H3 + H3.T))
    ed = np.linalg.eigvalsh(Hd)
    assert np.allclose(e3, ed, atol=2e-5 * np.abs(ed).max())


def _mix(x):
    z = (x + 0x9E3779B97F4A7C15) & MASK
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
    return z ^ (z >> 31)


def _r3(seed, kind, k1, k2):
    lo, hi = sorted([tuple(k1), tuple(k2)])
    x = _mix((seed ^ kind) & MASK)
    for v in lo + hi:
        x = _mix(x ^ v)
    return (x >> 11) * 2.0 ** -52 - 1.0


def _sign_below(bits, q):
    return bin(bits & ((1 << q) - 1)).count("1")


def _apply(bits, create, destroy):
    """a+_c... a_d... |bits>: create ascending product of `create` (applied
    last-to-first as a+_c1 a+_c2 ...), destroy (a_dn ... a_d1, d1 first).
    Returns (new bits, sign) or None."""
    p = 0
    b = bits
    for q in destroy:                       # a_d1 acts first
        if not (b >> q) & 1:
            return None
        p += _sign_below(b, q)
        b &= ~(1 << q)
    for q in reversed(create):              # a+_ck acts first
        if (b >> q) & 1:
            return None
        p += _sign_below(b, q)
        b |= 1 << q
    return b, (-1) ** p


def _dense_r(T, seed):
    """sum_{T,T'} R(T,T') A+_T A_T' on the basis of T, from s.p. m only."""
    ex = T.extra
    m2 = {"p": list(ex["sp_m2_p"]), "n": list(ex["sp_m2_n"])}
    nsp = {"p": len(m2["p"]), "n": len(m2["n"])}
    # basis index of (proton SD, neutron SD)
    sdp, sdn = list(ex["sd_bits_p"]), list(ex["sd_bits_n"])
    pst, nst = T.a["pstart"], T.a["nstart"]
    index = {}
    pconj = ex["psector_conj"]
    for isec in range(len(ex["psector_start"])):
        c = pconj[isec] - 1
        for ip in range(ex["psector_start"][isec] - 1, ex["psector_end"][isec]):
            for jn in range(ex["nsector_start"][c] - 1, ex["nsector_end"][c]):
                index[(int(sdp[ip]), int(sdn[jn]))] = int(pst[ip] + nst[jn] - 1)
    H = np.zeros((T.dim, T.dim))
    # triplet families: (kind, species of the three slots)
    fams = [(1, "ppp"), (2, "nnn"), (3, "ppn"), (4, "pnn")]

    def trips(sp):
        # all (created-slot tuples) of species pattern sp, sorted within species
        np_ = sp.count("p")
        nn_ = sp.count("n")
        for P in itertools.combinations(range(nsp["p"]), np_):
            for N in itertools.combinations(range(nsp["n"]), nn_):
                yield P, N
    for kind, sp in fams:
        tl = list(trips(sp))
        for (pb, nb_), i in index.items():
            for (Pd, Nd) in tl:
                if any(not (pb >> q) & 1 for q in Pd) or any(not (nb_ >> q) & 1 for q in Nd):
                    continue
                md = sum(m2["p"][q] for q in Pd) + sum(m2["n"][q] for q in Nd)
                for (Pc, Nc) in tl:
                    if sum(m2["p"][q] for q in Pc) + sum(m2["n"][q] for q in Nc) != md:
                        continue
                    rp = _apply(pb, list(Pc), list(Pd))
                    rn = _apply(nb_, list(Nc), list(Nd))
                    if rp is None or rn is None:
                        continue
                    f = index.get((rp[0], rn[0]))
                    if f is None:
                        continue
                    kc, kd = list(Pc) + list(Nc), list(Pd) + list(Nd)
                    H[f, i] += _r3(seed, kind, kc, kd) * rp[1] * rn[1]
    return H


@pytest.mark.parametrize("orb,z,n,jz2", [("sd", 2, 1, 1), ("sd", 1, 2, 1), ("sd", 3, 0, 1), ("sd", 2, 2, 4)])
def test_seeded_three_body_part_against_second_quantization(orb, z, n, jz2):
    spec = _spec(orb, z, n, jz2, spe=False)
    seed = 0x1234ABCD
    T = model.build_tables3(spec, w2=0.0, w3=1.0, seed=seed)
    H = oracle.dense_from_applyh(T)
    Hr = _dense_r(T, seed)
    assert np.abs(H - H.T).max() < 1e-6
    assert np.abs(H - Hr).max() < 2e-6 * max(1.0, np.abs(Hr).max()), np.abs(H - Hr).max()


def test_validator_accepts_three_body_tables():
    for orb, z, n, jz2 in SYSTEMS:
        T = model.build_tables3(_spec(orb, z, n, jz2), w2=1.0, w3=0.3, seed=9)
        assert engine.validate_tables(T) == (0, ""), (orb, z, n)


@pytest.mark.parametrize("name,how,status,needle", [
    ("p3b_op", "first:1000000", 2, "hmatppp"),
    ("p2b_cop", "first:500", 2, "proton pairs"),
    ("n2b_dop", "first:0", 1, "neutron pairs"),
    ("cppntriplet", "all:1000000", 2, "hmatppn"),
    ("p3b_phase", "first:2", 1, "p3b_phase"),
])
def test_validator_rejects_corrupted_three_body_tables(name, how, status, needle):
    T = model.build_tables3(_spec("sd", 3, 2, 1), w2=1.0, w3=0.3, seed=9)
    a3 = {k: v.copy() for k, v in T.a3.items()}
    where, val = how.split(":")
    if where == "all":
        a3[name][:] = int(val)
    else:
        a3[name][0] = int(val)
    st, msg = engine.validate_tables(model.Tables(T.a, T.s, T.extra, a3, dict(T.s3)))
    assert st == status and needle in msg, (st, msg)


def test_three_body_bundle_in_a_two_body_context_is_rejected():
    T = model.build_tables(_spec("sd", 2, 2, 0))
    a = dict(T.a)
    a["optype"] = a["optype"].copy()
    a["optype"][0] = 9
    st, msg = engine.validate_tables(model.Tables(a, T.s, T.extra))
    assert st == 1 and "three-body" in msg


def test_three_body_needs_three_particles():
    with pytest.raises(RuntimeError, match="three valence particles"):
        model.build_tables3(_spec("sd", 1, 1, 0), w2=1.0)


@pytest.mark.parametrize("orb,z,n,jz2", [("sd", 3, 2, 1), ("sd", 2, 3, 1), ("pf", 3, 1, 2)])
def test_three_body_jump_order_invariance(orb, z, n, jz2):
    from _perm import permute_jumps3
    T = model.build_tables3(_spec(orb, z, n, jz2), w2=1.0, w3=0.3, seed=4)
    T2 = permute_jumps3(T, np.random.default_rng(1))
    assert not np.array_equal(T.a3["p2b_cop"], T2.a3["p2b_cop"]) or not np.array_equal(T.a["p1b_isd"], T2.a["p1b_isd"])
    assert engine.validate_tables(T2) == (0, "")
    v = np.random.default_rng(2).standard_normal(T.dim)
    y, y2 = oracle.applyh(T, v), oracle.applyh(T2, v)
    assert np.abs(y - y2).max() < 1e-12 * np.abs(y).max()
