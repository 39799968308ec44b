"""The builder's haiku order inside a block and its pair orders are the
reference's: checked against the oracle's step-by-step restatements of
count_create_haikus / fill_blocks and count_create_pairs /
count_create_pnpairs / sortpair / find_pair_start / count_uncouplepn
(oracle/basis_order.py)."""
import numpy as np
import pytest

from bigstickpublick_b200 import model
from oracle import basis_order as bo

PSD = [(0, 1, 1, 1), (0, 1, 3, 1), (0, 2, 5, 1), (1, 0, 1, 1), (0, 2, 3, 1)]


def _cases():
    return [
        ("sd 2p2n", lambda: model.build_tables(model.sd_model(2, 2, seed=1))),
        ("sd 3p2n odd", lambda: model.build_tables(model.sd_model(3, 2, seed=3, jz2=1))),
        ("sd 4p5n odd", lambda: model.build_tables(model.sd_model(4, 5, seed=4, jz2=1))),
        ("pf 2p3n odd", lambda: model.build_tables(model.pf_model(2, 3, seed=5, jz2=1))),
        ("psd 2p1n mixed parity", lambda: model.build_tables(model.ModelSpec(
            PSD, 2, 1, 1, -1, *model.synthetic_interaction(PSD, 9), 1.0, 1.0))),
    ]


def _species(T, s):
    m2 = [int(x) for x in T.extra["sp_m2_" + s]]
    orb = T.extra["sp_orb_" + s]
    spec = T.extra["spec"]
    ls = [o[1] for o in spec.orbits]
    same = len({l % 2 for l in ls}) == 1
    par = [1 if same else (-1 if ls[o] % 2 else 1) for o in orb]
    nl = sum(1 for x in m2 if x < 0)
    return m2, par, nl


def _qn(bits, m2, par, off, n):
    j, p, k = 0, 1, 0
    for q in range(n):
        if bits >> q & 1:
            j += m2[off + q]
            p *= par[off + q]
            k += 1
    return k, (1 if p > 0 else 2), j


@pytest.mark.parametrize("name,mk", _cases(), ids=[c[0] for c in _cases()])
def test_sd_order_inside_blocks_is_the_reference_creation_order(name, mk):
    T = mk()
    for s, N in (("p", T.extra["spec"].np_), ("n", T.extra["spec"].nn)):
        m2, par, nl = _species(T, s)
        nr = len(m2) - nl
        hl = bo.create_haikus(nl, min(N, nl))
        hr = bo.create_haikus(nr, min(N, nr))
        bits = [int(b) for b in T.extra["sd_bits_" + s]]
        s0, s1 = T.extra[s + "sector_start"], T.extra[s + "sector_end"]
        lmask = (1 << nl) - 1
        for a, b in zip(s0, s1):
            i = int(a) - 1
            while i < int(b):
                L, R = bits[i] & lmask, bits[i] >> nl
                kl, kr = _qn(L, m2, par, 0, nl), _qn(R, m2, par, nl, nr)
                left = bo.block_haikus(hl[kl[0]], m2[:nl], par[:nl], kl[2], kl[1])
                right = bo.block_haikus(hr[kr[0]], m2[nl:], par[nl:], kr[2], kr[1])
                want = [l | (r << nl) for l in left for r in right]
                got = bits[i:i + len(want)]
                assert got == want, (name, s, i)
                i += len(want)


@pytest.mark.parametrize("name,mk", _cases(), ids=[c[0] for c in _cases()])
def test_pn_pair_layout_is_the_reference_sortpair_order(name, mk):
    T = mk()
    m2p, parp, nlp = _species(T, "p")
    m2n, parn, nln = _species(T, "n")
    pairs = bo.pn_pairs(m2p, parp, m2n, parn)
    ld = len(m2n) + 1
    cexp = np.zeros(ld * (len(m2p) + 1), dtype=np.int64)
    dexp = np.zeros_like(cexp)
    for first, n, nme in bo.sections(pairs, square=True):
        for pos in range(1, n + 1):
            p = pairs[first + pos - 2]
            sp = -(p["qp"] + 1) if p["qp"] < nlp else p["qp"] - nlp + 1
            sn = -(p["qn"] + 1) if p["qn"] < nln else p["qn"] - nln + 1
            idx = (sn + nln) + (sp + nlp) * ld
            cexp[idx] = (pos - 1) * n
            dexp[idx] = pos + nme
    assert np.array_equal(np.asarray(T.a["cpnpair"]), cexp)
    assert np.array_equal(np.asarray(T.a["dpnpair"]), dexp)
    assert T.s["nmatpn"] == sum(n * n for _, n, _ in bo.sections(pairs, square=True))


@pytest.mark.parametrize("name,mk", _cases(), ids=[c[0] for c in _cases()])
def test_pp_jump_labels_follow_the_reference_pair_order(name, mk):
    T = mk()
    if T.s["np2b"] == 0:
        pytest.skip("no proton pairs")
    m2, par, nl = _species(T, "p")
    pairs = bo.xx_pairs(m2, par)
    pos = {(p["q1"], p["q2"]): i + 1 for i, p in enumerate(pairs)}
    secs = bo.sections(pairs, square=False)
    sec_of = {}
    for k, (first, n, nme) in enumerate(secs):
        for c in range(first, first + n):
            sec_of[c] = k
    assert T.s["nmatpp"] == sum(n * (n + 1) // 2 for _, n, _ in secs)
    bits = [int(b) for b in T.extra["sd_bits_p"]]
    sd_of = {int(v): i for i, v in enumerate(T.a["pstart"])}
    isd, fsd, op = T.a["p2b_isd"], T.a["p2b_fsd"], T.a["p2b_op"]
    for x in range(len(op)):
        bi, bf = bits[sd_of[int(isd[x])]], bits[sd_of[int(fsd[x])]]
        ann = [q for q in range(len(m2)) if (bi & ~bf) >> q & 1]
        cre = [q for q in range(len(m2)) if (bf & ~bi) >> q & 1]
        if not ann:   # diagonal: a pair annihilated and created again
            continue
        if len(ann) == 2:
            cands = [(tuple(cre), tuple(ann))]
        else:         # one state moves, the other member of both pairs is a spectator
            common = [q for q in range(len(m2)) if (bi & bf) >> q & 1]
            cands = [(tuple(sorted((cre[0], q))), tuple(sorted((ann[0], q)))) for q in common]
        labels = set()
        for cp, dp in cands:
            c, d = pos[cp], pos[dp]
            first, n, nme = secs[sec_of[c]]
            iref = first - 1
            hi, lo = max(c, d), min(c, d)
            labels.add(nme + (hi - iref) * (hi - iref - 1) // 2 + lo - iref)
        assert int(op[x]) in labels, (name, x)


def test_sortpair_is_a_heap_sort_not_a_stable_sort():
    # the restated heap sort reorders equal keys; the builder must follow it,
    # not a stable sort, or the pair layouts above would differ
    m2 = [-5, -3, -1, 1, 3, 5, -1, 1]
    par = [1] * 8
    pairs = bo.xx_pairs(m2, par)
    ms = [p["m"] for p in pairs]
    assert ms == sorted(ms, reverse=True)
    gen = [(b - 1, a - 1) for a in range(2, 9) for b in range(1, a)]
    stable = sorted(gen, key=lambda t: -((m2[t[0]] + m2[t[1]]) // 2))
    assert [(p["q1"], p["q2"]) for p in pairs] != stable
