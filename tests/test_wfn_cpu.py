"""The .wfn eigenvector file (write_wfn_header / wfn_writeeigenvec,
src/bwfnlib.f90:77-134 and :373-546): byte layout, round trip, and the s.p.
state order of sort_spsqn (src/bspstates.f90:100-215)."""
import struct

import numpy as np
import pytest

from bigstickpublick_b200 import model, wfn


def test_sps_order_is_sort_spsqn():
    """sd.sps order (d3/2, d5/2, s1/2): all positive parity, so states are
    sorted by |m| only, stably by the selection sort with swap."""
    sps = wfn.sorted_sps(model.SD_ORBITS)
    assert len(sps) == 12
    assert [abs(x["m2"]) for x in sps] == sorted(abs(x["m2"]) for x in sps)
    # the selection sort with swap is not stable: the first |m| = 1 state it
    # selects is d3/2 m = -1/2 (the first |m| = 1 in extract_sps order)
    assert (sps[0]["orb"], sps[0]["m2"]) == (1, -1)
    assert all(x["w"] == 0 and x["par"] == 1 and x["group"] == 0 for x in sps)
    # every (orbit, m) exactly once
    assert sorted((x["orb"], x["m2"]) for x in sps) == sorted(
        (i + 1, m) for i, (_, _, j2, _) in enumerate(model.SD_ORBITS) for m in range(-j2, j2 + 1, 2))


def _restated_sort(orbits):
    """The three selection sorts of sort_spsqn written out directly."""
    sp = [(n, l, j2, m, i + 1) for i, (n, l, j2, w) in enumerate(orbits) for m in range(-j2, j2 + 1, 2)]
    for i in range(len(sp)):
        k = i
        for j in range(i + 1, len(sp)):
            if abs(sp[j][3]) < abs(sp[k][3]):
                k = j
        sp[i], sp[k] = sp[k], sp[i]
    return [(x[4], x[3]) for x in sp]


@pytest.mark.parametrize("orbits", [model.SD_ORBITS, model.PF_ORBITS])
def test_sps_matches_direct_restatement(orbits):
    assert [(x["orb"], x["m2"]) for x in wfn.sorted_sps(orbits)] == _restated_sort(orbits)


@pytest.mark.parametrize("lanc_prec", [4, 8])
def test_round_trip_and_layout(tmp_path, lanc_prec):
    spec = model.sd_model(2, 3, seed=1, jz2=1)
    T = model.build_tables(spec)
    rng = np.random.default_rng(0)
    k = 3
    V = rng.standard_normal((T.dim, k))
    V /= np.linalg.norm(V, axis=0)
    ev = np.array([-20.5, -19.25, -18.0])
    xj = np.array([1.5, 2.5, 0.5])
    xt2 = np.array([0.75, 3.75, 0.75])
    p = tmp_path / "s.wfn"
    wfn.write_wfn(p, spec, ev, V, xj, xt2, lanc_prec=lanc_prec)
    raw = p.read_bytes()
    magic, version, zero, after = struct.unpack_from("<4i", raw, 0)
    assert (magic, version, zero) == (31415926, 1, 0)
    h, states = wfn.read_wfn(p, lanc_prec=lanc_prec)
    assert h["dim"] == T.dim and h["nkeep"] == k and (h["np"], h["nn"]) == (2, 3)
    assert h["jz2"] == 1 and h["cparity"] == "+" and h["isoflag"] == 1
    assert (h["maxWtot"], h["allsameparity"], h["allsameW"], h["spinless"]) == (0, 1, 1, 0)
    assert len(h["orbits"][0]) == len(h["orbits"][1]) == 3
    assert h["orbits"][0][0] == (0, 3, 2, 1, 0)  # nr, 2j, l, par, w of d3/2
    assert len(h["sps"][0]) == 12
    # the after-header word points at the first vector record
    assert struct.unpack_from("<i", raw, after)[0] == 27182818
    rec = 20 + T.dim * (4 if lanc_prec == 4 else 8)
    assert len(raw) == after + k * rec
    dt = np.float32 if lanc_prec == 4 else np.float64
    for i, s in enumerate(states):
        assert s["index"] == i + 1
        assert s["e"] == np.float32(ev[i]) and s["xj"] == np.float32(xj[i]) and s["xt2"] == np.float32(xt2[i])
        assert np.array_equal(s["vec"], V[:, i].astype(dt))


def test_mixed_w_is_refused(tmp_path):
    spec = model.sd_model(1, 1, seed=1)
    spec.orbits = [(0, 2, 3, 0), (0, 2, 5, 1), (1, 0, 1, 2)]
    with pytest.raises(ValueError):
        wfn.header_bytes(spec, 10)
