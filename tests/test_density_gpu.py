"""bsg_density1b on the GPU: m-scheme one-body transition densities against
the oracle's restatement of applyP1Bdenbundled_g / applyN1Bdenbundled_g
(src/bdenslib3.f90:14-311), 'b' bundles, repeatability and table errors; and
the reduced densities of 25Mg against every block the reference prints in
examples/sd/output/mg25ref.res and mg25alt.res."""
import json
import os

import numpy as np
import pytest

from bigstickpublick_b200 import densities, model
from oracle import density1b as od

pytestmark = pytest.mark.gpu
GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "mg25.json")))


def _H(T):
    from bigstickpublick_b200.engine import Hamiltonian
    return Hamiltonian(T)


def _tables(np_, nn, jz, shell, seed=4):
    m = model.sd_model(np_, nn, seed=seed, jz2=jz) if shell == "sd" else model.pf_model(np_, nn, seed=seed, jz2=jz)
    return model.build_tables(m)


def _close(a, b, rel=1e-12):
    return np.abs(a - b).max() <= rel * max(1.0, np.abs(b).max())


@pytest.mark.parametrize("np_,nn,jz,shell,k", [(2, 2, 0, "sd", 1), (3, 2, 1, "sd", 5), (1, 0, 1, "sd", 3),
                                               (0, 3, 3, "sd", 2), (2, 1, 1, "pf", 4), (4, 4, 0, "sd", 32),
                                               (6, 6, 0, "sd", 4)])
def test_density1b_matches_oracle(np_, nn, jz, shell, k):
    T = _tables(np_, nn, jz, shell)
    X = np.random.default_rng(np_ * 10 + nn).standard_normal((T.dim, k))
    H = _H(T)
    md = H.density1b(X)
    Dp, Dn = od.bundled(T, X)
    assert _close(md["p"], Dp) and _close(md["n"], Dn)
    again = H.density1b(X)
    assert np.array_equal(again["p"], md["p"]) and np.array_equal(again["n"], md["n"])
    H.close()


def _split_with_backward(T):
    """Same densities through 'f' + 'b' bundles: per P1B bundle keep the
    jumps with isd > fsd (A) and isd == fsd (D); 'f' over A and D, 'b' over A
    (the jumps with isd < fsd are the conjugates of A, same phase)."""
    d = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in T.extra["density"].items()}
    keys = ["p1b_isd", "p1b_fsd", "p1b_cop", "p1b_dop", "p1b_phase"]
    new = {k: [] for k in keys}
    bun = {k: [] for k in ("optype", "hchar", "pxstart", "pxend", "nxstart", "nxend", "cstride")}
    for b in range(int(d["nbundles"])):
        if d["optype"][b] != 5:
            for k in bun:
                bun[k].append(d[k][b])
            continue
        j = np.arange(d["pxstart"][b] - 1, d["pxend"][b])
        A = j[d["p1b_isd"][j] > d["p1b_fsd"][j]]
        Dg = j[d["p1b_isd"][j] == d["p1b_fsd"][j]]
        start = len(new["p1b_isd"])
        for k in keys:
            new[k].extend(d[k][A].tolist() + d[k][Dg].tolist())
        for hc, lo, hi in ((ord("f"), start + 1, start + len(A) + len(Dg)), (ord("b"), start + 1, start + len(A))):
            if hi < lo:
                continue
            for k, v in (("optype", 5), ("hchar", hc), ("pxstart", lo), ("pxend", hi), ("nxstart", d["nxstart"][b]),
                         ("nxend", d["nxend"][b]), ("cstride", d["cstride"][b])):
                bun[k].append(v)
    dt = {"p1b_isd": "i8", "p1b_fsd": "i8", "p1b_cop": "i2", "p1b_dop": "i2", "p1b_phase": "i1"}
    for k in keys:
        d[k] = np.array(new[k], dtype=dt[k])
    for k, v in bun.items():
        d[k] = np.array(v, dtype=d[k].dtype)
    d["np1b"] = len(d["p1b_isd"])
    d["nbundles"] = len(d["optype"])
    return d


def _with_density(T, d):
    alt = model.Tables(T.a, T.s, dict(T.extra, density=d))
    return alt.density_ctypes(), alt


def test_backward_bundles_equal_forward():
    T = _tables(4, 3, 1, "sd")
    X = np.random.default_rng(7).standard_normal((T.dim, 6))
    H = _H(T)
    ref = H.density1b(X)
    d = _split_with_backward(T)
    assert (d["hchar"] == ord("b")).any()
    dt, keep = _with_density(T, d)
    got = H.density1b(X, density_tables=dt)
    assert _close(got["p"], ref["p"]) and _close(got["n"], ref["n"])
    H.close()


@pytest.mark.parametrize("field,value,code", [("p1b_cop", 99, "OOB"), ("pxend", 10 ** 9, "OOB"),
                                              ("p1b_phase", 3, "BAD_TABLE"), ("optype", 2, "BAD_TABLE")])
def test_bad_density_tables_are_refused(field, value, code):
    T = _tables(2, 2, 0, "sd")
    X = np.random.default_rng(1).standard_normal((T.dim, 2))
    H = _H(T)
    d = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in T.extra["density"].items()}
    d[field][0] = value
    dt, keep = _with_density(T, d)
    with pytest.raises(RuntimeError, match=code):
        H.density1b(X, density_tables=dt)
    # the context stays usable
    ok = H.density1b(X)
    assert _close(ok["p"], od.bundled(T, X)[0])
    H.close()


def _mg25(run):
    from bigstickpublick_b200.engine import angular_momentum_isospin
    r = GOLD["runs"][run]
    ss, ts = model.ModelSpec.scaling(*r["scaling"])
    orbits = [tuple(o) for o in GOLD["orbits"]]
    spec = model.ModelSpec(orbits, r["np"], r["nn"], r["jz2"], 1, GOLD["spe"], [tuple(t) for t in GOLD["tbme"]], ss, ts)
    T = model.build_tables(spec)
    H = _H(T)
    ev, vecs, rep = H.lanczos(nkeep=10, niter=400, matvec_prec=8, want_vectors=True, converge_tol=1e-12)
    J, Tv = angular_momentum_isospin(spec, vecs)
    red = densities.density1b(H, vecs, J, Tv)
    H.close()
    return r, red


@pytest.mark.parametrize("run", ["mg25ref", "mg25alt"])
def test_mg25_reduced_densities_equal_reference_res(run):
    """Every printed block (initial, final, Jt; Tt = 0 and 1) to the 5
    decimals of the .res file plus eigenvector convergence.  Transition
    densities carry the product of the two eigenvectors' arbitrary signs: one
    sign per state pair, taken from its largest printed entry."""
    r, red = _mg25(run)
    blocks = r["densities"]
    sign, big = {}, {}
    for b in blocks:
        key = (min(b["i"], b["f"]), max(b["i"], b["f"]))
        ours = red[(b["i"], b["f"])][b["Jt"]]
        for a, c, t0, t1 in b["rho"]:
            for tt, g in ((0, t0), (1, t1)):
                if abs(g) > big.get(key, 0.0):
                    big[key] = abs(g)
                    sign[key] = np.sign(ours[a - 1, c - 1, tt] * g)
    printed = {}
    for b in blocks:
        i, f, Jt = b["i"], b["f"], b["Jt"]
        assert Jt in red[(i, f)], (i, f, Jt)
        ours = red[(i, f)][Jt] * sign[(min(i, f), max(i, f))]
        # states 7 and 8 of mg25alt lie 0.6 keV apart with different J; the
        # reference's vectors of that pair are less converged
        tol = 1e-3 if run == "mg25alt" and {i, f} & {7, 8} else 5e-5
        for a, c, t0, t1 in b["rho"]:
            assert abs(ours[a - 1, c - 1, 0] - t0) < tol and abs(ours[a - 1, c - 1, 1] - t1) < tol, (i, f, Jt, a, c)
        printed[(i, f, Jt)] = {(a, c) for a, c, _, _ in b["rho"]}
    # nothing the reference left out (below 1e-6 or triangle-forbidden) is large here
    for (i, f), bl in red.items():
        for Jt, den in bl.items():
            keep = printed.get((i, f, Jt), set())
            for a in range(den.shape[0]):
                for c in range(den.shape[1]):
                    if (a + 1, c + 1) not in keep:
                        assert np.abs(den[a, c]).max() < 1e-5, (i, f, Jt, a, c)
