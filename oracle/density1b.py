"""ORACLE (test infrastructure only) -- one-body transition densities.

Two CPU restatements of <f| a+_c a_d |i> for every pair of states, used as the
checker of bsg_density1b:

* ``bundled``: the reference's traversal, applyP1Bdenbundled_g and
  applyN1Bdenbundled_g (src/bdenslib3.f90:14-311): per P1B / N1B bundle and
  jump, the sum over the conjugate SDs (arithmetic progressions of basis
  states, indexed exactly as there) of vec_f(statef) vec_i(statei) times the
  phase, into (cop, dop); 'b' bundles swap the states and the label.
* ``from_bits``: second quantization straight from the SD occupation bits,
  independent of the density jump tables: a_d then a+_c on every proton
  (neutron) SD of every basis state, phase from the occupied states below.

Both return (D_p, D_n) with D[f, i, c, d], c and d combined s.p. indices.
"""
import numpy as np


def _comb(lab, nl):
    return -lab - 1 if lab < 0 else nl + lab - 1


def bundled(tables, vecs):
    X = np.asarray(vecs, dtype=np.float64)
    if X.ndim == 1:
        X = X[:, None]
    s, a = tables.s, tables.a
    d = tables.extra["density"]
    k = X.shape[1]
    nlp, nqp = s["nhsps_pl"], s["nhsps_pl"] + s["nhsps_pr"]
    nln, nqn = s["nhsps_nl"], s["nhsps_nl"] + s["nhsps_nr"]
    Dp = np.zeros((k, k, nqp, nqp))
    Dn = np.zeros((k, k, nqn, nqn))
    pstart, nstart = a["pstart"], a["nstart"]
    for b in range(int(d["nbundles"])):
        op, hc, cs = int(d["optype"][b]), int(d["hchar"][b]), int(d["cstride"][b])
        if op == 5:      # P1B: jumps pxstart..pxend, neutron SDs nxstart..nxend
            j0, j1, c0, c1 = d["pxstart"][b], d["pxend"][b], d["nxstart"][b], d["nxend"][b]
            nc = (c1 + cs - c0) // cs
            first = nstart[c0 - cs] - 1 + cs          # nstart(c0 - cs + 1) - 1 + cs
            rows0 = first + cs * np.arange(nc) - 1    # + isd, 0-based
            pre, D, nl = "p1b_", Dp, nlp
        else:            # N1B: jumps nxstart..nxend, proton SDs pxstart..pxend
            j0, j1, c0, c1 = d["nxstart"][b], d["nxend"][b], d["pxstart"][b], d["pxend"][b]
            nc = (c1 + cs - c0) // cs
            pstride = pstart[c0 - 1 + cs] - pstart[c0 - 1] if nc > 1 else 0
            rows0 = pstart[c0 - 1] + pstride * np.arange(nc) - 1
            pre, D, nl = "n1b_", Dn, nln
        for j in range(j0 - 1, j1):
            ri = d[pre + "isd"][j] + rows0
            rf = d[pre + "fsd"][j] + rows0
            c, dd = _comb(int(d[pre + "cop"][j]), nl), _comb(int(d[pre + "dop"][j]), nl)
            ph = float(d[pre + "phase"][j])
            if hc == ord("b"):
                D[:, :, dd, c] += ph * (X[ri].T @ X[rf])
            else:
                D[:, :, c, dd] += ph * (X[rf].T @ X[ri])
    return Dp, Dn


def _phase(bits, c, d):
    """sign of a+_c a_d |bits> (ascending-label order)"""
    below = lambda b, q: bin(b & ((1 << q) - 1)).count("1")
    p = below(bits, d)
    p += below(bits & ~(1 << d), c)
    return -1.0 if p % 2 else 1.0


def from_bits(tables, vecs):
    X = np.asarray(vecs, dtype=np.float64)
    if X.ndim == 1:
        X = X[:, None]
    s, a, ex = tables.s, tables.a, tables.extra
    k = X.shape[1]
    # basis index of (proton SD, neutron SD) for every pair in the basis
    pst, nst = a["pstart"], a["nstart"]
    pairs = {}
    for ip in range(len(ex["psector_start"])):
        isn = ex["psector_conj"][ip] - 1
        for p in range(ex["psector_start"][ip] - 1, ex["psector_end"][ip]):
            for n in range(ex["nsector_start"][isn] - 1, ex["nsector_end"][isn]):
                pairs[(p, n)] = int(pst[p] + nst[n] - 1)
    out = []
    for sp in ("p", "n"):
        bits = [int(x) for x in ex["sd_bits_" + sp]]
        m2 = ex["sp_m2_" + sp]
        nq = len(m2)
        index = {b: i for i, b in enumerate(bits)}
        D = np.zeros((k, k, nq, nq))
        for (p, n), row in pairs.items():
            sd = p if sp == "p" else n
            b0 = bits[sd]
            for dq in range(nq):
                if not (b0 >> dq) & 1:
                    continue
                for cq in range(nq):
                    if m2[cq] != m2[dq] or (cq != dq and (b0 >> cq) & 1):
                        continue
                    b1 = (b0 & ~(1 << dq)) | (1 << cq)
                    t = index.get(b1)
                    if t is None:
                        continue
                    key = (t, n) if sp == "p" else (p, t)
                    rf = pairs.get(key)
                    if rf is None:
                        continue
                    D[:, :, cq, dq] += _phase(b0, cq, dq) * np.outer(X[rf], X[row])
        out.append(D)
    return out[0], out[1]


def apply1b_bundled(tables, ppot, npot, vin):
    """O vin by the reference's traversal, applyP1Bopbundled_g /
    applyN1Bopbundled_g (src/bdenslib3.f90:319-584): vout(statef) +=
    pot(cop, dop) * phase * vin(statei) per jump and conjugate SD; 'b' bundles
    vout(statei) += pot(dop, cop) * phase * vin(statef)."""
    x = np.asarray(vin, dtype=np.float64)
    one = x.ndim == 1
    X = x[:, None] if one else x
    s, a = tables.s, tables.a
    d = tables.extra["density"]
    nlp, nln = s["nhsps_pl"], s["nhsps_nl"]
    Y = np.zeros_like(X)
    pstart, nstart = a["pstart"], a["nstart"]
    for b in range(int(d["nbundles"])):
        op, hc, cs = int(d["optype"][b]), int(d["hchar"][b]), int(d["cstride"][b])
        if op == 5:
            if ppot is None:
                continue
            j0, j1, c0, c1 = d["pxstart"][b], d["pxend"][b], d["nxstart"][b], d["nxend"][b]
            nc = (c1 + cs - c0) // cs
            rows0 = nstart[c0 - cs] - 1 + cs + cs * np.arange(nc) - 1
            pre, pot, nl = "p1b_", ppot, nlp
        else:
            if npot is None:
                continue
            j0, j1, c0, c1 = d["nxstart"][b], d["nxend"][b], d["pxstart"][b], d["pxend"][b]
            nc = (c1 + cs - c0) // cs
            pstride = pstart[c0 - 1 + cs] - pstart[c0 - 1] if nc > 1 else 0
            rows0 = pstart[c0 - 1] + pstride * np.arange(nc) - 1
            pre, pot, nl = "n1b_", npot, nln
        for j in range(j0 - 1, j1):
            ri = d[pre + "isd"][j] + rows0
            rf = d[pre + "fsd"][j] + rows0
            c, dd = _comb(int(d[pre + "cop"][j]), nl), _comb(int(d[pre + "dop"][j]), nl)
            ph = float(d[pre + "phase"][j])
            if hc == ord("b"):
                Y[ri] += pot[dd, c] * ph * X[rf]
            else:
                Y[rf] += pot[c, dd] * ph * X[ri]
    return Y[:, 0] if one else Y


def apply1b_from_bits(tables, ppot, npot, vin):
    """O vin by second quantization on the SD bits (independent of the
    density tables): <f|O|i> = sum pot(c, d) <f|a+_c a_d|i>, i.e. the
    transpose of ``from_bits`` contracted with the operator."""
    x = np.asarray(vin, dtype=np.float64)
    one = x.ndim == 1
    X = x[:, None] if one else x
    # D[f, i, c, d] over unit vectors would be dim^2: build the action directly
    s, a, ex = tables.s, tables.a, tables.extra
    pst, nst = a["pstart"], a["nstart"]
    pairs = {}
    for ip in range(len(ex["psector_start"])):
        isn = ex["psector_conj"][ip] - 1
        for p in range(ex["psector_start"][ip] - 1, ex["psector_end"][ip]):
            for n in range(ex["nsector_start"][isn] - 1, ex["nsector_end"][isn]):
                pairs[(p, n)] = int(pst[p] + nst[n] - 1)
    Y = np.zeros_like(X)
    for sp, pot in (("p", ppot), ("n", npot)):
        if pot is None:
            continue
        bits = [int(v) for v in ex["sd_bits_" + sp]]
        index = {bb: i for i, bb in enumerate(bits)}
        nq = pot.shape[0]
        for (p, n), row in pairs.items():
            sd = p if sp == "p" else n
            b0 = bits[sd]
            for dq in range(nq):
                if not (b0 >> dq) & 1:
                    continue
                for cq in range(nq):
                    if pot[cq, dq] == 0.0 or (cq != dq and (b0 >> cq) & 1):
                        continue
                    t = index.get((b0 & ~(1 << dq)) | (1 << cq))
                    if t is None:
                        continue
                    rf = pairs.get((t, n) if sp == "p" else (p, t))
                    if rf is None:
                        continue
                    Y[rf] += pot[cq, dq] * _phase(b0, cq, dq) * X[row]
    return Y[:, 0] if one else Y
