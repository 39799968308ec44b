"""Reorderings of built tables that leave the Hamiltonian unchanged up to a
basis permutation, for the order-invariance tests.

A Fortran host hands over tables in its own orders: the jumps inside a
sector jump (the builder's order there is its own), the hmatpp / hmatnn
labels and the pairs inside an (M, parity) section.  The engine consumes any
valid table, so each of these orders may be changed freely:

* jumps: every sector jump's jump range (the ranges the opbundles point at)
  is permuted, all of its arrays together;
* labels: the hmatpp / hmatnn entries are relabeled by a permutation and the
  jump labels follow; the pn pairs of every (M, parity) section are put in a
  new order, which moves cpnpair / dpnpair and the square of hmatpn entries
  (src/btbmepn.f90:126-131, :417-487).
"""
import copy

import numpy as np

from bigstickpublick_b200 import model


def _clone(T):
    a3 = {k: v.copy() for k, v in T.a3.items()} if T.a3 is not None else None
    return model.Tables({k: v.copy() for k, v in T.a.items()}, dict(T.s), copy.copy(T.extra), a3,
                        dict(T.s3) if T.s3 is not None else None)


def permute_jumps(T, rng):
    """A random order inside every jump range of the opbundles."""
    T2 = _clone(T)
    a = T2.a
    fam = {  # jump family -> arrays, and the bundle ranges that index it
        "p1b": (["p1b_isd", "p1b_fsd", "p1b_cop", "p1b_dop", "p1b_phase"], 4, "px"),
        "n1b": (["n1b_isd", "n1b_fsd", "n1b_cop", "n1b_dop", "n1b_phase"], 4, "nx"),
        "p2b": (["p2b_isd", "p2b_fsd", "p2b_op", "p2b_phase"], 2, "px"),
        "n2b": (["n2b_isd", "n2b_fsd", "n2b_op", "n2b_phase"], 3, "nx"),
    }
    for name, (keys, optype, side) in fam.items():
        sel = a["optype"] == optype
        ranges = sorted({(int(s), int(e)) for s, e in zip(a[side + "start"][sel], a[side + "end"][sel])})
        for (s0, e0), (s1, e1) in zip(ranges, ranges[1:]):
            assert s1 > e0, f"{name}: overlapping jump ranges"
        n = len(a[keys[0]])
        perm = np.arange(n)
        for s, e in ranges:
            perm[s - 1:e] = s - 1 + rng.permutation(e - s + 1)
        for k in keys:
            a[k] = a[k][perm].copy()
    return T2


def _pn_sections(T):
    """pn pair sections from cpnpair / dpnpair: for each (M, parity) section
    the s.p. pairs (b, a) (cpnpair/dpnpair column-major indices) in their
    section position order, the section size n and its label offset.  The
    shells used here have one parity, so M alone labels a section."""
    ex = T.extra
    s = T.s
    nl, nr, pl, pr = s["nhsps_nl"], s["nhsps_nr"], s["nhsps_pl"], s["nhsps_pr"]
    ld = nl + nr + 1
    m2p, m2n = ex["sp_m2_p"], ex["sp_m2_n"]
    secs = {}
    for qp in range(pl + pr):
        a = -(qp + 1) if qp < pl else qp - pl + 1
        for qn in range(nl + nr):
            b = -(qn + 1) if qn < nl else qn - nl + 1
            idx = (b + nl) + (a + pl) * ld
            secs.setdefault(m2p[qp] + m2n[qn], []).append(idx)
    out = []
    cpn, dpn = T.a["cpnpair"], T.a["dpnpair"]
    for M, idxs in secs.items():
        n = len(idxs)
        pos = [int(cpn[i]) // n + 1 for i in idxs]
        order = [i for _, i in sorted(zip(pos, idxs))]
        nme = int(dpn[order[0]]) - 1
        out.append((order, n, nme))
    return out


def permute_labels(T, rng):
    """New hmatpp / hmatnn labels, and a new pair order in every pn section."""
    T2 = _clone(T)
    a = T2.a
    for kind, opk in (("pp", "p2b_op"), ("nn", "n2b_op")):
        h = a["hmat" + kind]
        perm = rng.permutation(len(h))            # old label l -> new label perm[l]
        newh = np.empty_like(h)
        newh[perm] = h
        a["hmat" + kind] = newh
        if len(a[opk]):
            a[opk] = (perm[a[opk] - 1] + 1).astype(a[opk].dtype)
    if T.s["np1b"] and T.s["nn1b"]:
        cpn, dpn, h = a["cpnpair"].copy(), a["dpnpair"].copy(), a["hmatpn"]
        newh = h.copy()
        for order, n, nme in _pn_sections(T):
            sig = rng.permutation(n)              # position p (0-based) -> sig[p]
            for p, idx in enumerate(order):
                cpn[idx] = sig[p] * n
                dpn[idx] = sig[p] + 1 + nme
            for c in range(n):
                for d in range(n):
                    newh[nme + sig[c] * n + sig[d]] = h[nme + c * n + d]
        a["cpnpair"], a["dpnpair"], a["hmatpn"] = cpn, dpn, newh
    return T2


def permute_jumps3(T, rng):
    """A random order inside every jump range of a three-body run's bundles:
    p3b (PPP), n3b (NNN), the pair-labelled p2b (PPN) and n2b (PNN), and the
    one-body jumps they pair with (n1b of PPN, p1b of PNN)."""
    T2 = _clone(T)
    a, a3 = T2.a, T2.a3
    fam = {  # jump family -> (arrays in a, arrays in a3), optype, side of the bundle range
        "p3b": ([], ["p3b_isd", "p3b_fsd", "p3b_op", "p3b_phase"], 7, "px"),
        "n3b": ([], ["n3b_isd", "n3b_fsd", "n3b_op", "n3b_phase"], 8, "nx"),
        "p2b": (["p2b_isd", "p2b_fsd", "p2b_phase"], ["p2b_cop", "p2b_dop"], 9, "px"),
        "n1b": (["n1b_isd", "n1b_fsd", "n1b_cop", "n1b_dop", "n1b_phase"], [], 9, "nx"),
        "p1b": (["p1b_isd", "p1b_fsd", "p1b_cop", "p1b_dop", "p1b_phase"], [], 10, "px"),
        "n2b": (["n2b_isd", "n2b_fsd", "n2b_phase"], ["n2b_cop", "n2b_dop"], 10, "nx"),
    }
    for name, (ka, k3, optype, side) in fam.items():
        sel = a["optype"] == optype
        ranges = sorted({(int(s), int(e)) for s, e in zip(a[side + "start"][sel], a[side + "end"][sel])})
        for (s0, e0), (s1, e1) in zip(ranges, ranges[1:]):
            assert s1 > e0, f"{name}: overlapping jump ranges"
        keys = [(a, k) for k in ka] + [(a3, k) for k in k3]
        n = len(keys[0][0][keys[0][1]])
        perm = np.arange(n)
        for s, e in ranges:
            perm[s - 1:e] = s - 1 + rng.permutation(e - s + 1)
        for d, k in keys:
            d[k] = d[k][perm].copy()
    return T2
