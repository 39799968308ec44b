"""ORACLE -- test infrastructure only.

Pure-Python restatements of the reference routines that fix three orders in
the tables: the order of haikus inside a block, the order of like-particle
pairs and the order of proton-neutron pairs.  They follow the reference's
loops step by step (no closed forms), so that the table builder's own
formulation of the same orders can be checked against them.

* create_haikus: count_create_haikus (src/bbasis_haikus.f90:327-411) for
  one W section and one template per particle number, the case of every
  untruncated space: the haikus of nh particles come from those of nh-1 in
  their order, with p from the section's last state down to the first, a new
  haiku for every free p until the first occupied one.
* block_haikus: fill_blocks (src/bbasis_blocks.f90:474-562), the haikus of one
  (nh, parity, Jz) in creation order.
* sortpair: the two heap sorts of src/btbme.f90:548-703, on M (leaving M
  descending) and then on parity inside every run of equal M.
* xx_pairs / pn_pairs: count_create_pairs (src/btbme.f90:208-308) and
  count_create_pnpairs (:324-423) followed by sortpair.
* sections: find_pair_start (src/btbme.f90:726-785) and the section loop of
  count_uncouplepn (src/btbmepn.f90:177-587): first pair (1-based) and first
  matrix element of every (M, parity) section.
"""


def create_haikus(nsps, nhmax):
    """haikus[nh] = occupation masks (bit p-1 for state p) in creation order."""
    haikus = [[0]]
    for nh in range(1, nhmax + 1):
        out = []
        for parent in haikus[nh - 1]:
            for p in range(nsps, 0, -1):
                if parent >> (p - 1) & 1:
                    break
                out.append(parent | (1 << (p - 1)))
        haikus.append(out)
    return haikus


def block_haikus(haikus_nh, m2, par, jz2, pidx):
    """The haikus of one block: parity index pidx (1: +, 2: -), 2Jz = jz2.
    m2, par: 2m and parity (+1/-1) of the section's states, state p at p-1."""
    out = []
    for h in haikus_nh:
        j, pp = 0, 1
        for q in range(len(m2)):
            if h >> q & 1:
                j += m2[q]
                pp *= par[q]
        if j == jz2 and (1 if pp > 0 else 2) == pidx:
            out.append(h)
    return out


def _heap(a, s, e, key, flip):
    """One heap sort pass of sortpair over a[s..e] (1-based, inclusive).
    flip=True is the M pass (child test and sift test with '>'), flip=False
    the parity pass (with '<')."""
    def below(x, y):
        return key(x) > key(y) if flip else key(x) < key(y)

    l = (e - s + 1) // 2 + s
    n = e
    while n >= s:
        if l > s:
            l -= 1
            tmp = a[l - 1]
        else:
            tmp = a[n - 1]
            a[n - 1] = a[s - 1]
            n -= 1
            if n == s:
                a[s - 1] = tmp
                break
        i = l
        j = l + l - (s - 1)
        while j <= n:
            if j < n and below(a[j - 1], a[j]):
                j += 1
            if below(tmp, a[j - 1]):
                a[i - 1] = a[j - 1]
                i = j
                j = j + j - (s - 1)
            else:
                j = n + 1
        a[i - 1] = tmp


def sortpair(pairs):
    """pairs: list of dicts with 'm' and 'par' (1: +, 2: -); sorted in place."""
    n = len(pairs)
    if n == 0:
        return pairs
    _heap(pairs, 1, n, lambda x: x["m"], True)
    istart, istop = 1, 1
    while istart <= n:
        m = pairs[istart - 1]["m"]
        if istart == n:
            istop = istart
        else:
            while pairs[istop]["m"] == m:
                istop += 1
                if istop == n:
                    break
        _heap(pairs, istart, istop, lambda x: x["par"], False)
        istart = istop + 1
        istop = istart
    return pairs


def xx_pairs(m2, par):
    """Like-particle pairs over the combined states (left then right, 0-based
    q): [{'q1','q2','m','par'}] in the reference's order."""
    ns = len(m2)
    out = []
    for a in range(2, ns + 1):          # asps
        for b in range(1, a):           # bsps
            out.append({"q1": b - 1, "q2": a - 1, "m": (m2[a - 1] + m2[b - 1]) // 2,
                        "par": (3 - par[a - 1] * par[b - 1]) // 2})
    return sortpair(out)


def pn_pairs(m2p, parp, m2n, parn):
    out = []
    for a in range(len(m2p)):
        for b in range(len(m2n)):
            out.append({"qp": a, "qn": b, "m": (m2p[a] + m2n[b]) // 2, "par": (3 - parp[a] * parn[b]) // 2})
    return sortpair(out)


def sections(pairs, square):
    """[(first pair 1-based, n pairs, first matrix element - 1)] per section."""
    secs = []
    for i, p in enumerate(pairs):
        if i == 0 or p["m"] != pairs[i - 1]["m"] or p["par"] != pairs[i - 1]["par"]:
            secs.append([i + 1, 0])
        secs[-1][1] += 1
    out, nme = [], 0
    for first, n in secs:
        out.append((first, n, nme))
        nme += n * n if square else n * (n + 1) // 2
    return out
