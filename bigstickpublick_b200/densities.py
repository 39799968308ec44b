"""One-body observables of Lanczos eigenstates: reduced transition densities,
one-body operators read from .opme files, and strength functions.

The m-scheme densities <f| a+_c a_d |i> come from the engine
(``Hamiltonian.density1b``, C ABI ``bsg_density1b``); this module couples them
to good Jt (and Tt for isospin interactions) the way the reference's
``coupled_densities`` does (src/bdensities.f90:69-181), with the density
definition it prints (src/bdenslib1.f90:618-631):

    rho_K(a+ b) = (Jf || (a+ b)_K || Ji) / sqrt(2K + 1)

Edmonds' reduced matrix element, divided by sqrt(2T + 1) as well when isospin
is good; the time-reversal relation rho_K(a+b, i->f) =
(-1)^(ja-jb+Ji-Jf [+Ti-Tf]) rho_K(b+a, f->i) holds for the results.
``density1b`` mirrors ``density1b_compute`` (src/bdenslib1.f90:83-443): J and
T of each state rounded by closest2J, Jt from |Jf-Ji| to Jf+Ji, blocks whose
Clebsch-Gordan coefficient (Ji Jz, Jt 0 | Jf Jz) vanishes flagged zero.
Angular momenta are passed doubled (2j, 2m) throughout, as the reference's
``cleb`` takes them.
"""
from math import factorial, sqrt

import numpy as np

CG_TOL = 5.0e-5     # cgtol of coupled_densities
DEN_TOL = 1.0e-6    # dentol of density1b_writeout: smaller entries are not printed


def cleb(j1, m1, j2, m2, j, m):
    """Clebsch-Gordan coefficient (j1/2 m1/2, j2/2 m2/2 | j/2 m/2), doubled
    arguments, by Racah's closed formula."""
    if m1 + m2 != m or abs(m1) > j1 or abs(m2) > j2 or abs(m) > j:
        return 0.0
    if (j1 + m1) % 2 or (j2 + m2) % 2 or (j + m) % 2 or (j1 + j2 + j) % 2:
        return 0.0
    if j > j1 + j2 or j < abs(j1 - j2):
        return 0.0
    a = (j1 + j2 - j) // 2
    b = (j1 - j2 + j) // 2
    c = (-j1 + j2 + j) // 2
    pre = (j + 1) * factorial(a) * factorial(b) * factorial(c) / factorial((j1 + j2 + j) // 2 + 1)
    pre *= (factorial((j1 + m1) // 2) * factorial((j1 - m1) // 2) * factorial((j2 + m2) // 2)
            * factorial((j2 - m2) // 2) * factorial((j + m) // 2) * factorial((j - m) // 2))
    s = 0.0
    for k in range(0, a + 1):
        d = [a - k, (j1 - m1) // 2 - k, (j2 + m2) // 2 - k, (j - j2 + m1) // 2 + k, (j - j1 - m2) // 2 + k]
        if min(d) < 0:
            continue
        den = factorial(k)
        for x in d:
            den *= factorial(x)
        s += (-1.0 if k % 2 else 1.0) / den
    return sqrt(pre) * s


def closest2j(even, x):
    """2J nearest to x among even (even=True) or odd values (closest2J)."""
    if even:
        return 2 * int(round(x))
    return 2 * int(round(x - 0.5)) + 1


def coupled_densities(orbit_j2, sp_p, sp_n, mp, mn, Jt, Ji, Ti, Jf, Tf, jz2, tz2, npart=(1, 1), isospin=True):
    """One (initial, final, Jt) block of reduced densities.

    orbit_j2: 2j per orbit; sp_p, sp_n: (orbit, 2m) per combined s.p. index;
    mp, mn: <f| a+_c a_d |i> per species; Ji, Ti, Jf, Tf, jz2, tz2 doubled
    (tz2 = Z - N valence).  Returns (zeroflag, den[norb, norb, 2]) with
    den[..., 0:2] the Tt = 0, 1 densities (isospin) or proton, neutron ones."""
    norb = len(orbit_j2)
    den = np.zeros((norb, norb, 2))
    cg = cleb(Ji, jz2, 2 * Jt, 0, Jf, jz2) * sqrt(2 * Jt + 1) / sqrt(Jf + 1)
    if abs(cg) < CG_TOL:
        return True, den
    cgt = [cleb(Ti, tz2, 2 * tt, 0, Tf, tz2) * sqrt((2 * tt + 1) / (Tf + 1)) for tt in (0, 1)]
    for it, (sp, m, tsign) in enumerate(((sp_p, mp, 1), (sp_n, mn, -1))):
        if npart[it] == 0:
            continue
        for qa, (a, ma) in enumerate(sp):
            ja = orbit_j2[a]
            for qb, (b, mb) in enumerate(sp):
                jb = orbit_j2[b]
                if ma != mb or 2 * Jt > ja + jb or 2 * Jt < abs(ja - jb):
                    continue
                x = m[qa, qb]
                if x == 0.0:
                    continue
                w = cleb(ja, ma, jb, -mb, 2 * Jt, 0) * (-1.0 if ((jb - mb) // 2) % 2 else 1.0)
                if isospin:
                    for tt in (0, 1):
                        if abs(cgt[tt]) < CG_TOL:
                            continue
                        den[a, b, tt] += w * tsign * x * cleb(1, tsign, 1, -tsign, 2 * tt, 0) / cgt[tt]
                else:
                    den[a, b, it] += w * x
    return False, den / cg


def tiled_pairs(k, call, block=16):
    """All k x k m-scheme density pairs from a routine that handles at most
    2*block states per call.  call(idx) returns {'p': D, 'n': D} for the
    states idx (D[f, i, c, d] over positions in idx); blocks of `block`
    states are taken two at a time, so every (f, i) pair is covered once."""
    if k <= 2 * block:
        return call(list(range(k)))
    nblk = (k + block - 1) // block
    out = None
    for bi in range(nblk):
        for bj in range(bi, nblk):
            idx = list(range(bi * block, min(k, (bi + 1) * block)))
            if bj != bi:
                idx += list(range(bj * block, min(k, (bj + 1) * block)))
            md = call(idx)
            if out is None:
                out = {sp: np.zeros((k, k) + md[sp].shape[2:]) for sp in md}
            for sp in md:
                ix = np.array(idx)
                out[sp][np.ix_(ix, ix)] = md[sp]
    return out


def reduced(tables, md, J, T=None, isospin=True):
    """Reduced densities of every (initial, final) pair from the m-scheme
    densities `md` ({'p': D_p, 'n': D_n}, D[f, i, c, d] as
    ``Hamiltonian.density1b`` returns them) of states with angular momentum J
    and isospin T.  Returns {(i, f): {Jt: den[norb, norb, 2]}}, 1-based state
    numbers, zero-flagged Jt left out, like density1b_compute."""
    spec = tables.extra["spec"]
    orbit_j2 = [o[2] for o in spec.orbits]
    ex = tables.extra
    sp_p = list(zip(ex["sp_orb_p"].tolist(), ex["sp_m2_p"].tolist()))
    sp_n = list(zip(ex["sp_orb_n"].tolist(), ex["sp_m2_n"].tolist()))
    odd = (spec.np_ + spec.nn) % 2 == 1
    J2 = [closest2j(not odd, x) for x in np.atleast_1d(J)]
    T2 = [closest2j(not odd, x) for x in np.atleast_1d(T)] if isospin else [0] * len(J2)
    tz2 = spec.np_ - spec.nn
    out = {}
    k = md["p"].shape[0]
    for i in range(k):
        for f in range(k):
            blocks = {}
            for Jt in range(abs(J2[f] - J2[i]) // 2, (J2[f] + J2[i]) // 2 + 1):
                zero, den = coupled_densities(orbit_j2, sp_p, sp_n, md["p"][f, i], md["n"][f, i], Jt, J2[i], T2[i],
                                              J2[f], T2[f], spec.jz2, tz2, (spec.np_, spec.nn), isospin)
                if not zero:
                    blocks[Jt] = den
            out[(i + 1, f + 1)] = blocks
    return out


def density1b(H, vecs, J, T=None, isospin=True):
    """Reduced one-body densities of every (initial, final) pair of the states
    `vecs` (dim x k) of the engine ``Hamiltonian`` H (tables from
    ``model.build_tables``); J, T e.g. from ``engine.angular_momentum_isospin``.
    The m-scheme densities come from the GPU (bsg_density1b)."""
    return reduced(H.tables, H.density1b(vecs), J, T, isospin)


# ---------------------------------------------------------------- operators
class OneBodyOperator:
    """A one-body operator as an .opme file gives it (readin1bodyop,
    src/bdenslib1.f90:1823-2071): reduced matrix elements <a||O||b> between
    orbits, of angular momentum `jop` and isospin `top` ('iso' files) or
    separate proton and neutron elements ('pns' / 'xpn' files)."""

    def __init__(self, kind, orbits, jop, top, iso=None, prot=None, neut=None):
        self.kind, self.orbits, self.jop, self.top = kind, orbits, jop, top
        self.iso = iso or {}
        self.prot = prot or {}
        self.neut = neut or {}


def read_opme(text):
    """Parse the text of an .opme file: first line 'iso', 'pns' or 'xpn'; the
    number of orbits; one line per orbit (index, n, l, j; xpn also gives the
    neutron index); 'J T' (iso) or 'J' (pn); then 'a b value' lines (pns:
    'a b proton neutron'; xpn: neutron orbits offset by the orbit count,
    charge-changing elements skipped)."""
    lines = [ln.split("!")[0] for ln in text.splitlines()]
    lines = [ln for ln in lines if ln.strip()]
    kind = lines[0].strip()[:3]
    if kind not in ("iso", "pns", "xpn"):
        raise ValueError("first line of an .opme file must start with iso, pns or xpn")
    norb = int(lines[1].split()[0])
    orbits = []
    for ln in lines[2:2 + norb]:
        t = ln.split()
        if kind == "xpn":
            t = [t[0]] + t[2:]
        orbits.append((int(t[1]), int(t[2]), int(round(2 * float(t[3])))))   # n, l, 2j
    t = lines[2 + norb].split()
    jop = int(t[0])
    top = int(t[1]) if kind == "iso" else 2
    op = OneBodyOperator(kind, orbits, jop, top)
    for ln in lines[3 + norb:]:
        t = ln.split()
        a, b = int(t[0]), int(t[1])
        if kind == "iso":
            op.iso[(a, b)] = float(t[2])
        elif kind == "pns":
            op.prot[(a, b)] = float(t[2])
            op.neut[(a, b)] = float(t[3])
        else:
            if (a <= norb) != (b <= norb):
                continue
            if a <= norb:
                op.prot[(a, b)] = float(t[2])
            else:
                op.neut[(a - norb, b - norb)] = float(t[2])
    return op


def onebody_operator(tables, op):
    """The M = 0 m-scheme matrix elements of `op` on the combined s.p.
    indices of `tables`, as decouple1bodyop builds pPOT_h / nPOT_h
    (src/bdenslib1.f90:2444-2597):

        pPOT(a ma, b mb) = (-1)^(jb-mb) (ja ma, jb -mb | J 0) <a||O||b>
                           / sqrt(2J+1) [/ sqrt(2T+1) (1/2 1/2, 1/2 -1/2 | T 0)]

    with an extra -1 and (1/2 -1/2, 1/2 1/2 | T 0) for neutrons of an isospin
    operator.  Returns (ppot, npot), None for a species without particles."""
    spec = tables.extra["spec"]
    orbit_j2 = [o[2] for o in spec.orbits]
    for k, (n, l, j2) in enumerate(op.orbits):
        o = spec.orbits[k]
        if (n, l, j2) != (o[0], o[1], o[2]):
            raise ValueError(f"orbit {k + 1} of the operator ({n} {l} {j2}/2) does not match the model space")
    if len(op.orbits) != len(spec.orbits):
        raise ValueError("operator and model space have different orbit counts")
    J, T = op.jop, op.top
    out = []
    for it, (npart, sps) in enumerate(((spec.np_, "p"), (spec.nn, "n"))):
        ex = tables.extra
        sp = list(zip(ex["sp_orb_" + sps].tolist(), ex["sp_m2_" + sps].tolist()))
        if npart == 0:
            out.append(None)
            continue
        pot = np.zeros((len(sp), len(sp)))
        for qa, (a, ma) in enumerate(sp):
            ja = orbit_j2[a]
            for qb, (b, mb) in enumerate(sp):
                jb = orbit_j2[b]
                if op.kind == "iso":
                    x = op.iso.get((a + 1, b + 1), 0.0)
                else:
                    x = (op.prot if it == 0 else op.neut).get((a + 1, b + 1), 0.0)
                if x == 0.0 or ma != mb or 2 * J > ja + jb or 2 * J < abs(ja - jb):
                    continue
                ph = -1.0 if ((jb - mb) // 2) % 2 else 1.0
                w = ph * cleb(ja, ma, jb, -mb, 2 * J, ma - mb) * x / sqrt(2 * J + 1)
                if op.kind == "iso":
                    tz = 1 if it == 0 else -1
                    w *= cleb(1, tz, 1, -tz, 2 * T, 0) / sqrt(2 * T + 1)
                    if it == 1:
                        w = -w
                pot[qa, qb] = w
        out.append(pot)
    return out[0], out[1]


def strength_function(H, pivot, niter=30):
    """Strength distribution of the (unnormalized) pivot O|psi>, as the
    reference's strength option prints it (src/blanczoslib.f90:1109-1142):
    `niter` Lanczos iterations from the normalized pivot, full
    reorthogonalization, and for every Ritz pair (E_k, y_k) the strength
    y_k(1)^2 |pivot|^2.  Returns (energies, strengths, total = |pivot|^2).
    Ritz vectors come back in the full basis; y_k(1) is their overlap with the
    normalized pivot."""
    p = np.asarray(pivot, dtype=np.float64)
    total = float(p @ p)
    ph = p / np.sqrt(total)
    k = min(niter, H.dim)
    ev, vecs, rep = H.lanczos(nkeep=k, niter=niter, matvec_prec=8, fixed_iter=True, want_vectors=True, pivot=ph)
    s = (vecs.T @ ph) ** 2 * total
    return ev, s, total
