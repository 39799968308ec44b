"""Reduced one-body transition densities of Lanczos eigenstates.

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
