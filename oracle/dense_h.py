"""ORACLE -- test infrastructure only (never imported by the product).

Independent dense M-scheme Hamiltonian from second quantization, for small
spaces.  It shares no code with the table builder: its own m-state order
(orbit order, m ascending), its own Slater-determinant enumeration and phases,
its own Clebsch-Gordan coefficients in exact rational arithmetic, and the
single-particle energies applied as a one-body operator (the reference folds
them into the two-body part with 1/(A-1), src/bsppot.f90:39-238; for a fixed
particle number the two are the same operator).

Physics conventions it encodes (the reference's isospin formalism,
src/binput_tbme.f90:36-56 and :1490-1540):
  V_pp(ij,kl) = sum_J z_ab z_cd <ja mi jb mj|JM><jc mk jd ml|JM> V_{J,T=1}(ab,cd)
  V_pn(ij,kl) = sum_J (z_ab z_cd / 2) <..|JM><..|JM> (V_{J,0} + V_{J,1})(ab,cd)
with z_ab = sqrt(1 + delta_ab) and the exchange phase
  V_JT(ba,cd) = (-1)^(ja+jb+J+T) V_JT(ab,cd).
"""
import itertools
import math
from fractions import Fraction

import numpy as np


def _fact(n):
    return math.factorial(n)


def cg(j1, m1, j2, m2, J, M):
    """<j1 m1 j2 m2 | J M>, all arguments doubled, exact then float."""
    if m1 + m2 != M or abs(m1) > j1 or abs(m2) > j2 or abs(M) > J:
        return 0.0
    if J > j1 + j2 or J < abs(j1 - j2) or (j1 + j2 + J) % 2:
        return 0.0
    a, b, c = (j1 + j2 - J) // 2, (j1 - j2 + J) // 2, (-j1 + j2 + J) // 2
    d = (j1 + j2 + J) // 2 + 1
    pre = Fraction((J + 1) * _fact(a) * _fact(b) * _fact(c), _fact(d))
    pre *= Fraction(_fact((j1 + m1) // 2) * _fact((j1 - m1) // 2) * _fact((j2 + m2) // 2) *
                    _fact((j2 - m2) // 2) * _fact((J + M) // 2) * _fact((J - M) // 2))
    s = Fraction(0)
    k = 0
    while True:
        t = [k, a - k, (j1 - m1) // 2 - k, (j2 + m2) // 2 - k,
             (J - j2 + m1) // 2 + k, (J - j1 - m2) // 2 + k]
        if t[1] < 0 or t[2] < 0 or t[3] < 0:
            break
        if t[4] >= 0 and t[5] >= 0:
            den = 1
            for x in t:
                den *= _fact(x)
            s += Fraction((-1) ** k, den)
        k += 1
    return float(s) * math.sqrt(float(pre))


class CoupledV:
    def __init__(self, orbits, tbme):
        self.j2 = [o[2] for o in orbits]
        self.v = {}
        for (a, b, c, d, J, T, val) in tbme:
            for key, sg in self._images(a - 1, b - 1, c - 1, d - 1, J, T):
                self.v.setdefault(key, sg * val)

    def _images(self, a, b, c, d, J, T):
        sab = (-1) ** ((self.j2[a] + self.j2[b]) // 2 + J + T)
        scd = (-1) ** ((self.j2[c] + self.j2[d]) // 2 + J + T)
        out = []
        for (p, q, sp) in ((a, b, 1), (b, a, sab)):
            for (r, s, sr) in ((c, d, 1), (d, c, scd)):
                out.append(((p, q, r, s, J, T), sp * sr))
                out.append(((r, s, p, q, J, T), sp * sr))
        return out

    def get(self, a, b, c, d, J, T):
        if a == b and (J + T) % 2 == 0:
            return 0.0
        if c == d and (J + T) % 2 == 0:
            return 0.0
        return self.v.get((a, b, c, d, J, T), 0.0)


def dense_h(orbits, np_, nn, jz2, spe, tbme, spe_scale=1.0, tbme_scale=1.0, maxdim=6000):
    """Dense H (float64) and the basis list [(proton bits, neutron bits)]."""
    states = [(o, m) for o, orb in enumerate(orbits) for m in range(-orb[2], orb[2] + 1, 2)]
    ns = len(states)
    V = CoupledV(orbits, tbme)
    j2 = [o[2] for o in orbits]
    spe = [spe_scale * e for e in spe]

    def sds(n):
        out = []
        for occ in itertools.combinations(range(ns), n):
            out.append((sum(1 << q for q in occ), sum(states[q][1] for q in occ)))
        return out

    psd, nsd = sds(np_), sds(nn)
    basis = [(pb, nb_) for (pb, pm) in psd for (nb_, nm) in nsd if pm + nm == jz2]
    dim = len(basis)
    if dim > maxdim:
        raise ValueError(f"dense oracle limited to dim <= {maxdim} (got {dim})")
    index = {b: i for i, b in enumerate(basis)}

    def zeta(a, b):
        return math.sqrt(2.0) if a == b else 1.0

    def vpp(i, j, k, l):
        (a, mi), (b, mj), (c, mk), (d, ml) = states[i], states[j], states[k], states[l]
        if mi + mj != mk + ml:
            return 0.0
        s = 0.0
        for J in range(0, 12):
            c1 = cg(j2[a], mi, j2[b], mj, 2 * J, mi + mj)
            if c1 == 0.0:
                continue
            c2 = cg(j2[c], mk, j2[d], ml, 2 * J, mk + ml)
            if c2 == 0.0:
                continue
            s += zeta(a, b) * zeta(c, d) * c1 * c2 * V.get(a, b, c, d, J, 1)
        return s * tbme_scale

    def vpn(i, j, k, l):
        (a, mi), (b, mj), (c, mk), (d, ml) = states[i], states[j], states[k], states[l]
        if mi + mj != mk + ml:
            return 0.0
        s = 0.0
        for J in range(0, 12):
            c1 = cg(j2[a], mi, j2[b], mj, 2 * J, mi + mj)
            if c1 == 0.0:
                continue
            c2 = cg(j2[c], mk, j2[d], ml, 2 * J, mk + ml)
            if c2 == 0.0:
                continue
            s += 0.5 * zeta(a, b) * zeta(c, d) * c1 * c2 * (V.get(a, b, c, d, J, 0) + V.get(a, b, c, d, J, 1))
        return s * tbme_scale

    def sign_below(bits, q):
        return -1 if bin(bits & ((1 << q) - 1)).count("1") % 2 else 1

    def ann(bits, q):
        if not bits >> q & 1:
            return None, 0
        return bits & ~(1 << q), sign_below(bits, q)

    def cre(bits, q):
        if bits >> q & 1:
            return None, 0
        return bits | (1 << q), sign_below(bits, q)

    pair_list = [(i, j) for i in range(ns) for j in range(i + 1, ns)]
    vxx = {}
    for (i, j) in pair_list:
        for (k, l) in pair_list:
            v = vpp(i, j, k, l)
            if v != 0.0:
                vxx[(i, j, k, l)] = v
    vxn = {}
    for i in range(ns):
        for j in range(ns):
            for k in range(ns):
                for l in range(ns):
                    v = vpn(i, j, k, l)
                    if v != 0.0:
                        vxn[(i, j, k, l)] = v

    def apply2(bits, i, j, k, l):
        # a+_i a+_j a_l a_k
        b1, s1 = ann(bits, k)
        if b1 is None:
            return None, 0
        b2, s2 = ann(b1, l)
        if b2 is None:
            return None, 0
        b3, s3 = cre(b2, j)
        if b3 is None:
            return None, 0
        b4, s4 = cre(b3, i)
        if b4 is None:
            return None, 0
        return b4, s1 * s2 * s3 * s4

    def apply1(bits, i, k):
        b1, s1 = ann(bits, k)
        if b1 is None:
            return None, 0
        b2, s2 = cre(b1, i)
        if b2 is None:
            return None, 0
        return b2, s1 * s2

    H = np.zeros((dim, dim))
    for col, (pb, nb_) in enumerate(basis):
        # one-body SPE
        e = sum(spe[states[q][0]] for q in range(ns) if pb >> q & 1)
        e += sum(spe[states[q][0]] for q in range(ns) if nb_ >> q & 1)
        H[col, col] += e
        # pp and nn
        for (i, j, k, l), v in vxx.items():
            fb, s = apply2(pb, i, j, k, l)
            if fb is not None:
                H[index[(fb, nb_)], col] += s * v
            fb, s = apply2(nb_, i, j, k, l)
            if fb is not None:
                H[index[(pb, fb)], col] += s * v
        # pn: a+_i(p) a+_j(n) a_l(n) a_k(p) = (a+_i a_k)_p (a+_j a_l)_n
        for (i, j, k, l), v in vxn.items():
            fp, sp = apply1(pb, i, k)
            if fp is None:
                continue
            fn, sn = apply1(nb_, j, l)
            if fn is None:
                continue
            H[index[(fp, fn)], col] += sp * sn * v
    return H, basis


def coupled_two_body_spectrum(orbits, spe, tbme, T, tbme_scale=1.0, spe_scale=1.0):
    """Eigenvalues of the J-T coupled two-particle problem (all J, given T),
    each with multiplicity (2J+1): the spectrum a 2-particle M-scheme
    calculation must reproduce, summed over M."""
    V = CoupledV(orbits, tbme)
    norb = len(orbits)
    evals = []
    for J in range(0, 12):
        pairs = [(a, b) for a in range(norb) for b in range(a, norb)
                 if abs(orbits[a][2] - orbits[b][2]) // 2 <= J <= (orbits[a][2] + orbits[b][2]) // 2
                 and not (a == b and (J + T) % 2 == 0)]
        if not pairs:
            continue
        n = len(pairs)
        M = np.zeros((n, n))
        for x, (a, b) in enumerate(pairs):
            for y, (c, d) in enumerate(pairs):
                M[x, y] = tbme_scale * V.get(a, b, c, d, J, T)
            M[x, x] += spe_scale * (spe[a] + spe[b])
        for e in np.linalg.eigvalsh(M):
            evals.append((float(e), J))
    return evals
