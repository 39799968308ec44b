"""Model spaces, interaction files and the host-side table build.

This is the Python face of libbsghost.so (the CPU stand-in for the Fortran
host's setup).  It reads the reference's isospin-format inputs:

* ``.sps`` orbit files (``iso``, number of orbits, then ``n l j w`` lines;
  src/binput.f90), and
* ``.int`` interaction files (first line ``nme spe_1 .. spe_norb [...]``, then
  ``a b c d J T V`` lines; reader src/binput_tbme.f90:898-1240, values read as
  real(4) at :936), with the scaling line ``xspe A0 A x`` giving
  TBME scale (A0/A)**x (src/binput_tbme.f90:1025-1032).

It also generates the seeded synthetic interactions used as stand-ins for
real ones: every canonical J-T coupled matrix element drawn N(0, 1 MeV) from a
SplitMix64 stream through Box-Muller.
"""
import ctypes as C
import os
import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi

# orbit lists (n, l, 2j, w) in the order of the reference's example files:
# sd.sps (examples/sd/sd.sps: d3/2, d5/2, s1/2) and fp0.sps
# (util/examples/fp0.sps: f7/2, p3/2, f5/2, p1/2)
SD_ORBITS = [(0, 2, 3, 2), (0, 2, 5, 2), (1, 0, 1, 2)]
PF_ORBITS = [(1, 3, 7, 3), (2, 1, 3, 3), (1, 3, 5, 3), (2, 1, 1, 3)]
# SPEs of the synthetic sd interaction, in sd.sps order (d3/2, d5/2, s1/2)
SD_SYNTH_SPE = [2.1, -3.9, -3.2]


def read_sps(path):
    """Parse an isospin .sps file -> list of (n, l, 2j, w)."""
    toks = open(path).read().split()
    if not toks or toks[0].lower() != "iso":
        raise ValueError(f"{path}: only isospin-format .sps files are supported")
    norb = int(float(toks[1]))
    orbs = []
    for i in range(norb):
        n, l, j, w = (float(x) for x in toks[2 + 4 * i: 6 + 4 * i])
        orbs.append((int(n), int(l), int(round(2 * j)), int(w)))
    return orbs


def read_int(path, norb):
    """Parse an isospin .int file -> (spe[norb], [(a,b,c,d,J,T,V)]).

    Comment lines start with '!' or '#'.  Values are rounded to float32 as the
    reference reads them into real(4) variables."""
    lines = []
    for raw in open(path):
        s = raw.strip()
        if not s or s[0] in "!#":
            continue
        lines.append(s)
    head = lines[0].split()
    nme = int(float(head[0]))
    spe = [float(np.float32(float(x))) for x in head[1:1 + norb]]
    tb = []
    for s in lines[1:1 + nme]:
        f = s.split()
        a, b, c, d, J, T = (int(x) for x in f[:6])
        tb.append((a, b, c, d, J, T, float(np.float32(float(f[6])))))
    return spe, tb


# ---------------------------------------------------------------- synthetic
class SplitMix64:
    """SplitMix64 stream with Box-Muller normals (fp64)."""

    MASK = (1 << 64) - 1

    def __init__(self, seed):
        self.state = seed & self.MASK

    def next_u64(self):
        self.state = (self.state + 0x9E3779B97F4A7C15) & self.MASK
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & self.MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & self.MASK
        return z ^ (z >> 31)

    def uniform(self):
        """uniform in (0, 1]"""
        return ((self.next_u64() >> 11) + 1) * (1.0 / 9007199254740992.0)

    def normal(self):
        u1, u2 = self.uniform(), self.uniform()
        return math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)

    def randint(self, lo, hi):
        """uniform integer in [lo, hi]"""
        return lo + int(self.uniform() * (hi - lo + 1) - 1e-12)


def canonical_tbme_keys(orbits):
    """All independent J-T coupled matrix elements (a<=b, c<=d, (a,b)<=(c,d),
    parity conserved, J allowed by both pairs, J+T odd when a==b or c==d).
    63 for sd, 195 for pf."""
    norb = len(orbits)
    pairs = [(a, b) for a in range(1, norb + 1) for b in range(a, norb + 1)]
    keys = []
    for i, (a, b) in enumerate(pairs):
        for (c, d) in pairs[i:]:
            la, lb, lc, ld = (orbits[x - 1][1] for x in (a, b, c, d))
            if (la + lb + lc + ld) % 2:
                continue
            ja, jb, jc, jd = (orbits[x - 1][2] for x in (a, b, c, d))
            jmin = max(abs(ja - jb), abs(jc - jd)) // 2
            jmax = min(ja + jb, jc + jd) // 2
            for J in range(jmin, jmax + 1):
                for T in (0, 1):
                    if a == b and (J + T) % 2 == 0:
                        continue
                    if c == d and (J + T) % 2 == 0:
                        continue
                    keys.append((a, b, c, d, J, T))
    return keys


def synthetic_interaction(orbits, seed, spe=None):
    """Seeded random isospin interaction: V_JT ~ N(0,1) MeV for every
    canonical coupled matrix element, written/rounded through '%.8e' and
    float32 like a .int file; SPEs given, or drawn N(0,1) from the stream."""
    rng = SplitMix64(seed)
    if spe is None:
        spe = [rng.normal() for _ in orbits]
    tb = []
    for k in canonical_tbme_keys(orbits):
        v = float(np.float32(float("%.8e" % rng.normal())))
        tb.append(k + (v,))
    spe = [float(np.float32(float("%.8e" % s))) for s in spe]
    return spe, tb


def write_int(path, spe, tbme, comment="synthetic"):
    with open(path, "w") as f:
        f.write(f"! {comment}\n")
        f.write("%d " % len(tbme) + " ".join("%.8e" % s for s in spe) + "\n")
        for (a, b, c, d, J, T, v) in tbme:
            f.write("%3d %3d %3d %3d %3d %3d %.8e\n" % (a, b, c, d, J, T, v))


# -------------------------------------------------------------- the model
@dataclass
class ModelSpec:
    orbits: list
    np_: int
    nn: int
    jz2: int = 0
    parity: int = 1
    spe: list = field(default_factory=list)
    tbme: list = field(default_factory=list)
    spe_scale: float = 1.0
    tbme_scale: float = 1.0

    @staticmethod
    def scaling(xspe, a0, a, x):
        """(spe scale, tbme scale) from the reference's scaling line."""
        if a == 0 or x == 0:
            return float(np.float32(xspe)), float(np.float32(a0))
        return float(np.float32(xspe)), float(np.float32((a0 / a) ** x))


_TABLE_FIELDS = [
    ("pstart", "i8", "nsd_p"), ("nstart", "i8", "nsd_n"),
    ("p1b_isd", "i8", "np1b"), ("p1b_fsd", "i8", "np1b"), ("p1b_cop", "i2", "np1b"),
    ("p1b_dop", "i2", "np1b"), ("p1b_phase", "i1", "np1b"),
    ("n1b_isd", "i8", "nn1b"), ("n1b_fsd", "i8", "nn1b"), ("n1b_cop", "i2", "nn1b"),
    ("n1b_dop", "i2", "nn1b"), ("n1b_phase", "i1", "nn1b"),
    ("p2b_isd", "i8", "np2b"), ("p2b_fsd", "i8", "np2b"), ("p2b_op", "i4", "np2b"),
    ("p2b_phase", "i1", "np2b"),
    ("n2b_isd", "i8", "nn2b"), ("n2b_fsd", "i8", "nn2b"), ("n2b_op", "i4", "nn2b"),
    ("n2b_phase", "i1", "nn2b"),
    ("hmatpp", "f4", "nmatpp"), ("hmatnn", "f4", "nmatnn"), ("hmatpn", "f4", "nmatpn"),
    ("optype", "i4", "nbundles"), ("hchar", "i4", "nbundles"),
    ("pxstart", "i8", "nbundles"), ("pxend", "i8", "nbundles"), ("nxstart", "i8", "nbundles"),
    ("nxend", "i8", "nbundles"), ("cstride", "i8", "nbundles"),
]
# one-body density tables (bsg_density_tables): name, dtype, length field
_DENSITY_FIELDS = [
    ("p1b_isd", "i8", "np1b"), ("p1b_fsd", "i8", "np1b"), ("p1b_cop", "i2", "np1b"),
    ("p1b_dop", "i2", "np1b"), ("p1b_phase", "i1", "np1b"),
    ("n1b_isd", "i8", "nn1b"), ("n1b_fsd", "i8", "nn1b"), ("n1b_cop", "i2", "nn1b"),
    ("n1b_dop", "i2", "nn1b"), ("n1b_phase", "i1", "nn1b"),
    ("optype", "i4", "nbundles"), ("hchar", "i4", "nbundles"),
    ("pxstart", "i8", "nbundles"), ("pxend", "i8", "nbundles"), ("nxstart", "i8", "nbundles"),
    ("nxend", "i8", "nbundles"), ("cstride", "i8", "nbundles"),
]
# three-body arrays (bsg_tables3): name, dtype, length field (None: computed)
_TABLE3_FIELDS = [
    ("p2b_cop", "i4", "np2b"), ("p2b_dop", "i4", "np2b"), ("n2b_cop", "i4", "nn2b"), ("n2b_dop", "i4", "nn2b"),
    ("p3b_isd", "i8", "np3b"), ("p3b_fsd", "i8", "np3b"), ("p3b_op", "i4", "np3b"), ("p3b_phase", "i1", "np3b"),
    ("n3b_isd", "i8", "nn3b"), ("n3b_fsd", "i8", "nn3b"), ("n3b_op", "i4", "nn3b"), ("n3b_phase", "i1", "nn3b"),
    ("hmatppp", "f4", "nmatppp"), ("hmatnnn", "f4", "nmatnnn"), ("hmatppn", "f4", "nmatppn"),
    ("hmatpnn", "f4", "nmatpnn"),
    ("cppntriplet", "i4", None), ("dppntriplet", "i4", None), ("cpnntriplet", "i4", None),
    ("dpnntriplet", "i4", None),
]
_CTYPES = {"i1": C.c_int8, "i2": C.c_int16, "i4": C.c_int32, "i8": C.c_int64,
           "f4": C.c_float, "f8": C.c_double, "u8": C.c_uint64}


def _np_from(ptr, n, dt):
    if n == 0 or not ptr:
        return np.zeros(0, dtype=dt)
    arr = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(_CTYPES[dt])), shape=(int(n),))
    return arr.astype(dt, copy=True)


class Tables:
    """The reference's module arrays for one Hamiltonian, as numpy arrays.

    ``as_ctypes()`` returns a ``bsg_tables`` view whose pointers reference
    these arrays (kept alive by this object)."""

    def __init__(self, arrays, scalars, extra, arrays3=None, scalars3=None):
        self.a = arrays
        self.s = scalars
        self.extra = extra
        # three-body run (build_tables3): the bsg_tables3 arrays and sizes
        self.a3 = arrays3
        self.s3 = scalars3
        self._c = None
        self._c3 = None

    @property
    def threebody(self):
        return self.a3 is not None

    def as_ctypes3(self):
        """``bsg_tables3`` view of the three-body arrays (None for a
        two-body Hamiltonian)."""
        if self.a3 is None:
            return None
        t = _abi.BsgTables3()
        for k, v in self.s3.items():
            setattr(t, k, v)
        for name, dt, _ in _TABLE3_FIELDS:
            arr = self.a3.get(name)
            setattr(t, name, None if arr is None or arr.size == 0 else arr.ctypes.data_as(C.POINTER(_CTYPES[dt])))
        self._c3 = t
        return t

    @property
    def dim(self):
        return int(self.s["dimbasis"])

    def as_ctypes(self):
        t = _abi.BsgTables()
        for k, v in self.s.items():
            setattr(t, k, v)
        for name, dt, _ in _TABLE_FIELDS + [("cpnpair", "i8", None), ("dpnpair", "i8", None),
                                             ("pspe_h", "f4", None), ("nspe_h", "f4", None)]:
            arr = self.a.get(name)
            if arr is None or arr.size == 0:
                setattr(t, name, None)
            else:
                setattr(t, name, arr.ctypes.data_as(C.POINTER(_CTYPES[dt])))
        self._c = t
        return t

    def density_ctypes(self):
        """``bsg_density_tables`` view of the one-body density jumps and
        P1B/N1B bundles (pointers into ``extra['density']``)."""
        d = self.extra["density"]
        t = _abi.BsgDensityTables()
        for k in ("np1b", "nn1b", "nbundles"):
            setattr(t, k, int(d[k]))
        for name, dt, _ in _DENSITY_FIELDS:
            arr = d[name]
            setattr(t, name, arr.ctypes.data_as(C.POINTER(_CTYPES[dt])) if arr.size else None)
        self._dc = t
        return t


def build_tables3(spec: ModelSpec, w2=1.0, w3=0.0, seed=0) -> Tables:
    """Three-body tables (bsg_host_build3): SPE plus PPP / PPN / PNN / NNN
    bundles with W = w2 * V2 / (A - 2) + w3 * R, V2 the two-body
    interaction of `spec` between three-particle states and R the seeded
    symmetric part of the builder (uniform in [-1, 1)).  With w3 = 0 the
    Hamiltonian equals the two-body one of `spec`."""
    return build_tables(spec, three=(w2, w3, seed))


def build_tables(spec: ModelSpec, three=None) -> Tables:
    """Run the host-side table builder (libbsghost.so) and copy its arrays.
    three: (w2, w3, seed) for a three-body build (build_tables3)."""
    lib = _abi.host_lib()
    orbs = (_abi.BsgOrbit * len(spec.orbits))(*[_abi.BsgOrbit(*o) for o in spec.orbits])
    tb = (_abi.BsgTbme * max(1, len(spec.tbme)))()
    for i, (a, b, c, d, J, T, v) in enumerate(spec.tbme):
        tb[i] = _abi.BsgTbme(a, b, c, d, J, T, v)
    spe = (C.c_double * len(spec.orbits))(*(spec.spe or [0.0] * len(spec.orbits)))
    ms = _abi.BsgModelSpec(len(spec.orbits), orbs, spec.np_, spec.nn, spec.jz2, spec.parity,
                           len(spec.tbme), tb, spe, spec.spe_scale, spec.tbme_scale)
    hp = C.POINTER(_abi.BsgHostTables)()
    if three is None:
        st = lib.bsg_host_build(C.byref(ms), C.byref(hp))
    else:
        s3 = _abi.BsgModel3Spec(float(three[0]), float(three[1]), int(three[2]) & ((1 << 64) - 1))
        st = lib.bsg_host_build3(C.byref(ms), C.byref(s3), C.byref(hp))
    if st != 0:
        raise RuntimeError(f"bsg_host_build: {_abi.STATUS_NAMES.get(st, st)}: "
                           f"{lib.bsg_host_last_error().decode()}")
    try:
        h = hp.contents
        t = h.t
        scal = {k: getattr(t, k) for k in (
            "dimbasis", "nsd_p", "nsd_n", "np1b", "nn1b", "np2b", "nn2b", "nmatpp", "nmatnn",
            "nmatpn", "nhsps_pl", "nhsps_pr", "nhsps_nl", "nhsps_nr", "call_spe", "nbundles")}
        arrs = {}
        for name, dt, nfield in _TABLE_FIELDS:
            arrs[name] = _np_from(getattr(t, name), scal[nfield], dt)
        arrs3 = scal3 = None
        if three is not None:
            u = h.t3.contents
            scal3 = {k: getattr(u, k) for k in ("np3b", "nn3b", "nmatppp", "nmatnnn", "nmatppn", "nmatpnn",
                                                "npairs_p", "npairs_n")}
            lens = dict(scal3, np2b=t.np2b, nn2b=t.nn2b)
            ntp = u.npairs_p * (t.nhsps_nl + t.nhsps_nr + 1)
            ntn = u.npairs_n * (t.nhsps_pl + t.nhsps_pr + 1)
            arrs3 = {}
            for name, dt, nfield in _TABLE3_FIELDS:
                n = lens[nfield] if nfield else (ntp if "ppn" in name else ntn)
                arrs3[name] = _np_from(getattr(u, name), n, dt)
        ncp = (t.nhsps_nl + t.nhsps_nr + 1) * (t.nhsps_pl + t.nhsps_pr + 1)
        arrs["cpnpair"] = _np_from(t.cpnpair, ncp, "i8")
        arrs["dpnpair"] = _np_from(t.dpnpair, ncp, "i8")
        if t.call_spe:
            arrs["pspe_h"] = _np_from(t.pspe_h, t.nsd_p, "f4")
            arrs["nspe_h"] = _np_from(t.nspe_h, t.nsd_n, "f4")
        extra = {
            "psector_start": _np_from(h.psector_start, h.nsectors_p, "i8"),
            "psector_end": _np_from(h.psector_end, h.nsectors_p, "i8"),
            "psector_jz2": _np_from(h.psector_jz2, h.nsectors_p, "i4"),
            "psector_conj": _np_from(h.psector_conj, h.nsectors_p, "i4"),
            "nsector_start": _np_from(h.nsector_start, h.nsectors_n, "i8"),
            "nsector_end": _np_from(h.nsector_end, h.nsectors_n, "i8"),
            "nsector_jz2": _np_from(h.nsector_jz2, h.nsectors_n, "i4"),
            "sp_orb_p": _np_from(h.sp_orb_p, h.nhsps_p, "i4"),
            "sp_m2_p": _np_from(h.sp_m2_p, h.nhsps_p, "i4"),
            "sp_orb_n": _np_from(h.sp_orb_n, h.nhsps_n, "i4"),
            "sp_m2_n": _np_from(h.sp_m2_n, h.nhsps_n, "i4"),
            "sd_bits_p": _np_from(h.sd_bits_p, t.nsd_p, "u8"),
            "sd_bits_n": _np_from(h.sd_bits_n, t.nsd_n, "u8"),
        }
        d = h.dt
        dens = {"np1b": d.np1b, "nn1b": d.nn1b, "nbundles": d.nbundles}
        for name, dt, nfield in _DENSITY_FIELDS:
            dens[name] = _np_from(getattr(d, name), dens[nfield], dt)
        extra["density"] = dens
        jac = {}
        ntb = max(1, len(spec.tbme))
        for kind, nm in ((0, "pp"), (1, "nn"), (2, "pn")):
            n = int(scal["nmat" + nm])
            dt_ = np.zeros((n, ntb), dtype=np.float64)
            ds_ = np.zeros((n, len(spec.orbits)), dtype=np.float64)
            if n:
                st = lib.bsg_host_me_jacobian(hp, kind, dt_.ctypes.data_as(_abi.f64p),
                                              ds_.ctypes.data_as(_abi.f64p))
                if st != 0:
                    raise RuntimeError("bsg_host_me_jacobian failed")
            jac[nm] = (dt_, ds_)
        extra["jacobian"] = jac
        extra["spec"] = spec
    finally:
        lib.bsg_host_free(hp)
    return Tables(arrs, scal, extra, arrs3, scal3)


def build_tables_many(specs, threads=None):
    """build_tables for many specs on host threads (the builder runs outside
    the GIL); results in the order of `specs`."""
    from concurrent.futures import ThreadPoolExecutor
    specs = list(specs)
    n = threads or min(len(specs), os.cpu_count() or 1) or 1
    with ThreadPoolExecutor(max_workers=n) as ex:
        return list(ex.map(build_tables, specs))


# ------------------------------------------------------------ presets
def sd_model(np_, nn, seed=None, jz2=0, interaction=None, spe_scale=1.0, tbme_scale=1.0):
    """sd-shell model: seeded synthetic interaction (seed) or given (spe, tbme)."""
    if interaction is None:
        spe, tb = synthetic_interaction(SD_ORBITS, seed, spe=SD_SYNTH_SPE)
    else:
        spe, tb = interaction
    return ModelSpec(SD_ORBITS, np_, nn, jz2, 1, spe, tb, spe_scale, tbme_scale)


def pf_model(np_, nn, seed, jz2=0):
    spe, tb = synthetic_interaction(PF_ORBITS, seed)
    return ModelSpec(PF_ORBITS, np_, nn, jz2, 1, spe, tb, 1.0, 1.0)


def _pair_diagonal_keys(orbits):
    return [k for k in canonical_tbme_keys(orbits) if k[0] == k[2] and k[1] == k[3]]


def jsq_spec(spec: ModelSpec) -> ModelSpec:
    """J^2 of the many-body space of `spec` as a two-body operator, in the
    reference's own representation (a one-body part on the orbits plus
    coupled J-T matrix elements; lanczos_output evaluates <J^2> the same way,
    src/blanczoslib.f90:1023-1603):
      J^2 = sum_i j_i^2 + sum_{i<j} 2 j_i.j_j,
      one-body e_a = j_a(j_a+1),
      <ab;JT| 2 j_1.j_2 |ab;JT> = J(J+1) - j_a(j_a+1) - j_b(j_b+1)  (diagonal).
    Same orbits, particle numbers, 2Jz and parity, hence the same basis as H."""
    def jj(o):
        j = spec.orbits[o - 1][2] / 2.0
        return j * (j + 1.0)
    spe = [(o[2] / 2.0) * (o[2] / 2.0 + 1.0) for o in spec.orbits]
    tb = [(a, b, c, d, J, T, J * (J + 1.0) - jj(a) - jj(b)) for (a, b, c, d, J, T) in _pair_diagonal_keys(spec.orbits)]
    return ModelSpec(spec.orbits, spec.np_, spec.nn, spec.jz2, spec.parity, spe, tb, 1.0, 1.0)


def tsq_spec(spec: ModelSpec) -> ModelSpec:
    """T^2 like jsq_spec: one-body 3/4 per nucleon, pair elements
    T(T+1) - 3/2 for every coupled pair."""
    spe = [0.75] * len(spec.orbits)
    tb = [(a, b, c, d, J, T, T * (T + 1.0) - 1.5) for (a, b, c, d, J, T) in _pair_diagonal_keys(spec.orbits)]
    return ModelSpec(spec.orbits, spec.np_, spec.nn, spec.jz2, spec.parity, spe, tb, 1.0, 1.0)


def j_from_jsq(x):
    """J from <J^2> = J(J+1)."""
    return 0.5 * (np.sqrt(1.0 + 4.0 * np.maximum(np.asarray(x, dtype=np.float64), 0.0)) - 1.0)


def chain_rule(tables, dhmat):
    """Gradient of one eigenvalue with respect to the coupled interaction.

    dhmat: {'pp','nn','pn'} arrays dE/dhmat(label) (from Hamiltonian.grad, one
    state), plus 'spe_p'/'spe_n' (dE/dpspe_h, dE/dnspe_h) when the tables use
    SPE bundles.  Returns (dE/dV for every line of the interaction file in
    spec.tbme order, dE/de for every orbit's SPE) through the builder's
    uncoupling coefficients (src/btbme.f90:1209-1551, src/btbmepn.f90:177-587,
    SPE subsumption src/bsppot.f90:39-238).
    """
    spec = tables.extra["spec"]
    jac = tables.extra["jacobian"]
    g_tb = np.zeros(max(1, len(spec.tbme)))
    g_spe = np.zeros(len(spec.orbits))
    for nm in ("pp", "nn", "pn"):
        jt, js = jac[nm]
        d = np.asarray(dhmat[nm], dtype=np.float64)
        if d.size:
            g_tb += d @ jt
            g_spe += d @ js
    if tables.s["call_spe"] and "spe_p" in dhmat:
        # pspe_h(ip) = spe_scale * sum of occupied orbit SPEs
        for key, orbk, bits in (("spe_p", "sp_orb_p", "sd_bits_p"), ("spe_n", "sp_orb_n", "sd_bits_n")):
            orb = tables.extra[orbk]
            b = tables.extra[bits]
            d = np.asarray(dhmat[key], dtype=np.float64)
            for q in range(len(orb)):
                occ = ((b >> np.uint64(q)) & np.uint64(1)).astype(bool)
                g_spe[orb[q]] += spec.spe_scale * d[occ].sum()
    return g_tb[:len(spec.tbme)], g_spe


def batch_member(seed):
    """One Hamiltonian of the seeded sd-shell batch: valence Z and N drawn
    uniformly in 2..8 from a SplitMix64 stream of `seed`, then the synthetic
    isospin interaction continued from the same stream (SPEs -3.9/-3.2/+2.1
    MeV); 2Jz = 0 for even A, 1 for odd A."""
    rng = SplitMix64(seed)
    np_ = rng.randint(2, 8)
    nn = rng.randint(2, 8)
    tb = []
    for k in canonical_tbme_keys(SD_ORBITS):
        tb.append(k + (float(np.float32(float("%.8e" % rng.normal()))),))
    spe = [float(np.float32(float("%.8e" % s))) for s in SD_SYNTH_SPE]
    return ModelSpec(SD_ORBITS, np_, nn, (np_ + nn) % 2, 1, spe, tb)
