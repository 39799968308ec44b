"""The reference's .wfn eigenvector file, written and read.

BIGSTICK's lanczos_output writes each kept state to ``<name>.wfn`` so that
its other tools (densities, transition strengths, overlaps) can read the
states back.  The file is Fortran unformatted stream (no record markers),
native little-endian:

* header (write_wfn_header, src/bwfnlib.f90:373-546): int32 magic 31415926,
  int32 version 1, int32 0, five int32 slots of which the first (byte 12,
  ``wfn_after_header_word * 4``) receives the 0-based byte position of the
  first vector record; int32 np(1), np(2); int32 isoflag, numorb(1),
  numorb(2); per species and orbit int32 nr, 2j, l, par, w; int32 nsps(1),
  nsps(2); per species and s.p. state int32 nr, 2j, 2m, l, w, par, orb, group
  (states in sort_spsqn order, src/bspstates.f90:100-215); int32 2Jz,
  ichar(cparity), maxWtot, allsameparity, allsameW, spinless (logicals as
  int32 0/1, wfn_write_logical :1433-1472); int64 dimbasis
  (wfn_write_bkint :1275-1283);
* int32 nkeep (wfn_write_nkeep :1041-1050);
* per state (wfn_writeeigenvec :77-134): int32 27182818, int32 index
  (1-based), float32 energy, float32 J, float32 T(T+1), then the dimbasis
  amplitudes in the Lanczos vector precision (lanc_prec: float32 as the
  reference ships it, or float64), in basis order.

The basis order is the table builder's (the reference's sector, SD and
block order; see bsg_host.h).  Untruncated spaces only: every orbit has the
same W, so setWzero (src/binput.f90:960-990) makes W = 0 and maxWtot = 0.
"""
import struct

import numpy as np

WFN_MAGIC = 31415926
WFN_VECMAGIC = 27182818
WFN_VERSION = 1
AFTER_HEADER_WORD = 3


def _orbit_par(l, allsamepar):
    return 1 if allsamepar else (-1 if l % 2 else 1)


def sorted_sps(orbits, allsamepar=None):
    """extract_sps + sort_spsqn (src/bspstates.f90:53-215) for one species:
    list of dicts nr, j2, m2, l, w, par, orb (1-based), group (0) in the
    reference's order (selection sorts with swap on parity, then |m|; W is
    zero for every state of an untruncated space)."""
    if allsamepar is None:
        allsamepar = len({l % 2 for _, l, _, _ in orbits}) == 1
    sp = []
    for i, (n, l, j2, w) in enumerate(orbits):
        for m in range(-j2, j2 + 1, 2):
            sp.append(dict(nr=n, j2=j2, m2=m, l=l, w=0, par=_orbit_par(l, allsamepar), orb=i + 1, group=0))
    n = len(sp)

    def selection(lo, hi, key):
        for i in range(lo, hi + 1):
            k, best = i, key(sp[i])
            for j in range(i + 1, hi + 1):
                if key(sp[j]) < best:
                    k, best = j, key(sp[j])
            if k != i:
                sp[i], sp[k] = sp[k], sp[i]

    if not allsamepar:  # on parity within each W (all W equal here)
        selection(0, n - 1, lambda x: x["par"])
    start = 0
    while start < n:  # on |m| within each (W, par)
        end = max(i for i in range(start, n) if sp[i]["w"] == sp[start]["w"] and sp[i]["par"] == sp[start]["par"])
        selection(start, end, lambda x: abs(x["m2"]))
        start = end + 1
    return sp


def header_bytes(spec, dim):
    """Bytes of write_wfn_header for a model spec (model.ModelSpec) and its
    basis dimension, the after-header offset already filled in (it points
    past the nkeep word that follows the header)."""
    if len({o[3] for o in spec.orbits}) != 1:
        raise ValueError("the .wfn writer covers untruncated spaces (every orbit with the same W)")
    allsamepar = len({o[1] % 2 for o in spec.orbits}) == 1
    i4 = lambda *v: struct.pack("<%di" % len(v), *v)
    out = [i4(WFN_MAGIC, WFN_VERSION, 0, 0, 0, 0, 0, 0)]
    out.append(i4(spec.np_, spec.nn))
    norb = len(spec.orbits)
    out.append(i4(1, norb, norb))  # isoflag, numorb(1), numorb(2)
    for _ in range(2):
        for (n, l, j2, w) in spec.orbits:
            out.append(i4(n, j2, l, _orbit_par(l, allsamepar), 0))
    sps = sorted_sps(spec.orbits, allsamepar)
    out.append(i4(len(sps), len(sps)))
    for _ in range(2):
        for x in sps:
            out.append(i4(x["nr"], x["j2"], x["m2"], x["l"], x["w"], x["par"], x["orb"], x["group"]))
    if allsamepar:
        cparity = "+"
    else:
        cparity = "+" if spec.parity >= 0 else "-"
    spinless = spec.orbits[0][2] % 2 == 0
    out.append(i4(spec.jz2, ord(cparity), 0, 1 if allsamepar else 0, 1, 1 if spinless else 0))
    out.append(struct.pack("<q", int(dim)))
    head = bytearray(b"".join(out))
    after_nkeep = len(head) + 4
    head[4 * AFTER_HEADER_WORD:4 * AFTER_HEADER_WORD + 4] = struct.pack("<i", after_nkeep)
    return bytes(head)


def write_wfn(path, spec, evals, vecs, xj, xt2, lanc_prec=4):
    """Write states as lanczos_output does: vecs dim x k (basis order of the
    builder), evals[k], xj[k] = J, xt2[k] = T(T+1); amplitudes in float32
    (lanc_prec 4, the reference's shipped precision) or float64 (8)."""
    vecs = np.asarray(vecs)
    if vecs.ndim == 1:
        vecs = vecs[:, None]
    dim, k = vecs.shape
    dt = np.dtype("<f4") if lanc_prec == 4 else np.dtype("<f8")
    with open(path, "wb") as f:
        f.write(header_bytes(spec, dim))
        f.write(struct.pack("<i", k))
        for i in range(k):
            f.write(struct.pack("<ii3f", WFN_VECMAGIC, i + 1, float(evals[i]), float(xj[i]), float(xt2[i])))
            f.write(np.ascontiguousarray(vecs[:, i], dtype=dt).tobytes())


def read_wfn(path, lanc_prec=4):
    """Read a .wfn file as the reference's reader does (wfn_read header, then
    wfn_readeigenvec, src/bwfnlib.f90:146-300, :690-800): returns (header
    dict, list of states dict(index, e, xj, xt2, vec))."""
    buf = open(path, "rb").read()
    pos = 0

    def i4(n=1):
        nonlocal pos
        v = struct.unpack_from("<%di" % n, buf, pos)
        pos += 4 * n
        return v if n > 1 else v[0]

    h = {}
    magic, version, _, after, *_ = i4(8)
    if magic != WFN_MAGIC:
        raise ValueError("WFN file is missing magic number")
    if version != WFN_VERSION:
        raise ValueError(f"WFN version {version} is not {WFN_VERSION}")
    h["after_header"] = after
    h["np"], h["nn"] = i4(2)
    h["isoflag"], n1, n2 = i4(3)
    h["orbits"] = [[i4(5) for _ in range(n)] for n in (n1, n2)]
    s1, s2 = i4(2)
    h["sps"] = [[i4(8) for _ in range(n)] for n in (s1, s2)]
    h["jz2"], par, h["maxWtot"], h["allsameparity"], h["allsameW"], h["spinless"] = i4(6)
    h["cparity"] = chr(par)
    h["dim"] = struct.unpack_from("<q", buf, pos)[0]
    pos += 8
    h["nkeep"] = i4()
    if pos != after:
        raise ValueError(f"after-header offset {after} does not match the header length {pos}")
    dt = np.dtype("<f4") if lanc_prec == 4 else np.dtype("<f8")
    states = []
    for _ in range(h["nkeep"]):
        vm, idx = struct.unpack_from("<ii", buf, pos)
        e, xj, xt2 = struct.unpack_from("<3f", buf, pos + 8)
        pos += 20
        if vm != WFN_VECMAGIC:
            raise ValueError("vector record is missing its magic number")
        vec = np.frombuffer(buf, dtype=dt, count=h["dim"], offset=pos).copy()
        pos += h["dim"] * dt.itemsize
        states.append(dict(index=idx, e=e, xj=xj, xt2=xt2, vec=vec))
    if pos != len(buf):
        raise ValueError("trailing bytes after the last state")
    return h, states
