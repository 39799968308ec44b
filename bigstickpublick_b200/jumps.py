"""Jump tables generated on the GPU (bsg_jumpgen_*).

The host table builder (libbsghost.so) produces the jumps on the CPU, as the
reference's set-up does (weld / master1bodyjumps / master2bodyjumps,
src/bjumplib_weld.f90:296-809, src/bjumplib_master.f90:436-1196).
``device_jumps`` produces the same arrays with the engine's GPU kernels from
the species' Slater determinants, in the builder's sector-jump order, and
sorts every PN bundle's ranges with the reference's shell sort
(sort_bundled_jumps, src/bsortjumpslib.f90:21-175): protons on fsd, neutrons
on isd.  The result is byte-identical to the host tables.
"""
import ctypes as C
import time

import numpy as np

from . import _abi


class _Species:
    """A bsg_species view of one species of built tables (arrays kept alive)."""

    def __init__(self, tables, spec, which):
        ex = tables.extra
        sfx = "p" if which == "p" else "n"
        self.bits = np.ascontiguousarray(ex["sd_bits_" + sfx], dtype=np.uint64)
        self.xstart = np.ascontiguousarray(tables.a["pstart" if which == "p" else "nstart"], dtype=np.int64)
        m2 = np.asarray(ex["sp_m2_" + sfx], dtype=np.int32)
        orb = np.asarray(ex["sp_orb_" + sfx], dtype=np.int32)
        ls = [o[1] for o in spec.orbits]
        allsame = len({l % 2 for l in ls}) == 1
        self.m2 = np.ascontiguousarray(m2)
        self.par = np.ascontiguousarray([1 if allsame else (-1 if ls[o] % 2 else 1) for o in orb], dtype=np.int32)
        self.nl = int(np.sum(m2 < 0))
        self.s0 = np.ascontiguousarray(ex[sfx + "sector_start"], dtype=np.int64)
        self.s1 = np.ascontiguousarray(ex[sfx + "sector_end"], dtype=np.int64)
        i32p, i64p = C.POINTER(C.c_int32), C.POINTER(C.c_int64)
        self.c = _abi.BsgSpecies(len(m2), self.nl, self.m2.ctypes.data_as(i32p), self.par.ctypes.data_as(i32p),
                                 len(self.bits), self.bits.ctypes.data_as(C.POINTER(C.c_uint64)),
                                 self.xstart.ctypes.data_as(i64p), len(self.s0), self.s0.ctypes.data_as(i64p),
                                 self.s1.ctypes.data_as(i64p))


class JumpGen:
    """The device copy of one species (bsg_jumpgen_create)."""

    def __init__(self, tables, spec, which, device=0):
        self.lib = _abi.gpu_lib()
        self.sp = _Species(tables, spec, which)
        h = C.c_void_p()
        st = self.lib.bsg_jumpgen_create(device, C.byref(self.sp.c), C.byref(h))
        if st != 0:
            raise RuntimeError(f"bsg_jumpgen_create: status {st}")
        self.h = h
        self.ms = 0.0

    def close(self):
        if getattr(self, "h", None):
            self.lib.bsg_jumpgen_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st, what):
        if st != 0:
            buf = C.create_string_buffer(256)
            self.lib.bsg_jumpgen_last_error(self.h, buf, 256)
            raise RuntimeError(f"{what}: status {st}: {buf.value.decode()}")

    def one(self, pairs, write=True):
        """One-body jumps of the sector jumps [(is, fs), ...] (0-based):
        (starts, arrays or None)."""
        n = len(pairs)
        is_ = np.ascontiguousarray([p[0] for p in pairs], dtype=np.int32)
        fs_ = np.ascontiguousarray([p[1] for p in pairs], dtype=np.int32)
        starts = np.zeros(n + 1, dtype=np.int64)
        ms = C.c_double()
        st = self.lib.bsg_jumpgen_one(self.h, n, is_.ctypes.data, fs_.ctypes.data, starts.ctypes.data,
                                      None, None, None, None, None, C.byref(ms))
        self._check(st, "bsg_jumpgen_one (count)")
        self.ms += ms.value
        if not write:
            return starts, None
        tot = int(starts[-1])
        out = {"isd": np.zeros(tot, np.int64), "fsd": np.zeros(tot, np.int64), "cop": np.zeros(tot, np.int16),
               "dop": np.zeros(tot, np.int16), "phase": np.zeros(tot, np.int8)}
        st = self.lib.bsg_jumpgen_one(self.h, n, is_.ctypes.data, fs_.ctypes.data, starts.ctypes.data,
                                      *[out[k].ctypes.data for k in ("isd", "fsd", "cop", "dop", "phase")],
                                      C.byref(ms))
        self._check(st, "bsg_jumpgen_one")
        self.ms += ms.value
        return starts, out

    def two(self, secs, write=True):
        n = len(secs)
        sec = np.ascontiguousarray(secs, dtype=np.int32)
        starts = np.zeros(n + 1, dtype=np.int64)
        ms = C.c_double()
        st = self.lib.bsg_jumpgen_two(self.h, n, sec.ctypes.data, starts.ctypes.data, None, None, None, None,
                                      C.byref(ms))
        self._check(st, "bsg_jumpgen_two (count)")
        self.ms += ms.value
        if not write:
            return starts, None
        tot = int(starts[-1])
        out = {"isd": np.zeros(tot, np.int64), "fsd": np.zeros(tot, np.int64), "op": np.zeros(tot, np.int32),
               "phase": np.zeros(tot, np.int8)}
        st = self.lib.bsg_jumpgen_two(self.h, n, sec.ctypes.data, starts.ctypes.data,
                                      *[out[k].ctypes.data for k in ("isd", "fsd", "op", "phase")], C.byref(ms))
        self._check(st, "bsg_jumpgen_two")
        self.ms += ms.value
        return starts, out

    def sort(self, ranges, by_fsd, arrs):
        """sort1bjumps on the distinct ranges [(start, len)] of arrs, in place."""
        uniq = sorted({(int(a), int(b)) for a, b in ranges})
        st0 = np.ascontiguousarray([r[0] for r in uniq], dtype=np.int64)
        ln = np.ascontiguousarray([r[1] for r in uniq], dtype=np.int64)
        ms = C.c_double()
        st = self.lib.bsg_jumpgen_sort1(self.h, len(uniq), st0.ctypes.data, ln.ctypes.data, 1 if by_fsd else 0,
                                        len(arrs["isd"]),
                                        *[arrs[k].ctypes.data for k in ("isd", "fsd", "cop", "dop", "phase")],
                                        C.byref(ms))
        self._check(st, "bsg_jumpgen_sort1")
        self.ms += ms.value


def device_jumps(tables, spec, device=0, density=True):
    """The jump arrays of `tables` generated on the GPU in the builder's
    order, PN ranges sorted: dict 'p1b_isd' ... 'n2b_phase' (the keys of
    tables.a), and 'density' (the same for the one-body density jumps) when
    asked; plus 'kernel_ms' and 'wall_s'."""
    t0 = time.perf_counter()
    ex = tables.extra
    npart, nneut = spec.np_, spec.nn
    pconj = [int(c) - 1 for c in ex["psector_conj"]]
    nps, nns = len(pconj), len(ex["nsector_start"])
    gp, gn = JumpGen(tables, spec, "p", device), JumpGen(tables, spec, "n", device)
    out = {}
    try:
        # one-body sector jumps: protons is >= fs with jumps, each with its
        # conjugate neutron sector jump (first appearance)
        p1, n1 = [], []
        if npart >= 1 and nneut >= 1:
            cand = [(i, f) for i in range(nps) for f in range(i + 1)]
            starts, _ = gp.one(cand, write=False)
            p1 = [c for c, a, b in zip(cand, starts[:-1], starts[1:]) if b > a]
            seen = set()
            for i, f in p1:
                k = (pconj[i], pconj[f])
                if k not in seen:
                    seen.add(k)
                    n1.append(k)
        sp1, jp1 = gp.one(p1)
        sn1, jn1 = gn.one(n1)
        # two-body: inside each sector with jumps
        p2 = n2 = []
        if npart >= 2:
            s2, _ = gp.two(list(range(nps)), write=False)
            p2 = [s for s, a, b in zip(range(nps), s2[:-1], s2[1:]) if b > a]
        if nneut >= 2:
            s2, _ = gn.two(list(range(nns)), write=False)
            n2 = [s for s, a, b in zip(range(nns), s2[:-1], s2[1:]) if b > a]
        _, jp2 = gp.two(p2)
        _, jn2 = gn.two(n2)
        # sort_bundled_jumps over the PN bundles
        a = tables.a
        pn = a["optype"] == 4
        gp.sort([(s - 1, e - s + 1) for s, e in zip(a["pxstart"][pn], a["pxend"][pn])], True, jp1)
        gn.sort([(s - 1, e - s + 1) for s, e in zip(a["nxstart"][pn], a["nxend"][pn])], False, jn1)
        for pre, d in (("p1b_", jp1), ("n1b_", jn1)):
            for k in ("isd", "fsd", "cop", "dop", "phase"):
                out[pre + k] = d[k]
        for pre, d in (("p2b_", jp2), ("n2b_", jn2)):
            for k in ("isd", "fsd", "op", "phase"):
                out[pre + k] = d[k]
        if density:
            pj = [(i, i) for i in range(nps)] if npart >= 1 else []
            nj = [(i, i) for i in range(nns) if i in pconj] if nneut >= 1 else []
            d = {}
            for pre, g, lst in (("p1b_", gp, pj), ("n1b_", gn, nj)):
                st, _ = g.one(lst, write=False)
                keep = [c for c, x, y in zip(lst, st[:-1], st[1:]) if y > x]
                _, arr = g.one(keep)
                for k in ("isd", "fsd", "cop", "dop", "phase"):
                    d[pre + k] = arr[k]
            out["density"] = d
        out["kernel_ms"] = gp.ms + gn.ms
    finally:
        gp.close()
        gn.close()
    out["wall_s"] = time.perf_counter() - t0
    return out
