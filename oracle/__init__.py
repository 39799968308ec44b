"""ORACLE -- test infrastructure only.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package, as the checker.  The product (bigstickpublick_b200) never
imports, links or calls it.

* liboracle.so (oracle_applyh.c): plain-C restatement of BIGSTICK's
  applyHbundled_omp / applyHbundled_block_omp loops, and of the three-body
  bundle loops (applyhPPP/PPN/PNN/NNNbundled_g); its owner-computes
  OpenMP partition (each thread the output rows getLoadDist gives it), used
  as the timed CPU baseline and, restricted to a few rows, as the checker of
  large systems; and the serial-path split routines of applyHbundled_g.
* dense_h.py: independent dense Hamiltonian from second quantization.
* lanczos.py: numpy restatement of lanczos_p / lanczos_block with full
  reorthogonalization, convergence test and thick restart.
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build(force=False):
    """Compile oracle_applyh.c into oracle/liboracle.so with gcc."""
    out = os.path.join(_HERE, "liboracle.so")
    src = os.path.join(_HERE, "oracle_applyh.c")
    if force or not os.path.exists(out) or os.path.getmtime(out) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-std=c11", "-O3", "-march=x86-64-v2", "-fopenmp", "-fPIC",
                               "-shared", src, "-o", out])
    return out


def lib():
    global _LIB
    if _LIB is None:
        path = build()
        L = C.CDLL(path)
        L.oracle_applyh.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        L.oracle_applyh.restype = C.c_int
        L.oracle_applyh_omp.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int]
        L.oracle_applyh_omp.restype = C.c_int
        L.oracle_count_ops.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
        L.oracle_count_ops.restype = None
        L.oracle_density.argtypes = [C.c_void_p] + [C.c_void_p] * 6
        L.oracle_density.restype = C.c_int
        L.oracle_row_ops.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_row_ops.restype = C.c_int64
        L.oracle_applyh_rows.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int64, C.c_int64]
        L.oracle_applyh_rows.restype = C.c_int
        L.oracle_applyh_owner.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                          C.c_void_p, C.c_int]
        L.oracle_applyh_owner.restype = C.c_int
        L.oracle_applyh3.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        L.oracle_applyh3.restype = C.c_int
        L.oracle_applyh3_bundles.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                             C.c_void_p, C.c_int64]
        L.oracle_applyh3_bundles.restype = C.c_int
        L.oracle_count_ops3.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
        L.oracle_count_ops3.restype = None
        _LIB = L
    return _LIB


def _tp(tables):
    t = tables.as_ctypes()
    return C.cast(C.pointer(t), C.c_void_p), t


def applyh(tables, vin, nb=1, accumulate_into=None):
    """H vin (one thread, reference loop order).  vin: float32 or float64 array
    of dim*nb (interleaved block layout); returns a new array (or accumulates
    into `accumulate_into`)."""
    vin = np.ascontiguousarray(vin)
    prec = 4 if vin.dtype == np.float32 else 8
    out = np.zeros_like(vin) if accumulate_into is None else accumulate_into
    p, keep = _tp(tables)
    if getattr(tables, "threebody", False):
        t3 = tables.as_ctypes3()
        st = lib().oracle_applyh3(p, C.cast(C.pointer(t3), C.c_void_p), vin.ctypes.data, out.ctypes.data, nb, prec)
    else:
        st = lib().oracle_applyh(p, vin.ctypes.data, out.ctypes.data, nb, prec)
    if st != 0:
        raise RuntimeError(f"oracle_applyh status {st}")
    return out


def applyh3_bundles(tables, vin, bundles, nb=1, out=None):
    """vout += H vin over the listed bundles (0-based) of a three-body run."""
    vin = np.ascontiguousarray(vin)
    prec = 4 if vin.dtype == np.float32 else 8
    if out is None:
        out = np.zeros_like(vin)
    lst = np.ascontiguousarray(bundles, dtype=np.int64)
    p, keep = _tp(tables)
    t3 = tables.as_ctypes3()
    st = lib().oracle_applyh3_bundles(p, C.cast(C.pointer(t3), C.c_void_p), vin.ctypes.data, out.ctypes.data, nb,
                                      prec, lst.ctypes.data, len(lst))
    if st != 0:
        raise RuntimeError(f"oracle_applyh3_bundles status {st}")
    return out


def count_ops3(tables):
    """(ppp, nnn, ppn, pnn) inner-loop updates per matvec of a three-body run."""
    ops = (C.c_int64 * 4)()
    p, keep = _tp(tables)
    lib().oracle_count_ops3(p, ops)
    return tuple(int(x) for x in ops)


def applyh_omp(tables, vin, nb=1, nthreads=None, out=None):
    vin = np.ascontiguousarray(vin)
    prec = 4 if vin.dtype == np.float32 else 8
    if out is None:
        out = np.zeros_like(vin)
    p, keep = _tp(tables)
    st = lib().oracle_applyh_omp(p, vin.ctypes.data, out.ctypes.data, nb, prec,
                                 nthreads or os.cpu_count())
    if st != 0:
        raise RuntimeError(f"oracle_applyh_omp status {st}")
    return out


def row_ops(tables):
    """The output rows and their work, as getLoadDist buckets it
    (src/bapplyhlibOMP.f90:213-327): (row_start, ops), row_start the distinct
    pstart values in ascending order, ops the inner-loop updates landing in
    each row.  Row r holds the basis states row_start[r]+1 .. row_start[r+1]
    (1-based; the last row ends at dim)."""
    n = int(tables.s["nsd_p"])
    rs = np.zeros(n, dtype=np.int64)
    ops = np.zeros(n, dtype=np.int64)
    p, keep = _tp(tables)
    m = lib().oracle_row_ops(p, rs.ctypes.data, ops.ctypes.data)
    return rs[:m].copy(), ops[:m].copy()


def owner_ranges(row_start, ops, dim, nparts):
    """Cut the rows into nparts contiguous runs of about equal work (the
    equal-weight bucket runs of getLoadDist, src/bapplyhlibOMP.f90:330-420):
    int64 array (nparts, 2) of [lo, hi) row-start bounds."""
    csum = np.cumsum(ops)
    total = int(csum[-1]) if len(csum) else 0
    cuts = [0]
    for k in range(1, nparts):
        cuts.append(max(cuts[-1], int(np.searchsorted(csum, total * k / nparts, side="left")) + 1))
    cuts.append(len(row_start))
    lo = [int(row_start[c]) if c < len(row_start) else dim for c in cuts[:-1]]
    hi = lo[1:] + [dim]
    return np.array([[a, b] for a, b in zip(lo, hi) if b > a], dtype=np.int64).reshape(-1, 2)


def applyh_rows(tables, vin, lo, hi, nb=1, out=None):
    """out += (H vin) on the rows with pstart value in [lo, hi) only (one
    owner's share of applyHbundled_omp, one thread); other entries of out are
    left as they are."""
    vin = np.ascontiguousarray(vin)
    prec = 4 if vin.dtype == np.float32 else 8
    if out is None:
        out = np.zeros_like(vin)
    p, keep = _tp(tables)
    st = lib().oracle_applyh_rows(p, vin.ctypes.data, out.ctypes.data, nb, prec, int(lo), int(hi))
    if st != 0:
        raise RuntimeError(f"oracle_applyh_rows status {st}")
    return out


def applyh_owner(tables, vin, ranges, nb=1, nthreads=None, out=None):
    """out += (H vin) on the row ranges `ranges` ((n, 2) [lo, hi) bounds),
    the ranges spread over nthreads OpenMP threads: applyHbundled_omp's
    owner-computes partition when the ranges are owner_ranges(...) of all
    rows."""
    vin = np.ascontiguousarray(vin)
    prec = 4 if vin.dtype == np.float32 else 8
    if out is None:
        out = np.zeros_like(vin)
    b = np.ascontiguousarray(ranges, dtype=np.int64).reshape(-1, 2)
    p, keep = _tp(tables)
    st = lib().oracle_applyh_owner(p, vin.ctypes.data, out.ctypes.data, nb, prec, len(b), b.ctypes.data,
                                   nthreads or os.cpu_count())
    if st != 0:
        raise RuntimeError(f"oracle_applyh_owner status {st}")
    return out


def count_ops(tables):
    """(spe, pp, nn, pn) inner-loop updates per matvec."""
    ops = (C.c_int64 * 4)()
    p, keep = _tp(tables)
    lib().oracle_count_ops(p, ops)
    return tuple(int(x) for x in ops)


def density(tables, psi):
    """dE/dhmat for a normalized eigenvector psi (restated two-body densities):
    dict with 'pp', 'nn', 'pn' (and 'spe_p', 'spe_n' when call_spe)."""
    psi = np.ascontiguousarray(psi, dtype=np.float64)
    s = tables.s
    out = {"pp": np.zeros(s["nmatpp"]), "nn": np.zeros(s["nmatnn"]), "pn": np.zeros(s["nmatpn"]),
           "spe_p": np.zeros(s["nsd_p"]), "spe_n": np.zeros(s["nsd_n"])}
    p, keep = _tp(tables)
    st = lib().oracle_density(p, psi.ctypes.data, out["pp"].ctypes.data, out["nn"].ctypes.data,
                              out["pn"].ctypes.data, out["spe_p"].ctypes.data, out["spe_n"].ctypes.data)
    if st != 0:
        raise RuntimeError(f"oracle_density status {st}")
    return out


def dense_from_applyh(tables, prec=8):
    """Dense H by applying the oracle matvec to unit vectors (small dims)."""
    n = tables.dim
    dt = np.float64 if prec == 8 else np.float32
    H = np.zeros((n, n), dtype=np.float64)
    e = np.zeros(n, dtype=dt)
    for i in range(n):
        e[:] = 0
        e[i] = 1
        H[:, i] = applyh(tables, e)
    return H
