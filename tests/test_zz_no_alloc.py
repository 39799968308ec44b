"""bsg_applyh_noalloc: the host-vector applyH that allocates no device memory.

It exists for callers that cannot allocate device memory at the time of the
matvec (a host whose device memory is a fixed pool owned by another
component, or a driver whose device footprint is fixed after set-up).  It
stages vectors through a fixed static device array, so its results must be
those of the ordinary bsg_applyh entry point.  This file is collected last so
that a stop-at-first-failure run has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from bigstickpublick_b200 import model

pytestmark = pytest.mark.gpu

MAX_BYTES = 8 << 20  # BSG_NOALLOC_MAX_VECTOR_BYTES


def _noalloc(H, vin, vout, nb, prec, flags=0):
    lib = H.lib
    lib.bsg_applyh_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int]
    lib.bsg_applyh_noalloc.restype = C.c_int
    return lib.bsg_applyh_noalloc(H.h, vin.ctypes.data, vout.ctypes.data, nb, prec, flags)


@pytest.mark.parametrize("builder", [lambda: model.sd_model(2, 2, seed=1),
                                     lambda: model.pf_model(2, 2, seed=5)])
@pytest.mark.parametrize("prec,nb", [(8, 1), (4, 1), (8, 3), (8, 4), (4, 8)])
def test_noalloc_matches_applyh_twice(builder, prec, nb):
    from bigstickpublick_b200.engine import Hamiltonian
    T = model.build_tables(builder())
    H = Hamiltonian(T)
    dt = np.float64 if prec == 8 else np.float32
    tol = 1e-12 if prec == 8 else 2e-5
    rng = np.random.default_rng(42 + nb)
    vin = rng.standard_normal(T.dim * nb).astype(dt)
    # first on a fresh context (its row tiles are not built yet)
    first = np.zeros_like(vin)
    assert _noalloc(H, vin, first, nb, prec) == 0
    ref = H.applyh(vin.reshape(T.dim, nb) if nb > 1 else vin).reshape(-1)  # existing entry point
    scale = np.abs(ref).max()
    assert np.abs(first - ref).max() / scale < tol
    # two calls in a row on the now cached tiles
    for _ in range(2):
        out = np.full_like(vin, np.nan)
        assert _noalloc(H, vin, out, nb, prec) == 0
        assert np.abs(out - ref).max() / scale < tol
    # accumulate flag: vout += H vin
    base = rng.standard_normal(T.dim * nb).astype(dt)
    acc = base.copy()
    assert _noalloc(H, vin, acc, nb, prec, flags=1) == 0
    assert np.abs(acc - (base + ref)).max() / (np.abs(base + ref).max()) < tol
    H.close()


def test_noalloc_rejects_oversize_vectors():
    from bigstickpublick_b200.engine import Hamiltonian
    T = model.build_tables(model.sd_model(6, 6, seed=2))
    H = Hamiltonian(T)
    nb = 16  # 93,710 x 16 x 8 B = 12 MB > the 8 MiB static staging limit
    assert T.dim * nb * 8 > MAX_BYTES
    vin = np.ones(T.dim * nb)
    out = np.zeros_like(vin)
    assert _noalloc(H, vin, out, nb, 8) == 7  # BSG_ERR_ARG
    buf = C.create_string_buffer(256)
    H.lib.bsg_last_error(H.h, buf, 256)
    assert b"static staging limit" in buf.value
    assert not out.any()
    H.close()


def _spe_rows(nrows, seed=3):
    """An SPE-only Hamiltonian of nrows proton SDs with one neutron SD each
    (rows of one state, so one 32-position row tile per row): H is the
    diagonal pspe + nspe (the SPE case of src/bapplyhlibOMP.f90:988-1011)."""
    rng = np.random.default_rng(seed)
    i8 = lambda *x: np.array(x, dtype=np.int64)
    a = {k: np.zeros(0, dtype=v.dtype) for k, v in model.build_tables(model.sd_model(1, 0, seed=12, jz2=1)).a.items()}
    a.update(pstart=np.arange(nrows, dtype=np.int64), nstart=i8(1),
             hmatpp=np.zeros(1, np.float32), hmatnn=np.zeros(1, np.float32), hmatpn=np.zeros(1, np.float32),
             cpnpair=i8(0), dpnpair=i8(0), pspe_h=rng.standard_normal(nrows).astype(np.float32),
             nspe_h=np.array([0.25], np.float32), optype=np.array([1], np.int32), hchar=np.array([ord("f")], np.int32),
             pxstart=i8(1), pxend=i8(nrows), nxstart=i8(1), nxend=i8(1), cstride=i8(1))
    s = dict(dimbasis=nrows, nsd_p=nrows, nsd_n=1, np1b=0, nn1b=0, np2b=0, nn2b=0, nmatpp=1, nmatnn=1, nmatpn=1,
             nhsps_pl=0, nhsps_pr=0, nhsps_nl=0, nhsps_nr=0, call_spe=1, nbundles=1)
    return model.Tables(a, s, {})


def test_noalloc_tile_limit_status_and_cached_tiles():
    """A fresh context with more row tiles than the static array holds is
    refused with BSG_ERR_ARG and a message; once an applyH on the context (at
    set-up, where allocation is allowed) has cached its tiles, the same call
    works and matches bsg_applyh, twice in a row."""
    from bigstickpublick_b200.engine import Hamiltonian
    T = _spe_rows(70000)
    H = Hamiltonian(T)
    vin = np.random.default_rng(1).standard_normal(T.dim)
    out = np.zeros_like(vin)
    assert _noalloc(H, vin, out, 1, 8) == 7  # BSG_ERR_ARG
    buf = C.create_string_buffer(256)
    H.lib.bsg_last_error(H.h, buf, 256)
    assert b"row tiles exceed" in buf.value
    assert not out.any()
    ref = H.applyh(vin)
    diag = T.a["pspe_h"].astype(np.float32) + np.float32(0.25)
    assert np.abs(ref - diag.astype(np.float64) * vin).max() < 1e-12
    for _ in range(2):
        got = np.full_like(vin, np.nan)
        assert _noalloc(H, vin, got, 1, 8) == 0
        assert np.array_equal(got, ref)
    H.close()
