"""GPU applyH parity against the oracle (restated applyHbundled_omp)."""
import numpy as np
import pytest

from bigstickpublick_b200 import model
import oracle

pytestmark = pytest.mark.gpu

CASES = [
    ("sd 1p1n", lambda: model.sd_model(1, 1, seed=11)),
    ("sd 1p0n call_spe", lambda: model.sd_model(1, 0, seed=12, jz2=1)),
    ("sd 2p2n", lambda: model.sd_model(2, 2, seed=1)),
    ("sd 3p2n jz=1", lambda: model.sd_model(3, 2, seed=3, jz2=1)),
    ("sd 0p3n jz=3", lambda: model.sd_model(0, 3, seed=4, jz2=3)),
    ("pf 2p2n", lambda: model.pf_model(2, 2, seed=5)),
]


@pytest.fixture(scope="module")
def built():
    from bigstickpublick_b200.engine import Hamiltonian
    out = {}
    for name, mk in CASES:
        T = model.build_tables(mk())
        out[name] = (T, Hamiltonian(T))
    return out


@pytest.mark.parametrize("name", [c[0] for c in CASES])
@pytest.mark.parametrize("prec", [8, 4])
@pytest.mark.parametrize("nb", [1, 2, 3, 4, 8, 16])
def test_applyh_matches_oracle(built, name, prec, nb):
    T, H = built[name]
    rng = np.random.default_rng(1234 + nb)
    dt = np.float64 if prec == 8 else np.float32
    vin = rng.standard_normal((T.dim, nb)).astype(dt)
    if nb == 1:
        vin = vin[:, 0].copy()
    ref = oracle.applyh(T, vin.reshape(-1), nb=nb).reshape(vin.shape)
    got = H.applyh(vin)
    scale = np.abs(ref).max() + 1e-30
    err = np.abs(got - ref).max() / scale
    tol = 1e-12 if prec == 8 else 2e-5   # fp64: summation order only; fp32: fp32 accumulation
    assert err < tol, f"{name} prec={prec} nb={nb}: rel err {err:.3e}"


@pytest.mark.parametrize("name", [c[0] for c in CASES])
def test_accumulate_flag(built, name):
    T, H = built[name]
    rng = np.random.default_rng(7)
    vin = rng.standard_normal(T.dim)
    base = rng.standard_normal(T.dim)
    out = base.copy()
    H.applyh(vin, out, accumulate=True)
    ref = base + oracle.applyh(T, vin)
    assert np.abs(out - ref).max() < 1e-12 * (np.abs(ref).max() + 1)


def test_device_pointer_path_and_determinism(built):
    import torch
    T, H = built["pf 2p2n"]
    x = torch.randn(T.dim, 4, dtype=torch.float32, device="cuda")
    y1 = H.applyh(x)
    y2 = H.applyh(x)
    torch.cuda.synchronize()
    assert torch.equal(y1, y2), "applyH must be bitwise repeatable (no atomics)"
    ref = oracle.applyh(T, x.cpu().numpy().reshape(-1), nb=4).reshape(T.dim, 4)
    err = np.abs(y1.cpu().numpy() - ref).max() / np.abs(ref).max()
    assert err < 2e-5


@pytest.mark.parametrize("prec,nb,acc", [(4, 1, False), (8, 1, True), (4, 4, False), (8, 2, True)])
def test_pinned_host_buffers_reused(built, prec, nb, acc):
    """Pinned host buffers reused call after call, as the drop-in's vec1/vec2
    are: every call must see that call's buffer contents, and the result
    must equal the same input from pageable memory bit for bit."""
    import torch
    T, H = built["sd 3p2n jz=1"]
    dt = torch.float64 if prec == 8 else torch.float32
    shape = (T.dim,) if nb == 1 else (T.dim, nb)
    hin = torch.empty(shape, dtype=dt, pin_memory=True)
    hout = torch.empty(shape, dtype=dt, pin_memory=True)
    xin, xout = hin.numpy(), hout.numpy()
    rng = np.random.default_rng(9)
    tol = 1e-12 if prec == 8 else 2e-5
    for step in range(4):
        xin[...] = rng.standard_normal(shape)
        base = rng.standard_normal(shape) if acc else np.zeros(shape)
        xout[...] = base
        H.applyh(xin, xout, accumulate=acc)
        ref = base + oracle.applyh(T, xin.reshape(-1).astype(np.float64), nb=nb).reshape(shape)
        assert np.abs(xout - ref).max() <= tol * (np.abs(ref).max() + 1), step
    if not acc:
        direct = np.zeros(shape, dtype=xin.dtype)
        H.applyh(np.ascontiguousarray(xin.copy()), direct)
        assert np.array_equal(direct, xout)
