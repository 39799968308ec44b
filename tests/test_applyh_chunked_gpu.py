"""Host-pointer applyH on outputs of 32 MB and more runs as row-range chunks,
each chunk's output copied back while the next chunks run.  Each output
element is still computed by exactly one row tile, so the result must equal
the device-pointer applyH (one launch over all tiles) bit for bit, in store
and accumulate modes, for dense blocks and the per-column path."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ham():
    from bigstickpublick_b200 import model
    from bigstickpublick_b200.engine import Hamiltonian
    T = model.build_tables(model.pf_model(4, 4, seed=3))
    H = Hamiltonian(T, device=0)
    yield T, H
    H.close()


# (nb, dtype): every case holds at least 32 MB of output at dim 1,963,461
@pytest.mark.parametrize("nb,dt", [(4, np.float64), (8, np.float32), (3, np.float64), (16, np.float32)])
@pytest.mark.parametrize("accumulate", [False, True])
def test_chunked_host_applyh_equals_device_applyh(ham, nb, dt, accumulate):
    import torch
    T, H = ham
    assert T.dim * nb * np.dtype(dt).itemsize >= 32 << 20
    rng = np.random.default_rng(nb + 10 * accumulate)
    vin = rng.standard_normal((T.dim, nb)).astype(dt)
    vout0 = rng.standard_normal((T.dim, nb)).astype(dt) if accumulate else None
    host = H.applyh(vin, None if vout0 is None else vout0.copy(), accumulate=accumulate)
    dvin = torch.from_numpy(vin).cuda()
    dvout = torch.from_numpy(vout0).cuda() if accumulate else None
    dev = H.applyh(dvin, dvout, accumulate=accumulate)
    torch.cuda.synchronize()
    assert np.array_equal(host, dev.cpu().numpy())
