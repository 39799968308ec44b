"""Jump tables generated on the GPU (bsg_jumpgen_*) against the host table
builder's, byte for byte: one-body and two-body jumps of every sector jump in
the builder's order, the PN bundles' ranges after the reference's shell sort
(sort1bjumps with its stride table), and the one-body density jumps."""
import numpy as np
import pytest

from bigstickpublick_b200 import model
from bigstickpublick_b200.jumps import device_jumps

pytestmark = pytest.mark.gpu

KEYS = [p + k for p in ("p1b_", "n1b_") for k in ("isd", "fsd", "cop", "dop", "phase")] + \
       [p + k for p in ("p2b_", "n2b_") for k in ("isd", "fsd", "op", "phase")]

CASES = [
    ("sd 2p2n", lambda: model.sd_model(2, 2, seed=1)),
    ("sd 3p2n jz=1", lambda: model.sd_model(3, 2, seed=3, jz2=1)),
    ("sd 0p3n jz=3", lambda: model.sd_model(0, 3, seed=4, jz2=3)),
    ("sd 1p1n", lambda: model.sd_model(1, 1, seed=11)),
    ("pf 2p2n", lambda: model.pf_model(2, 2, seed=5)),
    ("sd 6p6n", lambda: model.sd_model(6, 6, seed=2)),
    ("pf 4p4n", lambda: model.pf_model(4, 4, seed=3)),
    ("pf 3p2n jz=1", lambda: model.pf_model(3, 2, seed=7, jz2=1)),
]


@pytest.mark.parametrize("name", [c[0] for c in CASES])
def test_device_jumps_equal_host_tables(name):
    spec = dict(CASES)[name]()
    T = model.build_tables(spec)
    d = device_jumps(T, spec)
    for k in KEYS:
        assert d[k].dtype == T.a[k].dtype, k
        assert np.array_equal(d[k], T.a[k]), (name, k, len(d[k]), len(T.a[k]))
    dens = T.extra["density"]
    for k in ("p1b_isd", "p1b_fsd", "p1b_cop", "p1b_dop", "p1b_phase",
              "n1b_isd", "n1b_fsd", "n1b_cop", "n1b_dop", "n1b_phase"):
        assert np.array_equal(d["density"][k], dens[k]), (name, "density", k)


def test_device_jumps_pf6p6n():
    """The largest configuration: 2,031,840 one-body and 4,250,100 two-body
    jumps per species, the PN ranges sorted on the device."""
    spec = model.pf_model(6, 6, seed=5)
    T = model.build_tables(spec)
    d = device_jumps(T, spec, density=False)
    assert len(d["p1b_isd"]) == 2_031_840 and len(d["n2b_isd"]) == 4_250_100
    for k in KEYS:
        assert np.array_equal(d[k], T.a[k]), k
