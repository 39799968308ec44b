"""The oracle's own consistency: serial restatement vs its OpenMP baseline,
block layout vs separate vectors, operation counts."""
import numpy as np

from bigstickpublick_b200 import model
import oracle


def test_serial_equals_openmp_and_block_layout():
    T = model.build_tables(model.sd_model(3, 3, seed=5))
    rng = np.random.default_rng(0)
    nb = 3
    v = rng.standard_normal((T.dim, nb))
    blk = oracle.applyh(T, v.reshape(-1), nb=nb).reshape(T.dim, nb)
    omp = oracle.applyh_omp(T, v.reshape(-1), nb=nb, nthreads=4).reshape(T.dim, nb)
    for k in range(nb):
        single = oracle.applyh(T, np.ascontiguousarray(v[:, k]))
        assert np.abs(blk[:, k] - single).max() < 1e-12 * np.abs(single).max()
    assert np.abs(blk - omp).max() < 1e-12 * np.abs(blk).max()


def test_fp32_path_close_to_fp64():
    T = model.build_tables(model.pf_model(2, 2, seed=5))
    v = np.random.default_rng(1).standard_normal(T.dim)
    r64 = oracle.applyh(T, v)
    r32 = oracle.applyh(T, v.astype(np.float32))
    assert np.abs(r32 - r64).max() / np.abs(r64).max() < 1e-5


def test_op_counts_sd6p6n():
    T = model.build_tables(model.sd_model(6, 6, seed=2))
    spe, pp, nn, pn = oracle.count_ops(T)
    assert spe == 0 and pp == nn and pn == 26323832
