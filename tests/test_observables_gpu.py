"""J and T of Lanczos eigenstates (<J^2>, <T^2> with the operators of
model.jsq_spec / model.tsq_spec applied by the engine) against the labels the
reference prints for 25Mg (examples/sd/output/mg25ref.res, mg25alt.res)."""
import json
import os

import numpy as np
import pytest

from bigstickpublick_b200 import model

pytestmark = pytest.mark.gpu
GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "mg25.json")))


@pytest.mark.parametrize("run", ["mg25ref", "mg25alt"])
def test_mg25_j_and_t_equal_reference_labels(run):
    from bigstickpublick_b200.engine import Hamiltonian, angular_momentum_isospin
    r = GOLD["runs"][run]
    ss, ts = model.ModelSpec.scaling(*r["scaling"])
    orbits = [tuple(o) for o in GOLD["orbits"]]
    spec = model.ModelSpec(orbits, r["np"], r["nn"], r["jz2"], 1, GOLD["spe"], [tuple(t) for t in GOLD["tbme"]], ss, ts)
    H = Hamiltonian(model.build_tables(spec))
    ev, vecs, rep = H.lanczos(nkeep=10, niter=400, matvec_prec=8, want_vectors=True, converge_tol=1e-12)
    H.close()
    gold_e = np.array([s["E"] for s in r["states"]])
    assert np.abs(ev - gold_e).max() < 1.5e-5
    J, T = angular_momentum_isospin(spec, vecs)
    gold_j = np.array([s["J"] for s in r["states"]])
    gold_t = np.array([s["T"] for s in r["states"]])
    # states 7 and 8 of mg25alt lie 0.6 keV apart with different J: their
    # Lanczos vectors converge more slowly, hence the looser bound there
    tol = 2e-2 if run == "mg25alt" else 1e-3
    assert np.abs(J - gold_j).max() < tol, (J, gold_j)
    assert np.abs(T - gold_t).max() < 1e-3, (T, gold_t)
