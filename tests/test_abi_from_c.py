"""The C ABI driven from plain C (tests/abi_from_c.c): the program compiles
against include/bsg.h and include/bsg_host.h alone with -Wall -Werror, and on
the GPU its applyH output and eigenvalues are those of the Python engine (same
libraries, bitwise for applyH), of the oracle matvec and of the oracle's dense
diagonalization of the coupled interaction."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from bigstickpublick_b200 import model
import oracle
from oracle import dense_h

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "bigstickpublick_b200")
SRC = os.path.join(ROOT, "tests", "abi_from_c.c")


def _compile(tmp_path):
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    exe = str(tmp_path / "abi_from_c")
    cmd = ["gcc", "-std=c11", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           SRC, "-o", exe, "-L", PKG, "-lbsgpu", "-lbsghost", "-lm", "-Wl,-rpath," + PKG]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def _write_spec(path, spec):
    spe = spec.spe or [0.0] * len(spec.orbits)
    lines = [f"{len(spec.orbits)} {spec.np_} {spec.nn} {spec.jz2} {spec.parity} "
             f"{spec.spe_scale!r} {spec.tbme_scale!r}"]
    lines += [f"{nr} {l} {j2} {w} {float(e)!r}" for (nr, l, j2, w), e in zip(spec.orbits, spe)]
    lines.append(str(len(spec.tbme)))
    lines += [f"{a} {b} {c} {d} {J} {T} {float(v)!r}" for a, b, c, d, J, T, v in spec.tbme]
    path.write_text("\n".join(lines) + "\n")


def _parse(stdout):
    """dim and the eigenvalues (by index) from the program's "dim D" and
    "eval K E" lines."""
    dim, evals = None, {}
    for ln in stdout.splitlines():
        f = ln.split()
        if f and f[0] == "dim":
            dim = int(f[1])
        elif f and f[0] == "eval":
            evals[int(f[1])] = float(f[2])
    return dim, np.array([evals[k] for k in range(len(evals))])


def test_output_parser():
    out = "dim 640\neval 0 -23.153591760000001\neval 1 -22.7033493\niterations 40 converged 1\n"
    dim, ev = _parse(out)
    assert dim == 640 and ev.tolist() == [-23.153591760000001, -22.7033493]


def test_c_caller_builds_against_the_headers(tmp_path):
    exe = _compile(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr
    bad = tmp_path / "bad.txt"
    bad.write_text("3 1 1\n")
    r = subprocess.run([exe, str(bad), str(tmp_path / "out.bin")], capture_output=True, text=True)
    assert r.returncode == 1 and "malformed spec" in r.stderr


def test_c_caller_reports_a_builder_error(tmp_path):
    # more valence protons than proton states: the builder refuses, and the
    # program prints the builder's status and message (no GPU call is made)
    exe = _compile(tmp_path)
    spec = model.sd_model(13, 0, seed=1)
    p = tmp_path / "spec.txt"
    _write_spec(p, spec)
    r = subprocess.run([exe, str(p), str(tmp_path / "out.bin")], capture_output=True, text=True)
    assert r.returncode == 1 and r.stderr.startswith("bsg_host_build: "), r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("name,spec", [
    ("sd 2p2n", model.sd_model(2, 2, seed=1)),
    ("pf 2p1n odd", model.pf_model(2, 1, seed=5, jz2=1)),
], ids=["sd2p2n", "pf2p1n"])
def test_c_caller_matches_python_and_oracle(tmp_path, name, spec):
    from bigstickpublick_b200 import engine
    exe = _compile(tmp_path)
    p = tmp_path / "spec.txt"
    _write_spec(p, spec)
    out = tmp_path / "vout.bin"
    r = subprocess.run([exe, str(p), str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    dim, evals_c = _parse(r.stdout)
    assert evals_c.size == 5
    vout_c = np.fromfile(out, dtype=np.float64)
    assert vout_c.size == dim

    T = model.build_tables(spec)
    assert T.dim == dim
    vin = np.sin(0.1 * np.arange(dim) + 1.0)
    H = engine.Hamiltonian(T)
    vout_py = H.applyh(vin)
    assert np.array_equal(vout_c, vout_py), name
    want = oracle.applyh(T, vin)
    assert np.allclose(vout_c, want, rtol=1e-12, atol=1e-12 * np.abs(want).max()), name

    ev_py, _, _ = H.lanczos(nkeep=5, niter=300)
    assert np.allclose(evals_c, ev_py, rtol=0, atol=1e-10), (evals_c, ev_py)
    Hd, _ = dense_h.dense_h(spec.orbits, spec.np_, spec.nn, spec.jz2, spec.spe, spec.tbme,
                            spec.spe_scale, spec.tbme_scale)
    ev_dense = np.linalg.eigvalsh(Hd)
    # matrix elements are stored in float32 (the reference's hmat arrays)
    tol = 2e-5 * max(1.0, np.abs(ev_dense).max())
    assert abs(evals_c[0] - ev_dense[0]) < tol, (evals_c, ev_dense[:5])
    # the uniform pivot has no overlap with the other time-reversal class at
    # Jz = 0, so the states found need not be the five lowest; each is still
    # an eigenvalue of H
    gap = np.abs(evals_c[:, None] - ev_dense[None, :]).min(axis=1)
    assert gap.max() < tol, (evals_c, gap)
