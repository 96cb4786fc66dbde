"""The run-file driver bin/qd_run (cli/qd_run.cpp): parsing on CPU (--check
touches no device), and on the GPU a whole run from a run file against the
same case built by qd_b200.systems and propagated through the Python mirror of
the MEX entry point."""
import json
import os
import subprocess

import numpy as np
import pytest

from qd_b200 import systems as S

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(os.path.dirname(HERE), "quantum-dynamics_b200", "bin", "qd_run")

SMALL = """# F + H2, a small grid
r1.n = 32
r2.n = 24
theta.n = 12
theta.m = 11
time.total_steps = 40
CRP.n_energies = 9
CRP.n_gradient_points = 5
options.precision = {prec}
options.steps_to_copy_psi_from_device_to_host = {every}
output.crp = {crp}
output.psi = {psi}
"""


def _run(args, **kw):
    if not os.path.exists(BIN):
        pytest.skip("bin/qd_run is not built (quantum-dynamics_b200/build.py)")
    return subprocess.run([BIN] + args, capture_output=True, text=True, timeout=600, **kw)


def _write(tmp_path, text):
    p = tmp_path / "case.run"
    p.write_text(text)
    return str(p)


def test_check_resolves_the_run_file(tmp_path):
    f = _write(tmp_path, SMALL.format(prec="fp32", every=10, crp="c.csv", psi="p.bin"))
    r = _run([f, "--check"])
    assert r.returncode == 0, r.stderr
    d = json.loads(r.stdout)
    base = S.build_case("f+h2", 32, 24, 12, m=11, total_steps=40, n_energies=9,
                        n_gradient_points=5)
    assert d["r1"]["n"] == 32 and d["theta"] == {"n": 12, "m": 11, "grids": ""}
    assert d["r1"]["dr"] == base.r1.dr and d["r2"]["dr"] == base.r2.dr
    assert abs(d["r1"]["mass"] - base.r1.mass) <= 1e-12 * base.r1.mass
    assert abs(d["r1"]["k0"] - base.r1.k0) <= 1e-12 * base.r1.k0
    assert d["CRP"]["n_dividing_surface"] == base.CRP.n_dividing_surface
    assert d["precision"] == "fp32" and d["steps_to_copy_psi_from_device_to_host"] == 10


@pytest.mark.parametrize("line,msg", [("bogus = 1", "unknown key"),
                                      ("r1.n = 12.5", "integer"),
                                      ("r1.n = x", "not a number"),
                                      ("masses = 1 2", "needs 3 numbers"),
                                      ("options.precision = fp16", "fp64 or fp32"),
                                      ("no equals sign", "expected key = value")])
def test_bad_run_files_are_rejected(tmp_path, line, msg):
    f = _write(tmp_path, "r2.n = 24\n" + line + "\n")
    r = _run([f, "--check"])
    assert r.returncode == 2
    assert msg in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_run_file_matches_python_case(tmp_path, prec):
    crp, psi = tmp_path / "crp.csv", tmp_path / "psi.bin"
    f = _write(tmp_path, SMALL.format(prec=prec, every=20, crp=crp, psi=psi))
    r = _run([f])
    assert r.returncode == 0, r.stdout + r.stderr
    assert "step 20 norm" in r.stdout and "step 40 norm" in r.stdout
    from qd_b200 import TimeEvolutionMexCUDA
    base = S.build_case("f+h2", 32, 24, 12, m=11, total_steps=40, n_energies=9,
                        n_gradient_points=5, precision=0 if prec == "fp64" else 1)
    TimeEvolutionMexCUDA(base)
    # the inputs agree to rounding (host and GPU set-up); complex64 arithmetic
    # may round such inputs one ulp apart
    psi_tol, crp_tol = (1e-8, 1e-8) if prec == "fp64" else (1e-5, 1e-6)
    got = np.loadtxt(crp, delimiter=",", skiprows=1)
    assert np.abs(got[:, 1] - base.CRP.energies).max() < 1e-12
    assert np.abs(got[:, 2] - base.CRP.eta_sq).max() < 1e-12 * base.CRP.eta_sq.max()
    assert np.abs(got[:, 3] - base.CRP.CRP).max() < crp_tol
    p = np.fromfile(psi, dtype=np.complex128).reshape(base.psi.shape)
    assert np.abs(p - base.psi).max() < psi_tol * np.abs(base.psi).max()
