"""Shared test set-up: import paths, the gpu marker, golden-case loaders."""
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "quantum-dynamics_b200")
GOLDEN = os.path.join(REPO, "tests", "golden")
for p in (REPO, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def golden_case(name):
    """Rebuild the input struct of tests/golden/ref_<name>.npz and return
    (data, expected) where expected holds the reference's outputs."""
    from qd_b200.systems import Struct
    z = np.load(os.path.join(GOLDEN, f"ref_{name}.npz"))
    r1 = Struct(n=z["r1"].size, r=z["r1"].copy(), dr=float(z["r1_dr"]), mass=float(z["r1_mass"]),
                r0=0.0, k0=0.0, delta=0.0)
    r2 = Struct(n=z["r2"].size, r=z["r2"].copy(), dr=float(z["r2_dr"]), mass=float(z["r2_mass"]),
                r0=0.0, k0=0.0, delta=0.0)
    theta = Struct(n=z["x"].size, m=int(z["m"]), x=z["x"].copy(), w=z["w"].copy(),
                   legendre=np.ascontiguousarray(z["legendre"]))
    ne = z["energies"].size
    data = Struct(r1=r1, r2=r2, theta=theta, pot=np.ascontiguousarray(z["pot"]),
                  psi=np.ascontiguousarray(z["psi_in"]).copy(),
                  time=Struct(total_steps=int(z["total_steps"]), time_step=float(z["time_step"]),
                              steps=0),
                  options=Struct(wave_to_matlab=None, test_name=name,
                                 steps_to_copy_psi_from_device_to_host=0, precision=0),
                  dump1=Struct(dump=z["dump1"].copy()), dump2=Struct(dump=z["dump2"].copy()),
                  CRP=Struct(n_dividing_surface=int(z["n_dividing_surface"]),
                             n_gradient_points=int(z["n_gradient_points"]), n_energies=ne,
                             calculate_CRP=1, energies=z["energies"].copy(),
                             eta_sq=z["eta_sq"].copy(), CRP=np.zeros(ne)))
    expected = dict(psi=z["psi_out"], crp=z["crp_out"], steps=int(z["steps_out"]))
    return data, expected


GOLDEN_CASES = ["h_h2_16x12x8_p5", "f_h2_20x16x10_p11"]


def have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def qdlib():
    """libqd.so, built in-tree if missing."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("qd_build", os.path.join(PKG, "build.py"))
    qd_build = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(qd_build)
    qd_build.build()
    from qd_b200 import _abi
    return _abi.lib()
