"""Regenerate the golden fixtures in tests/golden/ (run where the reference
checkout is present, its location in QD_REFERENCE_DIR):

    QD_REFERENCE_DIR=<checkout> python tests/golden/make_golden.py

* grids/<n>-LegendreGauss.grids   copied verbatim from the reference's
  GaussLegendre/ tables (32-digit Gauss-Legendre nodes and weights).
* ref_<name>.npz                  input struct and outputs of the reference's
  own CPU propagator (common/timeEvol.C via common/TimeEvolutionMex.C,
  compiled unmodified against the shims in oracle/ref_shim) on small cases.
"""
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "quantum-dynamics_b200"))
from qd_b200 import systems as S  # noqa: E402
from oracle import pyoracle as O  # noqa: E402

REF = os.environ.get("QD_REFERENCE_DIR", "")
GRIDS_N = (8, 12, 40, 41, 64, 128)

# small cases: (name, builder kwargs)
CASES = [
    ("h_h2_16x12x8_p5", dict(system="h+h2", n1=16, n2=12, n_theta=8, m=6, total_steps=30,
                            n_energies=11, n_gradient_points=5, R=(0.5, 12.0), r=(0.4, 8.0),
                            r_surface=4.5)),
    ("f_h2_20x16x10_p11", dict(system="f+h2", n1=20, n2=16, n_theta=10, m=9, total_steps=25,
                              n_energies=9, n_gradient_points=11, R=(1.0, 12.0),
                              r=(0.5, 8.0), r_surface=4.0)),
]

FIELDS_IN = ["pot", "psi"]


def save_case(name, kw):
    base = S.build_case(**kw)
    data = S.copy_case(base)
    O.ref_time_evolution(data)
    out = dict(
        kw=repr(kw),
        r1=base.r1.r, r1_dr=base.r1.dr, r1_mass=base.r1.mass,
        r2=base.r2.r, r2_dr=base.r2.dr, r2_mass=base.r2.mass,
        x=base.theta.x, w=base.theta.w, m=base.theta.m, legendre=base.theta.legendre,
        pot=base.pot, psi_in=base.psi, dump1=base.dump1.dump, dump2=base.dump2.dump,
        time_step=base.time.time_step, total_steps=base.time.total_steps,
        n_dividing_surface=base.CRP.n_dividing_surface,
        n_gradient_points=base.CRP.n_gradient_points,
        energies=base.CRP.energies, eta_sq=base.CRP.eta_sq,
        psi_out=data.psi, crp_out=data.CRP.CRP, steps_out=data.time.steps)
    np.savez_compressed(os.path.join(HERE, f"ref_{name}.npz"), **out)
    print("wrote", name, "max|P| =", np.abs(data.CRP.CRP).max())


def main():
    if not REF or not os.path.isdir(REF):
        sys.exit("set QD_REFERENCE_DIR to the reference checkout (now: %r)" % REF)
    os.makedirs(os.path.join(HERE, "grids"), exist_ok=True)
    for n in GRIDS_N:
        src = os.path.join(REF, "GaussLegendre", f"{n}-LegendreGauss.grids")
        shutil.copy(src, os.path.join(HERE, "grids", os.path.basename(src)))
    O.build()
    if not O.ref_available():
        sys.exit("oracle/_ref/libqdref.so was not built")
    for name, kw in CASES:
        save_case(name, kw)


if __name__ == "__main__":
    main()
