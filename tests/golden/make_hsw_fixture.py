"""Regenerate tests/golden/hsw_tables.npz from the reference's HSW data files
(run where the reference checkout is present, its location in
QD_REFERENCE_DIR):

    QD_REFERENCE_DIR=<checkout> python tests/golden/make_hsw_fixture.py

The fixture holds the numbers of FH2/HSW/three.param, two.param, so.input and
so.param, in file order, as the arrays qd_hsw_create_from_tables and the
oracle (oracle/hsw_oracle.py) take, so that the GPU tests run where the
reference checkout is absent.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
from oracle.hsw_oracle import read_tables  # noqa: E402

if __name__ == "__main__":
    root = os.environ.get("QD_REFERENCE_DIR", "")
    if not root or not os.path.isdir(os.path.join(root, "FH2", "HSW")):
        sys.exit("set QD_REFERENCE_DIR to the reference checkout (now: %r)" % root)
    t = read_tables(os.path.join(root, "FH2", "HSW"))
    np.savez_compressed(os.path.join(HERE, "hsw_tables.npz"), **t)
    print({k: np.shape(v) for k, v in t.items()})
