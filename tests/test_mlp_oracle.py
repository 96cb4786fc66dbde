"""CPU checks of the FP64 restatement of the PES surrogate network
(oracle/mlp_oracle.py), the checker of the GPU training kernels."""
import numpy as np

from oracle import mlp_oracle as M
from qd_b200 import systems as S
from qd_b200.surrogate import training_set


def _net(seed=3):
    rng = np.random.default_rng(seed)
    w = rng.uniform(-0.3, 0.3, M.NPARAM).astype(np.float32)
    norm = np.array([0.1, 0.2, 0.05, 0.2, 0.3, 0.1, 0.01, 0.05], dtype=np.float32)
    return w, norm


def _data(n=40, seed=5):
    m = np.array([18.9984, 1.00783, 1.00783]) * S.AMU_ME
    return training_set(S.leps_f_h2(), m, n=n, seed=seed)


def test_gradient_matches_finite_differences():
    w, norm = _net()
    r12, r23, r13, V = _data()
    _, g = M.loss_and_grad(w.astype(np.float64), norm, r12, r23, r13, V, quant=False)
    rng = np.random.default_rng(9)
    for i in rng.choice(M.NPARAM, 25, replace=False):
        h = 1e-6
        wp = w.astype(np.float64).copy(); wp[i] += h
        wm = w.astype(np.float64).copy(); wm[i] -= h
        lp, _ = M.loss_and_grad(wp, norm, r12, r23, r13, V, quant=False)
        lm, _ = M.loss_and_grad(wm, norm, r12, r23, r13, V, quant=False)
        assert abs((lp - lm) / (2 * h) - g[i]) < 1e-6 * max(1.0, abs(g[i]))


def test_features_symmetric_under_exchange_of_the_diatom_atoms():
    w, norm = _net()
    r12, r23, r13, _ = _data()
    a = M.predict(w, norm, r12, r23, r13)
    b = M.predict(w, norm, r13, r23, r12)
    assert np.array_equal(a, b)


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.1415927], dtype=np.float32)
    q = M.bf16(x)
    assert q[0] == 1.0 and q[1] == 1.0 and q[2] == 1.0078125
    assert abs(q[3] + 3.140625) < 1e-12


def test_training_set_respects_cut_and_mask():
    r12, r23, r13, V = _data(n=2000)
    assert r12.size == 2000
    assert (np.minimum(np.minimum(r12, r23), r13) > 0.4).all()
    assert (V < 3.0 / S.HARTREE_EV).all()
