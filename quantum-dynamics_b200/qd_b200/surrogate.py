"""Learned PES surrogate (qd_mlp_* of libqd.so): a permutation-symmetric MLP
trained on geometries that the plain PES labels, evaluated on the GPU, with the
plain PES as its judge (|dV| on the grid, |dP(E)|) and its fallback.

No counterpart in the reference, whose Matlab drivers evaluate the PES routine
at every grid point (H3/H3PESJacobi.m:5-27).

    sur = Surrogate(seed=12345)
    r12, r23, r13, V = training_set(pes, masses, n=200000)
    sur.fit(r12, r23, r13, V)                   # 60000 Adam steps
    pot = sur.potential(R, r, x, masses)          # the Jacobi grid, on the GPU
"""
import ctypes as C
import math

import numpy as np

from . import _abi
from ._abi import check, lib
from .systems import HARTREE_EV, jacobi_to_internuclear


def _dp(a):
    return a.ctypes.data_as(_abi.c_double_p)


def _as64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Surrogate:
    """One MLP on the current GPU (qd_mlp handle)."""

    def __init__(self, seed=12345):
        h = C.c_void_p()
        check(lib().qd_mlp_create(C.byref(h), seed))
        self._h = h
        self.n_params = int(lib().qd_mlp_n_params())

    def close(self):
        if self._h:
            lib().qd_mlp_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- parameters ---------------------------------------------------------------
    def params(self):
        """(FP32 master weights, standardisation [feature means, stds, V mean, std])."""
        w = np.empty(self.n_params, dtype=np.float32)
        nm = np.empty(8, dtype=np.float32)
        check(lib().qd_mlp_get_params(self._h, w.ctypes.data_as(_abi.c_float_p),
                                      nm.ctypes.data_as(_abi.c_float_p)))
        return w, nm

    def set_params(self, w, norm=None):
        w = np.ascontiguousarray(w, dtype=np.float32)
        nm = None if norm is None else np.ascontiguousarray(norm, dtype=np.float32)
        check(lib().qd_mlp_set_params(self._h, w.ctypes.data_as(_abi.c_float_p),
                                      None if nm is None else nm.ctypes.data_as(_abi.c_float_p)))

    def save(self, path):
        w, nm = self.params()
        np.savez(path, w=w, norm=nm)

    def load(self, path):
        z = np.load(path)
        self.set_params(z["w"], z["norm"])

    # -- training ---------------------------------------------------------------------
    def fit_normalisation(self, r12, r23, r13, V):
        a, b, c, v = (_as64(x) for x in (r12, r23, r13, V))
        check(lib().qd_mlp_fit_normalisation(self._h, a.size, _dp(a), _dp(b), _dp(c), _dp(v)))

    def fit(self, r12, r23, r13, V, steps=60000, batch=4096, lr=2e-3, lr_end=1e-6,
            normalise=True):
        """Adam on the mean squared error of the standardised V; returns the
        mean loss of the last epoch."""
        if normalise:
            self.fit_normalisation(r12, r23, r13, V)
        a, b, c, v = (_as64(x) for x in (r12, r23, r13, V))
        loss = C.c_double()
        check(lib().qd_mlp_train(self._h, a.size, _dp(a), _dp(b), _dp(c), _dp(v), int(steps),
                                 int(batch), lr, lr_end, None, C.byref(loss)))
        return loss.value

    def loss_and_grad(self, r12, r23, r13, V):
        """Loss over all samples and its gradient (no update)."""
        a, b, c, v = (_as64(x) for x in (r12, r23, r13, V))
        g = np.empty(self.n_params, dtype=np.float32)
        loss = C.c_double()
        check(lib().qd_mlp_train(self._h, a.size, _dp(a), _dp(b), _dp(c), _dp(v), 0, 1, 0.0,
                                 0.0, g.ctypes.data_as(_abi.c_float_p), C.byref(loss)))
        return loss.value, g

    # -- evaluation -----------------------------------------------------------------------
    def __call__(self, r12, r23, r13):
        a, b, c = (_as64(x) for x in (r12, r23, r13))
        out = np.empty(a.size)
        check(lib().qd_mlp_eval(self._h, a.size, _dp(a), _dp(b), _dp(c), _dp(out)))
        return out.reshape(np.shape(r12))

    def potential(self, R, r, x, masses, vmax=2.5, rmin=0.4, cap=True):
        """V on the Jacobi grid, shape (n_theta, n_r, n_R), the mapping and the
        mask of qd_potential_jacobi, evaluated on the GPU."""
        R, r, x, m = (_as64(v) for v in (R, r, x, masses))
        a, b, t = _abi.QdRadial(), _abi.QdRadial(), _abi.QdAngle()
        a.n, a.r = R.size, _dp(R)
        b.n, b.r = r.size, _dp(r)
        t.n, t.x = x.size, _dp(x)
        out = np.empty((x.size, r.size, R.size))
        check(lib().qd_mlp_potential(self._h, C.byref(a), C.byref(b), C.byref(t), _dp(m), vmax,
                                     rmin, 1 if cap else 0, _dp(out)))
        return out


def training_set(pes, masses, n=200000, R=(0.5, 12.0), r=(0.4, 8.0), e_cut_ev=3.0, rmin=0.4,
                 seed=12345):
    """n geometries drawn uniformly over the (R, r, cos theta) box of the grid,
    kept where every internuclear distance exceeds rmin and the plain PES is
    below e_cut_ev above the asymptote (V = 0 at atom + diatom(r_e)), labelled
    by the plain PES.  Returns r12, r23, r13, V (bohr, hartree)."""
    rng = np.random.default_rng(seed)
    out = [[], [], [], []]
    have = 0
    while have < n:
        m = 2 * (n - have) + 1024
        Rs = rng.uniform(*R, m)
        rs = rng.uniform(*r, m)
        cs = rng.uniform(-1.0, 1.0, m)
        r12, r13, r23 = jacobi_to_internuclear(Rs, rs, cs, masses)
        ok = (r12 > rmin) & (r13 > rmin) & (r23 > rmin)
        r12, r13, r23 = r12[ok], r13[ok], r23[ok]
        V = pes(r12, r23, r13)
        keep = V < e_cut_ev / HARTREE_EV
        for lst, a in zip(out, (r12, r23, r13, V)):
            lst.append(a[keep])
        have += int(keep.sum())
    return tuple(np.concatenate(lst)[:n] for lst in out)


def judge(surrogate, pes, R, r, x, masses, vmax=2.5, rmin=0.4, e_cut_ev=3.0):
    """|dV| of the surrogate against the plain PES on the Jacobi grid, over the
    points where the plain PES is below e_cut_ev (the region it was trained
    on): (rms, max) in hartree, and both grids."""
    from .systems import potential_on_grid
    plain = potential_on_grid(R, r, x, masses, pes, vmax=vmax, rmin=rmin)
    sur = surrogate.potential(R, r, x, masses, vmax=vmax, rmin=rmin)
    sel = plain < e_cut_ev / HARTREE_EV
    d = np.abs(sur - plain)[sel]
    return float(math.sqrt(np.mean(d * d))), float(d.max()), sur, plain


def potential_with_fallback(surrogate, pes, R, r, x, masses, tol_rms_ev=5e-3, tol_max_ev=5e-2,
                            **kw):
    """The surrogate's grid if its |dV| against the plain PES (judge) is within
    tolerance, else the plain PES's grid.  Returns (pot, used_surrogate, rms, max)."""
    rms, mx, sur, plain = judge(surrogate, pes, R, r, x, masses, **kw)
    ok = rms * HARTREE_EV <= tol_rms_ev and mx * HARTREE_EV <= tol_max_ev
    return (sur if ok else plain), ok, rms, mx
