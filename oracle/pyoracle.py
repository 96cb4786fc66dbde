"""TEST INFRASTRUCTURE ONLY: Python access to the CPU oracle.

* `oracle_time_evolution(data)`  -- the C restatement (qd_oracle.c), FP64.
* `ref_time_evolution(data)`     -- the reference's own common/timeEvol.C +
  common/TimeEvolutionMex.C compiled against the shims (oracle/_ref), if built.
* `np_time_evolution(data)`      -- an independent numpy restatement, small
  sizes only, used to cross-check the two above.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use this.
"""
import ctypes as C
import os
import sys
import subprocess
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "quantum-dynamics_b200"))
from qd_b200 import _abi  # noqa: E402  (struct layout of include/qd.h)

ORACLE_SO = os.path.join(HERE, "_build", "libqdoracle.so")
REF_SO = os.path.join(HERE, "_ref", "libqdref.so")

_o = None
_r = None


def build():
    """make -C oracle (restatement always; reference build when its sources
    are present)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _o
    if _o is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        dp = C.POINTER(C.c_double)
        L.qdo_time_evolution.argtypes = [C.POINTER(_abi.QdData), dp, dp]
        L.qdo_time_evolution.restype = C.c_int
        L.qdo_fft2d.argtypes = [dp, C.c_int, C.c_int, C.c_int]
        L.qdo_gradient3d.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                     dp, dp, dp, C.c_int]
        L.qdo_momentum.argtypes = [dp, C.c_int, C.c_double]
        L.qdo_num_threads.restype = C.c_int
        L.qdo_create.argtypes = [C.POINTER(_abi.QdData)]
        L.qdo_create.restype = C.c_void_p
        L.qdo_destroy.argtypes = [C.c_void_p]
        L.qdo_run_steps.argtypes = [C.c_void_p, C.c_int, dp, dp]
        L.qdo_run_steps.restype = C.c_int
        L.qdo_energies.argtypes = [C.POINTER(_abi.QdData), dp]
        L.qdo_energies.restype = C.c_int
        _o = L
    return _o


def ref_available():
    return os.path.exists(REF_SO)


def ref_lib():
    global _r
    if _r is None:
        L = C.CDLL(REF_SO)
        L.qdref_time_evolution.argtypes = [C.POINTER(_abi.QdData), C.c_int, C.c_char_p, C.c_int]
        L.qdref_time_evolution.restype = C.c_int
        _r = L
    return _r


def _dp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def oracle_time_evolution(data, norms=False, energies=False):
    """Propagate data.time.total_steps steps in place with the C oracle.
    Returns (norms[steps], energies[steps, 4]) when requested."""
    n = int(data.time.total_steps)
    nb = np.zeros(n) if norms else None
    eb = np.zeros((n, 4)) if energies else None
    d = _abi.to_c(data)
    rc = lib().qdo_time_evolution(C.byref(d), _dp(nb), _dp(eb))
    if rc != 0:
        raise RuntimeError(f"oracle failed: {rc}")
    _abi.from_c(d, data)
    return nb, eb


def oracle_energies(data):
    """(E_kin, E_rot, E_pot, E_total) of data.psi by the reference's formulas."""
    out = np.zeros(4)
    d = _abi.to_c(data)
    if lib().qdo_energies(C.byref(d), _dp(out)) != 0:
        raise RuntimeError("oracle energies failed")
    return out


def ref_time_evolution(data, verbose=False):
    """Run the reference's own MEX entry point (built in oracle/_ref)."""
    d = _abi.to_c(data)
    err = C.create_string_buffer(1024)
    rc = ref_lib().qdref_time_evolution(C.byref(d), int(verbose), err, 1024)
    if rc != 0:
        raise RuntimeError("reference failed: " + err.value.decode())
    _abi.from_c(d, data)


def fft2d(a, sign):
    """Oracle 2-D DFT of a (n2, n1) complex128 C array (column-major n1 x n2)."""
    a = np.ascontiguousarray(a, dtype=np.complex128).copy()
    lib().qdo_fft2d(_dp(a.view(np.float64)), a.shape[1], a.shape[0], sign)
    return a


# ---------------------------------------------------------------------------
# Independent numpy restatement (small cases)
# ---------------------------------------------------------------------------

def np_time_evolution(data):
    """numpy restatement of common/timeEvol.C:619-685 (FP64).  psi layout
    (n_theta, n2, n1).  Uses numpy.fft; the asin-based complex sqrt of
    common/complex.h:149-159 is replaced by numpy's principal sqrt, which
    differs only on the negative real axis."""
    r1, r2, th = data.r1, data.r2, data.theta
    n1, n2, nth, nl = int(r1.n), int(r2.n), int(th.n), int(th.m) + 1
    dt = float(data.time.time_step)

    def mom(n, dr):
        L = n * dr
        k = np.concatenate([np.arange(0, n // 2 + 1), np.arange(-n // 2 + 1, 0)])
        return 2 * np.pi / L * k

    T1 = mom(n1, r1.dr) ** 2 / (2 * r1.mass)
    T2 = mom(n2, r2.dr) ** 2 / (2 * r2.mass)
    I1 = 1.0 / (2 * r1.mass * r1.r ** 2)
    I2 = 1.0 / (2 * r2.mass * r2.r ** 2)
    l = np.arange(nl)
    expV = np.exp(-1j * dt * data.pot)
    rot = np.exp(-1j * dt / 2 * (l * (l + 1))[:, None, None] * (I1[None, None, :] + I2[None, :, None]))
    kin = np.exp(-1j * dt * (T1[None, :] + T2[:, None])) / (n1 * n2)
    P = th.legendre                              # (nth, nl): P[k, l]
    WP = (l + 0.5)[None, :] * th.w[:, None] * P  # (nth, nl)
    d = None
    if data.dump1.dump is not None and data.dump2.dump is not None:
        d = data.dump2.dump[:, None] * data.dump1.dump[None, :]
    crp = data.CRP
    ne = int(crp.n_energies)
    fai = np.zeros((ne, nth, n1), complex)
    dfai = np.zeros((ne, nth, n1), complex)
    n2p = int(crp.n_dividing_surface) - 1
    npts = int(crp.n_gradient_points)
    coef = {3: ([1], 2), 5: ([8, -1], 12), 7: ([45, -9, 1], 60),
            9: ([672, -168, 32, -3], 840), 11: ([2100, -600, 150, -25, 2], 2520)}[npts]
    psi = data.psi
    n_acc = 0
    for step in range(int(data.time.total_steps)):
        if step == 0 and int(data.time.steps) == 0:
            psi /= np.sqrt(expV)
        psi *= expV
        lpsi = np.einsum("kji,kl->lji", psi, WP)
        lpsi *= rot
        lpsi = np.fft.fft2(lpsi, axes=(1, 2))
        lpsi *= kin[None]
        lpsi = np.fft.ifft2(lpsi, axes=(1, 2)) * (n1 * n2)
        lpsi *= rot
        psi[...] = np.einsum("lji,kl->kji", lpsi, P)
        if d is not None:
            psi *= d[None]
        if crp.calculate_CRP:
            n_acc += 1
            vs = psi[:, n2p, :]
            g = sum(c * (psi[:, n2p + m + 1, :] - psi[:, n2p - m - 1, :])
                    for m, c in enumerate(coef[0])) / (coef[1] * r2.dr)
            et = dt * np.exp(1j * crp.energies * dt * n_acc)
            fai += et[:, None, None] * vs[None]
            dfai += et[:, None, None] * g[None]
        data.time.steps += 1
    if crp.calculate_CRP:
        c3 = np.einsum("eki,eki->ek", np.conj(fai), dfai)
        ce = (th.w[None, :] * c3).sum(1)
        crp.CRP[:] = ce.imag / crp.eta_sq * r1.dr / r2.mass
    return data
