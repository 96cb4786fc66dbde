"""Host-side mirror of the reference's propagator entry points.

`TimeEvolutionMexCUDA(data)` / `TimeEvolutionMex(data)` take the same struct
as the reference's MEX functions (common-cuda/TimeEvolutionMexCUDA.C:20-83,
common/TimeEvolutionMex.C:18-78) -- fields r1, r2, theta, pot, psi, time,
options, dump1, dump2, CRP -- and, like them, propagate
`time.total_steps` steps updating `psi`, `time.steps` and `CRP.CRP` in place.
Both run on the GPU through libqd.so's C ABI; errors the reference reports
through insist()/mexErrMsgTxt raise `QdError` here.

`Propagator` keeps the wavepacket on the device across calls (the C ABI's
handle API).
"""
import ctypes as C
import numpy as np

from . import _abi
from ._abi import check, lib


def _check_layout(data):
    n1, n2, nth = int(data.r1.n), int(data.r2.n), int(data.theta.n)
    m = int(data.theta.m)
    if data.psi.dtype != np.complex128 or data.psi.shape != (nth, n2, n1) or \
            not data.psi.flags.c_contiguous:
        raise ValueError(f"psi must be C-contiguous complex128 of shape {(nth, n2, n1)}")
    if data.pot.dtype != np.float64 or data.pot.shape != (nth, n2, n1):
        raise ValueError(f"pot must be float64 of shape {(nth, n2, n1)}")
    if data.theta.legendre.shape != (nth, m + 1):
        raise ValueError(f"theta.legendre must have shape {(nth, m + 1)} "
                         "(the (m+1) x n Matlab matrix, column-major)")


def TimeEvolutionMexCUDA(data):
    """Propagate `data.time.total_steps` steps on the GPU, in place."""
    _check_layout(data)
    d = _abi.to_c(data)
    check(lib().qd_time_evolution(C.byref(d)))
    _abi.from_c(d, data)
    return data


# The CPU MEX of the reference has the same interface; here both run on the GPU.
TimeEvolutionMex = TimeEvolutionMexCUDA


class Propagator:
    """Device-resident propagation (qd_create / qd_propagate / qd_download)."""

    def __init__(self, data):
        _check_layout(data)
        self.data = data
        self._c = _abi.to_c(data)
        self._h = C.c_void_p()
        check(lib().qd_create(C.byref(self._c), C.byref(self._h)))

    def propagate(self, n_steps):
        check(lib().qd_propagate(self._h, int(n_steps)))
        return self

    def propagate_timed(self, n_steps, flush_bytes=0):
        """Propagate and return the device time in ms (CUDA events on the
        library's stream; optional L2 flush between steps, not timed)."""
        ms = C.c_double()
        check(lib().qd_propagate_timed(self._h, int(n_steps), int(flush_bytes), C.byref(ms)))
        return ms.value

    def psi(self):
        out = np.empty_like(self.data.psi)
        check(lib().qd_get_psi(self._h, out.ctypes.data_as(_abi.c_double_p)))
        return out

    def crp(self):
        out = np.empty(int(self.data.CRP.n_energies))
        check(lib().qd_get_crp(self._h, out.ctypes.data_as(_abi.c_double_p)))
        return out

    def norms(self, n):
        out = np.empty(int(n))
        check(lib().qd_get_norms(self._h, out.ctypes.data_as(_abi.c_double_p), int(n)))
        return out

    @property
    def steps(self):
        s = C.c_int32()
        check(lib().qd_steps(self._h, C.byref(s)))
        return s.value

    def download(self):
        """Write psi, time.steps and CRP.CRP back into `data`."""
        check(lib().qd_download(self._h))
        self.data.time.steps = self.steps
        return self.data

    def energies(self):
        out = np.empty(4)
        check(lib().qd_energies(self._h, out.ctypes.data_as(_abi.c_double_p)))
        return out

    def checkpoint(self, path):
        check(lib().qd_checkpoint(self._h, str(path).encode()))

    def restore(self, path):
        check(lib().qd_restore(self._h, str(path).encode()))

    def close(self):
        if self._h:
            lib().qd_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def legendre_matrix_gpu(n, m, x):
    """theta.legendre ((n, m+1) C array) computed on the GPU in FP64."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty((n, m + 1))
    check(lib().qd_legendre_matrix(int(n), int(m), x.ctypes.data_as(_abi.c_double_p),
                                   out.ctypes.data_as(_abi.c_double_p)))
    return out


def read_grids(directory, n):
    """Gauss-Legendre nodes/weights from a .grids file via the C ABI."""
    x = np.empty(n)
    w = np.empty(n)
    check(lib().qd_read_grids(str(directory).encode(), int(n),
                              x.ctypes.data_as(_abi.c_double_p),
                              w.ctypes.data_as(_abi.c_double_p)))
    return x, w


def kernel_launch_count():
    return int(lib().qd_kernel_launch_count())


def set_device(device):
    """CUDA device for the calling thread's later library calls."""
    check(lib().qd_set_device(int(device)))
