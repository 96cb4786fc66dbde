"""Host-side mirror of the reference's propagator entry points.

`TimeEvolutionMexCUDA(data)` / `TimeEvolutionMex(data)` take the same struct
as the reference's MEX functions (common-cuda/TimeEvolutionMexCUDA.C:20-83,
common/TimeEvolutionMex.C:18-78) -- fields r1, r2, theta, pot, psi, time,
options, dump1, dump2, CRP -- and, like them, propagate
`time.total_steps` steps updating `psi`, `time.steps` and `CRP.CRP` in place.
Both run on the GPU through libqd.so's C ABI; errors the reference reports
through insist()/mexErrMsgTxt raise `QdError` here.  Given a list of structs
they propagate them as one batch (same grid; see qd_create_batch).

`Propagator` keeps the wavepacket(s) on the device across calls (the C ABI's
handle API).
"""
import ctypes as C
import os
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


def _c_runs(runs):
    """ctypes array of QdData over a list of structs (keeps the views alive)."""
    for d in runs:
        _check_layout(d)
    views = [_abi.to_c(d) for d in runs]
    arr = (_abi.QdData * len(runs))(*views)
    arr._views = views
    return arr


def TimeEvolutionMexCUDA(data):
    """Propagate `time.total_steps` steps on the GPU, in place.  `data` is one
    struct or a list of structs propagated together as a batch."""
    runs = data if isinstance(data, (list, tuple)) else [data]
    arr = _c_runs(runs)
    rc = lib().qd_time_evolution_batch(arr, len(runs))
    for d, c in zip(runs, arr):      # time.steps also when a progress callback stopped the call
        _abi.from_c(c, d)
    check(rc)
    return data


# The CPU MEX of the reference has the same interface; here both run on the GPU.
TimeEvolutionMex = TimeEvolutionMexCUDA


class Propagator:
    """Device-resident propagation of one struct or a batch of structs
    (qd_create_batch / qd_propagate / qd_download)."""

    def __init__(self, data):
        self.runs = list(data) if isinstance(data, (list, tuple)) else [data]
        self.data = self.runs[0]
        self._c = _c_runs(self.runs)
        self._h = C.c_void_p()
        check(lib().qd_create_batch(self._c, len(self.runs), C.byref(self._h)))

    @property
    def n_runs(self):
        return len(self.runs)

    def propagate(self, n_steps):
        check(lib().qd_propagate(self._h, int(n_steps)))
        return self

    def propagate_timed(self, n_steps, flush_bytes=0):
        """Propagate and return the device time in ms (CUDA events on the
        library's stream; optional L2 flush between steps, not timed)."""
        ms = C.c_double()
        check(lib().qd_propagate_timed(self._h, int(n_steps), int(flush_bytes), C.byref(ms)))
        return ms.value

    def psi(self, run=0):
        out = np.empty_like(self.runs[run].psi)
        check(lib().qd_get_psi_run(self._h, int(run), out.ctypes.data_as(_abi.c_double_p)))
        return out

    def crp(self, run=0):
        out = np.empty(int(self.runs[run].CRP.n_energies))
        check(lib().qd_get_crp_run(self._h, int(run), out.ctypes.data_as(_abi.c_double_p)))
        return out

    def norms(self, n, run=0):
        out = np.empty(int(n))
        check(lib().qd_get_norms_run(self._h, int(run), out.ctypes.data_as(_abi.c_double_p),
                                     int(n)))
        return out

    @property
    def steps(self):
        s = C.c_int32()
        check(lib().qd_steps(self._h, C.byref(s)))
        return s.value

    def download(self):
        """Write psi, time.steps and CRP.CRP back into the struct(s)."""
        check(lib().qd_download(self._h))
        for d in self.runs:
            d.time.steps = self.steps
        return self.data

    def energies(self, run=0):
        """(E_kin, E_rot, E_pot, E_total) of the current wavepacket, hartree."""
        out = np.empty(4)
        check(lib().qd_energies_run(self._h, int(run), out.ctypes.data_as(_abi.c_double_p)))
        return out

    def set_energy_interval(self, every):
        """Energies inside the propagation on every step whose count is a
        multiple of `every` (0: off); read them with energy_log()."""
        check(lib().qd_set_energy_interval(self._h, int(every)))
        return self

    def energy_log(self, run=0, cap=1 << 20):
        """Recorded energies of one run: array (n, 5) of step, E_kin, E_rot,
        E_pot, E_total (hartree), oldest first."""
        out = np.empty((int(cap), 5))
        n = C.c_int32()
        check(lib().qd_get_energy_log_run(self._h, int(run), out.ctypes.data_as(_abi.c_double_p),
                                          int(cap), C.byref(n)))
        return out[:n.value].copy()

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


def _grid_structs(R, r, x):
    R = np.ascontiguousarray(R, dtype=np.float64)
    r = np.ascontiguousarray(r, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    a, b, t = _abi.QdRadial(), _abi.QdRadial(), _abi.QdAngle()
    a.n, a.r = R.size, R.ctypes.data_as(_abi.c_double_p)
    b.n, b.r = r.size, r.ctypes.data_as(_abi.c_double_p)
    t.n, t.x = x.size, x.ctypes.data_as(_abi.c_double_p)
    return (a, b, t), (R, r, x)


def potential_jacobi(R, r, x, masses, pes, vmax=2.5, rmin=0.4, cap=True):
    """V on the Jacobi grid (shape (n_theta, n_r, n_R)) through the PES
    callback convention of the reference's PES MEX functions: `pes(r12, r23,
    r13)` gets the three internuclear distances of every point with all of them
    > rmin (one call) and returns V; the others get vmax (H3/H3PESJacobi.m)."""
    (a, b, t), keep = _grid_structs(R, r, x)
    m = np.ascontiguousarray(masses, dtype=np.float64)
    out = np.empty((t.n, b.n, a.n))

    def cb(n, p12, p23, p13, pv, ctx):
        try:
            r12 = np.ctypeslib.as_array(p12, (n,))
            r23 = np.ctypeslib.as_array(p23, (n,))
            r13 = np.ctypeslib.as_array(p13, (n,))
            np.ctypeslib.as_array(pv, (n,))[:] = pes(r12, r23, r13)
            return 0
        except Exception:
            return 1
    fn = _abi.PES_FN(cb)
    check(lib().qd_potential_jacobi(C.byref(a), C.byref(b), C.byref(t),
                                    m.ctypes.data_as(_abi.c_double_p), fn, None, vmax, rmin,
                                    1 if cap else 0, out.ctypes.data_as(_abi.c_double_p)))
    return out


def leps_params(pes):
    """qd_leps of a systems.LEPS surface (atomic units)."""
    p = _abi.QdLeps()
    for name in ("ab", "bc", "ac"):
        d = getattr(pes, name)
        q = getattr(p, name)
        q.de, q.beta, q.re, q.sato = d.de, d.beta, d.re, d.sato
    return p


def potential_leps_gpu(R, r, x, masses, pes, vmax=2.5, rmin=0.4, cap=True):
    """The extended-LEPS surface `pes` (a systems.LEPS) on the Jacobi grid,
    evaluated on the GPU in FP64 (qd_potential_leps)."""
    (a, b, t), keep = _grid_structs(R, r, x)
    m = np.ascontiguousarray(masses, dtype=np.float64)
    out = np.empty((t.n, b.n, a.n))
    p = leps_params(pes)
    check(lib().qd_potential_leps(C.byref(a), C.byref(b), C.byref(t),
                                  m.ctypes.data_as(_abi.c_double_p), C.byref(p), vmax, rmin,
                                  1 if cap else 0, out.ctypes.data_as(_abi.c_double_p)))
    return out


def bkmp2_gpu(r1, r2, r3):
    """The BKMP2 H3 surface (qd_bkmp2_eval, the MEX value of
    H3/BKMP2Mex.C in hartree) at internuclear distances in bohr."""
    a, b, c = np.broadcast_arrays(*(np.asarray(v, dtype=np.float64) for v in (r1, r2, r3)))
    shape = a.shape
    a, b, c = (np.ascontiguousarray(v).ravel() for v in (a, b, c))
    out = np.empty(a.size)
    check(lib().qd_bkmp2_eval(a.size, _abi._ptr(a), _abi._ptr(b), _abi._ptr(c), _abi._ptr(out)))
    return out.reshape(shape)


def potential_bkmp2_gpu(R, r, x, masses, vmax=2.5, rmin=0.4, cap=True):
    """BKMP2 on the Jacobi grid (shape (n_theta, n_r, n_R)), shifted by
    -vH2Min as H3/H3PESBKMP2.m does (qd_potential_bkmp2)."""
    (ga, gb, gt), keep = _grid_structs(R, r, x)
    m = np.ascontiguousarray(masses, dtype=np.float64)
    out = np.empty((gt.n, gb.n, ga.n))
    check(lib().qd_potential_bkmp2(C.byref(ga), C.byref(gb), C.byref(gt),
                                   m.ctypes.data_as(_abi.c_double_p), vmax, rmin,
                                   1 if cap else 0, out.ctypes.data_as(_abi.c_double_p)))
    return out


class HswSurface:
    """The HSW surface of F + H2 on the GPU (qd_hsw_*; the reference's
    FH2/HSW/hswpot.F + sospline.F behind HSWMex.C).  Build it from the
    reference's data directory (`HswSurface(dir)`, the HSW_DATA_DIR of
    HSWMex.C) or from the file contents as arrays (`HswSurface(tables=...)`
    with keys ix, iy, iz, a, p, x, y, z, so, so_param)."""

    def __init__(self, data_dir=None, tables=None):
        self._h = C.c_void_p()
        if tables is None:
            if data_dir is None:
                raise ValueError("need a data directory or tables")
            check(lib().qd_hsw_create(os.fsencode(data_dir), C.byref(self._h)))
            return
        t = {k: np.asarray(v) for k, v in tables.items()}
        ix, iy, iz = (np.ascontiguousarray(t[k], dtype=np.int32) for k in ("ix", "iy", "iz"))
        a = np.ascontiguousarray(t["a"], dtype=np.float64)
        pp = np.ascontiguousarray(t["p"], dtype=np.float64)
        x, y, z = (np.ascontiguousarray(t[k], dtype=np.float64) for k in ("x", "y", "z"))
        so = np.ascontiguousarray(t["so"], dtype=np.float64)
        sp = np.ascontiguousarray(t["so_param"], dtype=np.float64)
        if so.shape != (x.size, y.size, z.size) or pp.size < 12 or sp.size < 3:
            raise ValueError("inconsistent HSW tables")
        i32 = _abi.c_int32_p
        check(lib().qd_hsw_create_from_tables(
            a.size, ix.ctypes.data_as(i32), iy.ctypes.data_as(i32), iz.ctypes.data_as(i32),
            _abi._ptr(a), _abi._ptr(pp), x.size, y.size, z.size, _abi._ptr(x), _abi._ptr(y),
            _abi._ptr(z), _abi._ptr(so), _abi._ptr(sp), C.byref(self._h)))

    def __call__(self, r_fh1, r_hh, r_fh2):
        """V (hartree) at internuclear distances (bohr), the argument order of
        the reference's pot(): r(F-H1), r(H1-H2), r(F-H2)."""
        a, b, c = np.broadcast_arrays(*(np.asarray(v, dtype=np.float64) for v in (r_fh1, r_hh, r_fh2)))
        a, b, c = (np.ascontiguousarray(v).ravel() for v in (a, b, c))
        out = np.empty(a.size)
        check(lib().qd_hsw_eval(self._h, a.size, _abi._ptr(a), _abi._ptr(b), _abi._ptr(c),
                                _abi._ptr(out)))
        return out.reshape(np.shape(np.broadcast_arrays(r_fh1, r_hh, r_fh2)[0]))

    def potential(self, R, r, x, masses, vmax=2.5, rmin=0.4, cap=True):
        """The surface on the Jacobi grid (shape (n_theta, n_r, n_R)), the
        mapping and masking of potential_jacobi (atom 1 = F)."""
        (ga, gb, gt), keep = _grid_structs(R, r, x)
        m = np.ascontiguousarray(masses, dtype=np.float64)
        out = np.empty((gt.n, gb.n, ga.n))
        check(lib().qd_potential_hsw(C.byref(ga), C.byref(gb), C.byref(gt),
                                     m.ctypes.data_as(_abi.c_double_p), self._h, vmax, rmin,
                                     1 if cap else 0, out.ctypes.data_as(_abi.c_double_p)))
        return out

    def close(self):
        if self._h:
            lib().qd_hsw_destroy(self._h)
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


def _radial(c):
    s = _abi.QdRadial()
    arr = np.ascontiguousarray(c.r, dtype=np.float64)
    s.n, s.r, s.dr, s.mass = int(c.n), _abi._ptr(arr), float(c.dr), float(c.mass)
    s.r0, s.k0, s.delta = float(getattr(c, "r0", 0.0)), float(getattr(c, "k0", 0.0)), \
        float(getattr(c, "delta", 0.0))
    s._keep = arr                                 # the pointer's array lives with the struct
    return s


def init_state_gpu(r1, r2, theta, j0, v0, v_diatom, K=0):
    """(psi, e_vj, phi): the initial wavepacket built on the GPU (qd_init_state);
    v_diatom is the diatom potential on r2.r (hartree)."""
    a, b = _radial(r1), _radial(r2)
    x = np.ascontiguousarray(theta.x, dtype=np.float64)
    t = _abi.QdAngle()
    t.n, t.x = x.size, x.ctypes.data_as(_abi.c_double_p)
    vd = np.ascontiguousarray(v_diatom, dtype=np.float64)
    psi = np.empty((x.size, int(r2.n), int(r1.n)), dtype=np.complex128)
    phi = np.empty(int(r2.n))
    e = C.c_double()
    check(lib().qd_init_state(C.byref(a), C.byref(b), C.byref(t), int(j0), int(v0), int(K),
                              vd.ctypes.data_as(_abi.c_double_p),
                              psi.ctypes.data_as(_abi.c_double_p), C.byref(e),
                              phi.ctypes.data_as(_abi.c_double_p)))
    return psi, e.value, phi


def eta_sq_gpu(r1, e_coll):
    """eta^2 at the collision energies, on the GPU (qd_eta_sq)."""
    a = _radial(r1)
    e = np.ascontiguousarray(e_coll, dtype=np.float64)
    out = np.empty(e.size)
    check(lib().qd_eta_sq(C.byref(a), e.size, e.ctypes.data_as(_abi.c_double_p),
                          out.ctypes.data_as(_abi.c_double_p)))
    return out
