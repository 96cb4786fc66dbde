"""ctypes mirror of include/qd.h (the library's C ABI).

The structs carry the fields of the reference's Matlab struct
(common/MatlabStructures.h:12-157) one for one; see include/qd.h.
"""
import ctypes as C
import os

c_double_p = C.POINTER(C.c_double)
c_int32_p = C.POINTER(C.c_int32)
c_float_p = C.POINTER(C.c_float)

QD_OK = 0
QD_ERR_INVALID = -1
QD_ERR_CUDA = -2
QD_ERR_NOMEM = -3
QD_ERR_PES = -4
QD_ERR_NONFINITE = -5
QD_ERR_UNSUPPORTED = -6
QD_ERR_IO = -7
QD_ERR_DEVICE = -8
QD_ERR_STOPPED = -9

QD_PREC_FP64 = 0
QD_PREC_FP32 = 1

PROGRESS_FN = C.CFUNCTYPE(C.c_int, C.c_int32, C.c_double, c_double_p, C.c_void_p)


class QdRadial(C.Structure):
    _fields_ = [("n", C.c_int32), ("r", c_double_p), ("dr", C.c_double),
                ("mass", C.c_double), ("r0", C.c_double), ("k0", C.c_double),
                ("delta", C.c_double)]


class QdAngle(C.Structure):
    _fields_ = [("n", C.c_int32), ("m", C.c_int32), ("x", c_double_p),
                ("w", c_double_p), ("legendre", c_double_p)]


class QdTime(C.Structure):
    _fields_ = [("total_steps", C.c_int32), ("time_step", C.c_double),
                ("steps", C.c_int32)]


class QdOptions(C.Structure):
    _fields_ = [("wave_to_matlab", C.c_char_p), ("test_name", C.c_char_p),
                ("steps_to_copy_psi_from_device_to_host", C.c_int32),
                ("precision", C.c_int32), ("progress", PROGRESS_FN),
                ("progress_ctx", C.c_void_p)]


class QdDump(C.Structure):
    _fields_ = [("dump", c_double_p)]


class QdCrp(C.Structure):
    _fields_ = [("n_dividing_surface", C.c_int32), ("n_gradient_points", C.c_int32),
                ("n_energies", C.c_int32), ("calculate_CRP", C.c_int32),
                ("energies", c_double_p), ("eta_sq", c_double_p), ("CRP", c_double_p)]


class QdCs(C.Structure):
    _fields_ = [("J", C.c_int32), ("K", C.c_int32)]


class QdData(C.Structure):
    _fields_ = [("r1", QdRadial), ("r2", QdRadial), ("theta", QdAngle),
                ("pot", c_double_p), ("psi", c_double_p), ("time", QdTime),
                ("options", QdOptions), ("dump1", QdDump), ("dump2", QdDump),
                ("CRP", QdCrp), ("cs", QdCs)]


PES_FN = C.CFUNCTYPE(C.c_int, C.c_int64, c_double_p, c_double_p, c_double_p, c_double_p,
                     C.c_void_p)


class QdLepsPair(C.Structure):
    _fields_ = [("de", C.c_double), ("beta", C.c_double), ("re", C.c_double),
                ("sato", C.c_double)]


class QdLeps(C.Structure):
    _fields_ = [("ab", QdLepsPair), ("bc", QdLepsPair), ("ac", QdLepsPair)]


def _ptr(a):
    """double* into a C-contiguous float64 numpy array (None -> NULL)."""
    if a is None:
        return None
    assert a.dtype.name in ("float64", "complex128") and a.flags.c_contiguous, \
        "arrays handed to the C ABI must be C-contiguous float64/complex128"
    return a.ctypes.data_as(c_double_p)


def to_c(data):
    """Build a QdData over the numpy arrays of a `Struct` (see systems.py).

    No copies: psi, CRP.CRP are written in place by the library, and the
    returned struct keeps references to the arrays it points into.
    """
    d = QdData()
    keep = []
    for name in ("r1", "r2"):
        src = getattr(data, name)
        dst = getattr(d, name)
        dst.n = int(src.n)
        dst.r = _ptr(src.r); keep.append(src.r)
        dst.dr = float(src.dr)
        dst.mass = float(src.mass)
        dst.r0 = float(getattr(src, "r0", 0.0))
        dst.k0 = float(getattr(src, "k0", 0.0))
        dst.delta = float(getattr(src, "delta", 0.0))
    th = data.theta
    d.theta.n = int(th.n)
    d.theta.m = int(th.m)
    d.theta.x = _ptr(th.x); d.theta.w = _ptr(th.w); d.theta.legendre = _ptr(th.legendre)
    keep += [th.x, th.w, th.legendre]
    d.pot = _ptr(data.pot); keep.append(data.pot)
    d.psi = _ptr(data.psi); keep.append(data.psi)
    d.time.total_steps = int(data.time.total_steps)
    d.time.time_step = float(data.time.time_step)
    d.time.steps = int(data.time.steps)
    opt = data.options
    d.options.steps_to_copy_psi_from_device_to_host = int(
        getattr(opt, "steps_to_copy_psi_from_device_to_host", 0))
    d.options.precision = int(getattr(opt, "precision", QD_PREC_FP64))
    tn = getattr(opt, "test_name", None)
    if tn:
        b = tn.encode(); keep.append(b); d.options.test_name = b
    cb = getattr(opt, "progress", None)
    if cb is not None:
        d.options.progress = cb; keep.append(cb)
    for name in ("dump1", "dump2"):
        arr = getattr(getattr(data, name), "dump", None)
        getattr(d, name).dump = _ptr(arr)
        keep.append(arr)
    crp = data.CRP
    d.CRP.n_dividing_surface = int(crp.n_dividing_surface)
    d.CRP.n_gradient_points = int(crp.n_gradient_points)
    d.CRP.n_energies = int(crp.n_energies)
    d.CRP.calculate_CRP = int(crp.calculate_CRP)
    d.CRP.energies = _ptr(crp.energies); d.CRP.eta_sq = _ptr(crp.eta_sq)
    d.CRP.CRP = _ptr(crp.CRP)
    keep += [crp.energies, crp.eta_sq, crp.CRP]
    cs = getattr(data, "cs", None)
    d.cs.J = int(getattr(cs, "J", 0)) if cs is not None else 0
    d.cs.K = int(getattr(cs, "K", 0)) if cs is not None else 0
    d._keep = keep
    return d


def from_c(d, data):
    """Copy the scalar in/out fields (time.steps) back into the Struct."""
    data.time.steps = int(d.time.steps)


HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(os.path.dirname(HERE), "lib")
LIB_PATH = os.path.join(LIB_DIR, "libqd.so")

_lib = None


def lib():
    """Load libqd.so (built in-tree by build.py).  Raises if it is missing:
    there is no CPU fallback for the propagator."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"libqd.so not found at {LIB_PATH}: build it with "
            f"`python quantum-dynamics_b200/build.py` (the propagator has no CPU path)")
    L = C.CDLL(LIB_PATH)
    P = C.POINTER
    H = C.c_void_p
    sig = {
        "qd_abi_version": (C.c_int, []),
        "qd_last_error": (C.c_char_p, []),
        "qd_kernel_launch_count": (C.c_int64, []),
        "qd_set_device": (C.c_int, [C.c_int32]),
        "qd_time_evolution": (C.c_int, [P(QdData)]),
        "qd_create": (C.c_int, [P(QdData), P(H)]),
        "qd_destroy": (C.c_int, [H]),
        "qd_propagate": (C.c_int, [H, C.c_int32]),
        "qd_propagate_timed": (C.c_int, [H, C.c_int32, C.c_int64, c_double_p]),
        "qd_get_psi": (C.c_int, [H, c_double_p]),
        "qd_get_crp": (C.c_int, [H, c_double_p]),
        "qd_download": (C.c_int, [H]),
        "qd_get_norms": (C.c_int, [H, c_double_p, C.c_int32]),
        "qd_energies": (C.c_int, [H, c_double_p]),
        "qd_steps": (C.c_int, [H, P(C.c_int32)]),
        "qd_set_profiling": (C.c_int, [H, C.c_int32]),
        "qd_kernel_times": (C.c_int, [H, c_double_p, C.c_int32, P(C.c_int32)]),
        "qd_kernel_choice": (C.c_int, [H, P(C.c_int32)]),
        "qd_checkpoint": (C.c_int, [H, C.c_char_p]),
        "qd_restore": (C.c_int, [H, C.c_char_p]),
        "qd_create_batch": (C.c_int, [P(QdData), C.c_int32, P(H)]),
        "qd_time_evolution_batch": (C.c_int, [P(QdData), C.c_int32]),
        "qd_n_runs": (C.c_int, [H, P(C.c_int32)]),
        "qd_get_psi_run": (C.c_int, [H, C.c_int32, c_double_p]),
        "qd_get_crp_run": (C.c_int, [H, C.c_int32, c_double_p]),
        "qd_get_norms_run": (C.c_int, [H, C.c_int32, c_double_p, C.c_int32]),
        "qd_energies_run": (C.c_int, [H, C.c_int32, c_double_p]),
        "qd_energies_noalloc": (C.c_int, [H, C.c_int32, c_double_p]),
        "qd_set_energy_interval": (C.c_int, [H, C.c_int32]),
        "qd_get_energy_log_run": (C.c_int, [H, C.c_int32, c_double_p, C.c_int32,
                                            P(C.c_int32)]),
        "qd_read_grids": (C.c_int, [C.c_char_p, C.c_int32, c_double_p, c_double_p]),
        "qd_legendre_matrix": (C.c_int, [C.c_int32, C.c_int32, c_double_p, c_double_p]),
        "qd_cs_legendre": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, c_double_p, c_double_p]),
        "qd_init_state": (C.c_int, [P(QdRadial), P(QdRadial), P(QdAngle), C.c_int32,
                                    C.c_int32, C.c_int32, c_double_p, c_double_p, c_double_p,
                                    c_double_p]),
        "qd_eta_sq": (C.c_int, [P(QdRadial), C.c_int32, c_double_p, c_double_p]),
        "qd_mlp_create": (C.c_int, [P(H), C.c_uint64]),
        "qd_mlp_destroy": (C.c_int, [H]),
        "qd_mlp_n_params": (C.c_int32, []),
        "qd_mlp_get_params": (C.c_int, [H, c_float_p, c_float_p]),
        "qd_mlp_set_params": (C.c_int, [H, c_float_p, c_float_p]),
        "qd_mlp_fit_normalisation": (C.c_int, [H, C.c_int64, c_double_p, c_double_p,
                                               c_double_p, c_double_p]),
        "qd_mlp_train": (C.c_int, [H, C.c_int64, c_double_p, c_double_p, c_double_p,
                                   c_double_p, C.c_int32, C.c_int32, C.c_double, C.c_double,
                                   c_float_p, c_double_p]),
        "qd_mlp_eval": (C.c_int, [H, C.c_int64, c_double_p, c_double_p, c_double_p,
                                  c_double_p]),
        "qd_mlp_potential": (C.c_int, [H, P(QdRadial), P(QdRadial), P(QdAngle), c_double_p,
                                       C.c_double, C.c_double, C.c_int32, c_double_p]),
        "qd_potential_jacobi": (C.c_int, [P(QdRadial), P(QdRadial), P(QdAngle), c_double_p,
                                          PES_FN, C.c_void_p, C.c_double, C.c_double,
                                          C.c_int32, c_double_p]),
        "qd_potential_leps": (C.c_int, [P(QdRadial), P(QdRadial), P(QdAngle), c_double_p,
                                        P(QdLeps), C.c_double, C.c_double, C.c_int32,
                                        c_double_p]),
        "qd_bkmp2_eval": (C.c_int, [C.c_int64, c_double_p, c_double_p, c_double_p,
                                    c_double_p]),
        "qd_potential_bkmp2": (C.c_int, [P(QdRadial), P(QdRadial), P(QdAngle), c_double_p,
                                         C.c_double, C.c_double, C.c_int32, c_double_p]),
        "qd_hsw_create": (C.c_int, [C.c_char_p, P(H)]),
        "qd_hsw_create_from_tables": (C.c_int, [C.c_int32, c_int32_p, c_int32_p, c_int32_p,
                                                c_double_p, c_double_p, C.c_int32, C.c_int32,
                                                C.c_int32, c_double_p, c_double_p, c_double_p,
                                                c_double_p, c_double_p, P(H)]),
        "qd_hsw_destroy": (C.c_int, [H]),
        "qd_hsw_eval": (C.c_int, [H, C.c_int64, c_double_p, c_double_p, c_double_p,
                                  c_double_p]),
        "qd_potential_hsw": (C.c_int, [P(QdRadial), P(QdRadial), P(QdAngle), c_double_p, H,
                                       C.c_double, C.c_double, C.c_int32, c_double_p]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


class QdError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"qd error {code}: {msg}")
        self.code = code


def check(rc):
    if rc != QD_OK:
        raise QdError(rc, lib().qd_last_error().decode(errors="replace"))
    return rc
