"""The library form of the propagator's two passes (cuFFT and cuBLAS, the
design of the reference's GPU code, common-cuda/evolutionCUDA2.cu), timed for
comparison with this library's kernels.  Loads lib/libqd_libcmp.so, which
the propagator itself never uses."""
import ctypes as C
import os

_LIB = None
COMPUTE = {"fp64": 0, "fp32_simt": 1, "tf32": 2, "fp32_bf16x9": 3}


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                            "lib", "libqd_libcmp.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is not built (quantum-dynamics_b200/build.py builds it)")
        L = C.CDLL(path)
        L.qdc_last_error.restype = C.c_char_p
        L.qdc_lspace_cufft.argtypes = [C.c_int] * 6 + [C.POINTER(C.c_double)]
        L.qdc_column_cublas.argtypes = [C.c_int] * 7 + [C.POINTER(C.c_double)]
        _LIB = L
    return _LIB


def _check(rc):
    if rc != 0:
        raise RuntimeError(lib().qdc_last_error().decode(errors="replace"))


def set_device(device):
    _check(lib().qdc_set_device(int(device)))


def lspace_cufft_ms(n1, n2, nl, runs, fp64=False, reps=10):
    """ms per step: Rot/2, 2-D FFT, kinetic phase, inverse 2-D FFT, Rot/2 over
    all l-slices of all runs (one cufftPlanMany, elementwise phase kernels)."""
    ms = C.c_double()
    _check(lib().qdc_lspace_cufft(n1, n2, nl, runs, 0 if fp64 else 1, reps, C.byref(ms)))
    return ms.value


def column_cublas_ms(n1, n2, nth, nl, runs, compute, reps=10):
    """ms per step: Legendre l -> theta GEMM, exp(-iVdt) x absorber, theta -> l
    GEMM (strided-batched over the runs); compute is a key of COMPUTE."""
    ms = C.c_double()
    _check(lib().qdc_column_cublas(n1, n2, nth, nl, runs, COMPUTE[compute], reps, C.byref(ms)))
    return ms.value
