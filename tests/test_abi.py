"""The C-ABI library: loads, exports every entry point of include/qd.h,
validates its input the way the reference's insist() checks do, and refuses
to run without a GPU (there is no CPU path).  No compute runs here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import REPO, GOLDEN, have_gpu
from qd_b200 import _abi, systems as S
from qd_b200.timeevolution import TimeEvolutionMexCUDA, _c_runs


def header_functions():
    src = open(os.path.join(REPO, "include", "qd.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(qd_[a-z_0-9]+)\s*\(", src)))


def test_exports_every_declared_symbol(qdlib):
    names = header_functions()
    assert len(names) >= 19
    for n in names:
        assert hasattr(qdlib, n), n
    assert qdlib.qd_abi_version() == 2


def test_read_grids_matches_python_reader(qdlib):
    from qd_b200.timeevolution import read_grids
    for n in (8, 41, 64):
        x, w = read_grids(os.path.join(GOLDEN, "grids"), n)
        xs, ws = S.read_grids(os.path.join(GOLDEN, "grids"), n)
        assert np.array_equal(x, xs) and np.array_equal(w, ws)
    x = np.empty(5); w = np.empty(5)
    rc = qdlib.qd_read_grids(b"/nonexistent", 5, x.ctypes.data_as(_abi.c_double_p),
                             w.ctypes.data_as(_abi.c_double_p))
    assert rc == _abi.QD_ERR_IO and b"does not exist" in qdlib.qd_last_error()


def _small():
    return S.build_case("h+h2", 16, 12, 8, m=6, total_steps=3, n_energies=5,
                        n_gradient_points=5)


@pytest.mark.parametrize("mutate,code,msg", [
    (lambda d: setattr(d.r1, "n", 15), _abi.QD_ERR_INVALID, b"even"),
    (lambda d: setattr(d.CRP, "n_gradient_points", 4), _abi.QD_ERR_INVALID, b"NPoints"),
    (lambda d: setattr(d.CRP, "n_dividing_surface", 1), _abi.QD_ERR_INVALID, b"dividing surface"),
    (lambda d: setattr(d.CRP, "n_dividing_surface", 12), _abi.QD_ERR_INVALID, b"dividing surface"),
    (lambda d: d.pot.__setitem__((0, 0, 0), np.nan), _abi.QD_ERR_NONFINITE, b"pot"),
    (lambda d: d.psi.__setitem__((1, 1, 1), np.inf), _abi.QD_ERR_NONFINITE, b"psi"),
    (lambda d: setattr(d.options, "precision", 7), _abi.QD_ERR_INVALID, b"precision"),
])
def test_invalid_input_rejected_before_device_work(qdlib, mutate, code, msg):
    d = _small()
    mutate(d)
    c = _abi.to_c(d)
    if d.r1.n == 15:
        c.r1.n = 15
    h = C.c_void_p()
    rc = qdlib.qd_create(C.byref(c), C.byref(h))
    assert rc == code
    assert msg in qdlib.qd_last_error()
    assert not h.value


@pytest.mark.parametrize("where", ["pot", "psi"])
def test_nonfinite_found_in_large_inputs(qdlib, where):
    # 128 x 128 x 64 points: the finiteness scan splits the arrays over host
    # threads; a NaN or Inf in the last part is still found
    d = S.build_case("h+h2", 128, 128, 64, m=63, total_steps=1, n_energies=5,
                     n_gradient_points=5)
    if where == "pot":
        d.pot[-1, -1, -1] = np.nan
    else:
        d.psi[-1, -1, -2] = complex(0.0, -np.inf)
    c = _abi.to_c(d)
    h = C.c_void_p()
    assert qdlib.qd_create(C.byref(c), C.byref(h)) == _abi.QD_ERR_NONFINITE
    assert where.encode() in qdlib.qd_last_error()
    assert not h.value


@pytest.mark.gpu
@pytest.mark.parametrize("where", ["pot", "psi"])
@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("shape", [(128, 128, 64), (256, 256, 128)])
def test_nonfinite_found_while_staging_large_inputs(qdlib, where, prec, shape):
    # arrays of 4 MiB or more are checked while they are copied into the
    # page-locked staging buffers of the upload (one staging buffer's worth and
    # several), in both precisions
    n1, n2, nth = shape
    d = S.build_case("h+h2", n1, n2, nth, m=63, total_steps=1, n_energies=5,
                     n_gradient_points=5)
    d.options.precision = prec
    assert d.pot.nbytes >= 4 << 20
    if where == "pot":
        d.pot[-1, -1, -3] = np.inf
    else:
        d.psi[-1, -2, -1] = complex(np.nan, 0.0)
    c = _abi.to_c(d)
    h = C.c_void_p()
    assert qdlib.qd_create(C.byref(c), C.byref(h)) == _abi.QD_ERR_NONFINITE
    assert where.encode() in qdlib.qd_last_error()
    assert not h.value


@pytest.mark.gpu
def test_kernel_choice_reports_the_tuned_kernels(qdlib):
    # a complex64 handle on a uniform energy grid: tensor-core column pass,
    # a register-FFT or other built l-space kernel, chirp-z accumulation
    from qd_b200 import Propagator
    d = S.build_case("f+h2", 128, 96, 64, m=63, total_steps=2, n_energies=9,
                     n_gradient_points=5)
    d.options.precision = 1
    with Propagator(d) as p:
        p.propagate(2)
        ch = (C.c_int32 * 4)()
        assert qdlib.qd_kernel_choice(p._h, ch) == 0
    assert ch[0] in (0, 1, 2, 4, 8, 9, 10, 11)
    assert ch[1] == 1
    assert 0 <= ch[2] < 4
    assert ch[3] == 1
    assert qdlib.qd_kernel_choice(None, ch) == _abi.QD_ERR_INVALID


@pytest.mark.gpu
def test_nonfinite_found_in_one_run_of_a_batch(qdlib):
    # a batch whose third run carries a NaN in its potential: create reports that run
    d = S.build_case("h+h2", 128, 128, 64, m=63, total_steps=1, n_energies=5,
                     n_gradient_points=5)
    runs = [S.copy_case(d) for _ in range(4)]
    runs[2].pot = d.pot.copy()                  # copy_case shares the potential
    runs[2].pot[3, 5, 7] = np.nan
    arr = _c_runs(runs)
    h = C.c_void_p()
    assert qdlib.qd_create_batch(arr, 4, C.byref(h)) == _abi.QD_ERR_NONFINITE
    assert b"run 2" in qdlib.qd_last_error()
    assert not h.value


def test_unsupported_fft_size(qdlib):
    d = S.build_case("h+h2", 14, 12, 8, m=6, total_steps=1, n_energies=5, n_gradient_points=5)
    c = _abi.to_c(d)
    h = C.c_void_p()
    assert qdlib.qd_create(C.byref(c), C.byref(h)) == _abi.QD_ERR_UNSUPPORTED


@pytest.mark.skipif(have_gpu(), reason="checks the no-GPU behaviour")
def test_fails_loudly_without_gpu(qdlib):
    d = _small()
    with pytest.raises(_abi.QdError) as e:
        TimeEvolutionMexCUDA(d)
    assert e.value.code == _abi.QD_ERR_CUDA
    assert "no CPU path" in str(e.value)


def test_struct_layout_matches_header():
    # sizes of the ctypes mirror equal the C struct sizes on x86-64
    assert C.sizeof(_abi.QdRadial) == 56
    assert C.sizeof(_abi.QdAngle) == 32
    assert C.sizeof(_abi.QdTime) == 24
    assert C.sizeof(_abi.QdCrp) == 40


def _jacobi_grid():
    x, _ = S.gauss_legendre(12)
    R = np.linspace(0.5, 12.0, 20)
    r = np.linspace(0.4, 8.0, 16)
    m = np.array([18.9984, 1.00783, 1.00783]) * S.AMU_ME
    return R, r, x, m


def test_pes_callback_matches_jacobi_mapping(qdlib):
    # the host PES callback path (no GPU): same points, same values as the
    # restatement of H3PESJacobi.m in systems.potential_on_grid
    from qd_b200.timeevolution import potential_jacobi
    R, r, x, m = _jacobi_grid()
    pes = S.leps_f_h2()
    got = potential_jacobi(R, r, x, m, pes)
    ref = S.potential_on_grid(R, r, x, m, pes)
    assert got.shape == ref.shape
    assert np.array_equal(got, ref)
    uncapped = potential_jacobi(R, r, x, m, pes, cap=False)
    assert uncapped.max() > 2.5 and np.array_equal(np.minimum(uncapped, 2.5), got)


def test_pes_callback_errors(qdlib):
    from qd_b200.timeevolution import potential_jacobi
    from qd_b200._abi import QdError, QD_ERR_PES
    R, r, x, m = _jacobi_grid()

    def raises(r12, r23, r13):
        raise RuntimeError("no surface here")
    with pytest.raises(QdError) as e:
        potential_jacobi(R, r, x, m, raises)
    assert e.value.code == QD_ERR_PES
    with pytest.raises(QdError) as e:
        potential_jacobi(R, r, x, m, lambda a, b, c: np.full(a.shape, np.nan))
    assert e.value.code == QD_ERR_PES


@pytest.mark.gpu
@pytest.mark.parametrize("K", [0, 1, 3])
def test_cs_legendre_on_gpu_matches_host(qdlib, K):
    # the device basis against the host restatement systems.cs_legendre
    x, w = S.gauss_legendre(24)
    m = 23 - K
    out = np.empty((24, m + 1))
    _abi.check(qdlib.qd_cs_legendre(24, K, m, x.ctypes.data_as(_abi.c_double_p),
                                    out.ctypes.data_as(_abi.c_double_p)))
    ref = S.cs_legendre(x, K, m)
    if K == 0:
        assert np.abs(out - S.legendre_p2(m, x)).max() < 1e-14
    assert np.abs(out - ref).max() < 1e-13
    # the reference's transform pair is the identity on the basis
    Q = np.sqrt(w)[:, None] * np.sqrt(np.arange(m + 1) + 0.5)[None, :] * out
    assert np.abs(Q.T @ Q - np.eye(m + 1)).max() < 1e-12


@pytest.mark.parametrize("K", [0, 1, 3])
def test_cs_legendre_host_is_orthonormal(K):
    # the host restatement used to build test inputs: orthonormal under the
    # quadrature for every K
    x, w = S.gauss_legendre(24)
    m = 23 - K
    Q = np.sqrt(w)[:, None] * np.sqrt(np.arange(m + 1) + 0.5)[None, :] * S.cs_legendre(x, K, m)
    assert np.abs(Q.T @ Q - np.eye(m + 1)).max() < 1e-12


def test_cs_legendre_rejects_bad_nodes(qdlib):
    x = np.array([0.0, 1.5])
    out = np.empty((2, 2))
    rc = qdlib.qd_cs_legendre(2, 1, 1, x.ctypes.data_as(_abi.c_double_p),
                              out.ctypes.data_as(_abi.c_double_p))
    assert rc == _abi.QD_ERR_INVALID and b"outside" in qdlib.qd_last_error()
