"""The CPU oracle against the reference's known answers and its own code.

Pins (reference file:line):
  * FFT normalisation + momentum grid: the harmonic-oscillator check in
    common/fftwinterface.C:132-188 (<V> = <T> = 0.25, norm 1);
  * Gauss-Legendre nodes/weights: GaussLegendre/<n>-LegendreGauss.grids;
  * the whole propagation: the reference's own common/timeEvol.C, run through
    the shims (oracle/_ref) when built here, else its committed outputs in
    tests/golden/ref_*.npz (bit-exact).
"""
import ctypes as C
import math
import os

import numpy as np
import pytest

from conftest import GOLDEN, GOLDEN_CASES, golden_case
from oracle import pyoracle as O
from qd_b200 import systems as S


def test_fft_harmonic_oscillator_kat():
    # common/fftwinterface.C:132-188 (Matlab script + its printed output)
    n = 1024
    x = np.linspace(-10, 10, n)
    dx = x[1] - x[0]
    assert abs(dx - 0.019550342130987) < 1e-15
    f = math.pi ** -0.25 * np.exp(-0.5 * x ** 2)
    assert abs(np.sum(np.abs(f) ** 2) * dx - 0.999999999999998) < 1e-14
    assert abs(np.sum(np.abs(f) ** 2 * 0.5 * x * x) * dx - 0.25) < 1e-14
    F = O.fft2d(f[None, :].astype(complex), -1)[0]
    assert abs(np.sum(np.abs(F) ** 2) / n * dx - 0.999999999999999) < 1e-13
    k = np.empty(n)
    O.lib().qdo_momentum(k.ctypes.data_as(C.POINTER(C.c_double)), n, n * dx)
    kk = (2 * math.pi / (n * dx)) * np.concatenate([np.arange(0, n // 2 + 1),
                                                      np.arange(-n // 2 + 1, 0)])
    # the reference accumulates the grid by repeated addition (fftwinterface.C:116-124)
    assert np.allclose(k, kk, rtol=0, atol=1e-10)
    # Matlab's check uses the exact grid; the accumulated one differs by ~1e-12
    assert abs(np.sum(np.abs(F) ** 2 * kk ** 2) / n * dx / 2 - 0.25) < 1e-14
    assert abs(np.sum(np.abs(F) ** 2 * k ** 2) / n * dx / 2 - 0.25) < 1e-12


@pytest.mark.parametrize("shape", [(64, 48), (30, 20), (12, 10), (8, 2)])
def test_fft2d_matches_dft_definition(shape):
    n2, n1 = shape
    rng = np.random.default_rng(1)
    a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    for sign, ref in ((-1, np.fft.fft2(a)), (+1, np.fft.ifft2(a) * a.size)):
        got = O.fft2d(a, sign)
        assert np.abs(got - ref).max() < 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("n", [8, 12, 40, 41, 64, 128])
def test_gauss_legendre_against_reference_tables(n):
    xg, wg = S.read_grids(os.path.join(GOLDEN, "grids"), n)
    x, w = S.gauss_legendre(n)
    assert np.abs(x - xg).max() < 2e-15
    assert np.abs(w - wg).max() < 2e-15
    assert np.all(np.diff(x) > 0)
    assert abs(w.sum() - 2.0) < 1e-13


@pytest.mark.parametrize("n", [12, 40, 64])
def test_legendre_orthogonality_on_quadrature(n):
    x, w = S.gauss_legendre(n)
    P = S.legendre_p2(n - 1, x)            # (n, m+1)
    G = P.T @ (w[:, None] * P)
    l = np.arange(n)
    assert np.abs(G - np.diag(1.0 / (l + 0.5))).max() < 1e-12


@pytest.mark.parametrize("npts", [3, 5, 7, 9, 11])
def test_gradient_stencils_exact_on_polynomials(npts):
    # Gradient3.F: a (npts)-point central difference is exact for degree npts-1
    n1, n2, n3 = 3, 24, 2
    dx = 0.1
    r = np.arange(n2) * dx
    deg = npts - 1
    F = np.empty((n3, n2, n1), complex)
    for k in range(n3):
        for i in range(n1):
            F[k, :, i] = (1 + i + 1j * k) * r ** deg + 0.5 * r
    n2p = 12
    V = np.zeros((n3, n1), complex)
    G = np.zeros((n3, n1), complex)
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    rc = O.lib().qdo_gradient3d(n1, n2, n3, n2p, dx, dp(F.view(np.float64)),
                                dp(V.view(np.float64)), dp(G.view(np.float64)), npts)
    assert rc == 0
    x0 = r[n2p - 1]
    for k in range(n3):
        for i in range(n1):
            c = 1 + i + 1j * k
            assert abs(V[k, i] - (c * x0 ** deg + 0.5 * x0)) < 1e-12
            assert abs(G[k, i] - (c * deg * x0 ** (deg - 1) + 0.5)) < 1e-9
    assert O.lib().qdo_gradient3d(n1, n2, n3, n2p, dx, dp(F.view(np.float64)),
                                  dp(V.view(np.float64)), dp(G.view(np.float64)), 4) != 0


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_oracle_bit_exact_against_reference_outputs(name):
    data, exp = golden_case(name)
    O.oracle_time_evolution(data)
    assert data.time.steps == exp["steps"]
    assert np.array_equal(data.psi, exp["psi"])
    assert np.array_equal(data.CRP.CRP, exp["crp"])


@pytest.mark.skipif(not O.ref_available(), reason="reference not built here (oracle/_ref)")
def test_oracle_bit_exact_against_reference_build():
    base = S.build_case("h+h2", 24, 16, 10, m=8, total_steps=12, n_energies=7,
                        n_gradient_points=7, r_surface=4.0)
    a, b = S.copy_case(base), S.copy_case(base)
    b.time.steps = a.time.steps = 0
    O.oracle_time_evolution(a)
    O.ref_time_evolution(b)
    assert np.array_equal(a.psi, b.psi) and np.array_equal(a.CRP.CRP, b.CRP.CRP)
    # resume semantics: steps > 0 skips the V(-dt/2) pre-step (timeEvol.C:664-665)
    a.time.total_steps = b.time.total_steps = 5
    O.oracle_time_evolution(a)
    O.ref_time_evolution(b)
    assert a.time.steps == b.time.steps == 17
    assert np.array_equal(a.psi, b.psi) and np.array_equal(a.CRP.CRP, b.CRP.CRP)


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_numpy_restatement_agrees(name):
    data, exp = golden_case(name)
    O.np_time_evolution(data)
    scale = np.abs(exp["psi"]).max()
    assert np.abs(data.psi - exp["psi"]).max() < 1e-12 * scale
    assert np.abs(data.CRP.CRP - exp["crp"]).max() < 1e-12 * max(np.abs(exp["crp"]).max(), 1e-30)


def test_oracle_unitary_without_absorbers():
    base = S.build_case("h+h2", 32, 24, 12, m=11, total_steps=40, n_energies=5)
    base.dump1.dump = None
    base.dump2.dump = None
    norms, _ = O.oracle_time_evolution(base, norms=True)
    # with n_l = n_theta the Legendre pair is unitary, so is every phase and FFT
    assert np.abs(norms - norms[0]).max() < 1e-12 * norms[0]


def ho_state(n=96, nth=4):
    """A 2-D harmonic-oscillator ground state (m = 1, omega = 1) in (R, r),
    independent of theta: the two-dimensional form of the known-answer check
    in common/fftwinterface.C:132-188 (<T> = <V> = 0.25 per dimension)."""
    from qd_b200.systems import Struct
    g = np.linspace(1.0, 21.0, n)
    dx = g[1] - g[0]
    x, w = S.gauss_legendre(nth)
    f = math.pi ** -0.25 * np.exp(-0.5 * (g - 11.0) ** 2)
    psi = (math.sqrt(0.5) * f[None, None, :] * f[None, :, None]
           * np.ones((nth, 1, 1))).astype(np.complex128)
    pot = (0.5 * (g[None, None, :] - 11.0) ** 2 + 0.5 * (g[None, :, None] - 11.0) ** 2
           ) * np.ones((nth, 1, 1))
    r1 = Struct(n=n, r=g.copy(), dr=dx, mass=1.0, r0=0.0, k0=0.0, delta=0.0)
    r2 = Struct(n=n, r=g.copy(), dr=dx, mass=1.0, r0=0.0, k0=0.0, delta=0.0)
    theta = Struct(n=nth, m=nth - 1, x=x, w=w, legendre=S.legendre_p2(nth - 1, x))
    return Struct(r1=r1, r2=r2, theta=theta, pot=np.ascontiguousarray(pot),
                  psi=np.ascontiguousarray(psi),
                  time=Struct(total_steps=1, time_step=0.01, steps=0),
                  options=Struct(wave_to_matlab=None, test_name="ho", precision=0,
                                 steps_to_copy_psi_from_device_to_host=0),
                  dump1=Struct(dump=None), dump2=Struct(dump=None),
                  CRP=Struct(n_dividing_surface=1, n_gradient_points=3, n_energies=1,
                             calculate_CRP=0, energies=np.zeros(1), eta_sq=np.ones(1),
                             CRP=np.zeros(1)))


def test_oracle_energies_harmonic_oscillator_kat():
    e = O.oracle_energies(ho_state())
    assert abs(e[0] - 0.5) < 1e-10      # kinetic, two dimensions
    assert abs(e[1]) < 1e-12            # l = 0 only
    assert abs(e[2] - 0.5) < 1e-10      # potential
