"""GPU propagation through the C ABI against the CPU oracle (which is pinned
bit-exactly to the reference's own common/timeEvol.C).

Tolerances of the path's precision contract: FP64 plain form -- wavepacket norm 1e-10 relative,
P(E) 1e-8 absolute; complex64 form -- |dP(E)| <= 1e-3 over energies where
eta^2 > 1e-3 max eta^2, norm 1e-5 relative.
"""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, golden_case
from oracle import pyoracle as O
from qd_b200 import systems as S, QD_PREC_FP32, QD_PREC_FP64
from qd_b200.timeevolution import TimeEvolutionMexCUDA, Propagator

pytestmark = pytest.mark.gpu

FP64_PSI_REL = 1e-10
FP64_CRP_ABS = 1e-8
FP32_CRP_ABS = 1e-3


def norm(data, psi):
    w = data.theta.w
    return float(np.sum(w[:, None, None] * np.abs(psi) ** 2) * data.r1.dr * data.r2.dr)


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_fp64_matches_reference_outputs(name):
    data, exp = golden_case(name)
    TimeEvolutionMexCUDA(data)
    assert data.time.steps == exp["steps"]
    assert rel(data.psi, exp["psi"]) < FP64_PSI_REL
    assert np.abs(data.CRP.CRP - exp["crp"]).max() < FP64_CRP_ABS


CASES = [
    # (system, n1, n2, nth, m, steps, npts, extra)
    ("h+h2", 64, 64, 40, 38, 60, 11, {}),
    ("f+h2", 48, 40, 24, 20, 40, 7, {}),            # 48 = 16*3, 40 = 8*5
    ("h+h2", 12, 10, 6, 5, 30, 3, {}),               # tiny odd-radix grid
    ("f+h2", 32, 96, 16, 15, 25, 9, dict(r=(0.5, 9.0))),  # radix-3 in r
    ("h+h2", 32, 24, 10, 12, 20, 5, {}),             # n_l > n_theta
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}-{c[1]}x{c[2]}x{c[3]}-m{c[4]}")
def test_fp64_matches_oracle(case):
    system, n1, n2, nth, m, steps, npts, extra = case
    base = S.build_case(system, n1, n2, nth, m=m, total_steps=steps, n_energies=17,
                        n_gradient_points=npts, **extra)
    a, b = S.copy_case(base), S.copy_case(base)
    norms, _ = O.oracle_time_evolution(a, norms=True)
    with Propagator(b) as p:
        p.propagate(steps)
        gnorms = p.norms(steps)
        p.download()
    assert b.time.steps == a.time.steps == steps
    assert rel(b.psi, a.psi) < FP64_PSI_REL
    assert np.abs(gnorms - norms).max() < FP64_PSI_REL * norms.max()
    assert np.abs(b.CRP.CRP - a.CRP.CRP).max() < FP64_CRP_ABS


def test_fp64_no_absorber_no_crp_and_resume():
    base = S.build_case("h+h2", 32, 32, 16, m=15, total_steps=10, n_energies=5)
    base.dump1.dump = None
    base.CRP.calculate_CRP = 0
    a, b = S.copy_case(base), S.copy_case(base)
    O.oracle_time_evolution(a)
    TimeEvolutionMexCUDA(b)
    assert rel(b.psi, a.psi) < FP64_PSI_REL
    assert np.all(b.CRP.CRP == 0)
    # second call resumes from steps = 10 without the pre-step
    O.oracle_time_evolution(a)
    TimeEvolutionMexCUDA(b)
    assert a.time.steps == b.time.steps == 20
    assert rel(b.psi, a.psi) < FP64_PSI_REL


def test_fp64_unitary_without_absorbers():
    base = S.build_case("h+h2", 32, 32, 16, m=15, total_steps=50, n_energies=5)
    base.dump1.dump = None
    base.dump2.dump = None
    with Propagator(base) as p:
        p.propagate(50)
        n = p.norms(50)
    assert np.abs(n - n[0]).max() < 1e-12 * n[0]


@pytest.mark.parametrize("prec", [QD_PREC_FP64, QD_PREC_FP32])
def test_norm_growth_is_reported(prec):
    # an absorber above 1 (a host-side input error) makes the norm grow; the
    # host-side unitarity guard stops the call with QD_ERR_NONFINITE
    from qd_b200._abi import QdError, QD_ERR_NONFINITE
    d = S.build_case("h+h2", 32, 24, 12, m=11, total_steps=5, n_energies=5,
                     n_gradient_points=5, precision=prec)
    d.dump1.dump = np.full_like(d.dump1.dump, 1.01)
    with pytest.raises(QdError) as exc:
        TimeEvolutionMexCUDA(d)
    assert exc.value.code == QD_ERR_NONFINITE
    assert "grew" in str(exc.value)


def test_handle_split_calls_equal_one_call():
    base = S.build_case("f+h2", 32, 32, 16, m=15, total_steps=30, n_energies=9,
                        n_gradient_points=5)
    a, b = S.copy_case(base), S.copy_case(base)
    O.oracle_time_evolution(a)
    with Propagator(b) as p:
        for n in (7, 1, 22):
            p.propagate(n)
        assert p.steps == 30
        p.download()
    assert rel(b.psi, a.psi) < FP64_PSI_REL
    assert np.abs(b.CRP.CRP - a.CRP.CRP).max() < FP64_CRP_ABS


_BUDGET_REF = {}


def _budget_reference():
    # the oracle's 200-step run of the budget case, computed once per session
    if not _BUDGET_REF:
        base = S.build_case("f+h2", 64, 64, 32, m=31, total_steps=200, n_energies=41,
                            n_gradient_points=11)
        a = S.copy_case(base)
        norms, _ = O.oracle_time_evolution(a, norms=True)
        _BUDGET_REF.update(base=base, a=a, norms=norms)
    return _BUDGET_REF["base"], _BUDGET_REF["a"], _BUDGET_REF["norms"]


@pytest.mark.parametrize("slice_kind", ["auto", "0", "8"])
def test_fp32_matches_oracle_within_budget(slice_kind, monkeypatch):
    # every l-space kernel choice (the autotuner's, the split kernels, the
    # register-FFT kernel with the flux preparation in its extra CTAs): the
    # flux rows written by the column pass's slow tiles reach P(E) intact
    if slice_kind != "auto":
        monkeypatch.setenv("QD_SLICE_CLUSTER", slice_kind)
    base, a, norms = _budget_reference()
    b = S.copy_case(base)
    b.options.precision = QD_PREC_FP32
    with Propagator(b) as p:
        p.propagate(200)
        gn = p.norms(200)
        p.download()
    eta = base.CRP.eta_sq
    sel = eta > 1e-3 * eta.max()
    assert np.abs(b.CRP.CRP - a.CRP.CRP)[sel].max() < FP32_CRP_ABS
    assert np.abs(gn - norms).max() < 1e-4 * norms.max()
    assert rel(b.psi, a.psi) < 1e-4


def test_legendre_matrix_on_gpu():
    from qd_b200.timeevolution import legendre_matrix_gpu
    x, _ = S.gauss_legendre(40)
    P = legendre_matrix_gpu(40, 38, x)
    assert np.abs(P - S.legendre_p2(38, x)).max() < 1e-14


@pytest.mark.parametrize("path", ["tc", "simt"])
def test_fp32_c0_grid_against_oracle(path, monkeypatch):
    # 64 x 64 x 40, n_l = 39: padded to 48 x 48 in the tensor-core pass
    monkeypatch.setenv("QD_COLUMN_PATH", path)
    base = S.case_c0(total_steps=150)
    a, b = S.copy_case(base), S.copy_case(base)
    b.options.precision = QD_PREC_FP32
    norms, _ = O.oracle_time_evolution(a, norms=True)
    with Propagator(b) as p:
        p.propagate(150)
        gn = p.norms(150)
        p.download()
    eta = base.CRP.eta_sq
    sel = eta > 1e-3 * eta.max()
    assert np.abs(b.CRP.CRP - a.CRP.CRP)[sel].max() < FP32_CRP_ABS
    assert np.abs(gn - norms).max() < 1e-4 * norms.max()
    assert rel(b.psi, a.psi) < 1e-4


@pytest.mark.parametrize("shape", [(32, 24, 128, 127), (24, 20, 80, 79), (32, 24, 128, 100)])
def test_fp32_large_angular_bases_against_fp64(shape):
    # n_theta up to 128: the tensor-core column pass with one CTA per SM (S = 96,
    # 128), at S = 128 with B1 and B2 streamed through one shared-memory buffer;
    # n_l < n_theta runs the orthonormal completion of GEMM2
    n1, n2, nth, m = shape
    base = S.build_case("f+h2", n1, n2, nth, m=m, total_steps=40, n_energies=9,
                        n_gradient_points=5, r=(0.5, 9.0))
    got = {}
    for prec in (QD_PREC_FP64, QD_PREC_FP32):
        d = S.copy_case(base)
        d.options.precision = prec
        with Propagator(d) as p:
            p.propagate(40)
            got[prec] = (p.psi(), p.crp(), p.norms(40))
    a, b = got[QD_PREC_FP64], got[QD_PREC_FP32]
    assert rel(b[0], a[0]) < 1e-4
    assert np.abs(b[1] - a[1]).max() < FP32_CRP_ABS
    assert np.abs(b[2] - a[2]).max() < 1e-4 * np.abs(a[2]).max()


def test_fp32_large_cs_batch_against_fp64():
    # centrifugal-sudden blocks of uneven n_j on n_theta = 128 in one batch: the
    # streamed operand images follow each tile's angular set
    base = _cs_base(24, 20, 128, steps=30)
    combos = [(0, 0, 0, 2), (4, 1, 0, 2), (4, 2, 0, 2), (8, 3, 0, 3)]
    runs = [S.cs_case(base, *c) for c in combos]
    got = {}
    for prec in (QD_PREC_FP64, QD_PREC_FP32):
        rs = [S.copy_case(r) for r in runs]
        for r in rs:
            r.options.precision = prec
        with Propagator(rs) as p:
            p.propagate(30)
            got[prec] = [(p.psi(i), p.crp(i)) for i in range(len(rs))]
    for (psi64, crp64), (psi32, crp32) in zip(got[QD_PREC_FP64], got[QD_PREC_FP32]):
        if np.abs(psi64).max() > 0:
            assert rel(psi32, psi64) < 1e-4
        assert np.abs(crp32 - crp64).max() < FP32_CRP_ABS


def test_fp32_tensor_core_and_simt_agree(monkeypatch):
    base = S.build_case("f+h2", 128, 96, 64, m=63, total_steps=20, n_energies=9,
                        n_gradient_points=7, r=(0.5, 9.0))
    out = {}
    for path in ("tc", "simt"):
        monkeypatch.setenv("QD_COLUMN_PATH", path)
        d = S.copy_case(base)
        d.options.precision = QD_PREC_FP32
        with Propagator(d) as p:
            p.propagate(20)
            out[path] = p.psi()
    assert rel(out["tc"], out["simt"]) < 2e-5


@pytest.mark.parametrize("shape", [(64, 64, 32), (128, 128, 64), (128, 96, 64), (48, 40, 24),
                                   (256, 192, 16)])
def test_fp32_l_space_pass_variants_agree(shape, monkeypatch):
    # fused slice kernel with 1, 2, 4 CTAs per slice and the register-FFT slice
    # kernel on 1 (8), 2 (9) and 4 (10) CTAs per slice, and its 4-CTA form with
    # 16 x 16 row transforms (11), where they are built, against the three-kernel
    # split pass;
    # the flux preparation rides in the fused launches, so P(E) is compared too
    n1, n2, nth = shape
    base = S.build_case("f+h2", n1, n2, nth, m=nth - 1, total_steps=8, n_energies=5,
                        n_gradient_points=5, r=(0.5, 9.0))
    out = {}
    for cl in ("0", "1", "2", "4", "8", "9", "10", "11"):
        monkeypatch.setenv("QD_SLICE_CLUSTER", cl)
        d = S.copy_case(base)
        d.options.precision = QD_PREC_FP32
        with Propagator(d) as p:
            p.propagate(8)
            out[cl] = (p.psi(), p.crp())
    ref = out["0"]
    for cl, (psi, crp) in out.items():
        assert rel(psi, ref[0]) < 2e-5, cl
        assert np.abs(crp - ref[1]).max() < 1e-6, cl


@pytest.mark.parametrize("shape,kind", [((64, 64, 32), "8"), ((128, 96, 64), "8"),
                                        ((128, 96, 64), "9"), ((256, 192, 16), "10"),
                                        ((256, 192, 16), "11")])
def test_fp32_register_fft_slice_batch_matches_fp64(shape, kind, monkeypatch):
    # the register-FFT slice kernel (one CTA, or a 2- or 4-CTA cluster per slice) on
    # a 3-run batch (flux preparation in its extra CTAs) against the FP64
    # plain form of the same runs, 40 steps
    n1, n2, nth = shape
    base = S.build_case("f+h2", n1, n2, nth, m=nth - 1, total_steps=40, n_energies=9,
                        n_gradient_points=5, r=(0.5, 9.0))
    runs = S.batch_cases(base, [(0, 0), (0, 1), (1, 0)])
    monkeypatch.setenv("QD_SLICE_CLUSTER", kind)
    got = {}
    for prec in (QD_PREC_FP64, QD_PREC_FP32):
        rs = [S.copy_case(r) for r in runs]
        for r in rs:
            r.options.precision = prec
        with Propagator(rs) as p:
            p.propagate(40)
            got[prec] = [(p.psi(i), p.crp(i)) for i in range(len(rs))]
    for (a, ca), (b, cb) in zip(got[QD_PREC_FP32], got[QD_PREC_FP64]):
        assert rel(a, b) < 1e-4
        assert np.abs(ca - cb).max() < FP32_CRP_ABS


def test_fp32_c1_full_run_within_pe_budget():
    # the F + H2 128 x 128 x 64 case over its full 10000 steps: complex64 with the
    # tensor-core Legendre pass against the FP64 plain form (which is pinned to
    # the oracle above), max |dP(E)| <= 1e-3 where eta^2 > 1e-3 max eta^2
    c1 = S.case_c1()
    out = {}
    for prec in (QD_PREC_FP64, QD_PREC_FP32):
        d = S.copy_case(c1)
        d.options.precision = prec
        with Propagator(d) as p:
            p.propagate(10000)
            out[prec] = (p.crp(), p.norms(10000))
    eta = c1.CRP.eta_sq
    sel = eta > 1e-3 * eta.max()
    dP = np.abs(out[QD_PREC_FP32][0] - out[QD_PREC_FP64][0])[sel].max()
    assert dP < FP32_CRP_ABS, dP
    assert np.abs(out[QD_PREC_FP32][1] - out[QD_PREC_FP64][1]).max() < 1e-3


def test_fp32_c4_block_within_pe_budget():
    # one centrifugal-sudden block (J = 8, K = 2, n_j = 126) on the full C4 grid
    # 256 x 192 x 128 over 3000 steps: complex64 (tensor-core column pass at
    # n_theta = 128 with streamed operand images, 256 x 192 slices) against the
    # FP64 plain form, max |dP(E)| <= 1e-3 where eta^2 > 1e-3 max eta^2
    base = S.build_case("f+h2", 256, 192, 128, m=127, r=(0.4, 8.0), total_steps=3000)
    run = S.cs_case(base, 8, 2, 0, 3)
    out = {}
    for prec in (QD_PREC_FP64, QD_PREC_FP32):
        d = S.copy_case(run)
        d.options.precision = prec
        with Propagator(d) as p:
            p.propagate(3000)
            out[prec] = (p.crp(), p.norms(3000), p.psi())
    eta = run.CRP.eta_sq
    sel = eta > 1e-3 * eta.max()
    dP = np.abs(out[QD_PREC_FP32][0] - out[QD_PREC_FP64][0])[sel].max()
    assert dP < FP32_CRP_ABS, dP
    assert np.abs(out[QD_PREC_FP32][1] - out[QD_PREC_FP64][1]).max() < 1e-3
    assert rel(out[QD_PREC_FP32][2], out[QD_PREC_FP64][2]) < 1e-3


def test_fp32_c2_cs_blocks_within_pe_budget():
    # two centrifugal-sudden blocks of the C2 batch (J = 5, K = 1 and J = 10,
    # K = 2) on its 128 x 96 x 64 grid, in one batch, over 3000 steps (the
    # packets are absorbed): complex64 against the FP64 plain form, max |dP(E)|
    # <= 1e-3 where eta^2 > 1e-3 max eta^2
    base = S.build_case("f+h2", 128, 96, 64, m=63, r=(0.4, 8.0), total_steps=3000)
    runs = [S.cs_case(base, 5, 1, 0, 1), S.cs_case(base, 10, 2, 0, 2)]
    out = {}
    for prec in (QD_PREC_FP64, QD_PREC_FP32):
        rs = [S.copy_case(r) for r in runs]
        for r in rs:
            r.options.precision = prec
        with Propagator(rs) as p:
            p.propagate(3000)
            out[prec] = [(p.crp(i), p.norms(3000, i)) for i in range(len(rs))]
    for r, (c64, n64), (c32, n32) in zip(runs, out[QD_PREC_FP64], out[QD_PREC_FP32]):
        assert np.abs(c64).max() > 0.1                 # both blocks carry a packet
        eta = r.CRP.eta_sq
        sel = eta > 1e-3 * eta.max()
        assert np.abs(c32 - c64)[sel].max() < FP32_CRP_ABS
        assert np.abs(n32 - n64).max() < 1e-3


def _three_runs(prec, steps=25):
    # same F + H2 grid, different initial states (v0, j0) -> different psi,
    # energies and eta^2; the potential table is shared
    runs = []
    for v0, j0 in ((0, 0), (0, 2), (1, 0)):
        d = S.build_case("f+h2", 48, 40, 24, m=23, total_steps=steps, n_energies=13,
                         n_gradient_points=7, j0=j0, v0=v0, precision=prec)
        runs.append(d)
    for d in runs[1:]:
        d.pot = runs[0].pot
    return runs


@pytest.mark.parametrize("prec", [QD_PREC_FP64, QD_PREC_FP32])
def test_batch_equals_individual_runs(prec):
    runs = _three_runs(prec)
    single = [S.copy_case(d) for d in runs]
    batch = [S.copy_case(d) for d in runs]
    for d in single:
        TimeEvolutionMexCUDA(d)
    TimeEvolutionMexCUDA(batch)
    tol = 1e-12 if prec == QD_PREC_FP64 else 1e-6
    for a, b in zip(single, batch):
        assert b.time.steps == a.time.steps == 25
        assert rel(b.psi, a.psi) < tol
        assert np.abs(b.CRP.CRP - a.CRP.CRP).max() < tol * max(1.0, np.abs(a.CRP.CRP).max())


def test_batch_fp64_matches_oracle_per_run():
    runs = _three_runs(QD_PREC_FP64, steps=20)
    with Propagator([S.copy_case(d) for d in runs]) as p:
        p.propagate(20)
        got = [(p.psi(r), p.crp(r), p.norms(20, r)) for r in range(3)]
    for r, d in enumerate(runs):
        a = S.copy_case(d)
        norms, _ = O.oracle_time_evolution(a, norms=True)
        assert rel(got[r][0], a.psi) < FP64_PSI_REL
        assert np.abs(got[r][1] - a.CRP.CRP).max() < FP64_CRP_ABS
        assert np.abs(got[r][2] - norms).max() < FP64_PSI_REL


@pytest.mark.parametrize("m", [23, 17])          # n_l = n_theta and n_l < n_theta
@pytest.mark.parametrize("prec,tol", [(QD_PREC_FP64, 1e-10), (QD_PREC_FP32, 1e-4)])
def test_energies_match_oracle(prec, tol, m):
    base = S.build_case("f+h2", 48, 40, 24, m=m, total_steps=15, n_energies=5,
                        precision=prec)
    a = S.copy_case(base)
    O.oracle_time_evolution(a)
    e_ref = O.oracle_energies(a)
    with Propagator(S.copy_case(base)) as p:
        p.propagate(15)
        e = p.energies()
    assert np.abs(e - e_ref).max() < tol * np.abs(e_ref).max(), (e, e_ref)


@pytest.mark.parametrize("prec", [QD_PREC_FP64, QD_PREC_FP32])
def test_checkpoint_restore_resumes_exactly(prec, tmp_path):
    base = S.build_case("h+h2", 32, 32, 16, m=15, total_steps=40, n_energies=9,
                        n_gradient_points=5, precision=prec)
    path = tmp_path / "state.qdck"
    with Propagator(S.copy_case(base)) as p:
        p.propagate(17)
        p.checkpoint(path)
        p.propagate(23)
        psi_a, crp_a = p.psi(), p.crp()
    with Propagator(S.copy_case(base)) as q:
        q.restore(path)
        assert q.steps == 17
        q.propagate(23)
        psi_b, crp_b = q.psi(), q.crp()
        assert q.steps == 40
    assert np.array_equal(psi_a, psi_b)
    assert np.array_equal(crp_a, crp_b)


@pytest.mark.parametrize("prec,tol", [(QD_PREC_FP64, 1e-10), (QD_PREC_FP32, 1e-5)])
def test_energies_harmonic_oscillator_kat(prec, tol):
    from test_oracle import ho_state
    d = ho_state()
    d.options.precision = prec
    with Propagator(d) as p:
        e = p.energies()
    assert abs(e[0] - 0.5) < tol and abs(e[2] - 0.5) < tol and abs(e[1]) < tol


@pytest.mark.parametrize("system", ["h+h2", "f+h2"])
def test_leps_potential_on_gpu(system):
    # the device LEPS evaluation against the host restatement of
    # H3PESJacobi.m + the LEPS algebra (systems.potential_on_grid)
    from qd_b200.timeevolution import potential_leps_gpu
    x, _ = S.gauss_legendre(40)
    R = np.linspace(0.5, 12.0, 64)
    r = np.linspace(0.4, 8.0, 64)
    amu = (1.00783, 1.00783, 1.00783) if system == "h+h2" else (18.9984, 1.00783, 1.00783)
    m = np.array(amu) * S.AMU_ME
    pes = S.leps_h_h2() if system == "h+h2" else S.leps_f_h2()
    for cap in (True, False):
        got = potential_leps_gpu(R, r, x, m, pes, cap=cap)
        ref = S.potential_on_grid(R, r, x, m, pes) if cap else None
        if cap:
            assert np.abs(got - ref).max() < 1e-13 * np.abs(ref).max()
        else:
            assert np.array_equal(np.minimum(got, 2.5), potential_leps_gpu(R, r, x, m, pes))


def _cs_base(n1=32, n2=32, nth=16, steps=30, **kw):
    return S.build_case("f+h2", n1, n2, nth, m=nth - 1, total_steps=steps, n_energies=9,
                        n_gradient_points=5, r=(0.5, 9.0), **kw)


def test_cs_block_fp64_matches_oracle():
    # centrifugal-sudden block J = 5, K = 2 (n_j = n_theta - 2, basis Pbar_j^2)
    base = _cs_base()
    run = S.cs_case(base, 5, 2, 0, 2)
    a, b = S.copy_case(run), S.copy_case(run)
    norms, _ = O.oracle_time_evolution(a, norms=True)
    with Propagator(b) as p:
        p.propagate(30)
        gn = p.norms(30)
        e_gpu = p.energies()
        p.download()
    assert rel(b.psi, a.psi) < FP64_PSI_REL
    assert np.abs(gn - norms).max() < FP64_PSI_REL * norms.max()
    assert np.abs(b.CRP.CRP - a.CRP.CRP).max() < FP64_CRP_ABS
    e_ref = O.oracle_energies(a)
    assert np.abs(e_gpu - e_ref).max() < 1e-10 * np.abs(e_ref).max()


@pytest.mark.parametrize("slice_kind", ["auto", "8"])
def test_cs_mixed_batch(slice_kind, monkeypatch):
    # one batch of blocks with different K (different angular bases and n_j):
    # FP64 against the oracle run by run; complex64 (tensor-core column pass,
    # per-run operand images) against FP64
    if slice_kind != "auto":
        monkeypatch.setenv("QD_SLICE_CLUSTER", slice_kind)
    base = _cs_base(64, 64, 32, steps=40)
    combos = [(0, 0, 0, 0), (5, 1, 0, 1), (5, 2, 0, 2), (10, 0, 1, 0), (10, 3, 0, 2)]
    runs = [S.cs_case(base, *c) for c in combos]
    got = {}
    for prec in (QD_PREC_FP64, QD_PREC_FP32):
        rs = [S.copy_case(r) for r in runs]
        for r in rs:
            r.options.precision = prec
        with Propagator(rs) as p:
            p.propagate(40)
            got[prec] = [(p.psi(i), p.crp(i)) for i in range(len(rs))]
    for r, (psi64, crp64), (psi32, crp32) in zip(runs, got[QD_PREC_FP64], got[QD_PREC_FP32]):
        a = S.copy_case(r)
        O.oracle_time_evolution(a)
        assert rel(psi64, a.psi) < FP64_PSI_REL
        assert np.abs(crp64 - a.CRP.CRP).max() < FP64_CRP_ABS
        if np.abs(a.psi).max() > 0:
            assert rel(psi32, psi64) < 1e-4
        assert np.abs(crp32 - crp64).max() < FP32_CRP_ABS


def test_fp32_cs_batch_equals_individual_runs():
    # centrifugal-sudden blocks of different K in one complex64 batch (one
    # potential table and one angular basis per run) against each block
    # propagated alone
    base = _cs_base(64, 64, 32, steps=40)
    runs = [S.cs_case(base, *c) for c in [(0, 0, 0, 0), (5, 1, 0, 1), (10, 2, 0, 2)]]
    for r in runs:
        r.options.precision = QD_PREC_FP32
    single = [S.copy_case(r) for r in runs]
    batch = [S.copy_case(r) for r in runs]
    for d in single:
        TimeEvolutionMexCUDA(d)
    TimeEvolutionMexCUDA(batch)
    for a, b in zip(single, batch):
        if np.abs(a.psi).max() > 0:
            assert rel(b.psi, a.psi) < 1e-5
        assert np.abs(b.CRP.CRP - a.CRP.CRP).max() < 1e-5 * max(1.0, np.abs(a.CRP.CRP).max())


@pytest.mark.parametrize("j0,v0,K", [(0, 0, 0), (2, 0, 0), (0, 1, 0), (2, 0, 1), (1, 0, 2)])
def test_initial_state_on_gpu(j0, v0, K):
    # the GPU builder (sinc-DVR by parallel Jacobi, packet, eta^2) against the
    # host restatement of InitWavePacket.m / H2VibRotWaveFunction.m / EtaSq.m
    from qd_b200.timeevolution import init_state_gpu, eta_sq_gpu
    base = S.build_case("f+h2", 64, 96, 24, m=23, total_steps=1, n_energies=31)
    pes = S.leps_f_h2()
    vd = pes.diatom(base.r2.r)
    psi, e_vj, phi = init_state_gpu(base.r1, base.r2, base.theta, j0, v0, vd, K=K)
    e_ref, phi_ref = S.diatom_vibrot(base.r2, pes.diatom, j0, v0)
    assert abs(e_vj - e_ref) < 1e-11 * max(1.0, abs(e_ref))
    assert np.abs(phi - phi_ref).max() < 1e-8 * np.abs(phi_ref).max()
    if K == 0:
        ref, _, _ = S.init_wavepacket(base.r1, base.r2, base.theta, j0, v0, pes.diatom)
    else:
        ref = S.cs_case(base, max(K, 1), K, v0, j0).psi
    assert np.abs(psi - ref).max() < 1e-8 * max(np.abs(ref).max(), 1e-300)
    e_coll = base.CRP.energies - base.CRP.eDiatomic
    assert np.abs(eta_sq_gpu(base.r1, e_coll) - S.eta_sq(base.r1, e_coll)).max() < \
        1e-12 * S.eta_sq(base.r1, e_coll).max()
