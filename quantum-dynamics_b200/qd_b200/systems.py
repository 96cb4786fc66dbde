"""Problem set-up: the Matlab-driver side of the reference (its layer L4/L5).

Builds the run-parameter struct that the propagator consumes -- grids,
Gauss-Legendre quadrature, Legendre matrix, potential on the Jacobi grid,
absorbers, initial wavepacket, eta^2(E) and the dividing surface -- with the
same field names, units and layouts as the reference's Matlab struct
(H3/main.m:41-139, FH2/HSW/main.m).  Arrays are numpy, C-contiguous:

    psi, pot      shape (n_theta, n2, n1)  == Matlab (n1, n2, n_theta) column-major
    theta.legendre shape (n_theta, m+1)    == Matlab (m+1, n_theta) column-major

The potential is the extended-LEPS form whose Coulomb/exchange/Sato algebra
follows ClH2/G3/clh2g3v.F:89-101 (no three-centre term).
"""
import math
import os
import numpy as np

BOHR_PER_ANGSTROM = 1.0 / 0.529177210903
HARTREE_EV = 27.211386245988
AMU_ME = 1822.888486209


class Struct:
    """Attribute bag with the role of a Matlab struct."""

    def __init__(self, **kw):
        self.__dict__.update(kw)

    def __repr__(self):
        return "Struct(" + ", ".join(sorted(self.__dict__)) + ")"


def matlab_int32(x):
    """Matlab's int32(): round half away from zero."""
    return int(math.floor(abs(x) + 0.5)) * (1 if x >= 0 else -1)


# ---------------------------------------------------------------------------
# Quadrature and angular basis
# ---------------------------------------------------------------------------

def gauss_legendre(n):
    """Gauss-Legendre nodes (ascending) and weights on [-1, 1], FP64.

    Newton iteration on P_n from the Tricomi initial guesses; matches the
    reference's tabulated GaussLegendre/<n>-LegendreGauss.grids to rounding.
    """
    x = np.empty(n)
    w = np.empty(n)
    for i in range(n):
        # i-th root from the top, Tricomi's approximation
        t = math.pi * (4 * (i + 1) - 1) / (4 * n + 2)
        z = math.cos(t) * (1 - (n - 1) / (8.0 * n ** 3))
        for _ in range(100):
            p0, p1 = 1.0, z
            for k in range(2, n + 1):
                p0, p1 = p1, ((2 * k - 1) * z * p1 - (k - 1) * p0) / k
            if n == 1:
                p1, p0 = z, 1.0
            dp = n * (z * p1 - p0) / (z * z - 1.0) if n > 1 else 1.0
            dz = p1 / dp
            z -= dz
            if abs(dz) < 1e-17:
                break
        p0, p1 = 1.0, z
        for k in range(2, n + 1):
            p0, p1 = p1, ((2 * k - 1) * z * p1 - (k - 1) * p0) / k
        if n == 1:
            p1, p0 = z, 1.0
        dp = n * (z * p1 - p0) / (z * z - 1.0) if n > 1 else 1.0
        x[n - 1 - i] = z
        w[n - 1 - i] = 2.0 / ((1.0 - z * z) * dp * dp)
    if n % 2 == 1:
        x[n // 2] = 0.0
    return x, w


def read_grids(directory, n):
    """Read "<n>-LegendreGauss.grids" (common/GaussLegendre2.m:1-31): the
    ceil(n/2) non-negative nodes with weights, mirrored to ascending x."""
    path = os.path.join(directory, f"{n}-LegendreGauss.grids")
    if not (1 <= n <= 599):
        raise ValueError("argument should be 1 <= n <= 599")
    if not os.path.exists(path):
        raise FileNotFoundError(f'"{path}" does not exist')
    vals = np.loadtxt(path, ndmin=2)
    xh, wh = vals[:, 0].copy(), vals[:, 1].copy()
    if n != 2 * xh.size - (n % 2):
        raise ValueError(f"{path}: {xh.size} lines do not describe n = {n}")
    if n % 2:
        x = np.concatenate([-xh[:0:-1], xh])
        w = np.concatenate([wh[:0:-1], wh])
    else:
        x = np.concatenate([-xh[::-1], xh])
        w = np.concatenate([wh[::-1], wh])
    return x, w


def write_grids(path, x, w):
    """Write the non-negative half in the .grids format (32 digits)."""
    n = x.size
    h = n // 2
    with open(path, "w") as f:
        for xi, wi in zip(x[h:], w[h:]):
            f.write(f"{xi:.32f}  {wi:.32f}  \n")


def legendre_p2(m, x):
    """P_0..P_m at x by the recurrence of common/LegendreP2.m:9-21.
    Returns shape (len(x), m+1); as C memory this is the reference's
    transposed (m+1) x n theta.legendre (H3/main.m:98-101)."""
    x = np.asarray(x, dtype=np.float64)
    v = np.zeros((x.size, m + 1))
    v[:, 0] = 1.0
    if m >= 1:
        v[:, 1] = x
    for i in range(2, m + 1):
        v[:, i] = (2 - 1 / i) * x * v[:, i - 1] - (1 - 1 / i) * v[:, i - 2]
    return np.ascontiguousarray(v)


def legendre_p(j, x):
    """P_j(x) (common/LegendreP.m)."""
    return legendre_p2(j, x)[:, j]


# ---------------------------------------------------------------------------
# Potential energy surfaces
# ---------------------------------------------------------------------------

class MorseSato:
    """One diatom of an extended-LEPS surface, in atomic units."""

    def __init__(self, de_ev, beta_inv_angstrom, re_angstrom, sato):
        self.de = de_ev / HARTREE_EV
        self.beta = beta_inv_angstrom / BOHR_PER_ANGSTROM
        self.re = re_angstrom * BOHR_PER_ANGSTROM
        self.sato = sato
        self.pf = 0.5 * self.de * (1.0 - sato) / (1.0 + sato)

    def coulomb_exchange(self, r):
        """Coulomb Q and exchange J integrals (clh2g3v.F:89-97): singlet
        de*y*(y-2), anti-Morse triplet pf*y*(y+2), y = exp(-beta (r - re))."""
        y = np.exp(-self.beta * (r - self.re))
        q = 0.5 * (self.de * (y - 2.0) + self.pf * (y + 2.0)) * y
        j = 0.5 * (self.de * (y - 2.0) - self.pf * (y + 2.0)) * y
        return q, j

    def morse(self, r):
        y = np.exp(-self.beta * (r - self.re))
        return self.de * (1.0 - y) ** 2


class LEPS:
    """A + BC extended-LEPS: V = QAB + QBC + QAC - sqrt(JAB^2 + JBC^2 + JAC^2
    - JAB JBC - JBC JAC - JAC JAB) + De(BC) (zero at A + BC(r_e))."""

    def __init__(self, ab, bc, ac):
        self.ab, self.bc, self.ac = ab, bc, ac

    def __call__(self, r_ab, r_bc, r_ac):
        q1, j1 = self.ab.coulomb_exchange(r_ab)
        q2, j2 = self.bc.coulomb_exchange(r_bc)
        q3, j3 = self.ac.coulomb_exchange(r_ac)
        rad = np.sqrt(np.maximum(j1 * (j1 - j2) + j2 * (j2 - j3) + j3 * (j3 - j1), 0.0))
        return self.bc.de + q1 + q2 + q3 - rad

    def diatom(self, r):
        """Asymptotic BC potential (A far away)."""
        return self.bc.morse(r)


def leps_h_h2():
    hh = MorseSato(4.7466, 1.9425, 0.7416, 0.17)
    return LEPS(hh, hh, hh)


def leps_f_h2():
    fh = MorseSato(6.12, 2.2187, 0.9170, 0.167)
    hh = MorseSato(4.7466, 1.9425, 0.7416, 0.106)
    return LEPS(fh, hh, fh)


def jacobi_to_internuclear(R, r, cos_theta, masses):
    """Reactant Jacobi (R, r, theta) -> (r12, r13, r23) for atoms 1 + (2 3)
    (H3/H3PESJacobi.m:5-24, f2 = m3/(m2+m3))."""
    f2 = masses[2] / (masses[1] + masses[2])
    f3 = 1.0 - f2
    r23 = r
    r12 = np.sqrt((f2 * r) ** 2 + R ** 2 - 2 * f2 * r * R * cos_theta)
    r13 = np.sqrt((f3 * r) ** 2 + R ** 2 + 2 * f3 * r * R * cos_theta)
    return r12, r13, r23


def potential_on_grid(R, r, x, masses, pes, vmax=2.5, rmin=0.4):
    """V(i, j, k) on the Jacobi grid, shape (n_theta, n2, n1); VMax where any
    internuclear distance <= rmin (H3/H3PESJacobi.m:13-27) and V capped at
    VMax elsewhere."""
    X = np.asarray(x)[:, None, None]
    Rr = np.asarray(R)[None, None, :]
    rr = np.asarray(r)[None, :, None]
    r12, r13, r23 = jacobi_to_internuclear(Rr, rr, X, masses)
    r12, r13, r23 = np.broadcast_arrays(r12, r13, r23)
    V = np.full(r12.shape, vmax, dtype=np.float64)
    ok = (r12 > rmin) & (r13 > rmin) & (r23 > rmin)
    V[ok] = np.minimum(pes(r12[ok], r23[ok], r13[ok]), vmax)
    return np.ascontiguousarray(V)


# ---------------------------------------------------------------------------
# Absorbers, initial state, eta^2
# ---------------------------------------------------------------------------

def woods_saxon(cd, xd, x):
    """common/WoodsSaxon.m:4-5."""
    return 1.0 / (1.0 + np.exp(cd * (np.asarray(x) - xd)))


def quadratic_absorber(x, x_start, strength):
    """Per-step damping exp(-strength ((x - x_start)/(x_max - x_start))^2)
    beyond x_start, 1 before it."""
    x = np.asarray(x, dtype=np.float64)
    u = np.clip((x - x_start) / (x[-1] - x_start), 0.0, None)
    return np.ascontiguousarray(np.exp(-strength * u * u))


def diatom_vibrot(r2, v_diatom, j_rot, v_vib):
    """Sinc-DVR eigenstate of the diatom (H3/H2VibRotWaveFunction.m:20-46).
    Returns (energy, psi(r)/sqrt(dr)); the eigenvector sign is fixed so that
    its largest-magnitude component is positive."""
    n = int(r2.n)
    dr, mu, r = r2.dr, r2.mass, r2.r
    i = np.arange(1, n + 1, dtype=np.float64)
    I, J = np.meshgrid(i, i, indexing="ij")
    with np.errstate(divide="ignore", invalid="ignore"):
        H = (-1.0) ** (I - J) * (2.0 / (I - J) ** 2 - 2.0 / (I + J) ** 2)
    H[np.diag_indices(n)] = np.pi ** 2 / 3 - 1.0 / (2 * i * i)
    H /= 2 * mu * dr * dr
    V = v_diatom(r) + j_rot * (j_rot + 1) / (2 * mu * r ** 2)
    H[np.diag_indices(n)] += V
    e, vecs = np.linalg.eigh(H)
    vec = vecs[:, v_vib]
    if vec[np.argmax(np.abs(vec))] < 0:
        vec = -vec
    return float(e[v_vib]), vec / math.sqrt(dr)


def init_wavepacket(r1, r2, theta, j_rot, v_vib, v_diatom):
    """psi = g(R) phi_vj(r) sqrt(j+1/2) P_j(x_k) (H3/InitWavePacket.m:1-31),
    g = (pi delta^2)^(-1/4) exp(-(R-R0)^2/(2 delta^2) - i k0 R)."""
    R = r1.r
    g = (1.0 / (math.pi * r1.delta ** 2)) ** 0.25 * np.exp(
        -(R - r1.r0) ** 2 / (2 * r1.delta ** 2) - 1j * r1.k0 * R)
    e_vj, phi = diatom_vibrot(r2, v_diatom, j_rot, v_vib)
    P = math.sqrt(j_rot + 0.5) * legendre_p(j_rot, theta.x)
    psi = P[:, None, None] * phi[None, :, None] * g[None, None, :]
    return np.ascontiguousarray(psi.astype(np.complex128)), e_vj, phi


def eta_sq(r1, e_coll):
    """common/EtaSq.m:12-15 (J. Chem. Phys. 110, 11221 (1999))."""
    kE = np.sqrt(2 * r1.mass * np.asarray(e_coll, dtype=np.complex128))
    eta = math.pi ** 0.25 * np.sqrt(2 * r1.mass * r1.delta / kE) * np.exp(
        -r1.delta ** 2 / 2 * (kE - r1.k0) ** 2)
    return np.ascontiguousarray(np.abs(eta) ** 2)


# ---------------------------------------------------------------------------
# Whole cases
# ---------------------------------------------------------------------------

def build_case(system="h+h2", n1=64, n2=64, n_theta=40, m=None,
               R=(0.5, 12.0), r=(0.4, 8.0), R0=8.0, delta=0.3, e0_ev=0.5,
               j0=0, v0=0, time_step=10.0, total_steps=2000,
               absorb_len=2.0, absorb_strength=0.3, r_surface=4.5,
               n_gradient_points=11, e_range_ev=(0.3, 1.5), n_energies=241,
               vmax=2.5, precision=0, grids_dir=None):
    """Build the struct of one J = 0 propagation.  Defaults are the H + H2
    LEPS case on a 64 x 64 x 40 grid (j_max = 38)."""
    if system == "h+h2":
        pes = leps_h_h2()
        m_amu = (1.00783, 1.00783, 1.00783)
    elif system == "f+h2":
        pes = leps_f_h2()
        m_amu = (18.9984, 1.00783, 1.00783)
    else:
        raise ValueError(system)
    masses = np.array(m_amu) * AMU_ME
    if m is None:
        m = n_theta - 2 if system == "h+h2" and n_theta == 40 else n_theta - 1

    rg1 = np.linspace(R[0], R[1], n1)
    rg2 = np.linspace(r[0], r[1], n2)
    mu_R = masses[0] * (masses[1] + masses[2]) / masses.sum()
    mu_r = masses[1] * masses[2] / (masses[1] + masses[2])
    k0 = math.sqrt(2 * mu_R * e0_ev / HARTREE_EV)
    r1 = Struct(n=n1, r=rg1, dr=rg1[1] - rg1[0], mass=mu_R, r0=R0, k0=k0, delta=delta)
    r2 = Struct(n=n2, r=rg2, dr=rg2[1] - rg2[0], mass=mu_r, r0=0.0, k0=0.0, delta=0.0)

    if grids_dir is not None:
        x, w = read_grids(grids_dir, n_theta)
    else:
        x, w = gauss_legendre(n_theta)
    theta = Struct(n=n_theta, m=m, x=x, w=w, legendre=legendre_p2(m, x))

    pot = potential_on_grid(rg1, rg2, x, masses, pes, vmax=vmax)
    psi, e_vj, _ = init_wavepacket(r1, r2, theta, j0, v0, pes.diatom)

    dump1 = Struct(dump=quadratic_absorber(rg1, R[1] - absorb_len, absorb_strength))
    dump2 = Struct(dump=quadratic_absorber(rg2, r[1] - absorb_len, absorb_strength))

    e_coll = np.linspace(e_range_ev[0], e_range_ev[1], n_energies) / HARTREE_EV
    n_div = matlab_int32((r_surface - rg2.min()) / r2.dr)
    CRP = Struct(eDiatomic=e_vj, n_dividing_surface=n_div,
                 n_gradient_points=n_gradient_points, n_energies=n_energies,
                 energies=np.ascontiguousarray(e_coll + e_vj),
                 eta_sq=eta_sq(r1, e_coll), CRP=np.zeros(n_energies),
                 calculate_CRP=1)
    time = Struct(total_steps=total_steps, time_step=time_step, steps=0)
    options = Struct(wave_to_matlab=None, test_name=f"{system} {n1}x{n2}x{n_theta}",
                     steps_to_copy_psi_from_device_to_host=0, precision=precision)
    return Struct(r1=r1, r2=r2, theta=theta, pot=pot, psi=psi, time=time,
                  options=options, dump1=dump1, dump2=dump2, CRP=CRP,
                  masses=masses, system=system)


def case_c0(**kw):
    """H + H2 J=0 LEPS, 64 x 64 x 40, j_max 38, dt 10 au, 2000 steps."""
    return build_case("h+h2", 64, 64, 40, m=38, **kw)


def case_c1(**kw):
    """F + H2 J=0 LEPS, 128 x 128 x 64 (j_max 63), dt 10 au, 10000 steps."""
    kw.setdefault("total_steps", 10000)
    return build_case("f+h2", 128, 128, 64, m=63, **kw)


def batch_cases(base, states):
    """Runs of one batch: `base` with the initial diatomic state (v0, j0)
    replaced per run (psi, CRP.energies, CRP.eta_sq); grid and potential are
    shared (the same pot array)."""
    pes = leps_f_h2() if base.system == "f+h2" else leps_h_h2()
    e_coll = base.CRP.energies - base.CRP.eDiatomic
    runs = []
    for v0, j0 in states:
        d = copy_case(base)
        d.psi, e_vj, _ = init_wavepacket(d.r1, d.r2, d.theta, j0, v0, pes.diatom)
        d.CRP.eDiatomic = e_vj
        d.CRP.energies = np.ascontiguousarray(e_coll + e_vj)
        d.CRP.eta_sq = eta_sq(d.r1, e_coll)
        d.CRP.CRP = np.zeros(int(d.CRP.n_energies))
        d.pot = base.pot
        runs.append(d)
    return runs


def case_c2_j0(n_runs=64, **kw):
    """F + H2 J = 0 batch on the 128 x 96 x 64 grid (n_l = 64): n_runs
    propagations with initial states cycling over (v0, j0) = (0,0), (0,1),
    (0,2), (1,0)."""
    kw.setdefault("total_steps", 10000)
    base = build_case("f+h2", 128, 96, 64, m=63, r=(0.4, 8.0), **kw)
    states = [((0, 0), (0, 1), (0, 2), (1, 0))[i % 4] for i in range(n_runs)]
    return batch_cases(base, states)


def cs_legendre(x, K, m):
    """theta.legendre of centrifugal-sudden block K: column l (l = 0..m) is
    Pbar_{K+l}^K(x_k) / sqrt(l + 1/2), Pbar_j^K the associated Legendre
    function normalised to one on [-1, 1] (no Condon-Shortley phase), so that
    the reference's transform pair (B with L, F with (l+1/2) w_k L) is the
    identity on the basis.  K = 0 is legendre_p2 itself.  Shape (n, m+1)."""
    if K == 0:
        return legendre_p2(m, x)
    x = np.asarray(x, dtype=np.float64)
    s = np.sqrt(1.0 - x * x)
    p0 = np.full(x.size, math.sqrt(0.5))
    for mm in range(1, K + 1):                        # Pbar_K^K
        p0 = p0 * math.sqrt((2 * mm + 1) / (2 * mm)) * s
    v = np.zeros((x.size, m + 1))
    v[:, 0] = p0
    if m >= 1:
        p1 = math.sqrt(2 * K + 3) * x * p0            # Pbar_{K+1}^K
        v[:, 1] = p1
    for l in range(2, m + 1):
        j = K + l
        a = math.sqrt((4 * j * j - 1) / (j * j - K * K))
        b = math.sqrt(((j - 1) ** 2 - K * K) / (4 * (j - 1) ** 2 - 1))
        v[:, l] = a * (x * v[:, l - 1] - b * v[:, l - 2])
    v /= np.sqrt(np.arange(m + 1) + 0.5)[None, :]
    return np.ascontiguousarray(v)


def cs_case(base, J, K, v0, j0, j_max=None):
    """The run of centrifugal-sudden block (J, K) with initial diatom state
    (v0, j0), built from a J = 0 case `base`: angular basis Pbar_j^K for
    j = K .. j_max (n_j = j_max - K + 1), the centrifugal term
    (J(J+1) - 2K^2)/(2 mu_R R^2) added to the potential, and the initial packet
    g(R) phi_{v0 j0}(r) Pbar_{j0}^K(theta) (zero when K > j0: no such state)."""
    pes = leps_f_h2() if base.system == "f+h2" else leps_h_h2()
    if j_max is None:
        j_max = int(base.theta.m)
    d = copy_case(base)
    m = j_max - K
    th = Struct(**vars(base.theta))
    th.m = m
    th.legendre = cs_legendre(th.x, K, m)
    d.theta = th
    d.cs = Struct(J=J, K=K)
    R = base.r1.r
    cent = (J * (J + 1) - 2 * K * K) / (2 * base.r1.mass * R * R)
    d.pot = np.ascontiguousarray(base.pot + cent[None, None, :])
    g = (1.0 / (math.pi * base.r1.delta ** 2)) ** 0.25 * np.exp(
        -(R - base.r1.r0) ** 2 / (2 * base.r1.delta ** 2) - 1j * base.r1.k0 * R)
    e_vj, phi = diatom_vibrot(base.r2, pes.diatom, j0, v0)
    if K <= j0:
        ang = cs_legendre(th.x, K, j0 - K)[:, j0 - K] * math.sqrt(j0 - K + 0.5)
    else:
        ang = np.zeros(th.x.size)
    d.psi = np.ascontiguousarray((ang[:, None, None] * phi[None, :, None] *
                                  g[None, None, :]).astype(np.complex128))
    e_coll = base.CRP.energies - base.CRP.eDiatomic
    d.CRP.eDiatomic = e_vj
    d.CRP.energies = np.ascontiguousarray(e_coll + e_vj)
    d.CRP.eta_sq = eta_sq(base.r1, e_coll)
    d.CRP.CRP = np.zeros(int(base.CRP.n_energies))
    return d


def case_c2(n_runs=64, **kw):
    """The batched F + H2 configuration on the 128 x 96 x 64 grid: centrifugal-
    sudden blocks J in (0, 5, 10, 15, 20), K = 0 .. min(J, 4) (n_j = 64 - K),
    crossed with the initial states (v0, j0) = (0,0), (0,1), (0,2), (1,0), in
    that order, the first n_runs of them."""
    kw.setdefault("total_steps", 10000)
    base = build_case("f+h2", 128, 96, 64, m=63, r=(0.4, 8.0), **kw)
    combos = [(J, K, v0, j0) for J in (0, 5, 10, 15, 20) for K in range(min(J, 4) + 1)
              for (v0, j0) in ((0, 0), (0, 1), (0, 2), (1, 0))]
    return [cs_case(base, *c) for c in combos[:n_runs]]


def case_c4(n_runs=32, **kw):
    """The large batched F + H2 configuration on the 256 x 192 x 128 grid
    (j_max 127): centrifugal-sudden blocks J in (0, 4, ..., 28) with
    K = 0 .. min(J, 3), then J = 30 with K = 0 .. 2 (32 blocks, J = 0-30,
    K <= 3, n_j = 128 - K), all from the initial state (v0, j0) = (0, 3) so
    that every block carries a packet; the first n_runs of them."""
    kw.setdefault("total_steps", 20000)
    base = build_case("f+h2", 256, 192, 128, m=127, r=(0.4, 8.0), **kw)
    combos = [(J, K) for J in range(0, 29, 4) for K in range(min(J, 3) + 1)]
    combos += [(30, K) for K in range(3)]
    return [cs_case(base, J, K, 0, 3) for J, K in combos[:n_runs]]


def copy_case(data):
    """Deep copy of the arrays that a propagation mutates (psi, CRP, time)."""
    import copy
    d = copy.copy(data)
    d.psi = data.psi.copy()
    d.time = Struct(**vars(data.time))
    d.CRP = Struct(**vars(data.CRP))
    d.CRP.CRP = data.CRP.CRP.copy()
    d.options = Struct(**vars(data.options))
    return d
