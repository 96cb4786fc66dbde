"""TEST INFRASTRUCTURE ONLY: FP64 Python restatement of the BKMP2 H3 surface
(Boothroyd, Keogh, Martin, Peterson 1996; the reference's H3/bkmp2.F, the
"jun21/95" parameter set that file uses), the checker of the GPU surface in
libqd.so (qd_bkmp2_*).  Only tests/ load this module.

Values only (the reference also forms dV/dr; the propagator needs V).  Parts
restated, with the reference lines:
* singlet H2 curve vH2opt95 (bkmp2.F:252-306), triplet curve with the
  Johnson short-range correction triplet95 (:176-250),
* London term h3lond95 (:356-392), asymmetric correction Vascal95 with
  acalc95 (:419-516),
* compact-geometry terms: compac95 (:518-551), casym95 (:553-653), csym95
  (:655-722),
* bending terms vbcb95 (:724-1417): Vbend with the B1a / B1b angular
  functions, and for compact geometries Cbend,
* sum of the parts (bkmp2:20-115).
H3/H3PESBKMP2.m:23-27 subtracts vH2Min = -0.174495770896975 from the MEX
value; `pes()` below does the same.

Parity: the reference is Fortran and no Fortran compiler exists here, so it
cannot be run; the restatement is pinned only through the H2 limit (the
vibrational levels listed in H3/H2WaveFunctionTest.m, from the DVR of
H2VibRotWaveFunction.m on this surface at R = 100 bohr).  Three-body values
are "parity unpinned" beyond agreeing with the independent GPU restatement.
"""
import math

import numpy as np

VH2MIN = -0.174495770896975          # H3/H3PESBKMP2.m:19

# vH2opt95 (bkmp2.F:262-285): alpha(r) = a0/r + sum_{i>=1} a_i r^(i-1)
H2_A = [0.03537359271649620, 2.013977588700072, -2.827452449964767, 2.713257715593500,
        -2.792039234205731, 2.166542078766724, -1.272679684173909, 0.5630423099212294,
        -0.1879397372273814, 0.04719891893374140, -0.008851622656489644,
        0.001224998776243630, -1.227820520228028e-04, 8.638783190083473e-06,
        -4.036967926499151e-07, 1.123286608335365e-08, -1.406619156782167e-10]
H2_R0, H2_DD, H2_C6, H2_C8, H2_C10 = 3.5284882, 0.160979391, 6.499027, 124.3991, 3285.828
# triplet95 (bkmp2.F:200-204)
TR_A = [-0.0298546962, -23.9604445036, -42.5185569474, 2.0382390988, -11.5214861455,
        1.5309487826]
TR_C = [-0.4106358351531854, -0.0770355790707090, 0.4303193846943223]
TR_RL, TR_RR = 0.95, 1.15
# Vascal95 (bkmp2.F:437-441)
AS = [0.3788951192e-02, 0.1478100901e-02, -.1848513849e-03, 0.9230803609e-05,
      -.1293180255e-06, 0.5237179303e+00, -.1112326215e-02]
# compac95 / csym95 / casym95 (bkmp2.F:526, 669-671, 570-575)
RR, RP = 1.15, 1.25
CSYM = [-.2071708868e+00, -.5672350377e+00, 0.9058780367e-02]
CASYM = [0.2210243144e+00, 0.4367417579e+00, 0.6994985432e-02, 0.1491096501e+01,
         0.1602896673e+01, -.2821747323e+01, 0.4948310833e+00, -.3540394679e-01,
         -.3305809954e+01, 0.3644382172e+01, -.9997570970e+00, 0.7989919534e-01,
         -.1075807322e-02]
# vbcb95 (bkmp2.F:762-858)
BETA1, BETA2, BETA3 = 0.52, 0.052, 0.79
# Vbend sets (a: with B1a, g: with B1b): p11 p12 p13 | p21..p24 | p31 p32 | p41..p44 | p51..p53
VBA = dict(p1=[-.1838073394e+03, 0.1334593242e+02, -.2358129537e+00],
           p2=[-.4668193478e+01, 0.7197506670e+01, 0.2162004275e+02, 0.2106294028e+02],
           p3=[0.4242962586e+01, 0.4453505045e+01],
           p4=[-.1456918088e+00, -.1692657366e-01, 0.1279520698e+01, -.4898940075e+00],
           p5=[0.1742295219e+03, 0.3142175348e+02, 0.5152903406e+01])
VBB = dict(p1=[-.4765732725e+02, 0.3648933563e+01, -.7141145244e-01],
           p2=[0.1002349176e-01, 0.9989856329e-02, -.4161953634e-02, 0.9075807910e-03],
           p3=[-.2693628729e+00, -.1399065763e-01],
           p4=[-.1417634346e-01, -.4870024792e-03, 0.1312231847e+00, -.4409850519e-01],
           p5=[0.5382970863e+02, 0.4587102824e+01, 0.1768550515e+01])
# Cbend sets (c: with B1a, d: with B1b): q1 (5) | q2 (4) | q3 (2) | q4 (4) | q5 (3) | q6 (3) | q7 (5) | q8 (4)
CBA = dict(q1=[0.1860299931e+04, -.6134458037e+03, 0.7337207161e+02, -.2676717625e+04,
               0.1344099415e+04],
           q2=[0.1538913137e+03, 0.4348007369e+02, 0.1719720677e+03, 0.2115963042e+03],
           q3=[-.7026089414e+02, -.1300938992e+03],
           q4=[0.1310273564e+01, -.6175149574e+00, -.2679089358e+02, 0.5577477171e+01],
           q5=[-.3543353539e+04, -.3740709591e+03, 0.7979303144e+02],
           q6=[-.1104230585e+04, 0.4603572025e+04, -.5593496634e+04],
           q7=[-.1069406434e+02, 0.1021807153e+01, 0.6669828341e-01, 0.4168542348e+02,
               0.1751608567e+02],
           q8=[0.9486883238e+02, -.1519334221e+02, 0.4024697252e+04, -.2225159395e+02])
CBB = dict(q1=[0.4203543357e+03, -.4922474096e+02, 0.3362942544e+00, -.3827423082e+03,
               0.1746726001e+03],
           q2=[0.1699995737e-01, 0.1513036778e-01, 0.2659119354e-01, -.5760387483e-02],
           q3=[0.1020622621e+02, 0.1050536271e-01],
           q4=[0.6836172780e+00, -.1627858240e+00, -.6925485045e+01, 0.1632567385e+01],
           q5=[0.1083595009e+04, 0.4641431791e+01, -.8233144461e+00],
           q6=[-.6157225942e+02, 0.3094361471e+03, -.3299631143e+03],
           q7=[0.8866227120e+01, -.1382126854e+01, 0.7620770145e-01, -.5145757859e+02,
               0.2046097265e+01],
           q8=[0.2540775558e+01, -.4889246569e+00, -.1127439280e+04, -.2269932295e+01])


def singlet(r):
    """vH2opt95 value."""
    rp = [1.0, r]
    for _ in range(14):
        rp.append(rp[-1] * r)                       # r^0 .. r^15
    r02 = H2_R0 * H2_R0
    r04 = r02 * r02
    r06 = r04 * r02
    rr2 = rp[2] + r02
    rr4 = rp[4] + r04
    rr6 = rp[6] + r06
    rr25 = rr2 * rr2 * rr2 * rr2 * rr2
    alpha = H2_A[0] / r + H2_A[1]
    for i in range(2, 17):
        alpha = alpha + H2_A[i] * rp[i - 1]
    ex = math.exp(alpha)
    vsr = H2_DD * (ex - 1.0) * (ex - 1.0) - H2_DD
    vlr = -H2_C6 / rr6 - H2_C8 / (rr4 * rr4) - H2_C10 / rr25
    return vsr + vlr


def triplet(r):
    a1, a2, a3, a4, a5, a6 = TR_A
    c1, c2, c3 = TR_C
    if r >= TR_RR:
        return a1 * (a2 + r + a3 * (r * r) + a5 * r ** (-a6)) * math.exp(-a4 * r)
    dr = r - TR_RL
    e1 = singlet(r)
    if r <= TR_RL:
        return e1 + c2 * dr + c3
    return e1 + c1 * dr * dr * dr + c2 * dr + c3


def london(r):
    q, j = [], []
    for ri in r:
        e1, e3 = singlet(ri), triplet(ri)
        q.append(0.5 * (e1 + e3))
        j.append(0.5 * (e1 - e3))
    sumq = q[0] + q[1] + q[2]
    sumj = (j[1] - j[0]) ** 2 + (j[2] - j[1]) ** 2 + (j[2] - j[0]) ** 2
    return sumq - math.sqrt(0.5 * sumj + 1e-12)


def acalc(r1, r2, r3):
    return abs((r1 - r2) * (r2 - r3) * (r3 - r1))


def vascal(r):
    r1, r2, r3 = r
    R = r1 + r2 + r3
    A = acalc(r1, r2, r3)
    A2 = A * A
    A3 = A2 * A
    A4 = A3 * A
    A5 = A4 * A
    aa1, aa2, aa3, aa4, aa5, aa6, aa7 = AS
    S = aa2 * A2 + aa3 * A3 + aa4 * A4 + aa5 * A5
    return S * math.exp(-aa1 * (R * R * R)) + aa7 * A2 * math.exp(-aa6 * R) / R


def compac(r):
    T = [0.0, 0.0, 0.0]
    n = 0
    for i, ri in enumerate(r):
        if ri < RR:
            n += 1
            top = RR - ri
            T[i] = top * top * top / (RP - ri)
    return n, T


def csym(r):
    v1, v2, v3 = CSYM
    Sr = r[0] + r[1] + r[2]
    e3 = math.exp(-v3 * (Sr * Sr * Sr))
    sg = 0.0
    for ri in r:
        if ri < RR:
            d = RR - ri
            sg += (d * d * d / (RP - ri)) * (v1 + v1 * v2 * ri)
    return sg * e3


def casym(r, T):
    u = CASYM
    A = acalc(*r)
    A2 = A * A
    sumt = T[0] + T[1] + T[2]
    Sr = r[0] + r[1] + r[2]
    Pr = r[0] * r[1] * r[2]
    Pr2 = Pr * Pr
    series = (1.0 + u[3] / Pr2 + u[4] / Pr + u[5] + u[6] * Pr + u[7] * Pr2
              + A * (u[8] / Pr2 + u[9] / Pr + u[10] + u[11] * Pr + u[12] * Pr2))
    term1 = u[0] / Pr ** u[1]
    eterm = math.exp(-u[2] * (Sr * Sr * Sr))
    return sumt * A2 * term1 * series * eterm


def bends(r, icompc, T):
    """(Vbnda, Vbndb, Cbnda, Cbndb) of vbcb95."""
    r1, r2, r3 = r
    t1 = r1 * r1 - r2 * r2 - r3 * r3
    t2 = r2 * r2 - r3 * r3 - r1 * r1
    t3 = r3 * r3 - r1 * r1 - r2 * r2
    c1 = t1 / (-2.0 * r2 * r3)
    c2 = t2 / (-2.0 * r3 * r1)
    c3 = t3 / (-2.0 * r1 * r2)
    s = c1 + c2 + c3
    B1a = 1.0 - s
    sumb = (4.0 * c1 ** 3 - 3.0 * c1) + (4.0 * c2 ** 3 - 3.0 * c2) + (4.0 * c3 ** 3 - 3.0 * c3)
    B1b = 1.0 - (0.625 * sumb + 0.375 * s)
    R = r1 + r2 + r3
    Rsq = R * R
    B2 = 1.0 / r1 + 1.0 / r2 + 1.0 / r3
    B3 = (r2 - r1) ** 2 + (r3 - r2) ** 2 + (r1 - r3) ** 2
    B3b = math.sqrt(B3 + 1e-12)
    exp1 = math.exp(-BETA1 * R)
    exp2 = math.exp(-BETA2 * Rsq)
    exp7 = math.exp(-BETA3 * R)

    def vbend(B1, p):
        B12 = B1 * B1
        B13 = B12 * B1
        B14 = B13 * B1
        B15 = B14 * B1
        asum = p["p1"][0] + p["p1"][1] * R + p["p1"][2] * Rsq
        bsum = p["p2"][0] * B12 + p["p2"][1] * B13 + p["p2"][2] * B14 + p["p2"][3] * B15
        csum = p["p3"][0] * B1 * exp1 + p["p3"][1] * B12 * exp2
        d1 = p["p4"][0] * exp1 + p["p4"][1] * exp2
        d2 = p["p4"][2] * exp1 + p["p4"][3] * exp2
        fsum = p["p5"][0] + p["p5"][1] * R + p["p5"][2] * Rsq
        return (B1 * asum * exp1 + bsum * exp2 + B2 * csum + (B1 * B3 * d1 + B1 * B3b * d2)
                + B1 * fsum * exp7)

    va, vb = vbend(B1a, VBA), vbend(B1b, VBB)
    if icompc == 0:
        return va, vb, 0.0, 0.0
    sumT = T[0] + T[1] + T[2]
    P = r1 * r2 * r3
    Psq = P * P
    e7 = math.exp(-BETA2 * (Rsq * R))

    def cbend(B1, q):
        B12 = B1 * B1
        B13 = B12 * B1
        B14 = B13 * B1
        B15 = B14 * B1
        asum = q["q1"][0] + q["q1"][1] * R + q["q1"][2] * Rsq + q["q1"][3] / R + q["q1"][4] / Rsq
        bsum = q["q2"][0] * B12 + q["q2"][1] * B13 + q["q2"][2] * B14 + q["q2"][3] * B15
        csum = q["q3"][0] * B1 * exp1 + q["q3"][1] * B12 * exp2
        d1 = q["q4"][0] * exp1 + q["q4"][1] * exp2
        d2 = q["q4"][2] * exp1 + q["q4"][3] * exp2
        fsum = (q["q5"][0] + q["q8"][2]) + q["q5"][1] * R + q["q5"][2] * Rsq   # feb27/91: c51 + c83
        gsum = q["q6"][0] + q["q6"][1] / R + q["q6"][2] / Rsq
        aasum = q["q7"][0] + q["q7"][1] * P + q["q7"][2] * Psq + q["q7"][3] / P + q["q7"][4] / Psq
        ffsum = q["q8"][0] * P + q["q8"][1] * Psq + q["q8"][3] / Psq
        return (B1 * asum * exp1 / P + bsum * exp2 + B2 * csum + (B1 * B3 * d1 + B1 * B3b * d2)
                + B1 * fsum * e7 / P + B1 * gsum * e7 + B1 * aasum * exp2 + B1 * ffsum * e7)

    return va, vb, sumT * cbend(B1a, CBA), sumT * cbend(B1b, CBB)


def bkmp2(r1, r2, r3):
    """The MEX value (hartree) at the three internuclear distances (bohr)."""
    r = (float(r1), float(r2), float(r3))
    lo, hi = min(r), max(r)
    mid = sum(r) - lo - hi
    if lo + mid + 1e-5 < hi or lo < 0.2:          # chgeom (bkmp2.F:1418-1446) stops there
        return float("nan")
    icompc, T = compac(r)
    vlon, vas = london(r), vascal(r)
    cal = cas = 0.0
    if icompc >= 1:
        cal, cas = csym(r), casym(r, T)
    vbnda, vbndb, cbnda, cbndb = bends(r, icompc, T)
    return vlon + vas + vbnda + vbndb + cal + cas + cbnda + cbndb


def pes(r1, r2, r3):
    """H3PESBKMP2.m: the MEX value minus vH2Min, elementwise."""
    a, b, c = np.broadcast_arrays(*(np.asarray(v, dtype=float) for v in (r1, r2, r3)))
    out = np.array([bkmp2(x, y, z) for x, y, z in zip(a.ravel(), b.ravel(), c.ravel())])
    return out.reshape(a.shape) - VH2MIN
