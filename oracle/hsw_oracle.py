"""TEST INFRASTRUCTURE ONLY: FP64 numpy restatement of the HSW surface of
F + H2 (the reference's FH2/HSW/hswpot.F and sospline.F), the checker of the
GPU surface in libqd.so (qd_hsw_*).  Only tests/ load this module.

Inputs are the numbers of the reference's four data files (three.param,
two.param, so.input, so.param), as read by `read_tables(dir)` or loaded from
the committed fixture tests/golden/hsw_tables.npz.

Steps restated (file:line of the reference):
* SW1 three-body sum over the three.param records with
  X_q = q exp(-b_q (q - q0)) and the powers by repeated multiplication
  (hswpot.F:133-183); extended-Rydberg two-body terms (hswpot.F:185-208).
* Spin-orbit correction: node slopes along each axis from clamped cubic
  splines (sospline.F:53-285), the end slopes of the value splines from the
  four-point Lagrange derivative (sospline.F:291-314), zero end slopes for the
  cross derivatives (SPLINF(2)), tridiagonal solve (sospline.F:316-335);
  tricubic Hermite evaluation in the cell found by the reference's search
  (sospline.F:338-425, node gathering FORMV :427-505).
* The valley test, clamping and angle folding, and the final shift by the
  single-precision constant 0.0006 (hswpot.F:46-98).
"""
import math
import os

import numpy as np

AUKCAL = 627.5095          # hswpot.F:17
SHIFT = float(np.float32(0.0006))   # hswpot.F:98, a default-real constant


def read_tables(d):
    """The four data files of directory d as arrays, in file order."""
    three = [ln.split() for ln in open(os.path.join(d, "three.param")) if ln.strip()]
    ix = np.array([int(r[1]) for r in three], np.int32)
    iy = np.array([int(r[2]) for r in three], np.int32)
    iz = np.array([int(r[3]) for r in three], np.int32)
    a = np.array([float(r[4]) for r in three])
    p = np.array([float(ln.split()[0]) for ln in open(os.path.join(d, "two.param"))
                  if ln.strip()])
    lines = [ln.split() for ln in open(os.path.join(d, "so.input")) if ln.strip()]
    nx, ny, nz = (int(v) for v in lines[0][:3])
    rec = np.array([[float(v) for v in r[:4]] for r in lines[1:1 + nx * ny * nz]])
    so = rec[:, 3].reshape(nx, ny, nz)
    x = rec[::ny * nz, 0].copy()
    y = rec[:ny * nz:nz, 1].copy()
    z = rec[:nz, 2].copy()
    sop = np.array([float(ln.split()[0]) for ln in open(os.path.join(d, "so.param"))
                    if ln.strip()])[:3]
    return dict(ix=ix, iy=iy, iz=iz, a=a, p=p[:12], x=x, y=y, z=z, so=so, so_param=sop)


def lagrange_slope(x, y, ip):
    d = 0.0
    for i in range(4):
        if i == ip:
            continue
        t = y[i]
        for j in range(4):
            if j != ip and j != i:
                t *= x[ip] - x[j]
        for j in range(4):
            if j != i:
                t /= x[i] - x[j]
        d += t
    for i in range(4):
        if i != ip:
            d += y[ip] / (x[ip] - x[i])
    return d


def spline_slopes(g, f, s0, sn):
    n = len(g)
    n2 = n - 2
    s = np.zeros(n)
    s[0], s[-1] = s0, sn
    h = [g[i + 1] - g[i] for i in range(n - 1)]
    lam = [h[i + 1] / (h[i] + h[i + 1]) for i in range(n2)]
    mu = [1.0 - lam[i] for i in range(n2)]
    b = [3.0 * lam[i] / h[i] * (f[i + 1] - f[i]) + 3.0 * mu[i] / h[i + 1] * (f[i + 2] - f[i + 1])
         for i in range(n2)]
    b[0] = b[0] - lam[0] * s0
    b[n2 - 1] = b[n2 - 1] - mu[n2 - 1] * sn
    piv = [2.0] * n2
    for i in range(1, n2):
        piv[i] = 2.0 - lam[i] * mu[i - 1] / piv[i - 1]
        b[i] = b[i] - lam[i] / piv[i - 1] * b[i - 1]
    xs = [0.0] * n2
    xs[n2 - 1] = b[n2 - 1] / piv[n2 - 1]
    for i in range(n2 - 2, -1, -1):
        xs[i] = (b[i] - xs[i + 1] * mu[i]) / piv[i]
    s[1:n - 1] = xs
    return s


class HswOracle:
    """The surface from the tables; pot(rhf1, rhh, rhf2) per point."""

    def __init__(self, t):
        self.ix, self.iy, self.iz = (np.asarray(t[k]) for k in ("ix", "iy", "iz"))
        a = np.asarray(t["a"], float)
        self.coef = a[:-6]
        self.b = a[-6:-3]
        self.q0 = a[-3:]
        self.p = np.asarray(t["p"], float)
        self.gx, self.gy, self.gz = (np.asarray(t[k], float) for k in ("x", "y", "z"))
        sp = np.asarray(t["so_param"], float)
        self.esocut, self.rsolim, self.rrsolm = sp[0] / AUKCAL, sp[1], sp[2]
        self.raddeg = 180.0 / math.acos(-1.0)
        F = np.asarray(t["so"], float)                         # [i][j][k]
        nx, ny, nz = F.shape
        T = np.zeros((8, nx, ny, nz))                          # t = dx + 2 dy + 4 dz
        T[0] = F

        def family(t_, src, ax, value):
            g = (self.gx, self.gy, self.gz)[ax]
            n = len(g)
            src_arr = np.moveaxis(T[src], ax, -1)
            out = np.moveaxis(T[t_], ax, -1)
            for idx in np.ndindex(src_arr.shape[:-1]):
                f = src_arr[idx]
                s0 = sn = 0.0
                if value:
                    s0 = lagrange_slope(g[:4], f[:4], 0)
                    sn = lagrange_slope(g[n - 4:], f[n - 4:], 3)
                out[idx] = spline_slopes(g, f, s0, sn)

        family(1, 0, 0, True)
        family(2, 0, 1, True)
        if nz > 1:
            family(4, 0, 2, True)
        family(3, 1, 1, False)
        if nz > 1:
            family(5, 1, 2, False)
            family(6, 2, 2, False)
            family(7, 3, 2, False)
        self.T = T

    def sw1(self, x, y, z):
        fx = x * math.exp(-(self.b[0] * (x - self.q0[0])))
        fy = y * math.exp(-(self.b[1] * (y - self.q0[1])))
        fz = z * math.exp(-(self.b[2] * (z - self.q0[2])))
        m = int(max(self.ix.max(), self.iy.max(), self.iz.max())) + 1
        px, py, pz = [1.0, fx], [1.0, fy], [1.0, fz]
        for _ in range(2, m):
            px.append(px[-1] * fx)
            py.append(py[-1] * fy)
            pz.append(pz[-1] * fz)
        fit = 0.0
        for c, i, j, k in zip(self.coef, self.ix, self.iy, self.iz):
            fit = fit + px[i] * py[j] * pz[k] * c
        p = self.p

        def ryd(r, d, c1, re, c2, c3, v0):
            s = r - re
            s2 = s * s
            s3 = s2 * s
            return -d * (1.0 + c1 * s + c2 * s2 + c3 * s3) * math.exp(-c1 * s) + v0

        return (fit + ryd(x, *p[0:6]) + ryd(y, *p[6:12]) + ryd(z, *p[0:6]))

    @staticmethod
    def _cell(g, c):
        for s in range(1, len(g)):
            if c < g[s]:
                return s
        return len(g) - 1

    @staticmethod
    def _hermite(t, h):
        t2 = t * t
        t3 = t * t2
        u0 = -2.0 * t3 + 3.0 * t2
        return [u0, -u0 + 1.0, h * (t3 - t2), h * (t3 - 2.0 * t2 + t)]

    def so(self, c0, c1, c2):
        is_, js, ks = self._cell(self.gx, c0), self._cell(self.gy, c1), self._cell(self.gz, c2)
        hx = self.gx[is_] - self.gx[is_ - 1]
        hy = self.gy[js] - self.gy[js - 1]
        hz = self.gz[ks] - self.gz[ks - 1]
        u = [self._hermite((c0 - self.gx[is_ - 1]) / hx, hx),
             self._hermite((c1 - self.gy[js - 1]) / hy, hy),
             self._hermite((c2 - self.gz[ks - 1]) / hz, hz)]
        f = 0.0
        for k in range(4):
            nk, dk = (ks - 1 if k & 1 else ks), k >> 1
            for j in range(4):
                nj, dj = (js - 1 if j & 1 else js), j >> 1
                ukj = u[2][k] * u[1][j]
                for i in range(4):
                    ni, di = (is_ - 1 if i & 1 else is_), i >> 1
                    f = f + self.T[di + 2 * dj + 4 * dk, ni, nj, nk] * ukj * u[0][i]
        return f

    def pot(self, rhf1, r, rhf2):
        v = self.sw1(rhf1, r, rhf2)
        rbig = math.sqrt(0.5 * (rhf1 * rhf1 + rhf2 * rhf2 - 0.5 * r * r))
        c = (rbig * rbig + 0.25 * r * r - rhf1 * rhf1) / rbig / r
        if abs(c) >= 1.0:
            c = math.copysign(1.0, c)
        gam = math.acos(c)
        so = 0.0
        if v > self.esocut and r < self.rsolim and rbig > self.rrsolm:
            c0 = min(max(rbig, self.gx[0]), self.gx[-1])
            c1 = min(max(r, self.gy[0]), self.gy[-1])
            c2 = gam * self.raddeg
            if c2 > 90.0:
                c2 = 180.0 - c2
            so = self.so(c0, c1, c2)
        return v + so + SHIFT

    def many(self, a, b, c):
        return np.array([self.pot(float(x), float(y), float(z)) for x, y, z in zip(a, b, c)])
