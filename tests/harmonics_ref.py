"""Independent known answer for geopotential fields (test infrastructure).

The potential of one spherical-harmonic term of degree n and order m, per unit GM of the body, is
    U = R^n / r^(2n+1) * H(x, y, z)
with H = Re[(x + i y)^m] A(z, r^2) (cosine term) or Im[(x + i y)^m] A(z, r^2) (sine term), where
r^(n-m) P_n^(m)(z / r) = A(z, r^2) = sum_k a_k z^(n-m-2k) r^(2k) and P_n^(m) is the m-th derivative of the
Legendre polynomial P_n (so r^n P_nm(sin lat) e^(i m lon) = (x + i y)^m A, P_nm without the Condon-Shortley
phase). H is a homogeneous harmonic polynomial of degree n with rational coefficients; it is built exactly
with fractions, differentiated exactly, and evaluated in extended precision (numpy longdouble), so the
gradient
    grad U = R^n (grad H / r^(2n+1) - (2n+1) H r / r^(2n+3))
carries no pole singularity and no angle. Zonal terms enter the model files as J_n = -C_n0.

This is the same kind of check as the reference's known-answer test (src/tests/test_geopotential.cpp:24-76,
which evaluates Legendre functions in spherical coordinates); the evaluation here is a different one.
"""
from __future__ import annotations

from fractions import Fraction
from math import comb, factorial

import numpy as np

Poly = dict  # {(i, j, k): Fraction} for x^i y^j z^k


def _mul(a: Poly, b: Poly) -> Poly:
    out: Poly = {}
    for (i1, j1, k1), c1 in a.items():
        for (i2, j2, k2), c2 in b.items():
            key = (i1 + i2, j1 + j2, k1 + k2)
            out[key] = out.get(key, Fraction(0)) + c1 * c2
    return {k: v for k, v in out.items() if v != 0}


def _diff(a: Poly, axis: int) -> Poly:
    out: Poly = {}
    for e, c in a.items():
        if e[axis] == 0:
            continue
        ne = list(e)
        ne[axis] -= 1
        out[tuple(ne)] = out.get(tuple(ne), Fraction(0)) + c * e[axis]
    return out


def _legendre_deriv(n: int, m: int):
    """Coefficients {power of t: Fraction} of the m-th derivative of the Legendre polynomial P_n."""
    p = {}
    for k in range(n // 2 + 1):
        p[n - 2 * k] = Fraction((-1) ** k * comb(n, k) * comb(2 * n - 2 * k, n), 2 ** n)
    for _ in range(m):
        p = {e - 1: c * e for e, c in p.items() if e > 0}
    return p


def harmonic_poly(n: int, m: int, sine: bool) -> Poly:
    """H(x, y, z) = r^n P_nm(z/r) cos(m lon) (sine=False) or sin(m lon) (sine=True), exactly."""
    a: Poly = {}
    for e, c in _legendre_deriv(n, m).items():   # t^e -> z^e r^(n-m-e), n-m-e even
        k = (n - m - e) // 2
        for p in range(k + 1):
            for q in range(k - p + 1):
                u = k - p - q
                w = Fraction(factorial(k), factorial(p) * factorial(q) * factorial(u))
                key = (2 * p, 2 * q, 2 * u + e)
                a[key] = a.get(key, Fraction(0)) + c * w
    ring: Poly = {}
    for j in range(m + 1):   # (x + i y)^m: real part from even j, imaginary from odd j
        if (j % 2 == 1) != sine:
            continue
        sign = (-1) ** (j // 2)
        ring[(m - j, j, 0)] = Fraction(sign * comb(m, j))
    return _mul(ring, a)


class _Compiled:
    def __init__(self, poly: Poly):
        self.exp = np.array(list(poly.keys()), dtype=np.int64).reshape(-1, 3)
        self.coef = np.array([np.longdouble(c.numerator) / np.longdouble(c.denominator) for c in poly.values()],
                             dtype=np.longdouble)

    def __call__(self, x, y, z):
        if len(self.coef) == 0:
            return np.zeros_like(x)
        t = (x[:, None] ** self.exp[None, :, 0]) * (y[:, None] ** self.exp[None, :, 1]) * \
            (z[:, None] ** self.exp[None, :, 2])
        return t @ self.coef


_CACHE: dict = {}


def term_field(n: int, m: int, sine: bool, R: float, r: np.ndarray) -> np.ndarray:
    """Gradient of R^n H / r^(2n+1) at body-frame points r[k][3] (longdouble result)."""
    key = (n, m, sine)
    if key not in _CACHE:
        h = harmonic_poly(n, m, sine)
        _CACHE[key] = (_Compiled(h), _Compiled(_diff(h, 0)), _Compiled(_diff(h, 1)), _Compiled(_diff(h, 2)))
    H, Hx, Hy, Hz = _CACHE[key]
    p = np.asarray(r, dtype=np.longdouble)
    x, y, z = p[:, 0], p[:, 1], p[:, 2]
    r2 = x * x + y * y + z * z
    rr = np.sqrt(r2)
    Rn = np.longdouble(R) ** n
    inv = 1 / rr ** (2 * n + 1)
    h = H(x, y, z)
    g = np.stack([Hx(x, y, z), Hy(x, y, z), Hz(x, y, z)], axis=1) * inv[:, None]
    g -= ((2 * n + 1) * h * inv / r2)[:, None] * p
    return Rn * g


def model_field(tab: np.ndarray, nz: int, nt: int, R: float, r: np.ndarray) -> np.ndarray:
    """Field of a packed coefficient table (J_n at n^2-4, C_nm at n^2-4+2m-1, S_nm at n^2-4+2m)."""
    out = np.zeros((len(r), 3), dtype=np.longdouble)
    for n in range(2, nz + 1):
        base = n * n - 4
        if tab[base] != 0:
            out -= np.longdouble(tab[base]) * term_field(n, 0, False, R, r)
        if n > nt:
            continue
        for m in range(1, n + 1):
            c, s = tab[base + 2 * m - 1], tab[base + 2 * m]
            if c != 0:
                out += np.longdouble(c) * term_field(n, m, False, R, r)
            if s != 0:
                out += np.longdouble(s) * term_field(n, m, True, R, r)
    return out


# The known-answer grid: one coefficient per case, spheres of radius 1828.1828 * (-2.2)^k (k = 1..17) about a
# body of radius 1415.9265 (the reference's test sizes, src/tests/test_geopotential.cpp:12-22), 18 x 35 directions
# including both poles; bound 1e-13 of the largest field magnitude on each sphere.
KAT_R = 1415.9265
KAT_N = 17
KAT_EPS = 1e-13


def kat_cases():
    for n in range(2, 9):
        for m in range(n + 1):
            for sine in ((False,) if m == 0 else (False, True)):
                tab = np.zeros(77)
                base = n * n - 4
                if m == 0:
                    tab[base] = 0.1919810 / n
                elif not sine:
                    tab[base + 2 * m - 1] = 0.114 / n
                else:
                    tab[base + 2 * m] = 0.0514 / n
                yield n, m, sine, tab, n, (n if m else 0)


def kat_spheres():
    rn = 1828.1828
    th = np.arange(KAT_N + 1) * np.pi / KAT_N
    ph = np.arange(2 * KAT_N + 1) * np.pi / KAT_N
    T, P = np.meshgrid(th, ph, indexing="ij")
    unit = np.stack([np.sin(T) * np.cos(P), np.sin(T) * np.sin(P), np.cos(T)], axis=-1).reshape(-1, 3)
    for _ in range(KAT_N):
        rn *= -2.2
        yield unit * rn


def near_axis_points(k: int, rn: float):
    """Points approaching the z axis at height +-rn: the field there must tend to the on-axis value."""
    pts = []
    for iz in (-1, 1):
        for iphi in range(2 * KAT_N + 1):
            xy = np.sqrt(np.finfo(float).tiny) * (3 * k + 5) / (2 * k + 4)
            a = iphi * np.pi / KAT_N
            x, y = xy * np.cos(a), xy * np.sin(a)
            while x * x or y * y:
                pts.append((x, y, iz * rn))
                x /= 2
                y /= 2
    return np.array(pts)
