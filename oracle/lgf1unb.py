"""1-D lattice Green's functions of one unbounded direction with a spectral
shift (test infrastructure: the CPU oracle, never shipped or timed).

A direction that stays unbounded while the two others are spectral reduces
the 3-D lattice Poisson problem to a 1-D one per wave-number pair: find G(n)
with  A G = delta_n  for the 1-D stencil A of the scheme shifted by the
symbol c of the two spectral directions.  The closed forms below are the
residue sums over the roots r (|r| < 1) of the stencil's characteristic
polynomial, restated from the reference's src/lgf_1unb2spe.hpp:
  lgf2  (:161-184)  3-point stencil, one real root;
  lgf4  (:186-280)  5-point stencil, two roots: real, repeated at c = 3, or a
                    conjugate pair;
  lgf6  (:282-370)  7-point stencil, one real root and a conjugate pair;
  lgf8  (:372-490)  9-point stencil, two real roots (repeated at c*) or a
                    second conjugate pair, and a conjugate pair;
  meh4 / meh6 left and full (:492-612), the Mehrstellen schemes, whose
                    symbol does not split as a sum: they take the two
                    spectral wave numbers (k1, k2) instead of c.
Every regime (c = 0, small c, real roots, repeated root, complex roots) and
its cut-off is the reference's, so values agree to rounding.  Scalar
functions; green.py evaluates them once per distinct (n, c) or (n, k1, k2).
"""
import cmath
import math

import numpy as np

# ---------------------------------------------------------------- helpers


def _horner(a, x):
    out = a[-1]
    for coef in reversed(a[:-1]):
        out = x * out + coef
    return out


def _log_series(x_minus_one, terms=12):
    """log(x) about x = 1 (lgf_1unb2spe.hpp:51-58)."""
    out = 0.0
    for i in range(terms):
        out += 1.0 / (terms - i)
        out *= -x_minus_one
    return -out


def _value_minus_inverse_series(x_minus_one, terms=12):
    """x - 1/x about x = 1 (lgf_1unb2spe.hpp:66-73)."""
    out = 0.0
    for _ in range(terms):
        out += 1.0
        out *= -x_minus_one
    return -out + x_minus_one


_LARGE_LAMBDA = [0, 1. / 2., 0, 1. / 8., 0, 1. / 16., 0, 5. / 128., 0, 7. / 256.]


def _r_from_lambda(lam):
    """r = lambda - sqrt(lambda^2 - 1) with |r| <= 1 (lgf_1unb2spe.hpp:80-92)."""
    if math.isinf(lam):
        return 0.0
    if abs(lam) > 1.0e2:
        return _horner(_LARGE_LAMBDA, 1.0 / lam)
    return (lam - cmath.sqrt(complex(lam - 1)) * cmath.sqrt(complex(lam + 1))).real


def _oscillatory(r, pp, w, n):
    """Contribution of a conjugate root pair (lgf_1unb2spe.hpp:102-105)."""
    K = 2j * r ** (w - 1) / pp
    an = abs(n)
    return abs(K) * abs(r) ** an * math.sin(cmath.phase(r) * an + cmath.phase(K))


# ---------------------------------------------------------------- symbols


def lgf2_symbol(k):
    return 4.0 * math.sin(k / 2.) ** 2


def lgf4_symbol(k):
    return 4.0 * (4. / 3. * math.sin(k / 2.) ** 2 - 1. / 12. * math.sin(k) ** 2)


def lgf6_symbol(k):
    return 4.0 * (3. / 2. * math.sin(k / 2.) ** 2 - 3. / 20. * math.sin(k) ** 2 + 1. / 90. * math.sin(1.5 * k) ** 2)


def lgf8_symbol(k):
    return 4.0 * (8. / 5. * math.sin(k / 2.) ** 2 - 1. / 5. * math.sin(k) ** 2 + 8. / 315. * math.sin(1.5 * k) ** 2
                  - 1. / 560. * math.sin(2. * k) ** 2)


# root of the reduced polynomial nearest 1, as a series in c
_SMALL_C = {
    4: [0, 0.5, 1. / 24., 1. / 144., 5. / 3456., 7. / 20736., 7. / 82944., 11. / 497664.],
    6: [0, 0.5, 1. / 24., 1. / 720., -1. / 1152., -149. / 518400., -259. / 6220800., 163. / 62208000.],
    8: [0, 0.5, 1. / 24., 1. / 720., 1. / 40320., 577. / 3628800., 389. / 6220800., 34987. / 3048192000.],
}


def _pp4(z, c):
    return -4. / 3. + z * ((5. + 2. * c) + z * (-4. + z / 3.))


def _pp6(z, c):
    return 3. / 20. + z * (-3. + z * ((49. / 6. + 3. * c) + z * (-6. + z * (3. / 4. - z / 15.))))


def _pp8(z, c):
    return -8. / 315. + z * (2. / 5. + z * (-24. / 5. + z * (205. / 18. + 4. * c + z * (-8. + z * (6. / 5. + z * (
        -8. / 45. + z / 70.))))))


def _small_root(order, c):
    """(r1 - 1, r1) of the real root nearest 1 for small c."""
    lm1 = _horner(_SMALL_C[order], c)
    rm1 = lm1 - math.sqrt(lm1 * lm1 + 2 * lm1)
    return rm1, rm1 + 1.0


# ---------------------------------------------------------------- LGF2


def lgf2(n, c):
    """lgf_1unb2spe.hpp:161-184."""
    if c < 0:
        raise ValueError("c must be nonnegative")
    an = abs(n)
    if c == 0.0:
        return -0.5 * an
    if c < 1.0e-3:
        rm1 = c / 2. - math.sqrt(c * c / 4. + c)
        return -math.exp(an * _log_series(rm1)) / _value_minus_inverse_series(rm1)
    r = 1 + c / 2. - math.sqrt(c * c / 4. + c)
    return -r ** an / (r - 1. / r)


# ---------------------------------------------------------------- LGF4

_SQ15 = math.sqrt(15.)
_L4_REPEAT = [
    [4. / (5. * _SQ15), 1. / 5.],
    [-14. / (75. * _SQ15), -2. / 25., -4. / (25. * _SQ15), -1. / 150.],
    [901. / (18750. * _SQ15), 74. / 3125., 253. / (3750. * _SQ15), 23. / 3750., 1. / (250. * _SQ15), 1. / 15000.],
    [-37313. / (2812500. * _SQ15), -11267. / 1640625., -3167. / (140625. * _SQ15), -1. / 375., -31. / (11250. * _SQ15),
     -31. / 281250., -1. / (28125. * _SQ15), -1. / 3150000.],
    [3885631. / (1012500000. * _SQ15), 1194829. / 590625000., 1118351. / (157500000. * _SQ15), 12571. / 13125000.,
     13751. / (11250000. * _SQ15), 127. / 1875000., 247. / (6750000. * _SQ15), 13. / 15750000.,
     1. / (6300000. * _SQ15), 1. / 1134000000.],
]
_L4_CSTAR = 3.0


def lgf4(n, c):
    """lgf_1unb2spe.hpp:186-280."""
    if c < 0:
        raise ValueError("c must be nonnegative")
    an = abs(n)
    if c == 0.0:
        r, K = 7.179676972449123e-2, -7.216878364870408e-2
        return -0.5 * an + K * (r ** an - 1.0)
    if c < 1e-3:
        rm1, r1 = _small_root(4, c)
        lam2 = 4.0 + math.sqrt(9.0 - 3.0 * c)
        r2 = lam2 - math.sqrt(lam2 * lam2 - 1.0)
        pp1 = 1. / 12. * _value_minus_inverse_series(rm1) * (r1 - r2) * (r1 - 1.0 / r2)
        pp2 = _pp4(r2, c)
        return math.exp((an + 1) * _log_series(rm1)) / pp1 + r2 ** (an + 1) / pp2
    if c < _L4_CSTAR - 1e-5:
        lam1 = 4.0 + math.sqrt(9.0 - 3.0 * c)
        lam2 = 4.0 - math.sqrt(9.0 - 3.0 * c)
        r1 = lam1 - math.sqrt(lam1 * lam1 - 1.0)
        r2 = lam2 - math.sqrt(lam2 * lam2 - 1.0)
        f1 = 12 * r1 ** (an + 1) / ((r1 - 1.0 / r1) * (r1 - 1.0 / r2))
        f2 = 12 * r2 ** (an + 1) / ((r2 - 1.0 / r1) * (r2 - 1.0 / r2))
        return (f1 - f2) / (r1 - r2)
    if c < _L4_CSTAR + 1e-5:
        r = 4.0 - _SQ15
        g = [_horner(a, float(an)) for a in _L4_REPEAT]
        return r ** an * _horner(g, c - _L4_CSTAR)
    lam = 4.0 - cmath.sqrt(complex(9.0 - 3.0 * c))
    r = lam - cmath.sqrt(lam * lam - 1.0)
    pp = 1j / 6. * r.imag * (r - 1. / r) * (r - 1. / r.conjugate())
    return _oscillatory(r, pp, 2, n)


# ---------------------------------------------------------------- LGF6


def _lgf6_roots(c):
    xi = float(np.cbrt(360. * c - 775. + 60. * math.sqrt(36. * c * c - 155. * c + 405.)))
    lam1 = 0.25 * (9. - 95. / xi + xi)
    r1 = lam1 - math.sqrt(lam1 * lam1 - 1.0)
    w = complex(-0.5, math.sqrt(3.) / 2.)
    lam2 = 0.25 * (9. - 95. / (w * xi) + (w * xi))
    r2 = lam2 - cmath.sqrt(lam2 * lam2 - 1.0)
    return r1, r2


def lgf6(n, c):
    """lgf_1unb2spe.hpp:282-370."""
    if c < 0:
        raise ValueError("c must be nonnegative")
    an = abs(n)
    if c == 0.0:
        a, p, t, f = 1.035017642406219e-1, 9.54295097909627e-2, -9.958762687216868e-1, -2.168575565241744e+0
        return -0.5 * an + a * p ** an * math.sin(an * t + f) - a * math.sin(f)
    if c < 1e-3:
        rm1, r1 = _small_root(6, c)
        _, r2 = _lgf6_roots(c)
        pp2 = _pp6(r2, c)
        d = (r1 - r2) * (r1 - 1.0 / r2)
        pp1 = -1. / 90. * _value_minus_inverse_series(rm1) * (d.real * d.real + d.imag * d.imag)
        return math.exp((an + 2) * _log_series(rm1)) / pp1 + _oscillatory(r2, pp2, 3, n)
    r1, r2 = _lgf6_roots(c)
    return r1 ** (an + 2) / _pp6(r1, c) + _oscillatory(r2, _pp6(r2, c), 3, n)


# ---------------------------------------------------------------- LGF8

_L8_CSTAR = 3.204471924659902
_L8_A = [
    [-0.1932304295173025, -9.940958723693284e-2],
    [5.528645180523051e-2, 6.381749748906844e-2, 1.920895723993029e-2, 1.647044339102893e-3],
    [-1.246195963786745e-2, -2.200316066032414e-2, -1.156690496243602e-2, -2.513956535483380e-3,
     -2.386943138091703e-4, -8.186599895557273e-6],
    [2.586595339831205e-3, 5.946351585490818e-3, 4.392324394119772e-3, 1.460419122054276e-3, 2.498408821419240e-4,
     2.281049273902400e-5, 1.054600142736557e-6, 1.937682182122062e-8],
    [-6.143387386724980e-4, -1.461770070530813e-3, -1.338631620906462e-3, -5.893614275050890e-4,
     -1.419718637870522e-4, -2.006233681173800e-5, -1.705558618042543e-6, -8.568226736629197e-8,
     -2.340119751996688e-9, -2.675335915571021e-11],
]
_L8_U = [
    [0.0015031218476240784],
    [-0.013198947960911374, -0.00309497626043345],
    [0.002223792419320104, 0.0003211726758356002, -3.489943855291188e-6],
    [8.218756082933073e-5, 0.00012939734109457704, 2.076196709989474e-5, 7.970739601754506e-7],
    [-0.00011284539233578474, -4.455888056601662e-5, -4.596415525190604e-6, -1.2515613302441402e-7,
     7.499072573978986e-10],
]
_L8_V = [
    [-0.07869060869097218],
    [0.005694070346472886, -0.00011828157312623746],
    [0.001748394270280815, 0.0007853940979982054, 6.08419435502199e-5],
    [-0.000574565978306078, -0.000152486888729598, -8.030910109571855e-6, 6.101311014540467e-8],
    [4.706634682161246e-5, -8.921284296708267e-6, -4.142946014756904e-6, -3.42884013573887e-7,
     -7.828815619884859e-9],
]


def _lgf8_roots(c):
    tmp1 = 1968941520. + c * (-879221700. + c * (223915104. - c * 44089920))
    xi = (1520225. - 273420. * c + 35. * cmath.sqrt(complex(tmp1))) ** (1. / 3.)
    dl = (xi + (-4655. + 3780. * c) / xi).real
    eta = cmath.sqrt(complex(dl / 9. - 434. / 81.))
    s1 = cmath.sqrt(-868. / 81. + 81088. / (729. * eta) - dl / 9.)
    s3 = cmath.sqrt(-868. / 81. - 81088. / (729. * eta) - dl / 9.)
    lams = (0.5 * (32. / 9. + eta - s1), 0.5 * (32. / 9. + eta + s1), 0.5 * (32. / 9. - eta - s3))
    return [lam - cmath.sqrt(lam + 1.0) * cmath.sqrt(lam - 1.0) for lam in lams]


def lgf8(n, c):
    """lgf_1unb2spe.hpp:372-490."""
    if c < 0:
        raise ValueError("c must be nonnegative")
    an = abs(n)
    if c == 0.0:
        rho1, th1, a1, phi1 = 1.2185576475724652e-01, 1.4667413886166037e+00, 8.2123351081853858e-02, -6.5666289805823130e-01
        r2, a2 = 9.6191214171019512e-02, 4.0692417408429382e-02
        return -0.5 * an + a1 * rho1 ** an * math.sin(an * th1 + phi1) - a1 * math.sin(phi1) + a2 * (1.0 - r2 ** an)
    if c < 1e-3:
        rm1, r1 = _small_root(8, c)
        roots = _lgf8_roots(c)
        r2 = roots[1].real
        pp2 = _pp8(r2, c)
        r3 = roots[2]
        pp3 = _pp8(r3, c)
        d = (r1 - r3) * (r1 - 1.0 / r3)
        pp1 = 1. / 560. * _value_minus_inverse_series(rm1) * (r1 - r2) * (r1 - 1 / r2) * (d.real ** 2 + d.imag ** 2)
        return (math.exp((an + 3) * _log_series(rm1)) / pp1 + r2 ** (an + 3) / pp2
                + _oscillatory(r3, pp3, 4, n))
    if c < _L8_CSTAR - 1e-5:
        roots = _lgf8_roots(c)
        r1, r2, r3 = roots[0].real, roots[1].real, roots[2]
        pp3 = _pp8(r3, c)
        d1 = (r1 - r3) * (r1 - 1. / r3)
        d2 = (r2 - r3) * (r2 - 1. / r3)
        f1 = 560. * r1 ** (an + 3) / ((r1 - 1. / r1) * (r1 - 1. / r2) * (d1.real ** 2 + d1.imag ** 2))
        f2 = 560. * r2 ** (an + 3) / ((r2 - 1. / r1) * (r2 - 1. / r2) * (d2.real ** 2 + d2.imag ** 2))
        return (f2 - f1) / (r2 - r1) + _oscillatory(r3, pp3, 4, n)
    if c < _L8_CSTAR + 1e-5:
        r0, rho1, th1 = 1.4016094393066413e-01, 1.2718191072648583e-01, 1.5912866598657263e+00
        r0n, p1n = r0 ** an, rho1 ** an
        cn, sn = math.cos(an * th1), math.sin(an * th1)
        nr = float(an)
        g = [r0n * _horner(_L8_A[j], nr) + p1n * (cn * _horner(_L8_U[j], nr) + sn * _horner(_L8_V[j], nr))
             for j in range(5)]
        return -_horner(g, c - _L8_CSTAR)
    roots = _lgf8_roots(c)
    r1, r3 = roots[1], roots[2]
    cr1, cr3 = r1.conjugate(), r3.conjugate()
    pp1 = (1j / 280. * r1.imag * (r1 - 1. / r1) * (r1 - 1. / cr1) * (r1 - r3) * (r1 - 1. / r3) * (r1 - cr3)
           * (r1 - 1. / cr3))
    return _oscillatory(r1, pp1, 4, n) + _oscillatory(r3, _pp8(r3, c), 4, n)


# ---------------------------------------------------------------- Mehrstellen 4 and 6


def _ysq(k1, k2):
    return math.sin(k1 / 2) ** 2, math.sin(k2 / 2) ** 2


def meh4_left(n, k1, k2):
    """lgf_1unb2spe.hpp:511-525."""
    if k1 == 0 and k2 == 0:
        return -0.5 * abs(n)
    y0, y1 = _ysq(k1, k2)
    a0 = -8. / 3. * (y0 * y1 - y0 - y1) + 2.0
    a1 = 2. / 3. * (y0 + y1) - 1.0
    lam = -a0 / (2. * a1) if a1 != 0.0 else math.copysign(math.inf, -a0) if a0 != 0.0 else math.nan
    if not math.isfinite(lam):
        return (1.0 if n == 0 else 0.0) / a0
    r = _r_from_lambda(lam)
    return (r / a1) * r ** abs(n) / (r * r - 1.0)


def meh4_full(n, k1, k2):
    """lgf_1unb2spe.hpp:530-549."""
    if k1 == 0 and k2 == 0:
        return -0.5 * abs(n) - (1. / 12. if n == 0 else 0.0)
    y0, y1 = _ysq(k1, k2)
    a0 = -8. / 3. * (y0 * y1 - y0 - y1) + 2.0
    a1 = 2. / 3. * (y0 + y1) - 1.0
    b0 = 5. / 6. - 1. / 3. * (y0 + y1)
    b1 = 1. / 12.
    lam = -a0 / (2 * a1) if a1 != 0.0 else math.copysign(math.inf, -a0) if a0 != 0.0 else math.nan
    if math.isfinite(lam):
        r = _r_from_lambda(lam)
        pr = b1 + b0 * r + b1 * r * r
        if n == 0:
            return (r / a1) * (b0 + 2. * b1 * r) / (r * r - 1.)
        return pr * r ** abs(n) / (a1 * (r * r - 1))
    return (b0 / a0 if n == 0 else 0.0) + (b1 / a0 if n == 1 else 0.0)


def meh6_left(n, k1, k2):
    """lgf_1unb2spe.hpp:576-588."""
    if k1 == 0 and k2 == 0:
        return -0.5 * abs(n)
    y0, y1 = _ysq(k1, k2)
    a0 = -8. / 5. * y0 * y1 + 8. / 3. * (y0 + y1) + 2.0
    a1 = -8. / 15. * y0 * y1 + 2. / 3. * (y0 + y1) - 1.0
    lam = -a0 / (2. * a1) if a1 != 0.0 else math.copysign(math.inf, -a0) if a0 != 0.0 else math.nan
    if not math.isfinite(lam):
        return -(1.0 if n == 0 else 0.0) / a0
    r = _r_from_lambda(lam)
    return (r / a1) * r ** abs(n) / (r * r - 1.0)


def meh6_full(n, k1, k2):
    """lgf_1unb2spe.hpp:593-610."""
    an = abs(n)
    if k1 == 0 and k2 == 0:
        return -0.5 * an - (-1. / 240. if an == 1 else 0.0) - (11. / 120. if n == 0 else 0.0)
    y0, y1 = _ysq(k1, k2)
    a0 = -8. / 5. * y0 * y1 + 8. / 3. * (y0 + y1) + 2.0
    a1 = -8. / 15. * y0 * y1 + 2. / 3. * (y0 + y1) - 1.0
    b0 = -1. / 15. * (y0 ** 2 + y1 ** 2) + 8. / 45. * y0 * y1 - 11. / 45. * (y0 + y1) + 97. / 120.
    b1 = -2. / 45. * (y0 + y1) + 1. / 10.
    b2 = -1. / 240.
    lam = -a0 / (2 * a1)
    r = _r_from_lambda(lam)
    pr = b0 * r ** 2 + b1 * (r + r ** 3) + b2 * (1.0 + r ** 4)
    base = pr * r ** (an - 1) / (a1 * (r * r - 1.0))
    return base + (b2 / a1 if an == 1 else 0.0) + ((b1 * a1 - b2 * a0) / (a1 * a1) if n == 0 else 0.0)
