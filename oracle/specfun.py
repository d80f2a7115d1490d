"""Special functions used by the Green's kernels, vectorised over numpy arrays.

Each follows the published method the reference cites, with the same
coefficients (the Green's spectra must agree to round-off with the
reference's, so the approximations have to be the same ones):

- modified Bessel K0/K1: rational approximations of Numerical Recipes 3rd ed.
  sec. 6.5.1 (reference src/bessel.hpp:9-85);
- exponential integral E1 used as ``expint_ei``: Chebyshev expansions on
  [-4, 4] and [4, inf) (reference src/expint.hpp:35-190);
- sine integral Si: Chebyshev-Pade fits published with GalSim
  (reference src/si.hpp:23-116);
- Ji0c, the Bessel-integral series of Humbert (1929) truncated at 50 terms in
  extended precision (reference src/ji0.hpp:23-75);
- the one-unbounded-direction LGF of the 2nd-order stencil in closed form
  (reference src/lgf_1unb2spe.hpp:53-180).
"""
import math

import numpy as np

C_GAMMA = 0.5772156649015328606


def _poly(coef, x):
    """Horner evaluation with coef[0] the constant term (bessel.hpp:12-16)."""
    ans = np.full_like(np.asarray(x, dtype=np.float64), coef[-1])
    for c in coef[-2::-1]:
        ans = ans * x + c
    return ans


# Numerical Recipes 3rd ed. sec. 6.5.1 coefficients (bessel.hpp:52-84)
_K0PI = [1.0, 2.346487949187396e-1, 1.187082088663404e-2, 2.150707366040937e-4, 1.425433617130587e-6]
_K0QI = [9.847324170755358e-1, 1.518396076767770e-2, 8.362215678646257e-5]
_K0P = [1.159315156584126e-1, 2.770731240515333e-1, 2.066458134619875e-2, 4.574734709978264e-4, 3.454715527986737e-6]
_K0Q = [9.836249671709183e-1, 1.627693622304549e-2, 9.809660603621949e-5]
_K0PP = [1.253314137315499, 1.475731032429900e1, 6.123767403223466e1, 1.121012633939949e2,
         9.285288485892228e1, 3.198289277679660e1, 3.595376024148513, 6.160228690102976e-2]
_K0QQ = [1.0, 1.189963006673403e1, 5.027773590829784e1, 9.496513373427093e1, 8.318077493230258e1,
         3.181399777449301e1, 4.443672926432041, 1.408295601966600e-1]
_K1PI = [0.5, 5.598072040178741e-2, 1.818666382168295e-3, 2.397509908859959e-5, 1.239567816344855e-7]
_K1QI = [9.870202601341150e-1, 1.292092053534579e-2, 5.881933053917096e-5]
_K1P = [-3.079657578292062e-1, -8.109417631822442e-2, -3.477550948593604e-3, -5.385594871975406e-5,
        -3.110372465429008e-7]
_K1Q = [9.861813171751389e-1, 1.375094061153160e-2, 6.774221332947002e-5]
_K1PP = [1.253314137315502, 1.457171340220454e1, 6.063161173098803e1, 1.147386690867892e2,
         1.040442011439181e2, 4.356596656837691e1, 7.265230396353690, 3.144418558991021e-1]
_K1QQ = [1.0, 1.125154514806458e1, 4.427488496597630e1, 7.616113213117645e1, 5.863377227890893e1,
         1.850303673841586e1, 1.857244676566022, 2.538540887654872e-2]


def besselk0(x):
    x = np.asarray(x, dtype=np.float64)
    out = np.empty_like(x)
    lo = x <= 1.0
    with np.errstate(divide="ignore", invalid="ignore"):
        z = x * x
        term = _poly(_K0PI, z) * np.log(x) / _poly(_K0QI, 1.0 - z)
        small = _poly(_K0P, z) / _poly(_K0Q, 1.0 - z) - term
        zi = 1.0 / x
        large = np.exp(-x) * _poly(_K0PP, zi) / (_poly(_K0QQ, zi) * np.sqrt(x))
    out[lo] = small[lo]
    out[~lo] = large[~lo]
    return out


def besselk1(x):
    x = np.asarray(x, dtype=np.float64)
    out = np.empty_like(x)
    lo = x <= 1.0
    with np.errstate(divide="ignore", invalid="ignore"):
        z = x * x
        term = _poly(_K1PI, z) * np.log(x) / _poly(_K1QI, 1.0 - z)
        small = x * (_poly(_K1P, z) / _poly(_K1Q, 1.0 - z) + term) + 1.0 / x
        zi = 1.0 / x
        large = np.exp(-x) * _poly(_K1PP, zi) / (_poly(_K1QQ, zi) * np.sqrt(x))
    out[lo] = small[lo]
    out[~lo] = large[~lo]
    return out


# Chebyshev coefficients of E1 on [-4,4] (argument x/4) and [4,inf) (argument 4/x)
_E1_A = [7.8737715392882774, -8.0314874286705335, 3.8797325768522250, -1.6042971072992259,
         0.5630905453891458, -0.1704423017433357, 0.0452099390015415, -0.0106538986439085,
         0.0022562638123478, -0.0004335700473221, 0.0000762166811878, -0.0000123417443064,
         0.0000018519745698, -0.0000002588698662, 0.0000000338604319, -0.0000000041611418,
         0.0000000004821606, -0.0000000000528465, 0.0000000000054945, -0.0000000000005433,
         0.0000000000000512, -0.0000000000000046, 0.0000000000000004]
_E1_B = [0.2155283776715125, 0.1028106215227030, -0.0045526707131788, 0.0003571613122851,
         -0.0000379341616932, 0.0000049143944914, -0.0000007355024922, 0.0000001230603606,
         -0.0000000225236907, 0.0000000044412375, -0.0000000009328509, 0.0000000002069297,
         -0.0000000000481502, 0.0000000000116891, -0.0000000000029474, 0.0000000000007691,
         -0.0000000000002070, 0.0000000000000573, -0.0000000000000163, 0.0000000000000047,
         -0.0000000000000014, 0.0000000000000004, -0.0000000000000001]


def _clenshaw(a, t):
    b2 = np.zeros_like(t)
    b1 = np.zeros_like(t)
    b0 = np.full_like(t, a[-1])
    for k in range(len(a) - 2, -1, -1):
        b2 = b1
        b1 = b0
        b0 = t * b1 - b2 + a[k]
    return 0.5 * (b0 - b2)


def expint_ei(x):
    """expint.hpp:35-190: E1 via two Chebyshev fits; 0 below -4."""
    x = np.asarray(x, dtype=np.float64)
    out = np.zeros_like(x)
    mid = (x >= -4.0) & (x <= 4.0)
    hi = x > 4.0
    if np.any(mid):
        xm = x[mid]
        v = _clenshaw(_E1_A, 2.0 * (0.25 * xm))
        with np.errstate(divide="ignore"):
            out[mid] = -(v + np.log(np.abs(xm)))
    if np.any(hi):
        xh = x[hi]
        arg = 4.0 / xh
        out[hi] = _clenshaw(_E1_B, 2.0 * (2.0 * arg - 1.0)) * np.exp(-xh)
    return out


def sine_integral(x):
    """si.hpp:23-116: Si(x) from Chebyshev-Pade fits (GalSim)."""
    x = np.asarray(x, dtype=np.float64)
    x2 = x * x
    out = np.empty_like(x)
    big = x2 > 16.0
    if np.any(big):
        xb = x[big]
        y = 1.0 / (xb * xb)
        f = (1. + y * (7.44437068161936700618e2 + y * (1.96396372895146869801e5 + y * (2.37750310125431834034e7 + y * (
            1.43073403821274636888e9 + y * (4.33736238870432522765e10 + y * (6.40533830574022022911e11 + y * (
                4.20968180571076940208e12 + y * (1.00795182980368574617e13 + y * (4.94816688199951963482e12 + y * (
                    -4.94701168645415959931e11))))))))))) / (xb * (1. + y * (7.46437068161927678031e2 + y * (
                        1.97865247031583951450e5 + y * (2.41535670165126845144e7 + y * (1.47478952192985464958e9 + y * (
                            4.58595115847765779830e10 + y * (7.08501308149515401563e11 + y * (5.06084464593475076774e12 + y * (
                                1.43468549171581016479e13 + y * (1.11535493509914254097e13)))))))))))
        g = y * (1. + y * (8.1359520115168615e2 + y * (2.35239181626478200e5 + y * (3.12557570795778731e7 + y * (
            2.06297595146763354e9 + y * (6.83052205423625007e10 + y * (1.09049528450362786e12 + y * (
                7.57664583257834349e12 + y * (1.81004487464664575e13 + y * (6.43291613143049485e12 + y * (
                    -1.36517137670871689e12))))))))))) / (1. + y * (8.19595201151451564e2 + y * (2.40036752835578777e5 + y * (
                        3.26026661647090822e7 + y * (2.23355543278099360e9 + y * (7.87465017341829930e10 + y * (
                            1.39866710696414565e12 + y * (1.17164723371736605e13 + y * (4.01839087307656620e13 + y * (
                                3.99653257887490811e13))))))))))
        out[big] = np.where(xb > 0.0, math.pi / 2.0, -math.pi / 2.0) - f * np.cos(xb) - g * np.sin(xb)
    sm = ~big
    if np.any(sm):
        xs = x[sm]
        s2 = xs * xs
        out[sm] = xs * (1. + s2 * (-4.54393409816329991e-2 + s2 * (1.15457225751016682e-3 + s2 * (
            -1.41018536821330254e-5 + s2 * (9.43280809438713025e-8 + s2 * (-3.53201978997168357e-10 + s2 * (
                7.08240282274875911e-13 + s2 * (-6.05338212010422477e-16)))))))) / (1. + s2 * (
                    1.01162145739225565e-2 + s2 * (4.99175116169755106e-5 + s2 * (1.55654986308745614e-7 + s2 * (
                        3.28067571055789734e-10 + s2 * (4.5049097575386581e-13 + s2 * (3.21107051193712168e-16)))))))
    return out


def _inv_fact_sq(n_kept=50):
    """ji0.hpp:23-35: 1/(n!)^2 for n = 0..n_kept in extended precision."""
    f = np.longdouble(1)
    out = [np.longdouble(1)] * (n_kept + 1)
    for i in range(1, n_kept + 1):
        fi = f * np.longdouble(i)
        out[i - 1] = np.longdouble(1) / (f * f)
        f = fi
    out[n_kept] = np.longdouble(1) / (f * f)
    return out


_INV_F_SQR = _inv_fact_sq()


def ji0c(x):
    """ji0.hpp:37-47: int_0^x (1 - J0(u))/u du as a 50-term series."""
    x = np.asarray(x, dtype=np.float64)
    q = (-(0.25 * x * x)).astype(np.longdouble)
    val = np.zeros(x.shape, dtype=np.longdouble)
    for n in range(50, 0, -1):
        val -= q ** n * _INV_F_SQR[n] / np.longdouble(n) * np.longdouble(0.5)
    return val.astype(np.float64)


# lgf_1unb2spe.hpp:53-75
def _log_series(xm1):
    out = np.zeros_like(xm1)
    for i in range(12):
        out = out + 1.0 / (12 - i)
        out = out * (-xm1)
    return -out


def _value_minus_inverse_series(xm1):
    out = np.zeros_like(xm1)
    for _ in range(12):
        out = out + 1.0
        out = out * (-xm1)
    return -out + xm1


def lgf2_symbol(k):
    return 4.0 * np.sin(k / 2.0) ** 2


def lgf4_symbol(k):
    return 4.0 * (4. / 3. * np.sin(k / 2.) ** 2 - 1. / 12. * np.sin(k) ** 2)


def lgf6_symbol(k):
    return 4.0 * (3. / 2. * np.sin(k / 2.) ** 2 - 3. / 20. * np.sin(k) ** 2 + 1. / 90. * np.sin(1.5 * k) ** 2)


def lgf8_symbol(k):
    return 4.0 * (8. / 5. * np.sin(k / 2.) ** 2 - 1. / 5. * np.sin(k) ** 2 + 8. / 315. * np.sin(1.5 * k) ** 2
                  - 1. / 560. * np.sin(2. * k) ** 2)


def lgf2_1unb(n, c):
    """lgf_1unb2spe.hpp:170-184: 1-D LGF of the 3-point stencil with shift c."""
    n = np.abs(np.asarray(n, dtype=np.float64))
    c = np.asarray(c, dtype=np.float64)
    if np.any(c < 0):
        raise ValueError("c must be nonnegative")
    out = np.empty(np.broadcast(n, c).shape)
    n, c = np.broadcast_arrays(n, c)
    z = c == 0.0
    sm = (c > 0.0) & (c < 1.0e-3)
    lg = c >= 1.0e-3
    out[z] = -0.5 * n[z]
    if np.any(sm):
        cs = c[sm]
        rm1 = cs / 2. - np.sqrt(cs * cs / 4. + cs)
        out[sm] = -np.exp(n[sm] * _log_series(rm1)) / _value_minus_inverse_series(rm1)
    if np.any(lg):
        cl = c[lg]
        r = 1 + cl / 2. - np.sqrt(cl * cl / 4. + cl)
        out[lg] = -r ** n[lg] / (r - 1. / r)
    return out
