"""Manufactured-solution validation driver (error norms against an analytic
solution), restating samples/validation/src/validation_3d.cpp:28-486 and the
manufactured functions of samples/validation/src/validation_3d.hpp:78-165.

``run_case`` returns the same (err2, errInf) pairs the reference writes into
``data/validation_3d_<Center>_<bccode>_typeGreen=<k>.txt``.
"""
import math

import numpy as np

from .plans import CELL_CENTER, NODE_CENTER, EVEN, ODD, PER, UNB, NONE

_C = 10.0


def _f_odd_odd(x, L, p):
    return np.sin((2 * math.pi / L * p["freq"]) * x)


def _d2_odd_odd(x, L, p):
    w = 2 * math.pi / L * p["freq"]
    return -w * w * np.sin(w * x)


def _f_even_even(x, L, p):
    return np.cos((math.pi / L * p["freq"]) * x)


def _d2_even_even(x, L, p):
    w = math.pi / L * p["freq"]
    return -w * w * np.cos(w * x)


def _f_odd_even(x, L, p):
    return np.sin((math.pi / L * (p["freq"] + .5)) * x)


def _d2_odd_even(x, L, p):
    w = math.pi / L * (p["freq"] + .5)
    return -w * w * np.sin(w * x)


def _f_even_odd(x, L, p):
    return np.cos((math.pi / L * (p["freq"] + .5)) * x)


def _d2_even_odd(x, L, p):
    w = math.pi / L * (p["freq"] + .5)
    return -w * w * np.cos(w * x)


def _bump(xx):
    with np.errstate(divide="ignore", over="ignore", invalid="ignore"):
        v = np.exp(_C * (1. - 1. / (1. - xx * xx)))
    return np.where(np.abs(xx) >= 1., 0.0, v)


def _f_unb_spietz(x, L, p):
    s = p["sigma"] * L
    x0 = (x - p["center"] * L) / s
    x1 = (x + p["center"] * L) / s
    x2 = (x - (2. - p["center"]) * L) / s
    return _bump(x0) + p["sign"][0] * _bump(x1) + p["sign"][1] * _bump(x2)


def _d2_bump(xsq, s):
    with np.errstate(divide="ignore", over="ignore", invalid="ignore"):
        v = (np.exp(_C * (1. - 1. / (1. - xsq))) * (2. * _C * (2. * (_C - 1.) * xsq + 3. * xsq * xsq - 1.))
             / (xsq - 1.) ** 4 / (s * s))
    return np.where(np.abs(xsq) >= 1., 0.0, v)


def _d2_unb_spietz(x, L, p):
    s = p["sigma"] * L
    x0 = ((x - p["center"] * L) / s) ** 2
    x1 = ((x + p["center"] * L) / s) ** 2
    x2 = ((x - (2. - p["center"]) * L) / s) ** 2
    return _d2_bump(x0, s) + p["sign"][0] * _d2_bump(x1, s) + p["sign"][1] * _d2_bump(x2, s)


def _f_cst(x, L, p):
    return np.ones_like(x)


def _f_zero(x, L, p):
    return np.zeros_like(x)


def manufactured(bcl, bcr, freq):
    """validation_3d.cpp:240-297: solution / RHS factor for one direction."""
    p = {"freq": float(freq), "sign": [0., 0.], "center": 0.5, "sigma": .5}
    if bcl == PER and bcr == PER:
        return _f_odd_odd, _d2_odd_odd, p
    if bcl == ODD and bcr == ODD:
        return _f_odd_odd, _d2_odd_odd, p
    if bcl == EVEN and bcr == EVEN:
        return _f_even_even, _d2_even_even, p
    if bcl == ODD and bcr == EVEN:
        return _f_odd_even, _d2_odd_even, p
    if bcl == EVEN and bcr == ODD:
        return _f_even_odd, _d2_even_odd, p
    if bcl == UNB:
        if bcr == ODD:
            p["center"], p["sign"][1] = .7, -1.
        elif bcr == EVEN:
            p["center"], p["sign"][1] = .7, +1.
        return _f_unb_spietz, _d2_unb_spietz, p
    if bcr == UNB:
        if bcl == ODD:
            p["center"], p["sign"][0] = .3, -1.
        elif bcl == EVEN:
            p["center"], p["sign"][0] = .3, +1.
        return _f_unb_spietz, _d2_unb_spietz, p
    return _f_cst, _f_zero, p


def make_case(center, res, bc, lda=1, L=(1.0, 1.0, 1.0)):
    """validation_3d.cpp:36-45: grid sizes and spacing of one validation case.

    ``bc`` is [[xl, xr], [yl, yr], [zl, zr]] (same BC for every component).
    Returns (nglob, h, bcv) with bcv[d][side][lia].
    """
    fact = 0 if center == CELL_CENTER else 1
    nglob = [res[0] + fact, res[1] + fact, 1 if res[2] == 1 else res[2] + fact]
    h = [L[0] / (nglob[0] - fact), L[1] / (nglob[1] - fact), 1.0 if nglob[2] == 1 else L[2] / (nglob[2] - fact)]
    bcv = [[[bc[d][s]] * lda for s in range(2)] for d in range(3)]
    return nglob, h, bcv


def rhs_and_solution(center, nglob, h, L, bcv, lda):
    """validation_3d.cpp:219-339: manufactured RHS and analytic solution, shape (lda, n0, n1, n2)."""
    shift = 0.5 if center == CELL_CENTER else 0.0
    xs = [(np.arange(nglob[d]) + shift) * h[d] for d in range(3)]
    rhs = np.zeros((lda,) + tuple(nglob))
    sol = np.ones((lda,) + tuple(nglob))
    freqs = [1, 2, 4]
    for lia in range(lda):
        fs = [manufactured(bcv[d][0][lia], bcv[d][1][lia], freqs[d]) for d in range(3)]
        S = [fs[d][0](xs[d], L[d], fs[d][2]) for d in range(3)]
        R = [fs[d][1](xs[d], L[d], fs[d][2]) for d in range(3)]
        sol[lia] = S[0][:, None, None] * S[1][None, :, None] * S[2][None, None, :]
        rhs[lia] = (R[0][:, None, None] * S[1][None, :, None] * S[2][None, None, :]
                    + S[0][:, None, None] * R[1][None, :, None] * S[2][None, None, :]
                    + S[0][:, None, None] * S[1][None, :, None] * R[2][None, None, :])
    return rhs, sol


def error_norms(field, sol, h, bcv):
    """validation_3d.cpp:390-429: err2 = sqrt(sum err^2 * vol), errInf = max |err| per component."""
    vol = 1.0
    for d in range(3):
        if bcv[d][0][0] != NONE and bcv[d][1][0] != NONE:
            vol *= h[d]
    out = []
    for lia in range(field.shape[0]):
        e = sol[lia] - field[lia]
        out.append((math.sqrt(float(np.sum(e * e * vol))), float(np.max(np.abs(e)))))
    return out


def run_case(center, res, bc, kernel, lda=1, L=(1.0, 1.0, 1.0), alpha=2.0):
    from .solver import OracleSolver
    nglob, h, bcv = make_case(center, res, bc, lda, L)
    s = OracleSolver(nglob, lda, bcv, h, L, center)
    s.green_type = kernel
    s.alpha = alpha
    s.setup()
    rhs, sol = rhs_and_solution(center, nglob, h, L, bcv, lda)
    field = s.solve(rhs)
    return nglob, error_norms(field, sol, h, bcv)
