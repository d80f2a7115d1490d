"""Vortex-tube Biot-Savart validation (ROT solve), restating
samples/solve_vtube/src/vtube.cpp:55-600 (tube case) and the case set-up of
samples/solve_vtube/src/main_vtube.cpp:140-230.

``run_tube`` returns the per-component (err2, errInf) the reference writes to
``data/vtube_CellCenter_0_<dir><xsign><ysign>_typeGreen=<k>.txt``.
"""
import math

import numpy as np

from .plans import CELL_CENTER, EVEN, ODD, UNB, SPE, ROT
from .validation import error_norms


def vort_inf(r, sigma):
    rho = r / sigma
    return 1.0 / (2 * math.pi * sigma * sigma) * np.exp(-rho * rho * 0.5)


def vel_inf(r, sigma):
    eps = 100 * np.finfo(np.float64).eps
    rho = r / sigma
    with np.errstate(divide="ignore", invalid="ignore"):
        v = 1.0 / (2 * math.pi * r) * (1.0 - np.exp(-rho * rho * 0.5))
    return np.where(r < eps, 0.0, v)


def tube_case(vdir, sym_x, sym_y):
    """main_vtube.cpp:140-200: per-component BCs, tube centres and image signs."""
    dir2, dir0, dir1 = vdir, (vdir + 1) % 3, (vdir + 2) % 3
    bcv = [[[UNB] * 3, [UNB] * 3] for _ in range(3)]
    xc, yc, xs, ys = 0.5, 0.5, 0.0, 0.0
    for ip in range(3):
        if ip == dir2:
            left = {dir0: ODD, dir1: ODD, dir2: EVEN}
            bcv[ip] = [[left[c] for c in range(3)], [left[c] for c in range(3)]]
        elif ip == dir1:
            if sym_y == 1:
                yc, ys = 0.25, 1.0
                left = {dir0: EVEN, dir1: ODD, dir2: EVEN}
            elif sym_y == -1:
                yc, ys = 0.25, -1.0
                left = {dir0: ODD, dir1: EVEN, dir2: ODD}
            else:
                left = None
            if left is not None:
                bcv[ip] = [[left[c] for c in range(3)], [UNB] * 3]
        else:
            if sym_x == 1:
                xc, xs = 0.25, 1.0
                left = {dir0: ODD, dir1: EVEN, dir2: EVEN}
            elif sym_x == -1:
                xc, xs = 0.25, -1.0
                left = {dir0: EVEN, dir1: ODD, dir2: ODD}
            else:
                left = None
            if left is not None:
                bcv[ip] = [[left[c] for c in range(3)], [UNB] * 3]
    return bcv, xc, yc, xs, ys


def tube_fields(vdir, nglob, h, L, xc, yc, xs, ys, sigma):
    """vtube.cpp:160-300: vorticity RHS and analytic velocity of the tube and its images."""
    dir2, dir0, dir1 = vdir, (vdir + 1) % 3, (vdir + 2) % 3
    pos = np.meshgrid(*[(np.arange(nglob[d]) + 0.5) * h[d] for d in range(3)], indexing="ij")
    rhs = np.zeros((3,) + tuple(nglob))
    sol = np.zeros((3,) + tuple(nglob))
    for sx, sy, w in ((-1, -1, 1.0), (1, -1, xs), (-1, 1, ys), (1, 1, xs * ys)):
        x = pos[dir0] + sx * (xc * L[dir0])
        y = pos[dir1] + sy * (yc * L[dir1])
        th = np.arctan2(y, x)
        r = np.sqrt(x * x + y * y)
        vort, vel = vort_inf(r, sigma), vel_inf(r, sigma)
        rhs[dir2] += -vort * w
        if dir2 == 0:
            sol[1] += -np.sin(th) * vel * w
            sol[2] += +np.cos(th) * vel * w
        elif dir2 == 1:
            sol[0] += +np.cos(th) * vel * w
            sol[2] += -np.sin(th) * vel * w
        else:
            sol[0] += -np.sin(th) * vel * w
            sol[1] += +np.cos(th) * vel * w
    return rhs, sol


def run_tube(vdir, sym_x, sym_y, res=16, kernel=0, sigma=0.1, order=SPE):
    from .solver import OracleSolver
    L = (1.0, 1.0, 1.0)
    nglob = [res] * 3
    h = [L[d] / nglob[d] for d in range(3)]
    bcv, xc, yc, xs, ys = tube_case(vdir, sym_x, sym_y)
    s = OracleSolver(nglob, 3, bcv, h, L, CELL_CENTER, orderdiff=order)
    s.green_type = kernel
    s.setup()
    rhs, sol = tube_fields(vdir, nglob, h, L, xc, yc, xs, ys, sigma)
    field = s.solve(rhs, ROT)
    return error_norms(field, sol, h, bcv)
