"""Shared helpers of the GPU tests: run a case through the C ABI (pyflups
front-end) and through the CPU oracle on the same input."""
import math
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from flups_b200 import pyflups as pf  # noqa: E402
from oracle.solver import OracleSolver  # noqa: E402


def to_user(a):
    """oracle array (lda, n0, n1, n2) -> C-ABI user layout (axis 0 fastest): [lda][n2][n1][n0]."""
    return np.ascontiguousarray(np.transpose(a, (0, 3, 2, 1)))


def from_user(u, lda, nglob):
    return np.transpose(u.reshape(lda, nglob[2], nglob[1], nglob[0]), (0, 3, 2, 1))


def make_solver(nglob, lda, bcv, h, L, center, kernel, odiff=0, precision=64, alpha=2.0):
    t = pf.Topology(0, lda, list(nglob))
    bc = [[bcv[d][s][:lda] for s in range(2)] for d in range(3)]
    s = pf.Solver(t, bc, list(h), list(L), order_diff=odiff, center_type=[center] * 3)
    s.set_green_type(kernel)
    s.set_alpha(alpha)
    if precision != 64:
        s.set_precision(precision)
    s.setup()
    return t, s


def gpu_solve(nglob, lda, bcv, h, L, center, kernel, rhs, type_=0, odiff=0, precision=64, alpha=2.0, device=False,
              xlast=True):
    """One solve through the C ABI.  device=False passes host (numpy) arrays,
    which 3-D problems solve in the reference's pass order with slab-streamed
    copies; device=True passes CUDA arrays (the x-last order of all-unbounded
    problems unless xlast=False)."""
    t, s = make_solver(nglob, lda, bcv, h, L, center, kernel, odiff, precision, alpha)
    s.set_xlast(xlast)
    u = to_user(rhs)
    if device:
        import torch
        du = torch.from_numpy(u).cuda()
        dout = torch.zeros_like(du)
        s.solve(dout, du, type_)
        torch.cuda.synchronize()
        out = dout.cpu().numpy()
    else:
        out = np.zeros_like(u)
        s.solve(out, u, type_)
    err = s.last_error()
    del s, t
    assert err == 0, f"CUDA error {err}"
    return from_user(out, lda, nglob)


def oracle_solve(nglob, lda, bcv, h, L, center, kernel, rhs, type_=0, odiff=0, alpha=2.0):
    import os

    import scipy.fft
    # the oracle's transforms on every host core (same results, shorter waits)
    with scipy.fft.set_workers(os.cpu_count() or 1):
        o = OracleSolver(nglob, lda, bcv, h, L, center, orderdiff=odiff)
        o.green_type = kernel
        o.alpha = alpha
        o.setup()
        return o.solve(rhs, type_)


def rel_l2(a, b):
    num = float(np.sqrt(np.sum((a - b) ** 2)))
    den = float(np.sqrt(np.sum(b ** 2)))
    return num / den if den > 0 else num


def rel_linf(a, b):
    den = float(np.max(np.abs(b)))
    return float(np.max(np.abs(a - b))) / den if den > 0 else float(np.max(np.abs(a - b)))
