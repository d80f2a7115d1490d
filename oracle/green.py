"""Green's kernels in their four splittings (3 unbounded, 2 unbounded + 1
spectral, 1 unbounded + 2 spectral, 3 spectral), vectorised with numpy.

Reference: src/green_kernels.hpp:26-773 (formulas),
src/green_functions.cpp:27-708 (which formula applies where, values at r=0
and k=0), src/green_functions.hpp:30-91 (LGF table files).
"""
import json
import math
from pathlib import Path

import numpy as np

from . import lgf1unb as l1
from . import specfun as sf
from .plans import (CHAT_2, HEJ_0, HEJ_2, HEJ_4, HEJ_6, HEJ_8, HEJ_10, LGF_2, LGF_4, LGF_6, LGF_8,
                    MEHR_4F, MEHR_4L, MEHR_6F, MEHR_6L)

KERNEL_DIR = Path(__file__).resolve().parent.parent / "flups_b200" / "kernel"

_C_1O4PI = 1.0 / (4.0 * math.pi)
_C_1O2PI = 1.0 / (2.0 * math.pi)
_C_1OPI = 1.0 / math.pi
_C_1O2PI2 = 1.0 / (2.0 * math.pi * math.pi)
_C_1OSQRT2 = 1.0 / math.sqrt(2.0)
_C_1OSQRTPI = 1.0 / math.sqrt(math.pi)

HEJ_REG = (HEJ_2, HEJ_4, HEJ_6, HEJ_8, HEJ_10)
LGF_ALL = (LGF_2, LGF_4, LGF_6, LGF_8)
MEHR_ALL = (MEHR_4L, MEHR_6L, MEHR_4F, MEHR_6F)

_FARFIELD = None


def _farfield_table():
    global _FARFIELD
    if _FARFIELD is None:
        _FARFIELD = json.loads((KERNEL_DIR / "farfield.json").read_text())
    return _FARFIELD


def farfield(name, n1, n2, n3=None):
    """Evaluate the far-field expansion ``name`` (lgf_3unb0spe.hpp:5-374)."""
    ent = _farfield_table()[name]
    n1 = np.asarray(n1, dtype=np.float64)
    n2 = np.asarray(n2, dtype=np.float64)
    n3 = np.zeros_like(n1) if n3 is None else np.asarray(n3, dtype=np.float64)
    n = np.sqrt(n1 * n1 + n2 * n2 + n3 * n3)
    out = np.zeros(n.shape)
    cache = {}

    def pw(key, base, e):
        k = (key, e)
        if k not in cache:
            cache[k] = base ** e if e != 0 else 1.0
        return cache[k]

    for c, a, b, d, e, p in ent["terms"]:
        out += (c * math.pi ** p) * pw(1, n1, a) * pw(2, n2, b) * pw(3, n3, d) * pw(0, n, e)
    for c, a, b, d, e, p in ent["log_terms"]:
        out += c * np.log(n)
    return out


def _table_name(kind, ndim):
    # green_functions.hpp:53-72
    order = {LGF_2: 2, LGF_4: 4, MEHR_4L: 4, MEHR_4F: 4, LGF_6: 6, MEHR_6L: 6, MEHR_6F: 6, LGF_8: 8}[kind]
    if ndim == 3:
        if kind in (MEHR_4L, MEHR_6L):
            return f"MEHR_{order}L_3d_32.ker"
        if kind in (MEHR_4F, MEHR_6F):
            return f"MEHR_{order}F_3d_32.ker"
        return f"LGF_{order}_3d_32.ker"
    if kind in (MEHR_4L, MEHR_6L):
        return "MEHR_4L6L_2d_32.ker"
    if kind in (MEHR_4F, MEHR_6F):
        return f"MEHR_{order}F_2d_32.ker"
    return f"LGF_{order}_2d_32.ker"


def lgf_table(kind, ndim):
    data = np.fromfile(KERNEL_DIR / _table_name(kind, ndim), dtype="<f8")
    return 32, data


def _farfield_name(kind, ndim):
    base = {LGF_2: "lgf_2", LGF_4: "lgf_4", LGF_6: "lgf_6", LGF_8: "lgf_8", MEHR_4L: "mehr_4l",
            MEHR_6L: "mehr_6l", MEHR_4F: "mehr_4f", MEHR_6F: "mehr_6f"}[kind]
    if ndim == 2 and kind in (MEHR_4L, MEHR_6L):
        base = "mehr_4l6l"
    return f"{base}_{ndim}unb0spe"


def lgf_3d(kind, ix, iy, iz, h):
    """green_kernels.hpp:70-133 and :203-257: table inside 32^3, expansion outside; -G/h."""
    N, data = lgf_table(kind, 3)
    ix = ix.astype(np.int64)
    iy = iy.astype(np.int64)
    iz = iz.astype(np.int64)
    inside = (ix < N) & (iy < N) & (iz < N)
    g = np.empty(ix.shape)
    g[inside] = data[(ix + iy * N + iz * N * N)[inside]]
    out = ~inside
    if np.any(out):
        g[out] = farfield(_farfield_name(kind, 3), ix[out], iy[out], iz[out])
    return -g / h


def lgf_2d(kind, ix, iy, iz):
    """green_kernels.hpp:134-201 and :258-329: i1/i2 = first/second nonzero index; -G."""
    N, data = lgf_table(kind, 2)
    ix = ix.astype(np.int64)
    iy = iy.astype(np.int64)
    iz = iz.astype(np.int64)
    i1 = np.where(ix == 0, iy, ix)
    i2 = np.where(ix == 0, iz, np.where(iy == 0, iz, iy))
    inside = (i1 < N) & (i2 < N)
    g = np.empty(ix.shape)
    g[inside] = data[(i1 + i2 * N)[inside]]
    out = ~inside
    if np.any(out):
        g[out] = farfield(_farfield_name(kind, 2), i1[out], i2[out])
    return -g


# ---------------------------------------------------------------- 3 unbounded
def green_3unb(kind, r, ia, ib, ic, h, length, hprod):
    """green_functions.cpp:27-167 (kernels green_kernels.hpp:26-69)."""
    with np.errstate(divide="ignore", invalid="ignore"):
        rho = r / length
        ex = np.exp(-rho * rho * .5)
        ef = _erf(rho * _C_1OSQRT2)
        pre = _C_1OSQRT2 * _C_1OSQRTPI
        if kind == HEJ_2:
            g = -_C_1O4PI / r * _erf(r / length * _C_1OSQRT2)
        elif kind == HEJ_4:
            g = -_C_1O4PI / r * (pre * rho * ex + ef)
        elif kind == HEJ_6:
            g = -_C_1O4PI / r * (pre * (7. / 4. * rho - 1. / 4. * rho ** 3) * ex + ef)
        elif kind == HEJ_8:
            g = -_C_1O4PI / r * (pre * (19. / 8 * rho - 2. / 3 * rho ** 3 + 1. / 24 * rho ** 5) * ex + ef)
        elif kind == HEJ_10:
            g = -_C_1O4PI / r * (pre * (187. / 64. * rho - 233. / 192. * rho ** 3 + 29. / 192. * rho ** 5
                                        - 1. / 192. * rho ** 7) * ex + ef)
        elif kind == HEJ_0:
            g = -_C_1O2PI2 * (1.0 / length) * sf.sine_integral(rho) / rho
        elif kind == CHAT_2:
            g = -_C_1O4PI / r
        elif kind in LGF_ALL or kind in MEHR_ALL:
            return lgf_3d(kind, ia, ib, ic, h)
        else:
            raise ValueError("Green Function type unknown.")
    s3 = math.sqrt(math.pi ** 3)
    g0 = {HEJ_2: -math.sqrt(2.0) / (4.0 * length * s3),
          HEJ_4: -3.0 * math.sqrt(2.0) / (8.0 * length * s3),
          HEJ_6: -15.0 * math.sqrt(2.0) / (32.0 * length * s3),
          HEJ_8: -35.0 * math.sqrt(2.0) / (64.0 * length * s3),
          HEJ_10: -315.0 * math.sqrt(2.0) / (512.0 * length * s3),
          HEJ_0: -1.0 / (2.0 * math.pi * math.pi * length),
          CHAT_2: -0.5 * (1.5 * _C_1O2PI * hprod) ** (2. / 3.) / hprod}[kind]
    return g, g0


def _erf(x):
    from scipy.special import erf
    return erf(x)


# ------------------------------------------------------ 2 unbounded, 1 spectral
def green_2unb1spe(kind, r, k, ia, ib, ic, length, r_eq2d, r_cut, k_cut):
    """green_functions.cpp:192-391 (kernels green_kernels.hpp:340-456)."""
    out = np.zeros(r.shape)
    m_r0 = r <= r_cut
    m_k0 = (~m_r0) & (k <= k_cut)
    m_g = ~(m_r0 | m_k0)
    sig = length

    def hej_k0(rr, poly):
        rho2 = (rr / sig) ** 2
        return _C_1O2PI * (np.log(rr) - poly(rho2) * np.exp(-rho2 * 0.5) + 0.5 * sf.expint_ei(rho2 * 0.5))

    def hej_r0(const):
        return -_C_1O2PI * (sf.C_GAMMA * .5 - math.log(math.sqrt(2.0) * sig) + const)

    hej = {HEJ_2: (lambda x: 0.0 * x, 0.0),
           HEJ_4: (lambda x: 0.5 + 0.0 * x, 0.5),
           HEJ_6: (lambda x: 0.75 - 0.125 * x, 0.75),
           HEJ_8: (lambda x: 11. / 12. - 7. / 24. * x + 1. / 48. * x * x, 11. / 12.),
           HEJ_10: (lambda x: 25. / 24. - 23. / 48. * x + 13. / 192. * x * x - 1. / 384. * x ** 3, 25. / 24.)}
    with np.errstate(divide="ignore", invalid="ignore"):
        if kind in hej:
            poly, c = hej[kind]
            if kind == HEJ_2:
                rk = r[m_k0]
                rho2 = (rk / sig) ** 2
                out[m_k0] = _C_1O2PI * (np.log(rk) + 0.5 * sf.expint_ei(rho2 * 0.5))
            else:
                out[m_k0] = hej_k0(r[m_k0], poly)
            out[m_r0] = hej_r0(c)
        elif kind == HEJ_0:
            def f(rr):
                rho = rr / sig
                tmp = _C_1O2PI * (sf.ji0c(rho) + math.log(2 * sig) - sf.C_GAMMA)
                return np.where(rho < 30.0, tmp, _C_1O2PI * np.log(rr))
            out[m_k0] = f(r[m_k0])
            out[m_r0] = f(r[m_r0])
        elif kind == CHAT_2:
            out[m_g] = -_C_1O2PI * sf.besselk0(np.abs(k[m_g]) * r[m_g])
            out[m_k0] = _C_1O2PI * np.log(r[m_k0])
            kk = k[m_r0]
            out[m_r0] = -(1.0 - kk * r_eq2d * sf.besselk1(kk * r_eq2d)) * _C_1OPI / ((kk * r_eq2d) * (kk * r_eq2d))
        elif kind in LGF_ALL or kind in MEHR_ALL:
            m = m_k0 | m_r0
            out[m] = lgf_2d(kind, ia[m], ib[m], ic[m])
        else:
            raise ValueError("Green Function type unknown.")
    return out


# ------------------------------------------------------ 1 unbounded, 2 spectral
def _lgf_1unb_other(kind, r, k0, k1, k2, h):
    """LGF_4/6/8 and MEHR kernels of one unbounded direction
    (green_kernels.hpp:591-671): the 1-D lattice Green's function at
    n = round(|r| / h), shifted by the symbol of the spectral wave numbers
    (one of k0, k1, k2 is zero).  Evaluated once per distinct argument."""
    r, k0, k1, k2 = np.broadcast_arrays(*(np.asarray(a, dtype=np.float64) for a in (r, k0, k1, k2)))
    n = np.round(np.abs(r) / h).astype(np.int64)
    if kind in (LGF_4, LGF_6, LGF_8):
        sym = {LGF_4: l1.lgf4_symbol, LGF_6: l1.lgf6_symbol, LGF_8: l1.lgf8_symbol}[kind]
        fn = {LGF_4: l1.lgf4, LGF_6: l1.lgf6, LGF_8: l1.lgf8}[kind]
        symv = np.vectorize(sym, otypes=[np.float64])
        c = symv(k0 * h) + symv(k1 * h) + symv(k2 * h)
        keys = np.stack([n.ravel().astype(np.float64), c.ravel()], axis=1)
        uniq, inv = np.unique(keys, axis=0, return_inverse=True)
        vals = np.array([fn(int(a), float(b)) for a, b in uniq])
    else:
        fn = {MEHR_4L: l1.meh4_left, MEHR_6L: l1.meh6_left, MEHR_4F: l1.meh4_full, MEHR_6F: l1.meh6_full}[kind]
        a0, a1, a2 = np.abs(k0), np.abs(k1), np.abs(k2)
        kmax = np.maximum(a0, np.maximum(a1, a2))
        kmid = a0 + a1 + a2 - kmax
        keys = np.stack([n.ravel().astype(np.float64), (kmax * h).ravel(), (kmid * h).ravel()], axis=1)
        uniq, inv = np.unique(keys, axis=0, return_inverse=True)
        vals = np.array([fn(int(a), float(b), float(c)) for a, b, c in uniq])
    return vals[inv.ravel()].reshape(r.shape)


def green_1unb2spe(kind, r, k, k0, k1, k2, h, length, k_cut):
    """green_functions.cpp:407-538 (kernels green_kernels.hpp:461-671)."""
    sig = length
    m0 = k <= k_cut
    out = np.zeros(r.shape)
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        if kind in HEJ_REG:
            rho = r / sig
            s = k * sig
            s2, rho2 = s * s, rho * rho
            sub = np.where(s * rho > 100., 0.0,
                           (1.0 - _erf(_C_1OSQRT2 * (s - rho))) * np.exp(-s * rho)
                           + (1.0 - _erf(_C_1OSQRT2 * (s + rho))) * np.exp(s * rho))
            base = -.25 * sig / s * sub
            pre = sig * math.sqrt(2.0) * _C_1OSQRTPI
            e = np.exp(-.5 * (s * s + rho * rho))
            erfr = 0.5 * r * _erf(r * _C_1OSQRT2 / sig)
            q = sig * _C_1OSQRT2 * _C_1OSQRTPI
            er = np.exp(-rho * rho * .5)
            if kind == HEJ_2:
                g = base
                g0 = erfr - (1. - er) * q
            elif kind == HEJ_4:
                g = base - pre * .25 * e
                g0 = erfr - (1. - er) * .5 * q
            elif kind == HEJ_6:
                g = base - pre * (5. / 16. + 1. / 16. * (s2 - rho2)) * e
                g0 = erfr - (3. - er * (rho2 + 3.)) * .125 * q
            elif kind == HEJ_8:
                g = base - pre * (11. / 32. + 1. / 12. * s2 - 0.125 * rho2 - 1. / 48. * s2 * rho2
                                  + 1. / 96. * (s2 * s2 + rho2 * rho2)) * e
                g0 = erfr - (5. / 16. - er * (-1. / 48. * rho2 * rho2 + .25 * rho2 + 5. / 16.)) * q
            else:
                g = base - pre * (93. / 256. + 73. / 768. * s2 - 47. / 256. * rho2 - 17. / 384. * s2 * rho2
                                  + 11. / 768. * s2 * s2 + 23. / 768. * rho2 * rho2
                                  + 1. / 256. * (s2 * rho2 * rho2 - s2 * s2 * rho2)
                                  + 1. / 768. * (s2 * s2 * s2 - rho2 * rho2 * rho2)) * e
                g0 = erfr - (35. / 128. - er * (1. / 384. * rho2 ** 3 - 23. / 384. * rho2 * rho2
                                                 + 47. / 128. * rho2 + 35. / 128.)) * q
        elif kind == CHAT_2:
            g = -0.5 * np.exp(-k * r) / k
            g0 = 0.5 * np.abs(r)
        elif kind == LGF_2:
            c = sf.lgf2_symbol(k0 * h) + sf.lgf2_symbol(k1 * h) + sf.lgf2_symbol(k2 * h)
            n = np.round(np.abs(r) / h)
            g = g0 = -h * sf.lgf2_1unb(n, c)
        elif kind in (LGF_4, LGF_6, LGF_8, MEHR_4L, MEHR_6L, MEHR_4F, MEHR_6F):
            g = g0 = -h * _lgf_1unb_other(kind, r, k0, k1, k2, h)
        elif kind == HEJ_0:
            raise ValueError("HEJ0 kernel not available for 1D unbounded problems.")
        else:
            raise ValueError("Green Function type unknown.")
    out[m0] = np.asarray(g0 * np.ones_like(r))[m0]
    out[~m0] = np.asarray(g * np.ones_like(r))[~m0]
    return out


# ----------------------------------------------------------- 3 spectral
def green_0unb3spe(kind, ksqr, k0, k1, k2, h, length):
    """green_functions.cpp:560-708 (kernels green_kernels.hpp:681-773)."""
    sig = length
    with np.errstate(divide="ignore", invalid="ignore"):
        s = ksqr * (sig * sig)
        e = np.exp(-s * 0.5)
        if kind == HEJ_2:
            return -e / ksqr
        if kind == HEJ_4:
            return -(1.0 + s * 0.5) * e / ksqr
        if kind == HEJ_6:
            return -(1.0 + s * 0.5 + s * s * 0.125) * e / ksqr
        if kind == HEJ_8:
            s2 = s * s
            return -(1.0 + s * 0.5 + s2 * 0.125 + s2 * s * (1. / 48.)) * e / ksqr
        if kind == HEJ_10:
            s2 = s * s
            return -(1.0 + s * 0.5 + s2 * 0.125 + s2 * s * (1. / 48.) + s2 * s2 * (1. / 384.)) * e / ksqr
        if kind in (CHAT_2, HEJ_0):
            return -1.0 / ksqr
        sym = {LGF_2: sf.lgf2_symbol, LGF_4: sf.lgf4_symbol, LGF_6: sf.lgf6_symbol, LGF_8: sf.lgf8_symbol}
        if kind in sym:
            f = sym[kind]
            return -h * h / (f(k0 * h) + f(k1 * h) + f(k2 * h))
        y0, y1, y2 = np.sin(k0 * h / 2.) ** 2, np.sin(k1 * h / 2.) ** 2, np.sin(k2 * h / 2.) ** 2
        left = -4. * (y0 + y1 + y2) + 8. / 3. * (y0 * y1 + y1 * y2 + y0 * y2)
        if kind in (MEHR_6L, MEHR_6F):
            left = left - 32. / 15. * y0 * y1 * y2
        if kind == MEHR_4L or kind == MEHR_6L:
            return h * h / left
        if kind == MEHR_4F:
            return h * h * (1. - 1. / 3. * (y0 + y1 + y2)) / left
        if kind == MEHR_6F:
            right = (1. - 1. / 3. * (y0 + y1 + y2) + 8. / 45. * (y0 * y1 + y1 * y2 + y0 * y2)
                     - 1. / 15. * (y0 * y0 + y1 * y1 + y2 * y2))
            return h * h * right / left
    raise ValueError("Green Function type unknown.")
