"""The solve sequence of the reference, on global-index numpy arrays.

Arrays are shaped (lda, n0, n1, n2) in global index order; the reference's
pencil transposes (SwitchTopo) reduce, on one rank, to zero padding and a
shift by ``fieldstart`` along the transformed direction, which is what
``_switch_in``/``_switch_out`` do.

Reference: src/Solver.cpp:23-202 (ctor), :219-469 (setup), :589-811 (dry run),
:980-1106 (Green), :1115-1154 (scaling), :1207-1272 (solve), :1402-1462
(do_FFT), :1471-1542 (do_mult); src/FFTW_plan_dim.cpp:497-720 (execute and
postprocess); src/dothemagic_std.ipp:56-83; src/dothemagic_rot.ipp:102-350.
"""
import math

import numpy as np
import scipy.fft as sfft

from . import green as gk
from .plans import (BACKWARD, BACKWARD_DIFF, EMPTY, ENFORCE_PERIOD, EVEN, FD2, FD4, FD6, FORWARD,
                    HEJ_0, MIXUNB, NOD, NULL_FIRST, NULL_LAST, ODD, PERPER, ROT, SPE, STD, SYMSYM,
                    UNBUNB, CHAT_2, Plan, sort_plans)


def _r2r(kind, x):
    fam, typ = kind
    f = sfft.dct if fam == "dct" else sfft.dst
    return f(x, type=typ, axis=-1)


def _as_complex(real_line):
    return real_line[..., 0::2] + 1j * real_line[..., 1::2]


def _as_real(cplx_line):
    out = np.empty(cplx_line.shape[:-1] + (2 * cplx_line.shape[-1],))
    out[..., 0::2] = cplx_line.real
    out[..., 1::2] = cplx_line.imag
    return out


def execute_plan(p, lia, line):
    """FFTW_plan_dim.cpp:635-720 on one component; ``line`` has the transform axis last.

    Returns the in-place result (stale entries the transform does not write are kept).
    """
    fi, fo, n_in = p.fftwstart_in[lia], p.fftwstart_out[lia], p.n_in[0 if p.type in (PERPER, UNBUNB) else lia]
    if p.type == EMPTY:
        return line
    if p.type in (SYMSYM, MIXUNB):
        out = line.copy()
        out[..., fo:fo + n_in] = _r2r(p.kind[lia], line[..., fi:fi + n_in])
        return out
    if p.isr2c:
        if p.sign == FORWARD:  # real line of 2*n_out -> complex n_out
            out = _as_complex(line)
            res = sfft.rfft(line[..., fi:fi + n_in], axis=-1)
            out[..., fo:fo + res.shape[-1]] = res
            return out
        out = _as_real(line)  # complex n_out -> real 2*n_out
        res = sfft.irfft(line[..., fi:fi + n_in // 2 + 1], n=n_in, axis=-1, norm="forward")
        out[..., fo:fo + n_in] = res
        return out
    out = line.copy()
    seg = line[..., fi:fi + n_in]
    res = sfft.fft(seg, axis=-1) if p.sign == FORWARD else sfft.ifft(seg, axis=-1, norm="forward")
    out[..., fo:fo + n_in] = res
    return out


def postprocess_plan(p, lia, line):
    """FFTW_plan_dim.cpp:497-622 on one component (transform axis last, current units)."""
    c = p.postpro[lia]
    first, last, period = bool(c & NULL_FIRST), bool(c & NULL_LAST), bool(c & ENFORCE_PERIOD)
    nloc = line.shape[-1]
    if first:
        line[..., 0] = 0.0
    if last:
        line[..., nloc - 1] = 0.0
    if period and not (first or last):
        nfftw = p.n_out - 1 if p.sign == FORWARD else p.n_in[lia]
        line[..., nfftw] = line[..., 0]
    return line


class OracleSolver:
    """Single-rank FP64 FLUPS solver on numpy arrays (mirror of class Solver)."""

    def __init__(self, nglob, lda, bc, h, L, center, orderdiff=NOD):
        # Solver.cpp:23-202; bc[d][side][lia]
        self.nglob = [int(v) for v in nglob]
        self.lda = lda
        self.h = [float(v) for v in h]
        self.L = [float(v) for v in L]
        self.center = center
        self.odiff = orderdiff
        self.green_type = CHAT_2
        self.alpha = 2.0
        self.bc = bc
        self.plan_fwd = sort_plans([Plan(lda, d, h, L, bc[d], FORWARD, False, center) for d in range(3)])
        self.plan_bwd = sort_plans([Plan(lda, d, h, L, bc[d], BACKWARD, False, center) for d in range(3)])
        self.plan_green = sort_plans([Plan(1, d, h, L, bc[d], FORWARD, True, center) for d in range(3)])
        self.plan_diff = None
        if orderdiff != NOD:
            swap = {EVEN: ODD, ODD: EVEN}
            diffbc = [[[swap.get(v, v) for v in bc[d][s]] for s in range(2)] for d in range(3)]
            self.plan_diff = [Plan(lda, p.dim, h, L, diffbc[p.dim], BACKWARD, False, center)
                              for p in self.plan_bwd]
        self.ndim = sum(1 for p in self.plan_fwd if p.type != EMPTY)
        if self.ndim < 2:
            raise ValueError("We only handle 2D and 3D field")
        self.sizes_before = self._dry_run(self.plan_fwd)
        self._dry_run(self.plan_bwd)
        self._dry_run(self.plan_green)
        if self.plan_diff is not None:
            self._dry_run(self.plan_diff)
        self.normfact = 1.0
        self.volfact = 1.0
        for p in self.plan_fwd:
            self.normfact *= p.normfact
            self.volfact *= p.volfact
        self.green = None

    def _dry_run(self, plans):
        """Solver.cpp:617-650: init the plans in order on the running size."""
        size = list(self.nglob)
        cplx = False
        before = []
        for ip in range(self.ndim):
            before.append(list(size))
            plans[ip].init(size, cplx)
            size[plans[ip].dim] = plans[ip].n_out
            cplx = cplx or plans[ip].isr2c
        self._spec_size, self._spec_complex = size, cplx
        return before

    # ------------------------------------------------------------ spectral info
    def spectral_info(self):
        """Solver.hpp:222-229."""
        kfact, koffset, symstart = [0.0] * 3, [0.0] * 3, [0.0] * 3
        for p in self.plan_fwd:
            kfact[p.dim], koffset[p.dim], symstart[p.dim] = p.kfact, p.koffset, p.symstart
        return kfact, koffset, symstart

    # ------------------------------------------------------------ green
    def setup(self):
        """Solver.cpp:219-469 minus the distributed bookkeeping: compute the Green spectrum."""
        self.green = self._compute_green()
        return self

    @staticmethod
    def _symid(ie, symstart):
        """Topology.hpp:415-430 on one direction (signed symmetric index)."""
        ie = np.asarray(ie)
        if symstart == 0.0:
            return ie.copy()
        alt = -np.maximum(np.abs(2.0 * symstart - ie).astype(np.int64), 1)
        return np.where(ie <= symstart, ie, alt)

    def _compute_green(self):
        # Solver.cpp:980-1106
        h = self.h
        kind = self.green_type
        length = self.alpha * h[0]
        if kind == HEJ_0:
            length = h[0] / math.pi
        reg_or_lgf2 = kind in gk.HEJ_REG + (HEJ_0, 1)
        if reg_or_lgf2 and ((self.ndim == 3 and (h[0] != h[1] or h[1] != h[2])) or
                            (self.ndim == 2 and h[0] != h[1])):
            raise ValueError("You are trying to use a regularized kernel or a LGF while not having dx=dy=dz.")
        pg = self.plan_green
        is_spec, symstart, hfact, kfact, koffset = [False] * 3, [0.0] * 3, [0.0] * 3, [0.0] * 3, [0.0] * 3
        for ip in range(self.ndim):
            p = pg[ip]
            d = p.dim
            is_spec[d] = p.is_spectral
            symstart[d] = p.symstart
            hfact[d] = h[d]
            if p.is_spectral:
                hfact[d], kfact[d], koffset[d] = 0.0, p.kfact, p.koffset
            if p.type == EMPTY:
                hfact[d] = 0.0
        nspec = sum(1 for d in range(self.ndim) if is_spec[d])
        nunb = self.ndim - nspec
        # Green topology 0 (Solver.cpp:727-781): walk back from the spectral size
        size = list(self._green_spec_size())
        cplx = self._green_spec_complex
        for ip in range(self.ndim - 1, -1, -1):
            if pg[ip].isr2c_done_by_fft:
                size[pg[ip].dim] *= 2
                cplx = False
        ax = [pg[0].dim, (pg[0].dim + 1) % 3, (pg[0].dim + 2) % 3]  # topology axis order
        idx = [self._symid(np.arange(size[d]), symstart[d]) for d in range(3)]
        I0, I1, I2 = np.meshgrid(idx[0], idx[1], idx[2], indexing="ij")
        I = [I0, I1, I2]
        X = [I[d] * hfact[d] for d in range(3)]
        K = [(I[d] + koffset[d]) * kfact[d] for d in range(3)]
        A = [np.abs(I[ax[0]]), np.abs(I[ax[1]]), np.abs(I[ax[2]])]
        g = np.zeros(size)
        if nunb == 3:
            # only |is| matters here: evaluate on the distinct values per direction, then expand
            uniq = [np.unique(np.abs(idx[d]), return_inverse=True) for d in range(3)]
            U = np.meshgrid(uniq[0][0], uniq[1][0], uniq[2][0], indexing="ij")
            UX = [U[d] * hfact[d] for d in range(3)]
            UA = [U[ax[0]], U[ax[1]], U[ax[2]]]
            r = np.sqrt(UX[0] ** 2 + UX[1] ** 2 + UX[2] ** 2)
            res = gk.green_3unb(kind, r, UA[0], UA[1], UA[2], hfact[ax[0]], length, hfact[0] * hfact[1] * hfact[2])
            gu, g0 = res if isinstance(res, tuple) else (res, None)
            g = gu[np.ix_(uniq[0][1].ravel(), uniq[1][1].ravel(), uniq[2][1].ravel())]
            if g0 is not None:
                g[0, 0, 0] = g0
        elif nunb == 2:
            r = np.sqrt(X[0] ** 2 + X[1] ** 2 + X[2] ** 2)
            k = K[0] + K[1] + K[2]
            hs = [hfact[ax[0]], hfact[ax[1]], hfact[ax[2]]]
            r_eq2d = (1.0 / math.sqrt(math.pi)) * math.sqrt(hs[0] * hs[1] + hs[1] * hs[2] + hs[2] * hs[0])
            r_cut = (hs[0] + hs[1] + hs[2]) * .2
            k_cut = (kfact[ax[0]] + kfact[ax[1]] + kfact[ax[2]]) * 0.2
            g = gk.green_2unb1spe(kind, r, k, A[0], A[1], A[2], length, r_eq2d, r_cut, k_cut)
            if kind == CHAT_2:
                g[0, 0, 0] = 0.25 * (1.0 / (2.0 * math.pi)) * (math.pi - 6.0 + 2.0 * math.log(0.5 * math.pi * r_eq2d * r_eq2d))
        elif nunb == 1:
            r = np.sqrt(X[0] ** 2 + X[1] ** 2 + X[2] ** 2)
            k = np.sqrt(K[0] ** 2 + K[1] ** 2 + K[2] ** 2)
            hh = hfact[ax[0]] + hfact[ax[1]] + hfact[ax[2]]
            k_cut = (kfact[ax[0]] + kfact[ax[1]] + kfact[ax[2]]) * 0.2
            g = gk.green_1unb2spe(kind, r, k, K[ax[0]], K[ax[1]], K[ax[2]], hh, length, k_cut)
        else:
            ksq = K[0] ** 2 + K[1] ** 2 + K[2] ** 2
            g = gk.green_0unb3spe(kind, ksq, K[ax[0]], K[ax[1]], K[ax[2]], h[0], length)
            if sum(koffset) < 0.2:
                g[0, 0, 0] = 0.0
        data = g.astype(np.complex128) if cplx else g
        # forward transforms of the Green's function (Solver.cpp:1058-1076)
        for ip in range(self.ndim):
            p = pg[ip]
            if is_spec[p.dim]:
                if p.isr2c:  # spectral r2c direction: the topology just becomes complex
                    data = data.astype(np.complex128) if not np.iscomplexobj(data) else data
                continue
            a = np.moveaxis(data, p.dim, -1)
            if p.type in (SYMSYM, MIXUNB) and np.iscomplexobj(a):
                res = a.copy()
                res.real = execute_plan(p, 0, np.ascontiguousarray(a.real))
            else:
                res = execute_plan(p, 0, a)
            data = np.moveaxis(res, -1, p.dim)
        data = data * self.volfact  # Solver.cpp:1115-1154
        is_reg = kind in gk.HEJ_REG or kind in gk.LGF_ALL or kind in gk.MEHR_ALL
        if self.ndim == 3 and nspec == 1 and is_reg:
            # Solver.cpp:1086-1101: overwrite k != 0 in the spectral direction with the 3-spectral kernel
            kf = [0.0] * 3
            for ip in range(3):
                kf[pg[ip].dim] = pg[ip].kfact
            sl = [slice(None)] * 3
            for d in range(3):
                if is_spec[d]:
                    sl[d] = slice(1, None)
            shp = data.shape
            idx = [self._symid(np.arange(shp[d]), symstart[d]) for d in range(3)]
            J0, J1, J2 = np.meshgrid(idx[0], idx[1], idx[2], indexing="ij")
            J = [J0, J1, J2]
            KK = [(J[d] + koffset[d]) * kf[d] for d in range(3)]
            ksq = KK[0] ** 2 + KK[1] ** 2 + KK[2] ** 2
            g3 = gk.green_0unb3spe(kind, ksq, KK[ax[0]], KK[ax[1]], KK[ax[2]], h[0], length)
            data = data.copy()
            data[tuple(sl)] = g3[tuple(sl)]
            if sum(koffset) < 0.2:  # green_functions.cpp:702-706, also run for the completion
                data[0, 0, 0] = 0.0 if not np.iscomplexobj(data) else complex(0.0, data[0, 0, 0].imag)
        return data

    def _green_spec_size(self):
        size = list(self.nglob)
        cplx = False
        for ip in range(self.ndim):
            p = self.plan_green[ip]
            size[p.dim] = p.n_out
            cplx = cplx or p.isr2c
        self._green_spec_complex = cplx
        return size

    # ------------------------------------------------------------ solve
    def do_fft(self, data, sign):
        """Solver.cpp:1402-1462 on (lda, n0, n1, n2) arrays."""
        if sign == FORWARD:
            for ip in range(self.ndim):
                p = self.plan_fwd[ip]
                data = self._switch_in(data, p)
                data = self._apply(p, data)
            return data
        plans = self.plan_bwd if sign == BACKWARD else self.plan_diff
        for ip in range(self.ndim - 1, -1, -1):
            p = plans[ip]
            data = self._apply(p, data)
            data = self._switch_out(data, self.plan_fwd[ip], self.sizes_before[ip][self.plan_fwd[ip].dim])
        return data

    @staticmethod
    def _switch_in(data, p):
        ax = 1 + p.dim
        n_prev = data.shape[ax]
        shape = list(data.shape)
        if p.isr2c:
            shape[ax] = 2 * p.n_out
        else:
            shape[ax] = p.n_out
        out = np.zeros(shape, dtype=data.dtype)
        sl = [slice(None)] * 4
        sl[ax] = slice(p.fieldstart, p.fieldstart + n_prev)
        out[tuple(sl)] = data
        return out

    @staticmethod
    def _switch_out(data, pf, n_prev):
        ax = 1 + pf.dim
        sl = [slice(None)] * 4
        sl[ax] = slice(pf.fieldstart, pf.fieldstart + n_prev)
        return np.ascontiguousarray(data[tuple(sl)])

    def _apply(self, p, data):
        if p.type == EMPTY:
            return data
        ax = 1 + p.dim
        comps = []
        for lia in range(self.lda):
            line = np.moveaxis(data[lia], ax - 1, -1)
            res = execute_plan(p, lia, line)
            res = postprocess_plan(p, lia, res)
            comps.append(np.moveaxis(res, -1, ax - 1))
        return np.stack(comps, axis=0)

    def do_mult(self, data, type_=STD):
        """Solver.cpp:1471-1542 with dothemagic_std/rot."""
        if type_ == STD:
            return data * (self.normfact * self.green)[None]
        kabs, koffset, symstart = self.spectral_info()
        kf = np.zeros((3, 3, 2))
        for ip in range(3):
            d = self.plan_fwd[ip].dim
            for lia in range(self.lda):
                ph = 0
                if self.plan_fwd[ip].imult[lia]:
                    ph -= 1
                if self.plan_diff[ip].imult[lia]:
                    ph += 1
                if ph == 0:
                    kf[d, lia] = (0.0, kabs[d])
                elif ph == 1:
                    kf[d, lia] = (-kabs[d], 0.0)
                else:
                    kf[d, lia] = (kabs[d], 0.0)
        shp = data.shape[1:]
        isym = [self._symid(np.arange(shp[d]), symstart[d]) for d in range(3)]
        I0, I1, I2 = np.meshgrid(isym[0], isym[1], isym[2], indexing="ij")
        I = [I0 + koffset[0], I1 + koffset[1], I2 + koffset[2]]
        h = self.h
        c43, c16, c32, c310, c130 = 4. / 3., 1. / 6., 3. / 2., 3. / 10., 1. / 30.

        def sym(d, f):
            # dothemagic_rot.ipp: spectral (o1) or finite-difference (o2/o4/o6) symbol of f = kfact
            if self.odiff == SPE:
                return I[d] * f
            a = I[d] * f * h[d]
            if self.odiff == FD2:
                return np.sin(a) / h[d]
            if self.odiff == FD4:
                return c43 * np.sin(a) / h[d] - c16 * np.sin(a * 2.0) / h[d]
            if self.odiff == FD6:
                return c32 * np.sin(a) / h[d] - c310 * np.sin(a * 2.0) / h[d] + c130 * np.sin(a * 3.0) / h[d]
            raise ValueError("The differenciation order asked does not exist")

        G = self.green
        nf = self.normfact
        if not np.iscomplexobj(data):
            # real spectral data (dothemagic_rot.ipp KIND 01..06): the symbol is of (re + im) of kfact
            def kr(d, c):
                return sym(d, kf[d, c, 0] + kf[d, c, 1])
            f0, f1, f2 = data[0], data[1], data[2]
            rot0 = f2 * kr(1, 2) - f1 * kr(2, 1)
            rot1 = f0 * kr(2, 0) - f2 * kr(0, 2)
            rot2 = f1 * kr(0, 1) - f0 * kr(1, 0)
            return np.stack([nf * rot0 * G, nf * rot1 * G, nf * rot2 * G])

        def kc(d, c):
            return sym(d, kf[d, c, 0]) + 1j * sym(d, kf[d, c, 1])
        f0, f1, f2 = data[0], data[1], data[2]
        rot0 = f2 * kc(1, 2) - f1 * kc(2, 1)
        rot1 = f0 * kc(2, 0) - f2 * kc(0, 2)
        rot2 = f1 * kc(0, 1) - f0 * kc(1, 0)
        return np.stack([nf * (rot0 * G), nf * (rot1 * G), nf * (rot2 * G)])

    def solve(self, rhs, type_=STD):
        """Solver.cpp:1207-1272: rhs (lda, n0, n1, n2) real -> field of the same shape."""
        if type_ == ROT and self.lda != 3:
            raise ValueError("You need vectors when using the ROT solver")
        if type_ == ROT and self.odiff not in (SPE, FD2, FD4, FD6):
            raise ValueError("ROT solve needs orderDiff in SPE/FD2/FD4/FD6")
        if self.green is None:
            self.setup()
        data = np.asarray(rhs, dtype=np.float64).reshape((self.lda,) + tuple(self.nglob))
        data = self.do_fft(data, FORWARD)
        data = self.do_mult(data, type_)
        data = self.do_fft(data, BACKWARD if type_ == STD else BACKWARD_DIFF)
        return np.ascontiguousarray(data.real if np.iscomplexobj(data) else data)
