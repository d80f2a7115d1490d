"""Per-direction transform tables: a restatement of FFTW_plan_dim (ctor and
init) and of its cell/node specialisations.

Reference: src/FFTW_plan_dim.cpp:77-161 (ctor: type, volfact, kfact,
isSpectral), src/FFTW_plan_dim.cpp:35-51 (sort_plans),
src/FFTW_plan_dim_cell.cpp:19-390 and src/FFTW_plan_dim_node.cpp:19-461 (init
tables: n_in, n_out, fieldstart, fftwstart_in/out, kind, koffset, symstart,
normfact, imult, postprocessing).
"""
import math

__all__ = [
    "EVEN", "ODD", "PER", "UNB", "NONE",
    "SYMSYM", "MIXUNB", "PERPER", "UNBUNB", "EMPTY",
    "NULL_FIRST", "NULL_LAST", "ENFORCE_PERIOD",
    "REDFT00", "REDFT01", "REDFT10", "REDFT11", "RODFT00", "RODFT01", "RODFT10", "RODFT11",
    "FORWARD", "BACKWARD", "BACKWARD_DIFF", "NODE_CENTER", "CELL_CENTER",
    "CHAT_2", "LGF_2", "HEJ_2", "HEJ_4", "HEJ_6", "HEJ_8", "HEJ_10", "HEJ_0",
    "LGF_4", "LGF_6", "LGF_8", "MEHR_4L", "MEHR_6L", "MEHR_4F", "MEHR_6F",
    "STD", "ROT", "NOD", "SPE", "FD2", "FD4", "FD6",
    "Plan", "sort_plans", "bc_to_type",
]

# flups_interface.h:46-110
EVEN, ODD, PER, UNB, NONE = 0, 1, 3, 4, 9
CHAT_2, LGF_2, HEJ_2, HEJ_4, HEJ_6, HEJ_8, HEJ_10, HEJ_0 = 0, 1, 2, 3, 4, 5, 6, 7
LGF_4, LGF_6, LGF_8, MEHR_4L, MEHR_6L, MEHR_4F, MEHR_6F = 8, 9, 10, 11, 12, 13, 14
STD, ROT = 0, 1
NOD, SPE, FD2, FD4, FD6 = 0, 1, 2, 4, 6
NODE_CENTER, CELL_CENTER = 0, 1
FORWARD, BACKWARD, BACKWARD_DIFF = -1, 1, 2

# FFTW_plan_dim.hpp:34-40 and :57-62
SYMSYM, MIXUNB, PERPER, UNBUNB, EMPTY = 2, 5, 6, 8, 18
NULL_FIRST, NULL_LAST, ENFORCE_PERIOD = 1, 2, 4

# FFTW r2r kinds, as (family, type): scipy.fft.dct/dst of that type
REDFT00, REDFT10, REDFT01, REDFT11 = ("dct", 1), ("dct", 2), ("dct", 3), ("dct", 4)
RODFT00, RODFT10, RODFT01, RODFT11 = ("dst", 1), ("dst", 2), ("dst", 3), ("dst", 4)


def bc_to_type(bcl, bcr):
    """FFTW_plan_dim.cpp:59-65: the plan type is the sum of both BCs of component 0."""
    return bcl + bcr


class Plan:
    """One direction's transform (FFTW_plan_dim.hpp:74-102 members)."""

    def __init__(self, lda, dim, h, L, bc, sign, is_green, center):
        # FFTW_plan_dim.cpp:77-161
        self.lda = lda
        self.dim = dim
        self.sign = sign
        self.is_green = is_green
        self.center = center
        self.bc = [list(bc[0][:lda]), list(bc[1][:lda])]
        t = self.bc[0][0] + self.bc[1][0]
        self.is_spectral = False
        if t <= SYMSYM:
            self.type, self.volfact, self.kfact = SYMSYM, 1.0, 2.0 * math.pi / (2.0 * L[dim])
            self.is_spectral = bool(is_green)
        elif t <= MIXUNB:
            self.type, self.volfact, self.kfact = MIXUNB, h[dim], 2.0 * math.pi / (4.0 * L[dim])
        elif t == PERPER:
            self.type, self.volfact, self.kfact = PERPER, 1.0, 2.0 * math.pi / L[dim]
            self.is_spectral = bool(is_green)
        elif t == UNBUNB:
            self.type, self.volfact, self.kfact = UNBUNB, h[dim], 2.0 * math.pi / (2.0 * L[dim])
        elif t == EMPTY:
            self.type, self.volfact, self.kfact = EMPTY, 1.0, 0.0
        else:
            raise ValueError("Invalid combination of BCs")
        for lia in range(lda):
            if self.bc[0][lia] + self.bc[1][lia] > self.type:
                raise ValueError("component bc not compatible with the plan type")
        self.n_in = [1] * lda
        self.fftwstart_in = [0] * lda
        self.fftwstart_out = [0] * lda
        self.postpro = [0] * lda
        self.imult = [False] * lda
        self.kind = [None] * lda
        self.normfact = 1.0
        self.n_out = 1
        self.fieldstart = 0
        self.symstart = 0.0
        self.koffset = 0.0
        self.isr2c = False

    # FFTW_plan_dim.hpp:96-99
    @property
    def isr2c_done_by_fft(self):
        return self.isr2c and not self.is_spectral

    def init(self, size, is_complex):
        """FFTW_plan_dim.cpp:183-209 dispatch to the centring-specific tables."""
        n = size[self.dim]
        cell = self.center == CELL_CENTER
        if self.type == SYMSYM:
            (self._r2r_cell if cell else self._r2r_node)(n, is_complex)
        elif self.type == MIXUNB:
            (self._mix_cell if cell else self._mix_node)(n, is_complex)
        elif self.type == PERPER:
            (self._per_cell if cell else self._per_node)(n, is_complex)
        elif self.type == UNBUNB:
            (self._unb_cell if cell else self._unb_node)(n, is_complex)

    # ------------------------------------------------------------------ cell
    def _r2r_cell(self, n, is_complex):
        # FFTW_plan_dim_cell.cpp:19-184
        assert not is_complex
        self.symstart, self.fieldstart, self.isr2c = 0.0, 0, False
        self.normfact *= 1.0 / (2.0 * n)
        for lia in range(self.lda):
            l, r = self.bc[0][lia], self.bc[1][lia]
            if self.is_green:
                self.postpro[lia], self.fftwstart_in[lia], self.fftwstart_out[lia] = 0, 0, 0
                self.imult[lia] = False
                if l != r:
                    self.n_in[lia], self.n_out, self.koffset = n, n, 0.5
                else:
                    self.n_in[lia], self.n_out, self.koffset = n, n + 1, 0.0
                return
            self.n_in[lia] = n
            if l == EVEN:
                self.imult[lia] = False
                if r == EVEN:
                    self.n_out, self.koffset = n + 1, 0.0
                    if self.sign == FORWARD:
                        self.kind[lia], self.postpro[lia] = REDFT10, NULL_LAST
                    else:
                        self.kind[lia], self.postpro[lia] = REDFT01, 0
                elif r == ODD:
                    self.n_out, self.koffset = n, 0.5
                    self.kind[lia], self.postpro[lia] = REDFT11, 0
                else:
                    raise ValueError("unable to init the solver required")
            elif l == ODD:
                self.imult[lia] = True
                if r == ODD:
                    self.n_out, self.koffset = n + 1, 0.0
                    if self.sign == FORWARD:
                        self.kind[lia], self.fftwstart_in[lia], self.fftwstart_out[lia] = RODFT10, 0, 1
                        self.postpro[lia] = NULL_FIRST
                    else:
                        self.kind[lia], self.fftwstart_in[lia], self.fftwstart_out[lia] = RODFT01, 1, 0
                        self.postpro[lia] = NULL_LAST
                elif r == EVEN:
                    self.n_out, self.koffset = n, 0.5
                    self.kind[lia], self.postpro[lia] = RODFT11, 0
                else:
                    raise ValueError("unable to init the solver required")
            else:
                raise ValueError("unable to init the solver required")

    def _mix_cell(self, n, is_complex):
        # FFTW_plan_dim_cell.cpp:195-290
        assert not is_complex
        self.isr2c = False
        if self.is_green:
            self.fieldstart = 0
        elif self.bc[0][0] == UNB:
            self.fieldstart = n
        elif self.bc[1][0] == UNB:
            self.fieldstart = 0
        self.symstart = 0.0
        self.normfact *= 1.0 / (4.0 * n)
        for lia in range(self.lda):
            l, r = self.bc[0][lia], self.bc[1][lia]
            if self.is_green:
                self.n_in[lia], self.n_out, self.koffset = 2 * n + 1, 2 * n + 1, 0.0
                self.fftwstart_in[lia] = self.fftwstart_out[lia] = 0
                self.postpro[lia], self.imult[lia], self.kind[lia] = 0, False, REDFT00
                continue
            self.n_in[lia], self.n_out, self.koffset = 2 * n, 2 * n + 1, 0.0
            if (l == EVEN and r == UNB) or (l == UNB and r == EVEN):
                self.imult[lia] = False
                self.fftwstart_in[lia] = self.fftwstart_out[lia] = 0
                if self.sign == FORWARD:
                    self.kind[lia], self.postpro[lia] = REDFT10, NULL_LAST
                else:
                    self.kind[lia], self.postpro[lia] = REDFT01, 0
            elif (l == UNB and r == ODD) or (l == ODD and r == UNB):
                self.imult[lia] = True
                if self.sign == FORWARD:
                    self.kind[lia], self.fftwstart_in[lia], self.fftwstart_out[lia] = RODFT10, 0, 1
                    self.postpro[lia] = NULL_FIRST
                else:
                    self.kind[lia], self.fftwstart_in[lia], self.fftwstart_out[lia] = RODFT01, 1, 0
                    self.postpro[lia] = NULL_LAST
            else:
                raise ValueError("unable to init the solver required")

    def _per_cell(self, n, is_complex):
        # FFTW_plan_dim_cell.cpp:301-343 (only n_in[0] is set: DFT plans use it alone)
        if is_complex:
            self.n_in[0], self.n_out, self.isr2c = n, n, False
        else:
            self.n_in[0], self.n_out, self.isr2c = n, n // 2 + 1, True
        self.fieldstart = 0
        self.symstart = n / 2.0 if is_complex else 0.0
        self.normfact *= 1.0 / n
        for lia in range(self.lda):
            self.postpro[lia] = 0
            self.fftwstart_in[lia] = self.fftwstart_out[lia] = 0
            self.imult[lia] = False

    def _unb_cell(self, n, is_complex):
        # FFTW_plan_dim_cell.cpp:354-390
        if is_complex:
            self.n_in[0], self.n_out, self.isr2c = 2 * n, 2 * n, False
        else:
            self.n_in[0], self.n_out, self.isr2c = 2 * n, n + 1, True
        self.fieldstart = 0
        self.symstart = float(n)
        self.normfact *= 1.0 / (2.0 * n)
        for lia in range(self.lda):
            self.fftwstart_in[lia] = self.fftwstart_out[lia] = 0
            self.postpro[lia], self.imult[lia] = 0, False

    # ------------------------------------------------------------------ node
    def _r2r_node(self, n, is_complex):
        # FFTW_plan_dim_node.cpp:19-216
        assert not is_complex
        self.symstart, self.fieldstart, self.isr2c = 0.0, 0, False
        self.normfact *= 1.0 / (2.0 * (n - 1))
        for lia in range(self.lda):
            l, r = self.bc[0][lia], self.bc[1][lia]
            if self.is_green:
                self.postpro[lia], self.fftwstart_in[lia], self.fftwstart_out[lia] = 0, 0, 0
                self.imult[lia] = False
                if l == EVEN and r == EVEN:
                    self.n_in[lia], self.n_out, self.koffset = n, n, 0.0
                elif l == EVEN and r == ODD:
                    self.n_in[lia], self.n_out, self.koffset = n - 1, n, 0.5
                elif l == ODD and r == ODD:
                    self.n_in[lia], self.n_out, self.koffset = n - 2, n, 0.0
                elif l == ODD and r == EVEN:
                    self.n_in[lia], self.n_out, self.koffset = n - 1, n, 0.5
                return
            if l == EVEN:
                self.imult[lia] = False
                if r == EVEN:
                    self.n_in[lia], self.n_out = n, n
                    self.postpro[lia], self.koffset, self.kind[lia] = 0, 0.0, REDFT00
                elif r == ODD:
                    self.n_in[lia], self.n_out, self.koffset = n - 1, n, 0.5
                    if self.sign == FORWARD:
                        self.kind[lia], self.postpro[lia] = REDFT01, NULL_LAST
                    else:
                        self.kind[lia], self.postpro[lia] = REDFT10, NULL_LAST
                else:
                    raise ValueError("unable to init the solver required")
            elif l == ODD:
                self.imult[lia] = True
                if r == ODD:
                    self.n_in[lia], self.n_out, self.koffset = n - 2, n, 0.0
                    self.fieldstart = 0
                    self.kind[lia] = RODFT00
                    self.fftwstart_in[lia] = self.fftwstart_out[lia] = 1
                    self.postpro[lia] = NULL_FIRST + NULL_LAST
                elif r == EVEN:
                    self.n_in[lia], self.n_out, self.koffset = n - 1, n, 0.5
                    self.fieldstart = 0
                    if self.sign == FORWARD:
                        self.kind[lia], self.fftwstart_in[lia], self.fftwstart_out[lia] = RODFT01, 1, 0
                        self.postpro[lia] = NULL_LAST
                    else:
                        self.kind[lia], self.fftwstart_in[lia], self.fftwstart_out[lia] = RODFT10, 0, 1
                        self.postpro[lia] = NULL_FIRST
                else:
                    raise ValueError("unable to init the solver required")
            else:
                raise ValueError("unable to init the solver required")

    def _mix_node(self, n, is_complex):
        # FFTW_plan_dim_node.cpp:227-334
        assert not is_complex
        self.isr2c = False
        if self.is_green:
            self.fieldstart = 0
        elif self.bc[0][0] == UNB:
            self.fieldstart = n - 1
        elif self.bc[1][0] == UNB:
            self.fieldstart = 0
        self.symstart = 0.0
        self.normfact *= 1.0 / (2.0 * ((2 * n - 1) - 1.0))
        for lia in range(self.lda):
            l, r = self.bc[0][lia], self.bc[1][lia]
            eu = (l == EVEN and r == UNB) or (l == UNB and r == EVEN)
            ou = (l == UNB and r == ODD) or (l == ODD and r == UNB)
            if self.is_green:
                if eu or ou:
                    self.n_in[lia] = 2 * n - 1
                    self.n_out = self.n_in[lia]
                    self.koffset = 0.0
                self.fftwstart_in[lia] = self.fftwstart_out[lia] = 0
                self.postpro[lia], self.imult[lia], self.kind[lia] = 0, False, REDFT00
                continue
            if eu:
                self.n_in[lia] = 2 * n - 1
                self.n_out, self.koffset = self.n_in[lia], 0.0
                self.fftwstart_in[lia] = self.fftwstart_out[lia] = 0
                self.postpro[lia], self.imult[lia], self.kind[lia] = 0, False, REDFT00
            elif ou:
                self.n_in[lia] = (2 * n - 1) - 2
                self.n_out, self.koffset = self.n_in[lia] + 2, 0.0
                self.imult[lia] = True
                self.kind[lia] = RODFT00
                self.fftwstart_in[lia] = self.fftwstart_out[lia] = 1
                self.postpro[lia] = NULL_FIRST + NULL_LAST
            else:
                raise ValueError("unable to init the solver required")

    def _per_node(self, n, is_complex):
        # FFTW_plan_dim_node.cpp:345-398
        for lia in range(self.lda):
            self.n_in[lia] = n - 1
        if is_complex:
            self.n_out, self.isr2c = n, False
        else:
            self.n_out, self.isr2c = self.n_in[0] // 2 + 1 + 1, True
        self.fieldstart = 0
        self.symstart = (n - 1) / 2.0 if is_complex else 0.0
        self.normfact *= 1.0 / (n - 1)
        for lia in range(self.lda):
            self.postpro[lia] = ENFORCE_PERIOD
            self.fftwstart_in[lia] = self.fftwstart_out[lia] = 0
            self.imult[lia] = False

    def _unb_node(self, n, is_complex):
        # FFTW_plan_dim_node.cpp:410-461
        if is_complex:
            self.n_in[0], self.n_out, self.isr2c = 2 * (n - 1), 2 * (n - 1), False
        else:
            self.n_in[0], self.n_out, self.isr2c = 2 * (n - 1), (2 * (n - 1)) // 2 + 1, True
        self.fieldstart = 0
        self.symstart = float(n - 1)
        self.normfact *= 1.0 / (2.0 * (n - 1))
        for lia in range(self.lda):
            self.postpro[lia] = 0
            self.fftwstart_in[lia] = self.fftwstart_out[lia] = 0
            self.imult[lia] = False


def sort_plans(plans):
    """FFTW_plan_dim.cpp:35-51: stable sort of the three directions by plan type."""
    order = sorted(range(3), key=lambda i: plans[i].type)  # Python's sort is stable
    return [plans[i] for i in order]
