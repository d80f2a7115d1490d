"""The reference's own solver, built from its sources (oracle/build_ref.py,
oracle/ref_build/), checked in three steps before it is trusted as a checker
or a CPU baseline:

1. the FFTW stand-in it runs on (oracle/ref_build/fft_shim.cpp) against
   scipy.fft for every transform kind FLUPS plans (c2c both signs, r2c,
   c2r, DCT/DST I-IV), lengths with radices 2/3/4/5/7 and Bluestein primes;
2. the reference build against the reference's golden error norms
   (samples/validation/data_ref, samples/solve_vtube/data_ref) with the
   reference's own rule (samples/validation/scripts/check_res.py:9-44);
3. the oracle restatement (oracle/solver.py) against the reference build on
   whole solution fields, including cases no golden covers (the 1-unbounded
   LGF_4/6/8 and MEHR kernels, finite-difference ROT orders).

CPU only; skipped where the reference tree or g++ is absent.
"""
import ctypes
import json
import re
from pathlib import Path

import numpy as np
import pytest
import scipy.fft as sfft

from oracle import build_ref
from oracle.plans import CELL_CENTER, NODE_CENTER, EVEN, ODD, PER, UNB, SPE, FD2, FD4, ROT
from oracle.solver import OracleSolver
from oracle.validation import error_norms, make_case, rhs_and_solution
from oracle.vtube import tube_case, tube_fields

REF = build_ref.DEFAULT_REF
pytestmark = pytest.mark.skipif(not (REF / "src").is_dir(), reason="reference sources absent")

GOLD = json.loads((Path(__file__).parent / "golden" / "validation_ref.json").read_text())
TOL = 1e-10


@pytest.fixture(scope="module")
def ref():
    build_ref.build_flups()
    from oracle import ref_lib
    return ref_lib


@pytest.fixture(scope="module")
def shim():
    lib = ctypes.CDLL(str(build_ref.build_fftshim()))
    P = ctypes.c_void_p
    dp = ctypes.POINTER(ctypes.c_double)
    lib.fftw_plan_dft_1d.restype = P
    lib.fftw_plan_dft_1d.argtypes = [ctypes.c_int, dp, dp, ctypes.c_int, ctypes.c_uint]
    lib.fftw_plan_dft_r2c_1d.restype = P
    lib.fftw_plan_dft_r2c_1d.argtypes = [ctypes.c_int, dp, dp, ctypes.c_uint]
    lib.fftw_plan_dft_c2r_1d.restype = P
    lib.fftw_plan_dft_c2r_1d.argtypes = [ctypes.c_int, dp, dp, ctypes.c_uint]
    lib.fftw_plan_r2r_1d.restype = P
    lib.fftw_plan_r2r_1d.argtypes = [ctypes.c_int, dp, dp, ctypes.c_int, ctypes.c_uint]
    lib.fftw_execute.argtypes = [P]
    lib.fftw_destroy_plan.argtypes = [P]
    return lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


LENGTHS = [1, 2, 3, 4, 5, 6, 7, 8, 9, 12, 14, 15, 16, 17, 20, 25, 30, 32, 34, 38, 48, 64, 96, 100, 128, 768]


@pytest.mark.parametrize("n", LENGTHS)
def test_shim_dft(shim, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    for sign in (-1, 1):
        a = np.ascontiguousarray(x.view(np.float64).copy())
        out = np.zeros_like(a)
        p = shim.fftw_plan_dft_1d(n, _ptr(a), _ptr(out), sign, 0)
        shim.fftw_execute(p)
        shim.fftw_destroy_plan(p)
        want = sfft.fft(x) if sign == -1 else sfft.ifft(x) * n
        assert _rel(out.view(np.complex128), want) < 1e-13, (n, sign)


@pytest.mark.parametrize("n", [v for v in LENGTHS if v > 1])
def test_shim_r2c_c2r(shim, n):
    rng = np.random.default_rng(100 + n)
    x = rng.standard_normal(n)
    out = np.zeros(2 * (n // 2 + 1))
    p = shim.fftw_plan_dft_r2c_1d(n, _ptr(x), _ptr(out), 0)
    shim.fftw_execute(p)
    shim.fftw_destroy_plan(p)
    X = sfft.rfft(x)
    assert _rel(out.view(np.complex128), X) < 1e-13
    back = np.zeros(n)
    inp = np.ascontiguousarray(X.view(np.float64).copy())
    p = shim.fftw_plan_dft_c2r_1d(n, _ptr(inp), _ptr(back), 0)
    shim.fftw_execute(p)
    shim.fftw_destroy_plan(p)
    assert _rel(back, sfft.irfft(X, n) * n) < 1e-13


# FFTW r2r kinds (fftw3.h) and their scipy.fft counterparts (unnormalised)
R2R = {3: ("dct", 1), 5: ("dct", 2), 4: ("dct", 3), 6: ("dct", 4), 7: ("dst", 1), 9: ("dst", 2), 8: ("dst", 3), 10: ("dst", 4)}


@pytest.mark.parametrize("kind", sorted(R2R))
def test_shim_r2r(shim, kind):
    fn, t = R2R[kind]
    for n in LENGTHS:
        if kind == 3 and n < 2:
            continue
        x = np.random.default_rng(kind * 1000 + n).standard_normal(n)
        out = np.zeros(n)
        p = shim.fftw_plan_r2r_1d(n, _ptr(x), _ptr(out), kind, 0)
        shim.fftw_execute(p)
        shim.fftw_destroy_plan(p)
        want = getattr(sfft, fn)(x, type=t)
        assert _rel(out, want) < 1e-12, (fn, t, n)


_PAT = re.compile(r"validation_3d_(CellCenter|NodeCenter)_(\d{6})_typeGreen=(\d+)\.txt")


def _close(gold, mine):
    if gold < 1e-14:
        return abs(gold - mine) < TOL
    return abs(gold - mine) / gold < TOL


@pytest.mark.parametrize("centre", ["CellCenter", "NodeCenter"])
def test_ref_build_validation_goldens(ref, centre):
    """The reference build reproduces every validation golden of one centring."""
    bad, n = [], 0
    for fn in sorted(GOLD["validation"]):
        m = _PAT.match(fn)
        if m.group(1) != centre:
            continue
        code, kernel = m.group(2), int(m.group(3))
        center = CELL_CENTER if centre == "CellCenter" else NODE_CENTER
        bc = [[int(code[0]), int(code[1])], [int(code[2]), int(code[3])], [int(code[4]), int(code[5])]]
        for row in GOLD["validation"][fn]:
            ng = int(row[0])
            r0 = ng - (0 if center == CELL_CENTER else 1)
            res = (r0, r0, 1 if code[4:] == "99" else r0)
            nglob, h, bcv = make_case(center, res, bc)
            rhs, sol = rhs_and_solution(center, nglob, h, (1.0, 1.0, 1.0), bcv, 1)
            s = ref.RefSolver(nglob, 1, bcv, h, (1.0, 1.0, 1.0), center, kernel)
            errs = error_norms(s.solve(rhs), sol, h, bcv)
            s.close()
            n += 1
            if not (_close(row[1], errs[0][0]) and _close(row[2], errs[0][1])):
                bad.append((fn, ng, row[1:3], errs[0]))
    assert n > 1000
    assert not bad, bad[:5]


def test_ref_build_vtube_goldens(ref):
    pat = re.compile(r"vtube_CellCenter_0_(\d)(-?\d)(-?\d)_typeGreen=0\.txt")
    n = 0
    for fn, rows in GOLD["vtube"].items():
        m = pat.match(fn)
        vdir, sx, sy = int(m.group(1)), int(m.group(2)), int(m.group(3))
        nglob, L = [16] * 3, (1.0, 1.0, 1.0)
        h = [1.0 / 16] * 3
        bcv, xc, yc, xs, ys = tube_case(vdir, sx, sy)
        rhs, sol = tube_fields(vdir, nglob, h, L, xc, yc, xs, ys, 0.1)
        s = ref.RefSolver(nglob, 3, bcv, h, L, CELL_CENTER, 0, odiff=SPE)
        errs = error_norms(s.solve(rhs, ROT), sol, h, bcv)
        s.close()
        for row in rows:
            for c in range(3):
                assert _close(row[1 + 2 * c], errs[c][0]), (fn, c)
                assert _close(row[2 + 2 * c], errs[c][1]), (fn, c)
                n += 1
    assert n == 81


# whole fields, oracle against the reference build: (grid, lda, bc per direction, centre, kernel, type, diff order)
FIELD_CASES = [
    ([16, 12, 20], 1, [[UNB, UNB], [UNB, UNB], [UNB, UNB]], CELL_CENTER, 1, 0, 0),
    ([17, 9, 13], 1, [[EVEN, ODD], [PER, PER], [UNB, UNB]], NODE_CENTER, 3, 0, 0),
    ([16, 16, 16], 1, [[PER, PER], [PER, PER], [UNB, UNB]], CELL_CENTER, 8, 0, 0),   # LGF_4, 1 unbounded
    ([16, 16, 16], 1, [[EVEN, ODD], [PER, PER], [UNB, UNB]], CELL_CENTER, 9, 0, 0),   # LGF_6
    ([16, 16, 16], 1, [[PER, PER], [EVEN, EVEN], [UNB, UNB]], CELL_CENTER, 10, 0, 0),  # LGF_8
    ([16, 16, 16], 1, [[PER, PER], [PER, PER], [UNB, UNB]], CELL_CENTER, 11, 0, 0),  # MEHR_4L
    ([16, 16, 16], 1, [[PER, PER], [PER, PER], [UNB, UNB]], CELL_CENTER, 12, 0, 0),  # MEHR_6L
    ([16, 16, 16], 1, [[PER, PER], [PER, PER], [UNB, UNB]], CELL_CENTER, 13, 0, 0),  # MEHR_4F
    ([16, 16, 16], 1, [[PER, PER], [PER, PER], [UNB, UNB]], CELL_CENTER, 14, 0, 0),  # MEHR_6F
    ([16, 16, 16], 3, [[UNB, UNB], [UNB, UNB], [UNB, UNB]], CELL_CENTER, 8, ROT, SPE),
    ([16, 12, 8], 3, [[UNB, UNB], [PER, PER], [UNB, UNB]], CELL_CENTER, 0, ROT, FD2),
    ([16, 16, 16], 3, [[UNB, UNB], [UNB, UNB], [PER, PER]], CELL_CENTER, 2, ROT, FD4),
]


@pytest.mark.parametrize("case", range(len(FIELD_CASES)))
def test_oracle_matches_ref_build(ref, case):
    nglob, lda, bc, center, kernel, typ, odiff = FIELD_CASES[case]
    fact = 0 if center == CELL_CENTER else 1
    hh = 1.0 / (nglob[0] - fact)  # the regularised and lattice kernels want one spacing
    h = [hh] * 3
    L = [hh * (nglob[d] - fact) for d in range(3)]
    bcv = [[[bc[d][s]] * lda for s in range(2)] for d in range(3)]
    rhs = np.random.default_rng(case).standard_normal((lda, *nglob))
    s = ref.RefSolver(nglob, lda, bcv, h, L, center, kernel, odiff=odiff)
    want = s.solve(rhs, typ)
    s.close()
    o = OracleSolver(nglob, lda, bcv, h, L, center, orderdiff=odiff)
    o.green_type = kernel
    o.setup()
    got = o.solve(rhs, typ)
    err = float(np.linalg.norm(got - want) / np.linalg.norm(want))
    assert err < 1e-12, err
