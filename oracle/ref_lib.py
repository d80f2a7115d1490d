"""The reference's own solver, compiled from its sources by oracle/build_ref.py
into oracle/_ref/libflups_ref.so, behind a small Python class.

Test infrastructure of the oracle: the checker in tests/ and the CPU
baseline of bench.py, never the product.  Arrays are numpy FP64 in the
oracle's order (lda, n0, n1, n2) with the z index fastest; the driver
(oracle/ref_build/ref_driver.cpp) copies them into the reference's user
topology and calls flups_solve (src/flups.h:452).
"""
import ctypes
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parent / "_ref" / "libflups_ref.so"
_lib = None


def available():
    return LIB.exists()


def _load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            raise FileNotFoundError(f"{LIB} is missing: build it with `python -m oracle.build_ref`")
        lib = ctypes.CDLL(str(LIB))
        lib.flups_ref_new.restype = ctypes.c_void_p
        lib.flups_ref_new.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                      ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                      ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_double, ctypes.c_int]
        lib.flups_ref_solve.restype = ctypes.c_double
        lib.flups_ref_solve.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        lib.flups_ref_free.restype = None
        lib.flups_ref_free.argtypes = [ctypes.c_void_p]
        _lib = lib
    return _lib


def _ints(v):
    return (ctypes.c_int * len(v))(*[int(x) for x in v])


def _doubles(v):
    return (ctypes.c_double * len(v))(*[float(x) for x in v])


class RefSolver:
    """One reference solver: flups_topo_new + flups_init + flups_set_greenType
    (+ flups_set_alpha) + flups_setup on construction.

    bc[d][side][lia] as in the oracle; center: CELL_CENTER / NODE_CENTER for
    all directions; kernel: the reference's GreenType value; odiff: DiffType."""

    def __init__(self, nglob, lda, bc, h, L, center, kernel, alpha=2.0, odiff=0):
        self._lib = _load()
        self.nglob = [int(v) for v in nglob]
        self.lda = int(lda)
        flat = [bc[d][s][l] for d in range(3) for s in range(2) for l in range(self.lda)]
        self._h = self._lib.flups_ref_new(_ints(self.nglob), self.lda, _ints(flat), _doubles(h), _doubles(L),
                                          _ints([center] * 3), int(kernel), float(alpha), int(odiff))
        self.last_seconds = None

    def solve(self, rhs, type_=0):
        """rhs: (lda, n0, n1, n2) FP64; returns the field in the same order.
        last_seconds: the wall time of the flups_solve call itself."""
        dense = np.ascontiguousarray(np.asarray(rhs, dtype=np.float64).reshape((self.lda, *self.nglob)).transpose(0, 3, 2, 1))
        out = np.empty_like(dense)
        self.last_seconds = self._lib.flups_ref_solve(self._h, dense.ctypes.data, out.ctypes.data, int(type_))
        return np.ascontiguousarray(out.transpose(0, 3, 2, 1))

    def close(self):
        if self._h:
            self._lib.flups_ref_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
