"""flups_solve_noalloc, the entry point for callers that cannot allocate
device memory while they run (graph capture in the global mode, real-time
loops, frameworks owning the memory pools): through the C ABI it must give
the same field as flups_solve, on two calls in a row, without changing the
device's free memory, and must refuse a solve whose scratch is above its
64 MiB limit.  Collected last so that a stop at the first failure has run
every other test before it."""
import ctypes

import numpy as np
import pytest

from gpu_helpers import make_solver, to_user
from oracle.plans import CELL_CENTER, NODE_CENTER, CHAT_2, HEJ_2, LGF_2

pytestmark = pytest.mark.gpu


def _lib():
    from flups_b200 import pyflups as pf
    lib = pf.load_library()
    lib.flups_solve_noalloc.restype = ctypes.c_int
    lib.flups_solve_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    return lib


def _rhs(nglob, lda, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((lda,) + tuple(nglob))


CASES = [
    # (name, nglob, lda, bcv, center, kernel, precision, tolerance)
    ("unb64_fast_fp64", [64] * 3, 1, [[[4], [4]]] * 3, CELL_CENTER, LGF_2, 64, 1e-12),
    ("unb64_fast_fp32", [64] * 3, 1, [[[4], [4]]] * 3, CELL_CENTER, HEJ_2, 32, 2e-6),
    ("mixed_bc_general_fp64", [17, 9, 9], 1, [[[0], [1]], [[3], [3]], [[4], [4]]], NODE_CENTER, CHAT_2, 64, 1e-12),
]


@pytest.mark.parametrize("name,nglob,lda,bcv,center,kernel,precision,tol", CASES, ids=[c[0] for c in CASES])
def test_noalloc_matches_solve_twice(name, nglob, lda, bcv, center, kernel, precision, tol):
    import torch
    lib = _lib()
    fact = 0 if center == CELL_CENTER else 1
    h = [1.0 / (nglob[0] - fact)] * 3
    L = [h[d] * (nglob[d] - fact) for d in range(3)]
    t, s = make_solver(nglob, lda, bcv, h, L, center, kernel, precision=precision)
    stream = torch.cuda.current_stream()
    s.set_stream(stream)
    rhs = torch.from_numpy(to_user(_rhs(nglob, lda, 11))).cuda()
    ref = torch.zeros_like(rhs)
    s.solve(ref, rhs)
    torch.cuda.synchronize()
    # the first call on a device looks up the scratch array (and loads its kernels): a set-up call
    outs = [torch.full_like(rhs, float("nan")) for _ in range(3)]
    assert lib.flups_solve_noalloc(s._solver, outs[0].data_ptr(), rhs.data_ptr(), 0) == 0
    torch.cuda.synchronize()
    free = [torch.cuda.mem_get_info()[0]]
    for out in outs[1:]:
        assert lib.flups_solve_noalloc(s._solver, out.data_ptr(), rhs.data_ptr(), 0) == 0
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
    # two calls in a row take no device memory
    assert free[0] == free[1] == free[2]
    den = float(torch.linalg.vector_norm(ref))
    for out in outs:
        assert torch.isfinite(out).all()
        assert float(torch.linalg.vector_norm(out - ref)) / den <= tol
    assert s.last_error() == 0


def test_noalloc_refuses_oversized_and_host_pointers():
    import torch
    lib = _lib()
    n = 256  # FP64 work arrays of 256^3 all-unbounded need ~800 MiB, above the 64 MiB scratch
    t, s = make_solver([n] * 3, 1, [[[4], [4]]] * 3, [1.0 / n] * 3, [1.0] * 3, CELL_CENTER, CHAT_2)
    rhs = torch.zeros((n, n, n), dtype=torch.float64, device="cuda")
    out = torch.zeros_like(rhs)
    assert lib.flups_solve_noalloc(s._solver, out.data_ptr(), rhs.data_ptr(), 0) == -3
    host = np.zeros((n, n, n))
    assert lib.flups_solve_noalloc(s._solver, host.ctypes.data, host.ctypes.data, 0) == -2
    assert s.last_error() == 0
