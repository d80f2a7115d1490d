"""flups_solve_noalloc, the entry point for callers that cannot allocate
device memory while they run: real-time loops that must not wait on the
allocator (cudaMalloc can synchronise the device and takes driver locks),
and frameworks that reserve the device memory for their own pools at
start-up, after which a cudaMalloc fails.

Through the C ABI it must give the same field as flups_solve (within the
tolerance of the other tests: 1e-12 relative L2 in FP64, 2e-6 in FP32) on
two calls in a row, agree with the FP64 oracle to the same tolerance,
leave the device's free memory unchanged, and refuse a solve whose scratch
is above its 64 MiB limit.  This file is collected last so that a run that
stops at the first failure has run every other test before it; it also
passes alone in a fresh process (the first call on a device does the
array's address look-up itself)."""
import ctypes

import numpy as np
import pytest

from gpu_helpers import from_user, make_solver, oracle_solve, to_user
from oracle.plans import CELL_CENTER, NODE_CENTER, CHAT_2, HEJ_2, LGF_2

pytestmark = pytest.mark.gpu

STD, ROT = 0, 1


def _lib():
    from flups_b200 import pyflups as pf
    lib = pf.load_library()
    lib.flups_solve_noalloc.restype = ctypes.c_int
    lib.flups_solve_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    return lib


def _rhs(nglob, lda, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((lda,) + tuple(nglob))


UNB = [[[4], [4]]] * 3
UNB_V = [[[4] * 3, [4] * 3]] * 3

CASES = [
    # (name, nglob, lda, bcv, center, kernel, precision, tolerance, type, derivative order)
    ("unb64_fast_fp64", [64] * 3, 1, UNB, CELL_CENTER, LGF_2, 64, 1e-12, STD, 0),
    ("unb64_fast_fp32", [64] * 3, 1, UNB, CELL_CENTER, HEJ_2, 32, 2e-6, STD, 0),
    ("mixed_bc_general_fp64", [17, 9, 9], 1, [[[0], [1]], [[3], [3]], [[4], [4]]], NODE_CENTER, CHAT_2, 64, 1e-12,
     STD, 0),
    ("rot_unb32_fp64", [32] * 3, 3, UNB_V, CELL_CENTER, LGF_2, 64, 1e-12, ROT, 1),
    ("rot_unb64_fp32", [64] * 3, 3, UNB_V, CELL_CENTER, HEJ_2, 32, 2e-6, ROT, 2),
]


@pytest.mark.parametrize("name,nglob,lda,bcv,center,kernel,precision,tol,type_,odiff", CASES,
                         ids=[c[0] for c in CASES])
def test_noalloc_matches_solve_twice(name, nglob, lda, bcv, center, kernel, precision, tol, type_, odiff):
    import torch
    lib = _lib()
    fact = 0 if center == CELL_CENTER else 1
    h = [1.0 / (nglob[0] - fact)] * 3
    L = [h[d] * (nglob[d] - fact) for d in range(3)]
    t, s = make_solver(nglob, lda, bcv, h, L, center, kernel, odiff=odiff, precision=precision)
    stream = torch.cuda.current_stream()
    s.set_stream(stream)
    rhs_host = _rhs(nglob, lda, 11)
    rhs = torch.from_numpy(to_user(rhs_host)).cuda()
    ref = torch.zeros_like(rhs)
    s.solve(ref, rhs, type_)
    torch.cuda.synchronize()
    # the first call on a device looks up the scratch array (and loads its kernels): a set-up call
    outs = [torch.full_like(rhs, float("nan")) for _ in range(3)]
    assert lib.flups_solve_noalloc(s._solver, outs[0].data_ptr(), rhs.data_ptr(), type_) == 0
    torch.cuda.synchronize()
    free = [torch.cuda.mem_get_info()[0]]
    for out in outs[1:]:
        assert lib.flups_solve_noalloc(s._solver, out.data_ptr(), rhs.data_ptr(), type_) == 0
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
    # two calls in a row take no device memory
    assert free[0] == free[1] == free[2]
    den = float(torch.linalg.vector_norm(ref))
    for out in outs:
        assert torch.isfinite(out).all()
        assert float(torch.linalg.vector_norm(out - ref)) / den <= tol
    assert s.last_error() == 0
    # and the field is the oracle's (the reference's FP64 solve restated)
    want = oracle_solve(nglob, lda, bcv, h, L, center, kernel, rhs_host, type_=type_, odiff=odiff)
    got = from_user(outs[-1].cpu().numpy(), lda, nglob)
    assert np.linalg.norm(got - want) / np.linalg.norm(want) <= tol


def test_noalloc_refuses_oversized_and_host_pointers():
    import torch
    lib = _lib()
    n = 256  # FP64 work arrays of 256^3 all-unbounded need ~800 MiB, above the 64 MiB scratch
    t, s = make_solver([n] * 3, 1, UNB, [1.0 / n] * 3, [1.0] * 3, CELL_CENTER, CHAT_2)
    rhs = torch.zeros((n, n, n), dtype=torch.float64, device="cuda")
    out = torch.zeros_like(rhs)
    assert lib.flups_solve_noalloc(s._solver, out.data_ptr(), rhs.data_ptr(), STD) == -3
    host = np.zeros((n, n, n))
    assert lib.flups_solve_noalloc(s._solver, host.ctypes.data, host.ctypes.data, STD) == -2
    assert s.last_error() == 0
