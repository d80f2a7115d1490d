"""flups_b200_solve_group: the solves of several solvers with unevenly sized
grids (and different boundary conditions, kernels, precisions, solver types)
as one CUDA graph whose member solves are independent branches.  Each
member's field must equal the same solver's plain solve of the same device
arrays bit for bit (same kernels, same order), on the first call (which
captures) and on replays; a member whose work arrays grow in between gets
the group recaptured."""
import numpy as np
import pytest

from gpu_helpers import make_solver, to_user
from oracle.plans import CELL_CENTER, NODE_CENTER, CHAT_2, HEJ_2, LGF_2

pytestmark = pytest.mark.gpu

UNB = [[[4], [4]]] * 3

MEMBERS = [
    # (nglob, lda, bcv, center, kernel, precision, type, derivative order)
    ([32, 32, 32], 1, UNB, CELL_CENTER, HEJ_2, 32, 0, 0),
    ([48, 40, 36], 1, UNB, CELL_CENTER, LGF_2, 64, 0, 0),
    ([33, 17, 17], 1, [[[0], [1]], [[3], [3]], [[4], [4]]], NODE_CENTER, CHAT_2, 64, 0, 0),
    ([64, 64, 64], 3, [[[4] * 3, [4] * 3]] * 3, CELL_CENTER, LGF_2, 32, 1, 1),
    ([128, 96, 64], 1, UNB, CELL_CENTER, HEJ_2, 32, 0, 0),
]


def _member(nglob, lda, bcv, center, kernel, precision, typ, odiff):
    fact = 0 if center == CELL_CENTER else 1
    h = [1.0 / (nglob[0] - fact)] * 3
    L = [h[d] * (nglob[d] - fact) for d in range(3)]
    return make_solver(nglob, lda, bcv, h, L, center, kernel, odiff=odiff, precision=precision)


def test_group_graph_equals_member_solves():
    import torch
    from flups_b200 import pyflups as pf
    rng = np.random.default_rng(3)
    keep, solvers, rhss, refs, outs, types = [], [], [], [], [], []
    for (nglob, lda, bcv, center, kernel, precision, typ, odiff) in MEMBERS:
        t, s = _member(nglob, lda, bcv, center, kernel, precision, typ, odiff)
        keep.append(t)
        rhs = torch.from_numpy(to_user(rng.standard_normal((lda,) + tuple(nglob)))).cuda()
        ref = torch.zeros_like(rhs)
        s.solve(ref, rhs, typ)
        torch.cuda.synchronize()
        assert s.last_error() == 0
        solvers.append(s)
        rhss.append(rhs)
        refs.append(ref)
        outs.append(torch.full_like(rhs, float("nan")))
        types.append(typ)
    stream = torch.cuda.Stream()
    for rep in range(3):
        for o in outs:
            o.fill_(float("nan"))
        torch.cuda.synchronize()
        assert pf.solve_group(solvers, outs, rhss, types, stream=stream) == 0
        stream.synchronize()
        for i, (o, r) in enumerate(zip(outs, refs)):
            assert torch.equal(o, r), (rep, i)
        if rep == 1:
            # member 1's work arrays grow (a batch of two): its group is captured again
            s = solvers[1]
            two = torch.cat([rhss[1], rhss[1]])
            tout = torch.zeros_like(two)
            s.solve_batch(tout, two, 2)
            torch.cuda.synchronize()
    assert all(s.last_error() == 0 for s in solvers)


def test_group_refuses_host_arrays_and_repeats():
    import torch
    from flups_b200 import pyflups as pf
    t, s = _member([32, 32, 32], 1, UNB, CELL_CENTER, HEJ_2, 32, 0, 0)
    rhs = torch.zeros((32, 32, 32), dtype=torch.float64, device="cuda")
    out = torch.zeros_like(rhs)
    host = np.zeros((32, 32, 32))
    assert pf.solve_group([s], [host], [host]) == -2
    assert pf.solve_group([s, s], [out, torch.zeros_like(rhs)], [rhs, rhs]) == -2
    assert pf.solve_group([s], [out], [rhs]) == 0
    torch.cuda.synchronize()
    assert s.last_error() == 0
