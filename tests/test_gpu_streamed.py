"""Host-array solves: the rhs upload and the field download run in slabs of
the last forward direction on the library's copy streams, overlapped with
the transforms of the other slabs.  The slab passes do the same per-line
arithmetic as whole-array passes, so a solve with host arrays must equal the
solve of the same data in device arrays in the same (reference) pass order
bit for bit: one call, async calls
back to back (each with its own input), a batch, an in-place call, a
vector ROT solve, and grids that run the general line pass instead of the
register DFTs."""
import numpy as np
import pytest

from gpu_helpers import make_solver, to_user
from oracle.plans import CELL_CENTER, NODE_CENTER, CHAT_2, HEJ_2, LGF_2

pytestmark = pytest.mark.gpu

UNB = [[[4], [4]]] * 3
CASES = [
    # (name, nglob, lda, bcv, center, kernel, precision)
    ("unb64_fast_fp64", [64] * 3, 1, UNB, CELL_CENTER, LGF_2, 64),
    ("unb64_fast_fp32", [64] * 3, 1, UNB, CELL_CENTER, HEJ_2, 32),
    ("unb_ragged_general", [24, 20, 18], 1, UNB, CELL_CENTER, CHAT_2, 64),
    ("mixed_bc_node", [17, 9, 9], 1, [[[0], [1]], [[3], [3]], [[4], [4]]], NODE_CENTER, CHAT_2, 64),
]


def _setup(nglob, lda, bcv, center, kernel, precision, odiff=0):
    fact = 0 if center == CELL_CENTER else 1
    h = [1.0 / (nglob[0] - fact)] * 3
    L = [h[d] * (nglob[d] - fact) for d in range(3)]
    t, s = make_solver(nglob, lda, bcv, h, L, center, kernel, odiff=odiff, precision=precision)
    # host arrays stream in the reference's pass order: device arrays in the same order
    s.set_xlast(False)
    return t, s


def _device_solve(s, u, type_=0, nbatch=1):
    import torch
    d_in = torch.from_numpy(u).cuda()
    d_out = torch.zeros_like(d_in)
    if nbatch == 1:
        s.solve(d_out, d_in, type_)
    else:
        s.solve_batch(d_out, d_in, nbatch, type_)
    torch.cuda.synchronize()
    return d_out.cpu().numpy()


@pytest.mark.parametrize("name,nglob,lda,bcv,center,kernel,precision", CASES, ids=[c[0] for c in CASES])
def test_host_equals_device(name, nglob, lda, bcv, center, kernel, precision):
    import torch
    t, s = _setup(nglob, lda, bcv, center, kernel, precision)
    rng = np.random.default_rng(5)
    u = to_user(rng.standard_normal((lda,) + tuple(nglob)))
    ref = _device_solve(s, u)
    out = np.full_like(u, np.nan)
    s.solve(out, u)
    assert s.last_error() == 0
    assert np.array_equal(out, ref)
    # pinned host arrays, async, three solves back to back with their own inputs
    us = [to_user(rng.standard_normal((lda,) + tuple(nglob))) for _ in range(3)]
    refs = [_device_solve(s, x) for x in us]
    h_in = [torch.from_numpy(x).pin_memory() for x in us]
    h_out = [torch.full_like(x, float("nan")).pin_memory() for x in h_in]
    s.set_async(True)
    for a, b in zip(h_out, h_in):
        s.solve(a, b)
    s.synchronize()
    s.set_async(False)
    for a, r in zip(h_out, refs):
        assert np.array_equal(a.numpy(), r)
    # in place: field and rhs are the same host array
    x = us[0].copy()
    s.solve(x, x)
    assert np.array_equal(x, refs[0])
    assert s.last_error() == 0


def test_host_batch_equals_device():
    t, s = _setup([32] * 3, 1, UNB, CELL_CENTER, LGF_2, 64)
    rng = np.random.default_rng(8)
    u = np.concatenate([to_user(rng.standard_normal((1, 32, 32, 32))) for _ in range(3)])
    ref = _device_solve(s, u, nbatch=3)
    out = np.zeros_like(u)
    s.solve_batch(out, u, 3)
    assert np.array_equal(out, ref)


def test_host_rot_equals_device():
    t, s = _setup([32] * 3, 3, [[[4, 4, 4], [4, 4, 4]]] * 3, CELL_CENTER, HEJ_2, 64, odiff=1)
    rng = np.random.default_rng(9)
    u = to_user(rng.standard_normal((3, 32, 32, 32)))
    ref = _device_solve(s, u, type_=1)
    out = np.zeros_like(u)
    s.solve(out, u, 1)
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("name,nglob,lda,bcv,center,kernel,precision", CASES[:3], ids=[c[0] for c in CASES[:3]])
def test_host_async_chain(name, nglob, lda, bcv, center, kernel, precision):
    """Async solves of pinned host arrays whose rhs is an earlier solve's field
    (in place, then field -> rhs), with device-array solves (plain and graph)
    queued between them on the same stream: after one synchronize every result
    equals the same chain run one device solve at a time."""
    import torch
    t, s = _setup(nglob, lda, bcv, center, kernel, precision)
    rng = np.random.default_rng(11)
    u0 = to_user(rng.standard_normal((lda,) + tuple(nglob)))
    ud = to_user(rng.standard_normal((lda,) + tuple(nglob)))
    r1 = _device_solve(s, u0)
    r2 = _device_solve(s, r1)
    r3 = _device_solve(s, r2)
    r4 = _device_solve(s, r3)
    rd = _device_solve(s, ud)
    h1 = torch.from_numpy(u0.copy()).pin_memory()
    h2 = torch.full_like(h1, float("nan")).pin_memory()
    h3 = torch.full_like(h1, float("nan")).pin_memory()
    d_in = torch.from_numpy(ud).cuda()
    d_out = torch.zeros_like(d_in)
    g_out = torch.zeros_like(d_in)
    s.solve_graph(g_out, d_in)      # first call: plain solve + capture
    torch.cuda.synchronize()
    g_out.zero_()
    s.set_async(True)
    s.solve(h1, h1)                 # h1 = S(u0), in place
    s.solve(h1, h1)                 # h1 = S(S(u0)), in place again
    s.solve(d_out, d_in)            # a device-array solve between them
    s.solve(h2, h1)                 # h2 = S^3(u0)
    s.solve_graph(g_out, d_in)      # a graph replay between them
    s.solve(h3, h2)                 # h3 = S^4(u0)
    s.synchronize()
    s.set_async(False)
    assert s.last_error() == 0
    assert np.array_equal(h1.numpy(), r2)
    assert np.array_equal(h2.numpy(), r3)
    assert np.array_equal(h3.numpy(), r4)
    assert np.array_equal(d_out.cpu().numpy(), rd)
    assert np.array_equal(g_out.cpu().numpy(), rd)
