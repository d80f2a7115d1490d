"""Batched solves replayed from CUDA graphs, the CTA-tile autotuner and the
two compiled column tiles, the x-slab overlap and the L2 prefetch: none of
them changes the per-line arithmetic, so
each must reproduce the plain solve bit for bit (one right-hand side and a
batch, FP32 and FP64, lines of 64 to 512 points)."""
import numpy as np
import pytest

from gpu_helpers import make_solver, to_user
from oracle.plans import CELL_CENTER, HEJ_2, LGF_2

pytestmark = pytest.mark.gpu

UNB = [[[4], [4]]] * 3


def _setup(n, kernel, precision):
    h = [1.0 / n] * 3
    return make_solver([n] * 3, 1, UNB, h, [1.0] * 3, CELL_CENTER, kernel, precision=precision)


def _rhs(n, nb, seed):
    rng = np.random.default_rng(seed)
    return np.concatenate([to_user(rng.standard_normal((1, n, n, n))) for _ in range(nb)])


@pytest.mark.parametrize("n,precision", [(32, 32), (64, 64), (128, 32), (256, 32)])
def test_tiles_bitwise_equal(n, precision):
    import torch
    t, s = _setup(n, HEJ_2, precision)
    rhs = torch.from_numpy(_rhs(n, 1, 3)).cuda()
    outs = []
    for tile in (0, 1, 2):
        s.set_col_tile(tile)
        out = torch.zeros_like(rhs)
        s.solve(out, rhs)
        torch.cuda.synchronize()
        outs.append(out.cpu().numpy())
    assert s.last_error() == 0
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[0], outs[2])


@pytest.mark.parametrize("precision", [32, 64])
def test_graph_and_autotune_match_plain_batch(precision):
    import torch
    n, nb = 64, 4
    t, s = _setup(n, LGF_2, precision)
    rhs = torch.from_numpy(_rhs(n, nb, 4)).cuda()
    ref = torch.zeros_like(rhs)
    s.solve_batch(ref, rhs, nb)
    torch.cuda.synchronize()
    s.set_autotune(True)
    tuned = torch.zeros_like(rhs)
    s.solve_batch(tuned, rhs, nb)
    torch.cuda.synchronize()
    assert torch.equal(tuned, ref)
    out = torch.full_like(rhs, float("nan"))
    for _ in range(2):
        out.fill_(float("nan"))
        s.solve_graph(out, rhs, nb)
        torch.cuda.synchronize()
        assert torch.equal(out, ref)
    # the graph reads the arrays' current contents
    rhs2 = torch.from_numpy(_rhs(n, nb, 5)).cuda()
    ref2 = torch.zeros_like(rhs2)
    s.solve_batch(ref2, rhs2, nb)
    rhs.copy_(rhs2)
    s.solve_graph(out, rhs, nb)
    torch.cuda.synchronize()
    assert torch.equal(out, ref2)
    assert s.last_error() == 0


@pytest.mark.parametrize("n,precision", [(64, 64), (128, 32), (200, 32)])
def test_overlapped_middle_passes_bitwise(n, precision):
    """The x-slab overlap of the y / fused z / y passes on three streams gives
    the plain solve's result in the same (reference) pass order bit for bit."""
    import torch
    t, s = _setup(n, LGF_2, precision)
    s.set_xlast(False)
    rhs = torch.from_numpy(_rhs(n, 1, 6)).cuda()
    ref = torch.zeros_like(rhs)
    s.solve(ref, rhs)
    torch.cuda.synchronize()
    s.set_overlap(True)
    out = torch.full_like(rhs, float("nan"))
    for _ in range(2):
        s.solve(out, rhs)
        torch.cuda.synchronize()
        assert torch.equal(out, ref)
    assert s.last_error() == 0


@pytest.mark.parametrize("n,precision,nb", [(256, 32, 1), (256, 64, 1), (128, 32, 8)])
def test_l2_prefetch_bitwise(n, precision, nb):
    """The TMA L2 prefetch of the next blocks' input (row and column passes
    whose input exceeds 64 MB) is a hint only: results with it on and off are
    identical, for one right-hand side and for a batch."""
    import torch
    t, s = _setup(n, LGF_2, precision)
    rhs = torch.from_numpy(_rhs(n, nb, 11)).cuda()
    s.set_prefetch(False)
    ref = torch.zeros_like(rhs)
    s.solve_batch(ref, rhs, nb) if nb > 1 else s.solve(ref, rhs)
    torch.cuda.synchronize()
    s.set_prefetch(True)
    out = torch.full_like(rhs, float("nan"))
    s.solve_batch(out, rhs, nb) if nb > 1 else s.solve(out, rhs)
    torch.cuda.synchronize()
    assert torch.equal(out, ref)
    assert s.last_error() == 0
