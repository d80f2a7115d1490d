"""x and y passes of the all-unbounded FP32 pair as one 16-CTA cluster kernel
per direction (the x spectrum of a z plane kept in the cluster's distributed
shared memory): the same transforms as the separate x and y passes, checked
against them (device arrays, vectors, batches, host arrays through the
z-slab streamed solve) and against the FP64 mode at 512^3."""
import numpy as np
import pytest

from gpu_helpers import make_solver, to_user
from oracle.plans import CELL_CENTER, LGF_2

pytestmark = pytest.mark.gpu

UNB = [[[4], [4]]] * 3


def _setup(n, precision, lda=1):
    bcv = [[[4] * lda, [4] * lda]] * 3
    return make_solver([n] * 3, lda, bcv, [1.0 / n] * 3, [1.0] * 3, CELL_CENTER, LGF_2, precision=precision)


def _rhs(n, ncomp, seed):
    rng = np.random.default_rng(seed)
    return to_user(rng.standard_normal((ncomp, n, n, n)))


def _rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def _solve(s, rhs, nb, xy):
    import torch
    s.set_xy_cluster(xy)
    d = torch.from_numpy(rhs).cuda()
    out = torch.full_like(d, float("nan"))
    s.solve_batch(out, d, nb) if nb > 1 else s.solve(out, d)
    torch.cuda.synchronize()
    assert s.last_error() == 0
    return out.cpu().numpy()


def test_plan_names_the_cluster_passes():
    t, s = _setup(256, 32)
    names = [(p["name"], p["fast"]) for p in s.plan_json()["passes"] if p["name"] != "green"]
    assert ("fwd01", 5) in names and ("bwd10", 5) in names, names
    assert ("fwd1n", 1) in names and ("bwd1n", 1) in names, names
    s.set_xy_cluster(False)
    names = [p["name"] for p in s.plan_json()["passes"]]
    assert "fwd01" not in names and "fwd0" in names and "fwd1" in names


@pytest.mark.parametrize("lda,nb", [(1, 1), (3, 1), (1, 3)])
def test_cluster_matches_separate_passes_256(lda, nb):
    t, s = _setup(256, 32, lda)
    rhs = _rhs(256, lda * nb, 5 + lda + nb)
    ref = _solve(s, rhs, nb, False)
    got = _solve(s, rhs, nb, True)
    assert np.all(np.isfinite(got))
    # same transforms; only the compiler's contraction of the split formulas may differ
    assert _rel(got, ref) <= 1e-6


def test_cluster_host_arrays_streamed():
    """Host arrays go through the z-slab streamed solve: the cluster kernels
    run per slab of planes and give the device-array result bit for bit."""
    import torch
    t, s = _setup(256, 32)
    rhs = _rhs(256, 1, 21)
    dev = _solve(s, rhs, 1, True)
    out = np.zeros_like(rhs)
    s.solve(out, rhs)
    assert s.last_error() == 0
    assert np.array_equal(out, dev)


def test_cluster_512_matches_fp64():
    """The headline size: FP32 with the cluster passes against the FP64 mode
    (itself pinned to the oracle at 1e-12)."""
    rhs = _rhs(512, 1, 3)
    t64, s64 = _setup(512, 64)
    ref = _solve(s64, rhs, 1, True)
    del s64, t64
    t, s = _setup(512, 32)
    got = _solve(s, rhs, 1, True)
    sep = _solve(s, rhs, 1, False)
    assert _rel(got, ref) <= 2e-6
    assert _rel(got, sep) <= 1e-6
