"""z-slab decomposed solve (flups_b200/slab.py) with 2 to 4 ranks' solvers
in one process on one GPU (the all-to-all done by device copies): every step
is the single-GPU pass on a slab of a rank's own arrays, so the assembled
field equals the one-rank solve bit for bit, FP32 and FP64.  The
torch.distributed transport needs one GPU per rank; its exchange logic is
covered on CPU (tests/test_slab_gloo.py)."""
import numpy as np
import pytest

from gpu_helpers import make_solver, to_user
from oracle.plans import CELL_CENTER, HEJ_2, LGF_2

pytestmark = pytest.mark.gpu

UNB = [[[4], [4]]] * 3


def _unset_solver(n, kernel, precision):
    from flups_b200 import pyflups as pf
    t = pf.Topology(0, 1, [n] * 3)
    s = pf.Solver(t, [[pf.BoundaryType.UNB, pf.BoundaryType.UNB]] * 3, [1.0 / n] * 3, [1.0] * 3,
                  center_type=[CELL_CENTER] * 3)
    s.set_green_type(kernel)
    s.set_alpha(2.0)
    if precision != 64:
        s.set_precision(precision)
    return t, s


@pytest.mark.parametrize("n,precision,world,kernel", [(64, 64, 2, HEJ_2), (128, 32, 3, LGF_2), (256, 32, 4, LGF_2),
                                                      (96, 32, 2, HEJ_2)])
def test_slab_solve_equals_one_rank(n, precision, world, kernel):
    import torch
    from flups_b200.slab import SlabRank, solve_local
    rng = np.random.default_rng(n + world)
    rhs = torch.from_numpy(to_user(rng.standard_normal((1, n, n, n)))).cuda()
    t, s = make_solver([n] * 3, 1, UNB, [1.0 / n] * 3, [1.0] * 3, CELL_CENTER, kernel, precision=precision)
    s.set_xlast(False)  # the slab steps run the reference's pass order
    ref = torch.zeros_like(rhs)
    s.solve(ref, rhs)
    torch.cuda.synchronize()
    assert s.last_error() == 0
    full = s.device_bytes(1)
    keep, ranks = [], []
    for r in range(world):
        tr, sr = _unset_solver(n, kernel, precision)
        keep.append((tr, sr))
        ranks.append(SlabRank(sr, r, world))
    rhs_parts = [rhs[0, r.z0:r.z1].contiguous() for r in ranks]
    out_parts = [torch.full_like(p, float("nan")) for p in rhs_parts]
    solve_local(ranks, out_parts, rhs_parts)
    got = torch.cat(out_parts).unsqueeze(0)
    assert all(sr.last_error() == 0 for _, sr in keep)
    assert torch.equal(got, ref)
    # a rank's arrays (planes, columns, its columns of the Green's spectrum)
    # are about 1/world of the one-rank solver's, plus row padding
    for r in ranks:
        assert r.s.device_bytes(1) < full * (1.0 / world + 0.45)


@pytest.mark.parametrize("n,precision,world,kernel", [(64, 64, 2, HEJ_2), (128, 32, 3, LGF_2), (256, 32, 4, LGF_2)])
def test_slab_connected_equals_one_rank(n, precision, world, kernel):
    """The y passes store into and load from every rank's column array
    directly (here all on one GPU): no exchange copies, same result."""
    import torch
    from flups_b200.slab import SlabRank, connect_local, solve_local_connected
    rng = np.random.default_rng(n + 7 * world)
    rhs = torch.from_numpy(to_user(rng.standard_normal((1, n, n, n)))).cuda()
    t, s = make_solver([n] * 3, 1, UNB, [1.0 / n] * 3, [1.0] * 3, CELL_CENTER, kernel, precision=precision)
    s.set_xlast(False)  # the slab steps run the reference's pass order
    ref = torch.zeros_like(rhs)
    s.solve(ref, rhs)
    torch.cuda.synchronize()
    keep, ranks = [], []
    for r in range(world):
        tr, sr = _unset_solver(n, kernel, precision)
        keep.append((tr, sr))
        ranks.append(SlabRank(sr, r, world))
    connect_local(ranks)
    rhs_parts = [rhs[0, r.z0:r.z1].contiguous() for r in ranks]
    for rep in range(2):
        out_parts = [torch.full_like(p, float("nan")) for p in rhs_parts]
        solve_local_connected(ranks, out_parts, rhs_parts)
        assert torch.equal(torch.cat(out_parts).unsqueeze(0), ref), rep
    assert all(sr.last_error() == 0 for _, sr in keep)
    # a bad table is refused
    assert ranks[0].s.slab_peers([0, 0], [0, 1, 2], [1, 1]) == -2


def test_slab_refuses_other_problems():
    from flups_b200 import pyflups as pf
    from flups_b200.slab import SlabRank
    t = pf.Topology(0, 3, [32] * 3)
    s = pf.Solver(t, [[pf.BoundaryType.UNB, pf.BoundaryType.UNB]] * 3, [1 / 32] * 3, [1.0] * 3)
    with pytest.raises(ValueError):
        SlabRank(s, 0, 2)


def test_slab_peers_refused_without_register_dft_y_passes():
    """50^3 unbounded has 100-point lines, which the register DFTs do not
    cover: the y passes run the general line pass, which cannot store into
    the owners' column arrays, so connecting the peers is refused (-2) and
    the all-to-all form still equals the one-rank solve."""
    import torch
    from flups_b200.slab import SlabRank, solve_local
    n, world = 50, 2
    rng = np.random.default_rng(5)
    rhs = torch.from_numpy(to_user(rng.standard_normal((1, n, n, n)))).cuda()
    t, s = make_solver([n] * 3, 1, UNB, [1.0 / n] * 3, [1.0] * 3, CELL_CENTER, HEJ_2, precision=64)
    s.set_xlast(False)  # the slab steps run the reference's pass order
    ref = torch.zeros_like(rhs)
    s.solve(ref, rhs)
    torch.cuda.synchronize()
    keep, ranks = [], []
    for r in range(world):
        tr, sr = _unset_solver(n, HEJ_2, 64)
        keep.append((tr, sr))
        ranks.append(SlabRank(sr, r, world))
    from flups_b200.slab import _split_table
    cols = [r.s.slab_columns_ptr() for r in ranks]
    pitches = [r.columns_shape[2] for r in ranks]
    for r in ranks:
        assert r.s.slab_peers(cols, _split_table(r.plan), pitches) == -2
    rhs_parts = [rhs[0, r.z0:r.z1].contiguous() for r in ranks]
    out_parts = [torch.full_like(p, float("nan")) for p in rhs_parts]
    solve_local(ranks, out_parts, rhs_parts)
    assert torch.equal(torch.cat(out_parts).unsqueeze(0), ref)
    assert all(sr.last_error() == 0 for _, sr in keep)
