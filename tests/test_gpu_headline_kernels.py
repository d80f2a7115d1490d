"""The kernel instances of the measured workloads, pinned to the oracle on
cheap grids that select them.

The 512^3 all-unbounded solve runs 512-point half-length r2c / c2r rows
(1024-point real lines), 1024-point y columns (forward and inverse) and the
1024-point fused z pass; a 1024-point line is the first whose second
Stockham stage has radix 32.  Anisotropic grids put one of these line
lengths in one direction and short lines in the others, so the oracle (FP64
numpy, the reference's FFTW calls of src/FFTW_plan_dim.cpp:681-716) finishes
in seconds.  The same is done for the longest lines the register DFTs take
(4096-point rows, 2048-point columns, 3 x 2^k up to 3072 / 1536), for the
node-centred DCT-III / DCT-II rows of n = 512 and the fused z pass of 257
nodes in 512-point lines (513 x 257 x 257 workload), for
the node-centred DCT-I / DST-I rows (EVEN/EVEN and ODD/ODD, 65 and 257
points) and for one full 256^3 solve.  Each case also checks, through the host plan
description, that the passes of the intended length run the register DFTs.
FP64 <= 1e-12 and FP32 <= 2e-6 relative L2 against the oracle.
"""
import numpy as np
import pytest

from gpu_helpers import from_user, make_solver, oracle_solve, rel_l2, to_user
from oracle.plans import CELL_CENTER, NODE_CENTER, CHAT_2, LGF_2, LGF_4, HEJ_4

pytestmark = pytest.mark.gpu

UNB3 = [[[4], [4]]] * 3
EO_PER_UNB = [[[0], [1]], [[3], [3]], [[4], [4]]]
EE_PER_UNB = [[[0], [0]], [[3], [3]], [[4], [4]]]
OO_PER_UNB = [[[1], [1]], [[3], [3]], [[4], [4]]]

# (name, nglob, bc, centring, kernel, line length M whose passes must run the register DFTs, axis)
CASES = [
    ("rows1024_512x32x32", [512, 32, 32], UNB3, CELL_CENTER, LGF_2, 1024, 0),
    ("cols1024_32x512x32", [32, 512, 32], UNB3, CELL_CENTER, LGF_2, 1024, 1),
    ("fused1024_32x32x512", [32, 32, 512], UNB3, CELL_CENTER, LGF_2, 1024, 2),
    ("rows4096_2048x16x16", [2048, 16, 16], UNB3, CELL_CENTER, LGF_2, 4096, 0),
    ("cols2048_16x1024x16", [16, 1024, 16], UNB3, CELL_CENTER, LGF_2, 2048, 1),
    ("fused2048_16x16x1024", [16, 16, 1024], UNB3, CELL_CENTER, LGF_2, 2048, 2),
    ("rows3072_1536x16x16", [1536, 16, 16], UNB3, CELL_CENTER, CHAT_2, 3072, 0),
    ("cols1536_16x768x16", [16, 768, 16], UNB3, CELL_CENTER, CHAT_2, 1536, 1),
    ("fused1536_16x16x768", [16, 16, 768], UNB3, CELL_CENTER, CHAT_2, 1536, 2),
    # 768- and 384-point x rows: with device arrays the fused rows of the
    # x-last order (FP64 3 x 2^k rows run a first radix of 24)
    ("xrows768_384x24x24", [384, 24, 24], UNB3, CELL_CENTER, CHAT_2, 768, 0),
    ("xrows384_192x24x24", [192, 24, 24], UNB3, CELL_CENTER, LGF_2, 384, 0),
    ("node513_dct_rows_eo_per_unb", [513, 33, 33], EO_PER_UNB, NODE_CENTER, HEJ_4, 1024, 0),
    # the fused z pass of the same workload: 257 nodes in a 512-point line
    # (L/2 + 1 loaded and stored)
    ("node_fused512_eo_per_unb_17x17x257", [17, 17, 257], EO_PER_UNB, NODE_CENTER, HEJ_4, 512, 2),
    # 256-point real-side columns (first radix 16): the node grid's periodic y
    # (257 nodes) and, with device arrays, the z columns of the x-last order
    ("node_yreal256_eo_per_unb_17x257x17", [17, 257, 17], EO_PER_UNB, NODE_CENTER, HEJ_4, 256, 1),
    ("zreal256_32x32x128", [32, 32, 128], UNB3, CELL_CENTER, LGF_2, 256, 2),
    # DCT-I / DST-I rows (node-centred EVEN/EVEN, ODD/ODD): the real DFT of the
    # extension through a register DFT of half its length
    ("node257_dct1_rows_ee_per_unb", [257, 17, 17], EE_PER_UNB, NODE_CENTER, HEJ_4, 512, 0),
    ("node257_dst1_rows_oo_per_unb", [257, 17, 17], OO_PER_UNB, NODE_CENTER, HEJ_4, 512, 0),
    ("node65_dct1_rows_ee_per_unb", [65, 17, 17], EE_PER_UNB, NODE_CENTER, HEJ_4, 128, 0),
    ("node65_dst1_rows_oo_per_unb", [65, 17, 17], OO_PER_UNB, NODE_CENTER, HEJ_4, 128, 0),
]


def _rhs(nglob, lda=1, seed=17):
    rng = np.random.default_rng(seed)
    x = [np.arange(n) / n for n in nglob]
    X, Y, Z = np.meshgrid(*x, indexing="ij")
    out = np.zeros((lda,) + tuple(nglob))
    for c in range(lda):
        for _ in range(6):
            cc = rng.uniform(0.2, 0.8, 3)
            s = rng.uniform(0.03, 0.08)
            out[c] += rng.uniform(-1, 1) * np.exp(-((X - cc[0]) ** 2 + (Y - cc[1]) ** 2 + (Z - cc[2]) ** 2) / s ** 2)
        out[c] += 1e-3 * rng.standard_normal(nglob)
    return out


def _grid(nglob, center):
    fact = 0 if center == CELL_CENTER else 1
    h = [1.0 / (nglob[0] - fact)] * 3
    L = [h[d] * (nglob[d] - fact) for d in range(3)]
    return h, L


def _solve(nglob, lda, bcv, center, kernel, precision, rhs, type_=0, odiff=0, device=False):
    """device=False: host arrays (the reference's pass order, slab-streamed);
    device=True: CUDA arrays (the x-last order of all-unbounded problems),
    whose passes plan_json describes."""
    h, L = _grid(nglob, center)
    t, s = make_solver(nglob, lda, bcv, h, L, center, kernel, odiff=odiff, precision=precision)
    plan = s.plan_json(type_)
    u = to_user(rhs)
    if device:
        import torch
        du = torch.from_numpy(u).cuda()
        dout = torch.zeros_like(du)
        s.solve(dout, du, type_)
        torch.cuda.synchronize()
        out = dout.cpu().numpy()
    else:
        s.set_xlast(False)
        plan = s.plan_json(type_)
        out = np.zeros_like(u)
        s.solve(out, u, type_)
    assert s.last_error() == 0
    return from_user(out, lda, nglob), plan


_REF = {}


def _oracle(name, nglob, lda, bcv, center, kernel, rhs, type_=0, odiff=0):
    if name not in _REF:
        h, L = _grid(nglob, center)
        _REF[name] = oracle_solve(nglob, lda, bcv, h, L, center, kernel, rhs, type_=type_, odiff=odiff)
    return _REF[name]


def _check_fast(plan, M, axis):
    sel = [p for p in plan["passes"] if p["name"] != "green" and p["axis"] == axis and p["st"][0]["M"] == M]
    assert sel, f"no pass of {M}-point lines along axis {axis}"
    assert all(p["fast"] for p in sel), sel


@pytest.mark.parametrize("device", [False, True], ids=["host", "device"])
@pytest.mark.parametrize("precision,tol", [(64, 1e-12), (32, 2e-6)], ids=["fp64", "fp32"])
@pytest.mark.parametrize("name,nglob,bcv,center,kernel,M,axis", CASES, ids=[c[0] for c in CASES])
def test_kernel_instance_matches_oracle(name, nglob, bcv, center, kernel, M, axis, precision, tol, device):
    """Host arrays run the reference's pass order (x rows r2c / c2r, the fused
    pass along z); device arrays of all-unbounded grids run the x-last order
    (z columns r2c / c2r of the user's doubles, the fused pass along x rows)."""
    rhs = _rhs(nglob)
    got, plan = _solve(nglob, 1, bcv, center, kernel, precision, rhs, device=device)
    _check_fast(plan, M, axis)
    if device and bcv is UNB3 and M <= 1024:
        assert plan["xlast"] == 1
        fused = [p for p in plan["passes"] if p["name"] == "fused"]
        assert fused[0]["axis"] == 0 and fused[0]["fast"] == 5
    ref = _oracle(name, nglob, 1, bcv, center, kernel, rhs)
    assert rel_l2(got, ref) <= tol


@pytest.mark.parametrize("precision,tol", [(64, 1e-12), (32, 2e-6)], ids=["fp64", "fp32"])
@pytest.mark.parametrize("nglob,device", [([32, 32, 384], False), ([384, 32, 32], True), ([192, 32, 32], True),
                                          ([64, 64, 64], True)],
                         ids=["z768_host", "x768_device", "x384_device", "64cube_device"])
def test_rot_lines_lgf4(nglob, device, precision, tol):
    """The ROT solve of the 384^3 vortex-ring workload (LGF_4, spectral curl)
    with 768-point lines along its fused direction: host arrays run the
    reference's order (fused column pass along z, col_rot_kernel), device
    arrays the x-last order where it applies (fused rows, row_rot_kernel:
    lines that fit one warp, i.e. up to 1024 points for powers of two, and
    768 (FP32) or 384 (FP64) points for 3 x 2^k)."""
    bcv = [[[4] * 3, [4] * 3]] * 3
    rhs = _rhs(nglob, lda=3, seed=23)
    got, plan = _solve(nglob, 3, bcv, CELL_CENTER, LGF_4, precision, rhs, type_=1, odiff=1, device=device)
    # the last direction: forward DFT, curl and Green's multiply, inverse DFT in one register-DFT pass
    fused = [p for p in plan["passes"] if p["name"] == "fused"]
    assert len(fused) == 1 and fused[0]["fast"] in (1, 5), fused
    if device and (precision == 32 or nglob[0] <= 256):
        assert plan["xlast"] == 1 and fused[0]["fast"] == 5 and fused[0]["axis"] == 0
    ref = _oracle(f"rot_{nglob}", nglob, 3, bcv, CELL_CENTER, LGF_4, rhs, type_=1, odiff=1)
    assert rel_l2(got, ref) <= tol


def test_full_256_cube_fp64_matches_oracle():
    """One full 256^3 all-unbounded FP64 solve (512-point lines in every
    direction, the instances the graph and slab tests only compare with the
    library itself) against the oracle."""
    n = 256
    nglob = [n] * 3
    rhs = _rhs(nglob, seed=29)
    ref = _oracle("full256", nglob, 1, UNB3, CELL_CENTER, CHAT_2, rhs)
    for device in (False, True):
        got, plan = _solve(nglob, 1, UNB3, CELL_CENTER, CHAT_2, 64, rhs, device=device)
        for axis in range(3):
            _check_fast(plan, 2 * n, axis)
        assert plan["xlast"] == (1 if device else 0)
        assert rel_l2(got, ref) <= 1e-12


# grids whose directions are all unbounded or periodic (line lengths the
# register DFTs take in every direction): device arrays run the x-last order
# (z first, the fused pass along x rows)
PPU = [[[3], [3]], [[3], [3]], [[4], [4]]]
UPU = [[[4], [4]], [[3], [3]], [[4], [4]]]
PUP = [[[3], [3]], [[4], [4]], [[3], [3]]]
MIXED = [
    ("per_per_unb_64x48x32", [64, 48, 32], PPU, HEJ_4),
    ("unb_per_unb_48x64x32", [48, 64, 32], UPU, LGF_2),
    ("per_unb_per_64x32x48", [64, 32, 48], PUP, CHAT_2),
]


@pytest.mark.parametrize("precision,tol", [(64, 1e-12), (32, 2e-6)], ids=["fp64", "fp32"])
@pytest.mark.parametrize("name,nglob,bcv,kernel", MIXED, ids=[c[0] for c in MIXED])
def test_mixed_periodic_unbounded_xlast(name, nglob, bcv, kernel, precision, tol):
    rhs = _rhs(nglob)
    got, plan = _solve(nglob, 1, bcv, CELL_CENTER, kernel, precision, rhs, device=True)
    assert plan["xlast"] == 1
    fused = [p for p in plan["passes"] if p["name"] == "fused"]
    assert fused[0]["axis"] == 0 and fused[0]["fast"] == 5
    ref = _oracle(name, nglob, 1, bcv, CELL_CENTER, kernel, rhs)
    assert rel_l2(got, ref) <= tol


def _bc3(codes):
    return [[[c[0]] * 3, [c[1]] * 3] for c in codes]


# ROT with periodic directions: the x-last order when the reference's first
# (real-to-complex) direction is x (periodic x), else the reference's order
ROT_MIXED = [
    ("rot_per_per_unb_64x48x32", [64, 48, 32], _bc3([(3, 3), (3, 3), (4, 4)]), 1),
    ("rot_per_unb_per_48x32x64", [48, 32, 64], _bc3([(3, 3), (4, 4), (3, 3)]), 1),
    ("rot_unb_per_unb_24x48x32", [24, 48, 32], _bc3([(4, 4), (3, 3), (4, 4)]), 0),
]


@pytest.mark.parametrize("precision,tol", [(64, 1e-12), (32, 2e-6)], ids=["fp64", "fp32"])
@pytest.mark.parametrize("name,nglob,bcv,xlast", ROT_MIXED, ids=[c[0] for c in ROT_MIXED])
def test_mixed_rot(name, nglob, bcv, xlast, precision, tol):
    rhs = _rhs(nglob, lda=3, seed=29)
    got, plan = _solve(nglob, 3, bcv, CELL_CENTER, LGF_4, precision, rhs, type_=1, odiff=1, device=True)
    assert plan["xlast"] == xlast
    ref = _oracle(name, nglob, 3, bcv, CELL_CENTER, LGF_4, rhs, type_=1, odiff=1)
    assert rel_l2(got, ref) <= tol
