"""The register-resident power-of-two DFT kernels (flups_b200/csrc/fast_dft.cu)
against the oracle and against the general line-pass kernel, on grids where
they are selected (checked through the host-side plan description)."""
import numpy as np
import pytest

from gpu_helpers import from_user, make_solver, oracle_solve, rel_l2, to_user
from oracle.plans import CELL_CENTER, NODE_CENTER, CHAT_2, LGF_2, HEJ_2, HEJ_4

pytestmark = pytest.mark.gpu

UNB3 = [[[4], [4]]] * 3
PPU = [[[3], [3]], [[3], [3]], [[4], [4]]]


def _rhs(nglob, lda=1, seed=3):
    rng = np.random.default_rng(seed)
    x = [np.arange(n) / n for n in nglob]
    X, Y, Z = np.meshgrid(*x, indexing="ij")
    out = np.zeros((lda,) + tuple(nglob))
    for c in range(lda):
        for _ in range(4):
            cc = rng.uniform(0.3, 0.7, 3)
            s = rng.uniform(0.05, 0.1)
            out[c] += rng.uniform(-1, 1) * np.exp(-((X - cc[0]) ** 2 + (Y - cc[1]) ** 2 + (Z - cc[2]) ** 2) / s ** 2)
    return out


def _run(nglob, lda, bcv, center, kernel, precision, fast):
    n0 = nglob[0] - (0 if center == CELL_CENTER else 1)
    h = [1.0 / n0] * 3
    L = [h[d] * (nglob[d] - (0 if center == CELL_CENTER else 1)) for d in range(3)]
    t, s = make_solver(nglob, lda, bcv, h, L, center, kernel, precision=precision)
    from flups_b200 import pyflups as pf
    pf.load_library().flups_b200_set_fast_kernels(s._solver, int(fast))
    plan = s.plan_json()
    rhs = _rhs(nglob, lda)
    u = to_user(rhs)
    out = np.zeros_like(u)
    s.solve(out, u)
    assert s.last_error() == 0
    ref = oracle_solve(nglob, lda, bcv, h, L, center, kernel, rhs)
    return from_user(out, lda, nglob), ref, plan


CASES = [
    ("unb64_chat2", [64] * 3, 1, UNB3, CELL_CENTER, CHAT_2),
    ("unb32_hej2", [32] * 3, 1, UNB3, CELL_CENTER, HEJ_2),
    ("unb128_lgf2", [128] * 3, 1, UNB3, CELL_CENTER, LGF_2),
    ("unb_aniso", [128, 64, 32], 1, UNB3, CELL_CENTER, CHAT_2),
    ("ppu64_hej4", [64] * 3, 1, PPU, CELL_CENTER, HEJ_4),
    ("node65_unb", [65] * 3, 1, UNB3, NODE_CENTER, CHAT_2),
    ("vector3_unb64", [64] * 3, 3, [[[4] * 3, [4] * 3]] * 3, CELL_CENTER, LGF_2),
    # 3 x 2^k lines (radix-3 first stage): 96, 192, 384 points
    ("unb48_hej2_r3", [48] * 3, 1, UNB3, CELL_CENTER, HEJ_2),
    ("unb96_48_192_r3", [96, 48, 192], 1, UNB3, CELL_CENTER, LGF_2),
    ("ppu96_hej4_r3", [96, 96, 48], 1, PPU, CELL_CENTER, HEJ_4),
    # EVEN x (DCT line pass), UNB y and z: y is an r2c / c2r column pass
    ("euu64_col_r2c", [64] * 3, 1, [[[0], [0]], [[4], [4]], [[4], [4]]], CELL_CENTER, HEJ_2),
    ("euu48_col_r2c_r3", [48, 48, 96], 1, [[[0], [0]], [[4], [4]], [[4], [4]]], CELL_CENTER, LGF_2),
    ("ppu48_rows48", [48] * 3, 1, PPU, CELL_CENTER, CHAT_2),
    # node-centred EVEN/ODD x (DCT-III / DCT-II rows), PER y (r2c / c2r columns with the periodic copy), UNB z
    ("node_eo_per_unb65", [65] * 3, 1, [[[0], [1]], [[3], [3]], [[4], [4]]], NODE_CENTER, HEJ_4),
    ("node_eo_per_unb_129x65", [129, 65, 65], 1, [[[0], [1]], [[3], [3]], [[4], [4]]], NODE_CENTER, HEJ_4),
    # cell-centred ODD/ODD x (DST rows), PER y and z
    ("oopp64", [64] * 3, 1, [[[1], [1]], [[3], [3]], [[3], [3]]], CELL_CENTER, CHAT_2),
    # half-length DCT / DST rows: II/III (EVEN/EVEN, node ODD/EVEN), IV (EVEN/ODD, ODD/EVEN cell)
    ("eepp128_dct23", [128, 32, 32], 1, [[[0], [0]], [[3], [3]], [[3], [3]]], CELL_CENTER, HEJ_2),
    ("eopu64_dct4", [64] * 3, 1, [[[0], [1]], [[3], [3]], [[4], [4]]], CELL_CENTER, HEJ_4),
    ("oeuu96_dst4_r3", [96, 48, 48], 1, [[[1], [0]], [[4], [4]], [[4], [4]]], CELL_CENTER, LGF_2),
    ("node_oe_per_unb65_dst23", [65, 33, 33], 1, [[[1], [0]], [[3], [3]], [[4], [4]]], NODE_CENTER, CHAT_2),
    ("vector3_eopu64_dct4", [64, 32, 32], 3, [[[0, 0, 0], [1, 1, 1]], [[3] * 3, [3] * 3], [[4] * 3, [4] * 3]],
     CELL_CENTER, HEJ_2),
    # 768-point lines: FP32 first radix 48 (two stages) in the x rows (half length 384) and the y columns
    ("unb_384x32x32_r48", [384, 32, 32], 1, UNB3, CELL_CENTER, HEJ_2),
    ("unb_32x384x32_r48", [32, 384, 32], 1, UNB3, CELL_CENTER, LGF_2),
    # node EVEN/EVEN x: DCT-I rows through the extended-row DFT
    ("node_ee_unb65_dct1", [65, 33, 33], 1, [[[0], [0]], [[4], [4]], [[4], [4]]], NODE_CENTER, CHAT_2),
]


@pytest.mark.parametrize("name,nglob,lda,bcv,center,kernel", CASES, ids=[c[0] for c in CASES])
def test_fast_fp64_matches_oracle(name, nglob, lda, bcv, center, kernel):
    got, ref, plan = _run(nglob, lda, bcv, center, kernel, 64, True)
    assert any(p["fast"] for p in plan["passes"] if p["name"] != "green"), "fast kernels not selected"
    assert rel_l2(got, ref) <= 1e-12


@pytest.mark.parametrize("name,nglob", [(c[0], c[1]) for c in CASES if c[0].endswith("_r48")])
def test_radix48_lines_run_the_register_dft(name, nglob):
    """The 768-point lines of the radix-48 cases run the register DFT (not the
    general line pass) in FP32, so the parity cases above check that path."""
    case = next(c for c in CASES if c[0] == name)
    _, _, plan = _run(case[1], case[2], case[3], case[4], case[5], 32, True)
    long_passes = [p for p in plan["passes"] if p["name"] != "green" and p["st"][0]["M"] == 768]
    assert long_passes and all(p["fast"] for p in long_passes), long_passes


@pytest.mark.parametrize("name,nglob,lda,bcv,center,kernel", CASES, ids=[c[0] for c in CASES])
def test_fast_fp32_matches_oracle_and_general_engine(name, nglob, lda, bcv, center, kernel):
    got, ref, _ = _run(nglob, lda, bcv, center, kernel, 32, True)
    gen, _, plan = _run(nglob, lda, bcv, center, kernel, 32, False)
    assert not any(p["fast"] for p in plan["passes"])
    assert rel_l2(got, ref) <= 2e-6
    assert rel_l2(gen, ref) <= 2e-6
    assert rel_l2(got, gen) <= 2e-6


@pytest.mark.parametrize("n,odiff,kernel", [(32, 1, LGF_2), (48, 2, HEJ_2), (64, 4, CHAT_2)])
def test_rot_fused_matches_oracle(n, odiff, kernel):
    """ROT solves whose last direction runs through the register DFTs do the
    curl and Green's multiply inside that pass (three components per CTA):
    FP64 against the oracle (<= 1e-12), FP32 against the FP64 mode (<= 2e-6)."""
    from gpu_helpers import gpu_solve
    nglob = [n] * 3
    bcv = [[[4] * 3, [4] * 3]] * 3
    h = [1.0 / n] * 3
    L = [1.0] * 3
    rhs = _rhs(nglob, 3, seed=11)
    got = gpu_solve(nglob, 3, bcv, h, L, CELL_CENTER, kernel, rhs, type_=1, odiff=odiff)
    ref = oracle_solve(nglob, 3, bcv, h, L, CELL_CENTER, kernel, rhs, type_=1, odiff=odiff)
    assert rel_l2(got, ref) <= 1e-12
    got32 = gpu_solve(nglob, 3, bcv, h, L, CELL_CENTER, kernel, rhs, type_=1, odiff=odiff, precision=32)
    assert rel_l2(got32, got) <= 2e-6


XLAST_CASES = [
    ("unb64", [64] * 3, NODE_CENTER, CHAT_2),
    ("unb_aniso", [128, 64, 32], CELL_CENTER, LGF_2),
    ("unb96_r3", [96, 48, 48], CELL_CENTER, HEJ_2),
    ("unb_node65", [65, 33, 33], NODE_CENTER, HEJ_4),
]


@pytest.mark.parametrize("name,nglob,center,kernel", XLAST_CASES, ids=[c[0] for c in XLAST_CASES])
def test_xlast_order_matches_oracle_and_reference_order(name, nglob, center, kernel):
    """All-unbounded solves of device arrays in the x-last order (z r2c
    columns of the user's doubles, y columns, fused x rows) against the oracle
    and against the reference's order on the same device arrays: FP64 within
    1e-12 of both, FP32 within 2e-6."""
    from gpu_helpers import gpu_solve
    n0 = nglob[0] - (0 if center == CELL_CENTER else 1)
    h = [1.0 / n0] * 3
    L = [h[d] * (nglob[d] - (0 if center == CELL_CENTER else 1)) for d in range(3)]
    rhs = _rhs(nglob)
    ref = oracle_solve(nglob, 1, UNB3, h, L, center, kernel, rhs)
    for precision, tol in ((64, 1e-12), (32, 2e-6)):
        xl = gpu_solve(nglob, 1, UNB3, h, L, center, kernel, rhs, precision=precision, device=True)
        xf = gpu_solve(nglob, 1, UNB3, h, L, center, kernel, rhs, precision=precision, device=True, xlast=False)
        assert rel_l2(xl, ref) <= tol
        assert rel_l2(xf, ref) <= tol
        assert rel_l2(xl, xf) <= tol


@pytest.mark.parametrize("n,odiff,kernel", [(32, 1, LGF_2), (48, 2, HEJ_2), (64, 4, CHAT_2)])
def test_rot_xlast_matches_oracle(n, odiff, kernel):
    """ROT solves of device arrays in the x-last order (fused rows, three
    component warps per row meeting at a named barrier for the curl): FP64
    against the oracle (<= 1e-12), FP32 against the FP64 mode (<= 2e-6)."""
    from gpu_helpers import gpu_solve
    nglob = [n] * 3
    bcv = [[[4] * 3, [4] * 3]] * 3
    h = [1.0 / n] * 3
    L = [1.0] * 3
    rhs = _rhs(nglob, 3, seed=13)
    ref = oracle_solve(nglob, 3, bcv, h, L, CELL_CENTER, kernel, rhs, type_=1, odiff=odiff)
    got = gpu_solve(nglob, 3, bcv, h, L, CELL_CENTER, kernel, rhs, type_=1, odiff=odiff, device=True)
    assert rel_l2(got, ref) <= 1e-12
    got32 = gpu_solve(nglob, 3, bcv, h, L, CELL_CENTER, kernel, rhs, type_=1, odiff=odiff, precision=32, device=True)
    assert rel_l2(got32, got) <= 2e-6
