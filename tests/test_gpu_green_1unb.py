"""One unbounded direction with the higher-order lattice Green's functions
(LGF_4/6/8) and the Mehrstellen kernels (MEHR_4L/6L/4F/6F): the GPU's FP64
set-up (flups_b200/csrc/lgf1unb.cuh) and solve against the oracle, whose
1-D closed forms are pinned to the reference's own header
(tests/test_oracle_lgf1unb.py).  Reference: src/green_functions.cpp:456-482,
src/green_kernels.hpp:591-671, src/lgf_1unb2spe.hpp:161-612.
FP64 <= 1e-12 relative L2, FP32 <= 2e-6."""
import numpy as np
import pytest

from gpu_helpers import gpu_solve, oracle_solve, rel_l2
from oracle.plans import CELL_CENTER, NODE_CENTER, LGF_4, LGF_6, LGF_8, MEHR_4L, MEHR_6L, MEHR_4F, MEHR_6F

pytestmark = pytest.mark.gpu

KERNELS = [("LGF_4", LGF_4), ("LGF_6", LGF_6), ("LGF_8", LGF_8), ("MEHR_4L", MEHR_4L), ("MEHR_6L", MEHR_6L),
           ("MEHR_4F", MEHR_4F), ("MEHR_6F", MEHR_6F)]
BCS = [
    ("per_per_unb", [[[3], [3]], [[3], [3]], [[4], [4]]]),
    ("even_odd_unb", [[[0], [0]], [[1], [1]], [[4], [4]]]),
    ("eo_per_unb", [[[0], [1]], [[3], [3]], [[4], [4]]]),
]


def _rhs(nglob, seed):
    rng = np.random.default_rng(seed)
    x = [np.arange(n) / n for n in nglob]
    X, Y, Z = np.meshgrid(*x, indexing="ij")
    out = np.zeros((1,) + tuple(nglob))
    for _ in range(3):
        c = rng.uniform(0.3, 0.7, 3)
        out[0] += rng.uniform(-1, 1) * np.exp(-((X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2) / 0.02)
    return out + 1e-3 * rng.standard_normal(out.shape)


@pytest.mark.parametrize("center", [CELL_CENTER, NODE_CENTER], ids=["cell", "node"])
@pytest.mark.parametrize("bname,bcv", BCS, ids=[b[0] for b in BCS])
@pytest.mark.parametrize("kname,kernel", KERNELS, ids=[k[0] for k in KERNELS])
def test_one_unbounded_kernel_matches_oracle(kname, kernel, bname, bcv, center):
    n = 16
    nglob = [n + (0 if center == CELL_CENTER else 1)] * 3
    h = [1.0 / n] * 3
    L = [1.0] * 3
    rhs = _rhs(nglob, 7)
    ref = oracle_solve(nglob, 1, bcv, h, L, center, kernel, rhs)
    got = gpu_solve(nglob, 1, bcv, h, L, center, kernel, rhs)
    assert np.isfinite(ref).all()
    assert rel_l2(got, ref) <= 1e-12
    if bname == "per_per_unb" and center == CELL_CENTER:
        got32 = gpu_solve(nglob, 1, bcv, h, L, center, kernel, rhs, precision=32)
        assert rel_l2(got32, ref) <= 2e-6
