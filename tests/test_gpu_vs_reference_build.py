"""The CUDA path against the reference's own solver (its sources compiled by
oracle/build_ref.py into oracle/_ref/libflups_ref.so, which travels with the
repository), on the same inputs: whole solution fields, FP64 mode at
<= 1e-12 relative L2 (FP32 mode at <= 2e-6), host and device arrays (the two
pass orders).  The cases cover the measured workloads' families: all
unbounded (LGF_2 and CHAT_2), the node-centred EVEN/ODD - PER - UNB grid
(HEJ_4), a periodic/unbounded mix (x-last order), the vortex-ring ROT solve
(LGF_4, spectral curl) and one-unbounded lattice kernels.  Skipped where the
reference build is absent."""
import numpy as np
import pytest

from gpu_helpers import gpu_solve, rel_l2
from oracle import ref_lib
from oracle.plans import CELL_CENTER, NODE_CENTER, CHAT_2, LGF_2, LGF_4, HEJ_4

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_lib.available(), reason="reference build (oracle/_ref) absent")]

MEHR_4F, LGF_8 = 13, 10


def _bc(codes, lda=1):
    return [[[c[0]] * lda, [c[1]] * lda] for c in codes]


# (name, nglob, lda, bc, centring, kernel, type, diff order)
CASES = [
    ("unb_lgf2_64x48x32", [64, 48, 32], 1, _bc([(4, 4)] * 3), CELL_CENTER, LGF_2, 0, 0),
    ("unb_chat2_48cube", [48, 48, 48], 1, _bc([(4, 4)] * 3), CELL_CENTER, CHAT_2, 0, 0),
    ("node_eo_per_unb_hej4_129x33x33", [129, 33, 33], 1, _bc([(0, 1), (3, 3), (4, 4)]), NODE_CENTER, HEJ_4, 0, 0),
    ("per_per_unb_hej4_64x48x32", [64, 48, 32], 1, _bc([(3, 3), (3, 3), (4, 4)]), CELL_CENTER, HEJ_4, 0, 0),
    ("rot_unb_lgf4_32cube", [32, 32, 32], 3, _bc([(4, 4)] * 3, 3), CELL_CENTER, LGF_4, 1, 1),
    ("per_per_unb_mehr4f_32x32x48", [32, 32, 48], 1, _bc([(3, 3), (3, 3), (4, 4)]), CELL_CENTER, MEHR_4F, 0, 0),
    ("eo_per_unb_lgf8_32x32x48", [32, 32, 48], 1, _bc([(0, 1), (3, 3), (4, 4)]), CELL_CENTER, LGF_8, 0, 0),
]

_REF = {}


def _grid(nglob, center):
    fact = 0 if center == CELL_CENTER else 1
    hh = 1.0 / (nglob[0] - fact)
    return [hh] * 3, [hh * (nglob[d] - fact) for d in range(3)]


def _rhs(nglob, lda, seed):
    rng = np.random.default_rng(seed)
    x = [np.arange(n) / n for n in nglob]
    X, Y, Z = np.meshgrid(*x, indexing="ij")
    out = np.zeros((lda,) + tuple(nglob))
    for c in range(lda):
        for _ in range(5):
            cc = rng.uniform(0.25, 0.75, 3)
            s = rng.uniform(0.05, 0.1)
            out[c] += rng.uniform(-1, 1) * np.exp(-((X - cc[0]) ** 2 + (Y - cc[1]) ** 2 + (Z - cc[2]) ** 2) / s ** 2)
    return out


def _reference(name, nglob, lda, bcv, center, kernel, typ, odiff, rhs):
    if name not in _REF:
        h, L = _grid(nglob, center)
        s = ref_lib.RefSolver(nglob, lda, bcv, h, L, center, kernel, alpha=2.0, odiff=odiff)
        _REF[name] = s.solve(rhs, typ)
        s.close()
    return _REF[name]


@pytest.mark.parametrize("device", [False, True], ids=["host", "device"])
@pytest.mark.parametrize("precision,tol", [(64, 1e-12), (32, 2e-6)], ids=["fp64", "fp32"])
@pytest.mark.parametrize("name,nglob,lda,bcv,center,kernel,typ,odiff", CASES, ids=[c[0] for c in CASES])
def test_matches_reference_build(name, nglob, lda, bcv, center, kernel, typ, odiff, precision, tol, device):
    rhs = _rhs(nglob, lda, seed=len(name))
    h, L = _grid(nglob, center)
    got = gpu_solve(nglob, lda, bcv, h, L, center, kernel, rhs, type_=typ, odiff=odiff, precision=precision,
                    device=device)
    want = _reference(name, nglob, lda, bcv, center, kernel, typ, odiff, rhs)
    assert rel_l2(got, want) <= tol
