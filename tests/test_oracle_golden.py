"""Pin the CPU oracle against the reference's own golden vectors.

The reference's validation goldens (samples/validation/data_ref, 2452 files)
hold error norms of its solver against manufactured solutions; the vortex-tube
goldens (samples/solve_vtube/data_ref, 27 files) do the same for the
Biot-Savart (ROT) solve.  The comparison rule is the reference's
(samples/validation/scripts/check_res.py:9-44): relative difference < 1e-10,
absolute difference when the golden value is below 1e-14.
"""
import json
import re
from pathlib import Path

import pytest

from oracle.plans import CELL_CENTER, NODE_CENTER
from oracle.validation import run_case
from oracle.vtube import run_tube

GOLD = json.loads((Path(__file__).parent / "golden" / "validation_ref.json").read_text())
TOL = 1e-10
_PAT = re.compile(r"validation_3d_(CellCenter|NodeCenter)_(\d{6})_typeGreen=(\d+)\.txt")


def _close(ref, mine):
    if ref < 1e-14:
        return abs(ref - mine) < TOL
    return abs(ref - mine) / ref < TOL


def _cases():
    for fn in sorted(GOLD["validation"]):
        m = _PAT.match(fn)
        yield fn, m.group(1), m.group(2), int(m.group(3))


@pytest.mark.parametrize("centre", ["CellCenter", "NodeCenter"])
def test_validation_goldens(centre):
    """Every BC combination x kernel x resolution of the reference's goldens."""
    bad = []
    n = 0
    for fn, cname, code, kernel in _cases():
        if cname != centre:
            continue
        center = CELL_CENTER if cname == "CellCenter" else NODE_CENTER
        bc = [[int(code[0]), int(code[1])], [int(code[2]), int(code[3])], [int(code[4]), int(code[5])]]
        for row in GOLD["validation"][fn]:
            ng = int(row[0])
            r0 = ng - (0 if center == CELL_CENTER else 1)
            res = (r0, r0, 1 if code[4:] == "99" else r0)
            _, errs = run_case(center, res, bc, kernel)
            n += 1
            if not (_close(row[1], errs[0][0]) and _close(row[2], errs[0][1])):
                bad.append((fn, ng, row[1:3], errs[0]))
    assert n > 1000
    assert not bad, bad[:5]


def test_vtube_goldens():
    pat = re.compile(r"vtube_CellCenter_0_(\d)(-?\d)(-?\d)_typeGreen=0\.txt")
    n = 0
    for fn, rows in GOLD["vtube"].items():
        m = pat.match(fn)
        errs = run_tube(int(m.group(1)), int(m.group(2)), int(m.group(3)))
        for row in rows:
            for c in range(3):
                assert _close(row[1 + 2 * c], errs[c][0]), (fn, c)
                assert _close(row[2 + 2 * c], errs[c][1]), (fn, c)
                n += 1
    assert n == 81
