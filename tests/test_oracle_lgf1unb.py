"""The oracle's 1-D lattice Green's functions of one unbounded direction
(oracle/lgf1unb.py) against the reference's own header compiled here
(src/lgf_1unb2spe.hpp through oracle/build_ref.py): the committed golden
values of tests/golden/lgf1unb_ref.json (made by make_lgf1unb_ref.py) cover
every regime of lgf2/4/6/8 and of the Mehrstellen meh4/meh6 left and full.
The oracle must agree to 1e-12 (relative to max(1, |value|))."""
import json
from pathlib import Path

import pytest

from oracle import lgf1unb as l1

GOLD = Path(__file__).resolve().parent / "golden" / "lgf1unb_ref.json"
FN = {2: l1.lgf2, 4: l1.lgf4, 6: l1.lgf6, 8: l1.lgf8,
      41: l1.meh4_left, 42: l1.meh4_full, 61: l1.meh6_left, 62: l1.meh6_full}


def _rows():
    return json.loads(GOLD.read_text())["rows"]


@pytest.mark.parametrize("kind", sorted(FN))
def test_oracle_matches_reference_header(kind):
    rows = [r for r in _rows() if r[0] == kind]
    assert len(rows) >= 80
    for k, n, a, b, v in rows:
        got = FN[k](n, a) if k < 10 else FN[k](n, a, b)
        assert abs(got - v) <= 1e-12 * max(1.0, abs(v)), (k, n, a, b, v, got)
