"""Golden values of the reference's 1-D lattice Green's functions of one
unbounded direction (src/lgf_1unb2spe.hpp: lgf2/4/6/8 and the Mehrstellen
meh4/meh6 left and full), computed by the reference's own header compiled
with oracle/build_ref.py, at arguments that cover every regime of the
closed forms (c = 0, small c, real roots, the repeated roots at c = 3 and
c* = 3.2044..., complex roots; Mehrstellen wave-number pairs up to pi,
including one where the leading coefficient nearly vanishes).

    python tests/golden/make_lgf1unb_ref.py   (needs the reference tree and g++)

Writes tests/golden/lgf1unb_ref.json: rows [kind, n, a, b, value].
"""
import json
import math
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.build_ref import build_lgf1unb  # noqa: E402

NS = [0, 1, 2, 3, 4, 5, 7, 10, 16, 31, 64]
CS = {
    2: [0.0, 1e-6, 5e-4, 0.002, 0.3, 1.0, 4.0, 8.0],
    4: [0.0, 1e-6, 5e-4, 0.002, 0.3, 1.0, 2.5, 3.0 - 2e-5, 3.0 - 5e-6, 3.0, 3.0 + 5e-6, 3.0 + 2e-5, 3.5, 6.0, 10.6],
    6: [0.0, 1e-6, 5e-4, 0.002, 0.3, 1.0, 2.5, 3.0, 3.5, 6.0, 11.0],
    8: [0.0, 1e-6, 5e-4, 0.002, 0.3, 1.0, 2.5, 3.204471924659902 - 2e-5, 3.204471924659902 - 5e-6,
        3.204471924659902 + 5e-6, 3.204471924659902 + 2e-5, 3.5, 6.0, 11.3],
}
KS = [(0.0, 0.0), (1e-3, 0.0), (0.1, 0.0), (0.5, 0.3), (1.0, 1.0), (math.pi / 2, 0.7), (2.5, 1.0), (3.0, 2.9),
      (math.pi, 0.0), (math.pi, math.pi / 2), (math.pi, math.pi)]


def main():
    exe = build_lgf1unb()
    if exe is None:
        raise SystemExit("the reference tree or g++ is missing")
    lines = []
    for kind, cs in CS.items():
        for c in cs:
            for n in NS:
                lines.append(f"{kind} {n} {c!r} 0.0")
    for kind in (41, 42, 61, 62):
        for k1, k2 in KS:
            for n in NS:
                lines.append(f"{kind} {n} {k1!r} {k2!r}")
    out = subprocess.run([str(exe)], input="\n".join(lines) + "\n", capture_output=True, text=True, check=True).stdout
    rows = []
    for l in out.splitlines():
        k, n, a, b, v = l.split()
        rows.append([int(k), int(n), float(a), float(b), float(v)])
    dst = Path(__file__).resolve().parent / "lgf1unb_ref.json"
    dst.write_text(json.dumps({"source": "src/lgf_1unb2spe.hpp compiled by oracle/build_ref.py", "rows": rows}) + "\n")
    print(f"{len(rows)} rows -> {dst}")


if __name__ == "__main__":
    main()
