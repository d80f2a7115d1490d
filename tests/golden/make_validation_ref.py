"""Collect the reference's validation goldens into one committed fixture.

Source: samples/validation/data_ref/validation_3d_<Center>_<bccode>_typeGreen=<k>.txt
(error norms err2/errInf of the reference solver against manufactured
solutions, one line per resolution) and samples/solve_vtube/data_ref/*.txt.
Run once where the reference tree is present:

    python tests/golden/make_validation_ref.py /path/to/reference
"""
import json
import sys
from pathlib import Path


def read_dir(d):
    out = {}
    for f in sorted(Path(d).glob("*.txt")):
        rows = []
        for line in f.read_text().splitlines():
            parts = line.split()
            if not parts:
                continue
            rows.append([parts[0]] + [float(v) for v in parts[1:]])
        out[f.name] = rows
    return out


def main():
    ref = Path(sys.argv[1])
    data = {"validation": read_dir(ref / "samples/validation/data_ref"),
            "vtube": read_dir(ref / "samples/solve_vtube/data_ref")}
    dst = Path(__file__).with_name("validation_ref.json")
    dst.write_text(json.dumps(data, separators=(",", ":")))
    print(f"{len(data['validation'])} validation files, {len(data['vtube'])} vtube files -> {dst}")


if __name__ == "__main__":
    main()
