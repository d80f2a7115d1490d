"""Build libflups_b200.so in-tree with nvcc for sm_100a.

    python -m flups_b200.build          (or flups_b200.build.build())

Steps: turn kernel/farfield.json into a C include of coefficient tables,
then compile csrc/*.cu and csrc/*.cpp into flups_b200/libflups_b200.so.
"""
import json
import math
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libflups_b200.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def gen_farfield():
    data = json.loads((PKG / "kernel" / "farfield.json").read_text())
    lines = ["// generated from kernel/farfield.json by build.py -- do not edit"]
    entries = []
    for name, ent in data.items():
        coefs = [t[0] * math.pi ** t[5] for t in ent["terms"]]
        exps = []
        for t in ent["terms"]:
            exps += [int(t[1]), int(t[2]), int(t[3]), int(t[4])]
        logc = sum(t[0] for t in ent["log_terms"])
        lines.append(f"static const double ff_{name}_c[] = {{{', '.join(repr(c) for c in coefs)}}};")
        lines.append(f"static const int ff_{name}_e[] = {{{', '.join(str(e) for e in exps)}}};")
        entries.append(f'    {{"{name}", {ent["ndim"]}, {len(coefs)}, ff_{name}_c, ff_{name}_e, {logc!r}}},')
    lines.append("static const FarTable kFarTables[] = {")
    lines += entries
    lines.append("};")
    BUILD.mkdir(exist_ok=True)
    out = BUILD / "farfield_data.inc"
    text = "\n".join(lines) + "\n"
    if not out.exists() or out.read_text() != text:
        out.write_text(text)
    return out


def sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def build(verbose=False, extra=()):
    gen_farfield()
    objs, jobs = [], []
    for src in sources():
        obj = BUILD / (src.stem + ".o")
        deps = [src] + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp")) + \
            list((PKG.parent / "include").glob("*.h")) + [BUILD / "farfield_data.inc"]
        if not obj.exists() or any(d.stat().st_mtime > obj.stat().st_mtime for d in deps):
            cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", str(BUILD),
                   "-I", str(PKG.parent / "include"), "--expt-relaxed-constexpr", *extra]
            if src.suffix == ".cpp":
                cmd += ["-x", "cu"]
            cmd += ["-c", str(src), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            jobs.append(cmd)
        objs.append(obj)
    # the translation units are independent: compile them side by side
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
        for r in ex.map(lambda c: subprocess.run(c), jobs):
            if r.returncode != 0:
                raise subprocess.CalledProcessError(r.returncode, r.args)
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [NVCC, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart", "-ldl"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))
