"""Compile the pieces of the reference that build from their own sources
here, into oracle/_ref/ (git-ignored; test infrastructure only).

    python -m oracle.build_ref [REFERENCE_ROOT]

lgf1unb: the reference's header of 1-D lattice Green's functions
(src/lgf_1unb2spe.hpp) with the driver oracle/ref_lgf1unb.cpp.  The header
includes "defines.hpp", which pulls in FFTW, MPI and h3lpr (absent here);
-I oracle/ref_shim -I- makes the quoted include find oracle/ref_shim's
stand-in first (the header itself only uses printf and abort from it).
Returns the path of the built binary, or None when the reference or g++ is
missing (the GPU box has no reference tree).
"""
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
DEFAULT_REF = Path("/root/reference")


def build_lgf1unb(ref=DEFAULT_REF):
    src = Path(ref) / "src" / "lgf_1unb2spe.hpp"
    gxx = shutil.which("g++")
    if not src.exists() or gxx is None:
        return None
    OUT.mkdir(exist_ok=True)
    exe = OUT / "lgf1unb"
    drv = HERE / "ref_lgf1unb.cpp"
    if exe.exists() and exe.stat().st_mtime > max(drv.stat().st_mtime, src.stat().st_mtime):
        return exe
    cmd = [gxx, "-O2", "-std=c++17", "-I", str(HERE / "ref_shim"), "-I-", "-I", str(src.parent), str(drv), "-o", str(exe)]
    subprocess.run(cmd, check=True, stderr=subprocess.DEVNULL)
    return exe


def build(ref=DEFAULT_REF):
    return {"lgf1unb": build_lgf1unb(ref)}


if __name__ == "__main__":
    print(build(Path(sys.argv[1]) if len(sys.argv) > 1 else DEFAULT_REF))
