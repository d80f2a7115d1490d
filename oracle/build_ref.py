"""Compile the reference's own code from its sources, where it lies, into
oracle/_ref/ (git-ignored; test infrastructure only).  Nothing of the
reference is copied into this repository.

    python -m oracle.build_ref [REFERENCE_ROOT]

flups: the reference's solver library, every src/*.cpp compiled unmodified
against the stand-ins in oracle/ref_build/ (an FFTW-API subset on our own
FP64 FFT, a one-rank MPI, minimal h3lpr headers; FFTW, MPI and h3lpr are not
installed here), linked with oracle/ref_build/ref_driver.cpp into
oracle/_ref/libflups_ref.so.  Built with hidden visibility and -Bsymbolic:
only the driver's flups_ref_* entry points are exported, so the reference's
own flups_* names cannot clash with the product library in one process.
KERNEL_PATH points the lattice kernels at flups_b200/kernel (the same .ker
tables, present wherever the repository is).

lgf1unb: the reference's header of 1-D lattice Green's functions
(src/lgf_1unb2spe.hpp) with the driver oracle/ref_lgf1unb.cpp.  The header
includes "defines.hpp", which pulls in FFTW, MPI and h3lpr (absent here);
-I oracle/ref_shim -I- makes the quoted include find oracle/ref_shim's
stand-in first (the header itself only uses printf and abort from it).

Each builder returns the path of what it built, or None when the reference
or g++ is missing (the GPU box has no reference tree; there the library
built here travels with the repository).
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


def build_flups(ref=DEFAULT_REF, jobs=8):
    src_dir = Path(ref) / "src"
    gxx = shutil.which("g++")
    lib = OUT / "libflups_ref.so"
    if not src_dir.is_dir() or gxx is None:
        return lib if lib.exists() else None
    shim = HERE / "ref_build"
    kernels = HERE.parent / "flups_b200" / "kernel"
    srcs = sorted(src_dir.glob("*.cpp")) + [shim / "ref_driver.cpp", shim / "fft_shim.cpp", shim / "mpi_shim.cpp"]
    deps = srcs + sorted(src_dir.glob("*.h*")) + sorted(src_dir.glob("*.ipp")) + sorted(shim.rglob("*.h*"))
    if lib.exists() and lib.stat().st_mtime > max(p.stat().st_mtime for p in deps):
        return lib
    obj_dir = OUT / "obj"
    obj_dir.mkdir(parents=True, exist_ok=True)
    flags = ["-O3", "-std=c++17", "-fopenmp", "-fPIC", "-fvisibility=hidden", "-I", str(shim), "-I", str(src_dir),
             f"-DKERNEL_PATH={kernels}"]
    objs, procs = [], []
    for s in srcs:
        o = obj_dir / (("ref_" if s.parent == src_dir else "shim_") + s.stem + ".o")
        objs.append(o)
        procs.append(subprocess.Popen([gxx, *flags, "-c", str(s), "-o", str(o)], stderr=subprocess.PIPE))
        if len(procs) >= jobs:
            _wait(procs.pop(0))
    for p in procs:
        _wait(p)
    subprocess.run([gxx, "-shared", "-fopenmp", "-Wl,-Bsymbolic", "-o", str(lib), *map(str, objs)], check=True)
    return lib


def _wait(p):
    _, err = p.communicate()
    if p.returncode != 0:
        raise RuntimeError("reference build failed:\n" + err.decode(errors="replace")[-4000:])


def build_fftshim():
    """oracle/ref_build/fft_shim.cpp alone, its FFTW-API names exported, so that
    the tests can check the stand-in FFT against scipy.fft before trusting the
    reference build that runs on it."""
    gxx = shutil.which("g++")
    src = HERE / "ref_build" / "fft_shim.cpp"
    lib = OUT / "libfftshim.so"
    if gxx is None:
        return lib if lib.exists() else None
    if lib.exists() and lib.stat().st_mtime > max(src.stat().st_mtime, (HERE / "ref_build" / "fftw3.h").stat().st_mtime):
        return lib
    OUT.mkdir(exist_ok=True)
    subprocess.run([gxx, "-O2", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-I", str(HERE / "ref_build"), str(src),
                    "-o", str(lib)], check=True)
    return lib


def build(ref=DEFAULT_REF):
    return {"lgf1unb": build_lgf1unb(ref), "flups": build_flups(ref), "fftshim": build_fftshim()}


if __name__ == "__main__":
    print(build(Path(sys.argv[1]) if len(sys.argv) > 1 else DEFAULT_REF))
