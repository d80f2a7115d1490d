"""The C-ABI library loads and exports every entry point include/*.h declares.

CPU-only: no call here touches CUDA except through a child process that must
fail loudly when no device is present.
"""
import ctypes
import re
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
LIB = ROOT / "flups_b200" / "libflups_b200.so"


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(flups_\w+)\s*\(", text, flags=re.M):
            if "static inline" in text[max(0, m.start() - 0):m.end()].split("\n")[0]:
                continue
            names.add(m.group(1))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    if not LIB.exists():
        subprocess.run([sys.executable, "-m", "flups_b200.build"], cwd=ROOT, check=True)
    return ctypes.CDLL(str(LIB))


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 56
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_topology_layout_math():
    sys.path.insert(0, str(ROOT))
    from flups_b200 import pyflups as pf
    t = pf.Topology(0, 3, [17, 9, 5])
    assert [t.get_nglob(d) for d in range(3)] == [17, 9, 5]
    assert [t.get_nmem(d) for d in range(3)] == [17, 9, 5]  # 8-byte alignment: no padding for doubles
    assert t.memsize == 17 * 9 * 5 * 3
    t2 = pf.Topology(1, 1, [16, 16, 16], is_complex=True, alignment=64)
    # 16 complex doubles = 256 bytes along the axis: already a multiple of 64
    assert t2.get_nmem(1) == 16 and t2.is_complex
    t3 = pf.Topology(0, 1, [17, 8, 8], alignment=64)
    assert t3.get_nmem(0) == 24  # padded to 64 bytes (src/Topology.cpp:81-98)


def test_pencil_dirs():
    sys.path.insert(0, str(ROOT))
    from flups_b200 import pyflups as pf
    B = pf.BoundaryType
    # plan types: UNB/UNB=8, PER/PER=6, EVEN/ODD=1 -> sorted 2, 1, 0
    assert pf.pencil_dirs([[B.UNB, B.UNB], [B.PER, B.PER], [B.EVEN, B.ODD]]) == [2, 1, 0]
    assert pf.pencil_dirs([[B.UNB, B.UNB]] * 3) == [0, 1, 2]


def test_no_device_fails_loudly():
    """Without a GPU the solver must refuse to run (there is no CPU fallback)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "from flups_b200 import pyflups as pf\n"
        "t = pf.Topology(0, 1, [8, 8, 8])\n"
        "B = pf.BoundaryType\n"
        "s = pf.Solver(t, [[B.UNB, B.UNB]] * 3, [1/8]*3, [1.0]*3)\n"
        "s.setup()\n" % str(ROOT)
    )
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True)
    assert r.returncode != 0
    assert "no CUDA device" in r.stderr
