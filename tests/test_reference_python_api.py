"""The reference's own Python front-end (python_api/pyflups: flups_wrapper.py
binds the C symbols with ctypes, flups.py wraps them in classes) loaded
unmodified on top of libflups_b200.so, as a user of the reference would: the
library found through FLUPS_LIB_PATH under the name it looks for
(libflups.so).  mpi4py is not in this image, so a one-rank stand-in module
provides COMM_WORLD.  Everything up to flups_setup runs on the CPU: topology
getters, solver construction with the spectral information, the index
helper, hdf5_dump and print_data; the values must equal those of the
library's own front-end (flups_b200/pyflups.py).  Skipped where the
reference tree is absent (it is read, never copied)."""
import importlib
import os
import sys
import types
from pathlib import Path

import numpy as np
import pytest

REF_API = Path("/root/reference/python_api")
LIB = Path(__file__).resolve().parent.parent / "flups_b200" / "libflups_b200.so"

pytestmark = pytest.mark.skipif(not (REF_API / "pyflups" / "flups_wrapper.py").exists() or not LIB.exists(),
                                reason="the reference's python_api tree or the built library is absent")


def _fake_mpi4py():
    """A one-rank mpi4py: COMM_WORLD with a null handle (the library takes a
    size-1 communicator and ignores the handle)."""
    class Comm:
        handle = 0

        def Get_rank(self):
            return 0

        def Get_size(self):
            return 1

        def Barrier(self):
            return None

    mpi = types.ModuleType("mpi4py.MPI")
    mpi.Comm = Comm
    mpi.COMM_WORLD = Comm()
    mpi.Comm.f2py = staticmethod(lambda h: mpi.COMM_WORLD)
    mpi.Comm.fromhandle = staticmethod(lambda h: mpi.COMM_WORLD)
    pkg = types.ModuleType("mpi4py")
    pkg.MPI = mpi
    return pkg, mpi


@pytest.fixture()
def ref_pyflups(tmp_path, monkeypatch):
    (tmp_path / "libflups.so").symlink_to(LIB)
    monkeypatch.setenv("FLUPS_LIB_PATH", str(tmp_path))
    pkg, mpi = _fake_mpi4py()
    monkeypatch.setitem(sys.modules, "mpi4py", pkg)
    monkeypatch.setitem(sys.modules, "mpi4py.MPI", mpi)
    monkeypatch.syspath_prepend(str(REF_API))
    for name in [m for m in sys.modules if m == "pyflups" or m.startswith("pyflups.")]:
        monkeypatch.delitem(sys.modules, name)
    mod = importlib.import_module("pyflups")
    yield mod
    for name in [m for m in sys.modules if m == "pyflups" or m.startswith("pyflups.")]:
        sys.modules.pop(name, None)


def test_reference_front_end_runs_on_the_new_library(ref_pyflups, tmp_path, monkeypatch, capfd):
    rp = ref_pyflups
    from flups_b200 import pyflups as ours
    nglob = [16, 12, 8]
    topo = rp.Topology(0, 1, nglob, [1, 1, 1])
    mine = ours.Topology(0, 1, nglob)
    for d in range(3):
        assert topo.get_nglob(d) == mine.get_nglob(d) == nglob[d]
        assert topo.get_nmem(d) == mine.get_nmem(d)
    assert topo.memsize == mine.memsize and topo.locsize == mine.locsize and topo.is_complex == mine.is_complex
    # a solver with mixed boundary conditions: EVEN/ODD x, PER y, UNB z
    B = rp.BoundaryType
    bc = [[B.EVEN, B.ODD], [B.PER, B.PER], [B.UNB, B.UNB]]
    h = [1.0 / 16] * 3
    L = [1.0, 0.75, 0.5]
    s = rp.Solver(topo, bc, h, L, rp.DiffType.NOD, [rp.CenterType.CELL_CENTER] * 3)
    s.set_green_type(rp.GreenType.HEJ_4)
    s.set_alpha(2.0)
    kf, ko, ss = s.get_spectral_info()
    OB = ours.BoundaryType
    so = ours.Solver(mine, [[OB.EVEN, OB.ODD], [OB.PER, OB.PER], [OB.UNB, OB.UNB]], h, L)
    kf2, ko2, ss2 = so.get_spectral_info()
    assert np.allclose(kf, kf2, rtol=0, atol=0) and np.allclose(ko, ko2, rtol=0, atol=0) and np.allclose(ss, ss2)
    assert s.get_alloc_size() == so.get_alloc_size()
    # the index helper of the reference's front-end (flups_locID)
    nmem = [topo.get_nmem(d) for d in range(3)]
    assert rp.locID(0, 3, 2, 1, 0, 0, nmem, 1) == 3 + nmem[0] * (2 + nmem[1] * 1)
    # field output: flups_hdf5_dump writes ./data/<name> (raw doubles + XDMF here, no HDF5)
    monkeypatch.chdir(tmp_path)
    data = np.arange(topo.memsize, dtype=np.float64)
    rp.hdf5_dump(topo, "field", data)
    back = np.fromfile(tmp_path / "data" / "field.bin", dtype=np.float64)
    assert np.array_equal(back, data)
    xmf = (tmp_path / "data" / "field.xmf").read_text()
    assert "field.bin" in xmf and f"{nmem[2]} {nmem[1]} {nmem[0]}" in xmf
    capfd.readouterr()
    small = rp.Topology(0, 1, [3, 2, 1], [1, 1, 1])
    rp.print_data(small, np.arange(small.memsize, dtype=np.float64))
    out = capfd.readouterr().out
    assert out.count("\n") == 2 and "+5.000000e+00" in out
    del s, so, topo, mine, small
