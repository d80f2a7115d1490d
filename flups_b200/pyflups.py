"""Python front-end of libflups_b200.so, mirroring the reference's object
interface (python_api/pyflups/flups.py: Topology, Profiler, Solver with
set_green_type / set_alpha / setup / solve / get_alloc_size /
get_spectral_info) over the same C symbols.

Differences: no mpi4py (one rank; ``comm`` is ignored), arrays may be numpy
arrays (host) or CUDA torch tensors (device pointers are passed through), and
the added calls set_precision / solve_batch / device_bytes map to
include/flups_b200.h.  The library must be built (``python -m
flups_b200.build``); importing without it raises.
"""
import ctypes
from ctypes import POINTER, c_bool, c_double, c_int, c_size_t, c_void_p
from enum import IntEnum
from pathlib import Path

import numpy as np

_LIB_PATH = Path(__file__).resolve().parent / "libflups_b200.so"


class BoundaryType(IntEnum):
    EVEN = 0
    ODD = 1
    PER = 3
    UNB = 4
    NONE = 9


class GreenType(IntEnum):
    CHAT_2 = 0
    LGF_2 = 1
    HEJ_2 = 2
    HEJ_4 = 3
    HEJ_6 = 4
    HEJ_8 = 5
    HEJ_10 = 6
    HEJ_0 = 7
    LGF_4 = 8
    LGF_6 = 9
    LGF_8 = 10
    MEHR_4L = 11
    MEHR_6L = 12
    MEHR_4F = 13
    MEHR_6F = 14


class SolverType(IntEnum):
    STD = 0
    ROT = 1


class DiffType(IntEnum):
    NOD = 0
    SPE = 1
    FD2 = 2
    FD4 = 4
    FD6 = 6


class CenterType(IntEnum):
    NODE_CENTER = 0
    CELL_CENTER = 1


FLUPS_FORWARD, FLUPS_BACKWARD, FLUPS_BACKWARD_DIFF, FLUPS_ALIGNMENT = -1, 1, 2, 8

_lib = None


def load_library(path=None):
    """Load libflups_b200.so and declare the C signatures; raises if absent."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else _LIB_PATH
    if not p.exists():
        raise ImportError(f"{p} is missing: build it with `python -m flups_b200.build` (there is no CPU fallback)")
    lib = ctypes.CDLL(str(p))
    vp, ip, dp = c_void_p, POINTER(c_int), POINTER(c_double)
    sig = {
        "flups_malloc": (vp, [c_size_t]),
        "flups_free": (None, [vp]),
        "flups_topo_new": (vp, [c_int, c_int, ip, ip, c_bool, ip, c_int, ctypes.c_ssize_t]),
        "flups_topo_free": (None, [vp]),
        "flups_topo_get_isComplex": (c_bool, [vp]),
        "flups_topo_get_lda": (c_int, [vp]),
        "flups_topo_get_axis": (c_int, [vp]),
        "flups_topo_get_nglob": (c_int, [vp, c_int]),
        "flups_topo_get_nloc": (c_int, [vp, c_int]),
        "flups_topo_get_nmem": (c_int, [vp, c_int]),
        "flups_topo_get_nproc": (c_int, [vp, c_int]),
        "flups_topo_get_istartGlob": (None, [vp, ip]),
        "flups_topo_get_locsize": (c_size_t, [vp]),
        "flups_topo_get_memsize": (c_size_t, [vp]),
        "flups_topo_cmpt_rank_fromid": (c_int, [vp, c_int, c_int]),
        "flups_topo_cmpt_start_id_from_rank": (c_int, [vp, c_int, c_int]),
        "flups_init": (vp, [vp, POINTER(POINTER(c_int)), dp, dp, c_int, ip]),
        "flups_init_timed": (vp, [vp, POINTER(POINTER(c_int)), dp, dp, c_int, ip, vp]),
        "flups_cleanup_solver": (None, [vp]),
        "flups_cleanup_backend": (None, []),
        "flups_set_greenType": (None, [vp, c_int]),
        "flups_set_alpha": (None, [vp, c_double]),
        "flups_set_stream": (None, [vp, vp]),
        "flups_setup": (None, [vp, c_bool]),
        "flups_solve": (None, [vp, vp, vp, c_int]),
        "flups_solve_batch": (None, [vp, vp, vp, c_int, c_int]),
        "flups_get_allocSize": (c_size_t, [vp]),
        "flups_get_spectralInfo": (None, [vp, dp, dp, dp]),
        "flups_pencilDirs": (None, [POINTER(POINTER(c_int)), ip]),
        "flups_set_precision": (None, [vp, c_int]),
        "flups_get_precision": (c_int, [vp]),
        "flups_set_async": (None, [vp, c_int]),
        "flups_synchronize": (None, [vp]),
        "flups_b200_set_autotune": (None, [vp, c_int]),
        "flups_b200_set_col_tile": (None, [vp, c_int]),
        "flups_b200_set_overlap": (None, [vp, c_int]),
        "flups_b200_set_prefetch": (None, [vp, c_int]),
        "flups_b200_set_xlast": (None, [vp, c_int]),
        "flups_b200_slab_info": (c_int, [vp, POINTER(ctypes.c_int64)]),
        "flups_b200_slab_own": (c_int, [vp, c_int, c_int, c_int, c_int]),
        "flups_b200_slab_planes": (vp, [vp]),
        "flups_b200_slab_columns": (vp, [vp]),
        "flups_b200_slab_forward": (c_int, [vp, vp]),
        "flups_b200_slab_fused": (c_int, [vp, c_int]),
        "flups_b200_slab_backward": (c_int, [vp, vp, c_int]),
        "flups_b200_slab_peers": (c_int, [vp, c_int, POINTER(vp), ip, POINTER(ctypes.c_int64)]),
        "flups_b200_ipc_handle": (c_int, [vp, vp]),
        "flups_b200_ipc_open": (c_int, [vp, POINTER(vp)]),
        "flups_b200_ipc_close": (c_int, [vp]),
        "flups_get_innerBuffer": (vp, [vp]),
        "flups_get_innerTopo_physical": (vp, [vp]),
        "flups_get_innerTopo_spectral": (vp, [vp]),
        "flups_do_copy": (None, [vp, vp, vp, c_int]),
        "flups_do_FFT": (None, [vp, vp, c_int]),
        "flups_do_mult": (None, [vp, vp, c_int]),
        "flups_solve_graph": (c_int, [vp, vp, vp, c_int, c_int]),
        "flups_b200_solve_group": (c_int, [POINTER(vp), c_int, POINTER(vp), POINTER(vp), ip, vp]),
        "flups_get_last_error": (c_int, [vp]),
        "flups_get_device_bytes": (c_size_t, [vp, c_int]),
        "flups_b200_plan_json": (c_int, [vp, c_int, c_int, ctypes.c_char_p, c_int]),
        "flups_set_pass_timing": (None, [vp, c_int]),
        "flups_get_pass_stats": (c_int, [vp, c_int, dp, dp, POINTER(ctypes.c_long), ctypes.c_char_p, c_int]),
        "flups_profiler_new_n": (vp, [ctypes.c_char_p]),
        "flups_profiler_free": (None, [vp]),
        "flups_profiler_disp": (None, [vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _ptr(a):
    """Raw address of a numpy array or a torch tensor (host or device)."""
    if hasattr(a, "data_ptr"):
        return c_void_p(a.data_ptr())
    return c_void_p(a.ctypes.data)


class Topology:
    """src/flups.h:210-349 (pyflups Topology)."""

    def __init__(self, axis, lda, nglob, nproc=(1, 1, 1), is_complex=False, axproc=None, alignment=FLUPS_ALIGNMENT,
                 comm=None):
        lib = load_library()
        ng = (c_int * 3)(*nglob)
        npr = (c_int * 3)(*nproc)
        axp = (c_int * 3)(*axproc) if axproc is not None else None
        self._topo = lib.flups_topo_new(axis, lda, ng, npr, bool(is_complex), axp, alignment, 0)

    def __del__(self):
        if getattr(self, "_topo", None) and _lib is not None:
            _lib.flups_topo_free(self._topo)
            self._topo = None

    @classmethod
    def _borrowed(cls, ptr):
        """A topology owned by a solver (flups_get_innerTopo_*): never freed here."""
        t = cls.__new__(cls)
        t._topo = None
        t._view = ptr
        return t

    @property
    def _ptr(self):
        return self._topo if self._topo else getattr(self, "_view", None)

    @property
    def lda(self):
        return _lib.flups_topo_get_lda(self._ptr)

    @property
    def axis(self):
        return _lib.flups_topo_get_axis(self._ptr)

    @property
    def is_complex(self):
        return bool(_lib.flups_topo_get_isComplex(self._ptr))

    def get_nglob(self, dim):
        return _lib.flups_topo_get_nglob(self._ptr, dim)

    def get_nloc(self, dim):
        return _lib.flups_topo_get_nloc(self._ptr, dim)

    def get_nmem(self, dim):
        return _lib.flups_topo_get_nmem(self._ptr, dim)

    def get_nproc(self, dim):
        return _lib.flups_topo_get_nproc(self._ptr, dim)

    def get_istart(self):
        a = (c_int * 3)()
        _lib.flups_topo_get_istartGlob(self._ptr, a)
        return np.array(a[:])

    @property
    def locsize(self):
        return _lib.flups_topo_get_locsize(self._ptr)

    @property
    def memsize(self):
        return _lib.flups_topo_get_memsize(self._ptr)


class Profiler:
    def __init__(self, name="default"):
        self._prof = load_library().flups_profiler_new_n(name.encode())

    def __del__(self):
        if getattr(self, "_prof", None) and _lib is not None:
            _lib.flups_profiler_free(self._prof)
            self._prof = None

    def display(self):
        _lib.flups_profiler_disp(self._prof)

    @property
    def _ptr(self):
        return self._prof


class Solver:
    """src/flups.h:369-578 (pyflups Solver).

    ``boundary_conditions[d][side]`` is one BoundaryType, or a list with one
    BoundaryType per component.
    """

    def __init__(self, topology, boundary_conditions, h, L, order_diff=DiffType.NOD, center_type=None, profiler=None):
        lib = load_library()
        self._topology = topology
        lda = topology.lda
        self._bc_arrays = []
        for d in range(3):
            for s in range(2):
                v = boundary_conditions[d][s]
                vals = list(v) if isinstance(v, (list, tuple)) else [v] * lda
                self._bc_arrays.append((c_int * lda)(*[int(x) for x in vals]))
        self._bc = (POINTER(c_int) * 6)(*[ctypes.cast(a, POINTER(c_int)) for a in self._bc_arrays])
        hh = (c_double * 3)(*h)
        LL = (c_double * 3)(*L)
        ct = (c_int * 3)(*[int(c) for c in (center_type or [CenterType.CELL_CENTER] * 3)])
        if profiler is None:
            self._solver = lib.flups_init(topology._ptr, self._bc, hh, LL, int(order_diff), ct)
        else:
            self._solver = lib.flups_init_timed(topology._ptr, self._bc, hh, LL, int(order_diff), ct, profiler._ptr)

    def __del__(self):
        if getattr(self, "_solver", None) and _lib is not None:
            _lib.flups_cleanup_solver(self._solver)
            self._solver = None

    def set_green_type(self, green_type):
        _lib.flups_set_greenType(self._solver, int(green_type))

    def set_alpha(self, alpha):
        _lib.flups_set_alpha(self._solver, float(alpha))

    def set_precision(self, bits):
        _lib.flups_set_precision(self._solver, int(bits))

    def set_stream(self, stream):
        """stream: a torch.cuda.Stream or a raw cudaStream_t address."""
        raw = getattr(stream, "cuda_stream", stream)
        _lib.flups_set_stream(self._solver, c_void_p(raw))

    def set_async(self, flag):
        _lib.flups_set_async(self._solver, int(bool(flag)))

    def synchronize(self):
        _lib.flups_synchronize(self._solver)

    # ---- advanced API (src/flups.h:473-578)
    def get_inner_buffer(self):
        """The solver's inner buffer (managed memory: host- and device-accessible)
        as a numpy array of doubles, sized for both inner layouts."""
        ptr = _lib.flups_get_innerBuffer(self._solver)
        topo_s = self.get_inner_topo_spectral()
        n = max(topo_s.memsize, self._topology.memsize)
        return np.ctypeslib.as_array((ctypes.c_double * n).from_address(ptr))

    def get_inner_topo_physical(self):
        return Topology._borrowed(_lib.flups_get_innerTopo_physical(self._solver))

    def get_inner_topo_spectral(self):
        return Topology._borrowed(_lib.flups_get_innerTopo_spectral(self._solver))

    def do_copy(self, topology, data, sign):
        _lib.flups_do_copy(self._solver, topology._ptr, _ptr(data), int(sign))

    def do_fft(self, data, sign):
        _lib.flups_do_FFT(self._solver, _ptr(data), int(sign))

    def do_mult(self, data, solver_type=SolverType.STD):
        _lib.flups_do_mult(self._solver, _ptr(data), int(solver_type))

    def set_autotune(self, on):
        _lib.flups_b200_set_autotune(self._solver, int(bool(on)))

    def set_overlap(self, on):
        """Overlap the per-x-slab middle passes on three streams (device arrays, STD)."""
        _lib.flups_b200_set_overlap(self._solver, int(bool(on)))

    def set_prefetch(self, on):
        """L2 prefetch of the next blocks' input in the row / column passes (default on)."""
        _lib.flups_b200_set_prefetch(self._solver, int(bool(on)))

    def set_xlast(self, on):
        """Pass order of all-unbounded 3-D device-array solves: x last (default) or the reference's x first."""
        _lib.flups_b200_set_xlast(self._solver, int(bool(on)))

    # ---- one rank's share of a z-slab decomposed solve (flups_b200/slab.py drives it)
    def slab_info(self):
        """(code, spectrum extents (nx, ny, nz), plane-array row pitch, user planes, column-array row pitch,
        bytes per real); code 0 when the problem qualifies."""
        info = (ctypes.c_int64 * 7)()
        code = _lib.flups_b200_slab_info(self._solver, info)
        return code, (info[0], info[1], info[2]), info[3], info[4], info[5], info[6]

    def slab_own(self, z0, z1, x0, x1):
        """Before setup: the planes [z0, z1) and spectrum columns [x0, x1) this solver owns."""
        return _lib.flups_b200_slab_own(self._solver, int(z0), int(z1), int(x0), int(x1))

    def slab_planes_ptr(self):
        return _lib.flups_b200_slab_planes(self._solver)

    def slab_columns_ptr(self):
        return _lib.flups_b200_slab_columns(self._solver)

    def slab_forward(self, rhs):
        return _lib.flups_b200_slab_forward(self._solver, _ptr(rhs))

    def slab_fused(self, solver_type=SolverType.STD):
        return _lib.flups_b200_slab_fused(self._solver, int(solver_type))

    def slab_backward(self, field, solver_type=SolverType.STD):
        return _lib.flups_b200_slab_backward(self._solver, _ptr(field), int(solver_type))

    def slab_peers(self, cols, xs, pitches):
        """Every rank's column array (device addresses), the column split xs (n + 1 values) and
        the arrays' row pitches; an empty list goes back to the plane array."""
        n = len(cols)
        c = (c_void_p * max(1, n))(*[c_void_p(int(p)) for p in cols])
        x = (c_int * (n + 1))(*[int(v) for v in xs] if n else [0])
        pt = (ctypes.c_int64 * max(1, n))(*[int(v) for v in pitches])
        return _lib.flups_b200_slab_peers(self._solver, n, c, x, pt)

    def set_col_tile(self, tile):
        """0 default/tuned, 1: 256-thread tiles, 2: 128-thread tiles (cross-checks)."""
        _lib.flups_b200_set_col_tile(self._solver, int(tile))

    def solve_graph(self, field, rhs, nbatch=1, solver_type=SolverType.STD):
        """Device arrays only; replays a captured CUDA graph after the first call."""
        rc = _lib.flups_solve_graph(self._solver, _ptr(field), _ptr(rhs), int(nbatch), int(solver_type))
        if rc != 0:
            raise RuntimeError(f"flups_solve_graph returned {rc} (CUDA error {self.last_error()})")
        return field

    def setup(self, change_comm=False):
        _lib.flups_setup(self._solver, bool(change_comm))

    def solve(self, field, rhs, solver_type=SolverType.STD):
        _lib.flups_solve(self._solver, _ptr(field), _ptr(rhs), int(solver_type))
        return field

    def solve_batch(self, field, rhs, nbatch, solver_type=SolverType.STD):
        _lib.flups_solve_batch(self._solver, _ptr(field), _ptr(rhs), int(nbatch), int(solver_type))
        return field

    def get_alloc_size(self):
        return _lib.flups_get_allocSize(self._solver)

    def device_bytes(self, nbatch=1):
        return _lib.flups_get_device_bytes(self._solver, int(nbatch))

    def last_error(self):
        return _lib.flups_get_last_error(self._solver)

    def plan_json(self, solver_type=SolverType.STD, nbatch=1):
        """Host-only description of the per-direction tables and the passes of one solve (no GPU needed)."""
        import json
        n = _lib.flups_b200_plan_json(self._solver, int(solver_type), int(nbatch), None, 0)
        buf = ctypes.create_string_buffer(n)
        _lib.flups_b200_plan_json(self._solver, int(solver_type), int(nbatch), buf, n)
        return json.loads(buf.value.decode())

    def set_pass_timing(self, on):
        _lib.flups_set_pass_timing(self._solver, int(bool(on)))

    def pass_stats(self):
        """Per pass of one solve: name, accumulated ms, algorithmic bytes per launch, timed launches."""
        n = _lib.flups_get_pass_stats(self._solver, 0, None, None, None, None, 0)
        ms, by, ca = (c_double * n)(), (c_double * n)(), (ctypes.c_long * n)()
        names = ctypes.create_string_buffer(32 * n)
        _lib.flups_get_pass_stats(self._solver, n, ms, by, ca, names, 32)
        out = []
        for k in range(n):
            nm = names.raw[32 * k:32 * (k + 1)].split(b"\0")[0].decode()
            out.append({"name": nm, "ms_total": ms[k], "bytes": by[k], "calls": ca[k]})
        return out

    def get_spectral_info(self):
        kf, ko, ss = (c_double * 3)(), (c_double * 3)(), (c_double * 3)()
        _lib.flups_get_spectralInfo(self._solver, kf, ko, ss)
        return np.array(kf[:]), np.array(ko[:]), np.array(ss[:])


def pencil_dirs(boundary_conditions):
    """flups_pencilDirs (src/flups.h:570)."""
    lib = load_library()
    arrs = [(c_int * 1)(int(boundary_conditions[d][s])) for d in range(3) for s in range(2)]
    bc = (POINTER(c_int) * 6)(*[ctypes.cast(a, POINTER(c_int)) for a in arrs])
    dirs = (c_int * 3)()
    lib.flups_pencilDirs(bc, dirs)
    return list(dirs)


def solve_group(solvers, fields, rhss, types=None, stream=None):
    """flups_b200_solve_group: the solves of several solvers (device arrays,
    different grids allowed) as one CUDA graph on `stream` (a torch stream or
    None); returns the library's code (0 on success)."""
    n = len(solvers)
    types = [int(SolverType.STD)] * n if types is None else [int(t) for t in types]
    sv = (c_void_p * n)(*[s._solver for s in solvers])
    fv = (c_void_p * n)(*[_ptr(f).value for f in fields])
    rv = (c_void_p * n)(*[_ptr(r).value for r in rhss])
    tv = (c_int * n)(*types)
    st = c_void_p(stream.cuda_stream) if stream is not None else None
    return _lib.flups_b200_solve_group(sv, n, fv, rv, tv, st)
