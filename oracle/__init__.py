"""CPU FP64 oracle for the FLUPS single-rank solve path.

TEST INFRASTRUCTURE ONLY.  This package restates, in numpy/scipy, the
algorithm of the reference solver (vortexlab-uclouvain/flups): the
per-direction transform tables (src/FFTW_plan_dim*.cpp), the Green's function
setup (src/green_functions.cpp, src/green_kernels.hpp), the spectral multiply
(src/dothemagic_std.ipp, src/dothemagic_rot.ipp) and the solve sequence
(src/Solver.cpp).  Each function cites the reference file:line it follows.

It is the checker for the CUDA library in ``flups_b200``: only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of ``bench.py`` may
import it.  The product never calls into it.

FFTW (the reference's transform library, unpinned version >= 3.3.8, not
vendored) is replaced by ``scipy.fft``: FFTW's REDFT00/10/01/11 and
RODFT00/10/01/11 kinds are scipy's unnormalised ``dct``/``dst`` types I-IV,
and FFTW's unnormalised r2c/c2r/c2c are scipy's ``rfft``/``irfft``/``fft``/
``ifft`` with ``norm="forward"`` on the inverse.

Parity pin: ``oracle.validation`` re-runs the reference's manufactured-solution
driver (samples/validation/src/validation_3d.cpp) and the tests compare its
error norms with the reference's golden files
(samples/validation/data_ref/*.txt, committed as tests/golden/validation_ref.json)
with the reference's own rule (scripts/check_res.py: 1e-10 relative).
"""
from .plans import *  # noqa: F401,F403
from .solver import OracleSolver  # noqa: F401
