"""B200-native FLUPS solve path.

The product is the shared library ``libflups_b200.so`` (hand-written CUDA for
sm_100a behind the reference's C ABI, headers in ``include/``); this package
holds its sources (``csrc/``), build recipe (``build.py``), the lattice
Green's function data (``kernel/``) and a Python front-end (``pyflups``).
"""
__all__ = ["pyflups"]
