// Stand-in for the reference's src/defines.hpp when its 1-D lattice Green's
// function header (src/lgf_1unb2spe.hpp) is compiled alone for the oracle's
// golden values: that header only needs printf and abort from it.  Found
// first because oracle/build_ref.py compiles with -I oracle/ref_shim -I-.
#pragma once
#include <cstdio>
#include <cstdlib>
