// Golden values of the reference's own 1-D lattice Green's functions
// (src/lgf_1unb2spe.hpp, compiled unmodified by oracle/build_ref.py): reads
// lines "kind n a b" from stdin and prints "kind n a b value" with 17
// significant digits.  kind 2/4/6/8: lgf<kind>(n, c = a); kind 41/61 (42/62):
// meh4/meh6 left (full) at (n, k1 = a, k2 = b).  Test infrastructure only.
#include <cstdio>

#include "lgf_1unb2spe.hpp"

int main() {
    int kind, n;
    double a, b;
    while (std::scanf("%d %d %lf %lf", &kind, &n, &a, &b) == 4) {
        double v = 0.0;
        switch (kind) {
            case 2: v = LGFOneUnbounded::lgf2(n, a); break;
            case 4: v = LGFOneUnbounded::lgf4(n, a); break;
            case 6: v = LGFOneUnbounded::lgf6(n, a); break;
            case 8: v = LGFOneUnbounded::lgf8(n, a); break;
            case 41: v = LGFOneUnbounded::meh4_left(n, a, b); break;
            case 42: v = LGFOneUnbounded::meh4_full(n, a, b); break;
            case 61: v = LGFOneUnbounded::meh6_left(n, a, b); break;
            case 62: v = LGFOneUnbounded::meh6_full(n, a, b); break;
            default: return 1;
        }
        std::printf("%d %d %.17g %.17g %.17g\n", kind, n, a, b, v);
    }
    return 0;
}
