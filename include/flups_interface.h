/*
 * flups_interface.h -- enums and constants of the FLUPS C API.
 *
 * Values are fixed by the reference interface (vortexlab-uclouvain/flups,
 * src/flups_interface.h:14-110) so that code compiled against the reference
 * header passes the same integers to this library.
 */
#ifndef FLUPS_INTERFACE_H_
#define FLUPS_INTERFACE_H_

/* transform signs (src/flups_interface.h:14-26) */
#define FLUPS_FORWARD -1
#define FLUPS_BACKWARD 1
#define FLUPS_BACKWARD_DIFF 2

/* alignment in bytes of the user topologies (src/flups_interface.h:32) */
#define FLUPS_ALIGNMENT 8

/* boundary conditions (src/flups_interface.h:46-52) */
enum BoundaryType { EVEN = 0, ODD = 1, PER = 3, UNB = 4, NONE = 9 };

/* Green's kernels (src/flups_interface.h:58-74) */
enum GreenType {
    CHAT_2 = 0,
    LGF_2 = 1,
    HEJ_2 = 2,
    HEJ_4 = 3,
    HEJ_6 = 4,
    HEJ_8 = 5,
    HEJ_10 = 6,
    HEJ_0 = 7,
    LGF_4 = 8,
    LGF_6 = 9,
    LGF_8 = 10,
    MEHR_4L = 11,
    MEHR_6L = 12,
    MEHR_4F = 13,
    MEHR_6F = 14
};

/* solve kinds: STD = grad^2 phi = f, ROT = grad^2 phi = curl f (src/flups_interface.h:85-88) */
enum SolverType { STD = 0, ROT = 1 };

/* derivative used by ROT (src/flups_interface.h:95-101) */
enum DiffType { NOD = 0, SPE = 1, FD2 = 2, FD4 = 4, FD6 = 6 };

/* data location (src/flups_interface.h:107-110) */
enum CenterType { NODE_CENTER = 0, CELL_CENTER = 1 };

#endif
