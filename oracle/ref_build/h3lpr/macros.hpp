// Minimal stand-in for the h3lpr helper library's macros.hpp, enough for the
// reference's solver sources (src/defines.hpp and the files including it):
// assertions that print and abort (kept on in every build of the oracle),
// warnings to stderr, verbose logs and begin/end traces compiled out, and the
// small min/max/alignment helpers.  Like the library it stands in for, it
// brings in the system headers some reference sources use without including
// them (stat/mkdir, OpenMP).  Test infrastructure of the oracle only.
#pragma once
#include <stdint.h>
#include <sys/stat.h>
#include <sys/types.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include <cstdio>
#include <cstdlib>

#define m_min(a, b) (((a) < (b)) ? (a) : (b))
#define m_max(a, b) (((a) > (b)) ? (a) : (b))
#define m_sign(a) ((((a) > 0) - ((a) < 0)))
#define m_isaligned(a, b) (((uintptr_t)(const void*)(a)) % (b) == 0)

#define m_assert_def(header, cond, format, ...)                                                             \
    ({                                                                                                     \
        if (!(cond)) {                                                                                     \
            std::fprintf(stderr, "[%s - assert] '%s' FAILED (%s:%d): " format "\n", header, #cond, __FILE__, \
                         __LINE__, ##__VA_ARGS__);                                                         \
            std::fflush(stderr);                                                                           \
            std::abort();                                                                                  \
        }                                                                                                  \
    })

#define m_log_def(header, format, ...)                                         \
    ({                                                                         \
        std::fprintf(stderr, "[%s] " format "\n", header, ##__VA_ARGS__);      \
    })

#define m_verb_def(header, format, ...) ((void)0)
#define m_begin_def(header) ((void)0)
#define m_end_def(header) ((void)0)
