// Minimal stand-in for the h3lpr helper library's ptr.hpp: m_ptr, an aligned
// zero-filled allocation whose raw pointer is returned by operator() and
// released by free() (POSIX allocations are released with std::free, which
// the reference's m_free relies on; the object does not own them).  Test
// infrastructure of the oracle only.
#pragma once
#include <stdlib.h>
#include <string.h>

#include <cstddef>
#include <cstdio>

namespace H3LPR {
enum AllocType { H3LPR_ALLOC_POSIX, H3LPR_ALLOC_MPI };

template <AllocType A, typename T, size_t ALIGN>
class m_ptr {
   public:
    m_ptr() = default;
    explicit m_ptr(size_t bytes) { calloc(bytes); }
    void calloc(size_t bytes) {
        void* p = nullptr;
        if (posix_memalign(&p, ALIGN < sizeof(void*) ? sizeof(void*) : ALIGN, bytes ? bytes : ALIGN) != 0) {
            std::fprintf(stderr, "h3lpr stand-in: allocation of %zu bytes failed\n", bytes);
            abort();
        }
        memset(p, 0, bytes);
        ptr_ = static_cast<T>(p);
    }
    void free() {
        if (ptr_) ::free((void*)ptr_);
        ptr_ = nullptr;
    }
    T operator()() const { return ptr_; }

   private:
    T ptr_ = nullptr;
};
}  // namespace H3LPR
