// Explicit vector memory accesses: one instruction per complex value (or
// per pair of twiddles), written as PTX so that a complex value is never
// moved as two scalar accesses.  Shared-memory addresses are 32-bit
// shared-window addresses; all accesses are volatile so that they keep their
// order relative to barriers and to each other.
#pragma once
#include <cuda_runtime.h>

namespace flb {

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// ---- shared memory
__device__ __forceinline__ void lds(unsigned a, float2& v) {
    asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(a));
}
__device__ __forceinline__ void lds(unsigned a, double2& v) {
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(a));
}
__device__ __forceinline__ void lds(unsigned a, float4& v) {
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a));
}
__device__ __forceinline__ void sts(unsigned a, const float2& v) {
    asm volatile("st.shared.v2.f32 [%0], {%1, %2};" ::"r"(a), "f"(v.x), "f"(v.y) : "memory");
}
__device__ __forceinline__ void sts(unsigned a, const double2& v) {
    asm volatile("st.shared.v2.f64 [%0], {%1, %2};" ::"r"(a), "d"(v.x), "d"(v.y) : "memory");
}

// ---- global memory (default caching)
__device__ __forceinline__ void ldg(const float2* p, float2& v) {
    asm volatile("ld.global.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p));
}
__device__ __forceinline__ void ldg(const double2* p, double2& v) {
    asm volatile("ld.global.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
}
__device__ __forceinline__ void stg(float2* p, const float2& v) {
    asm volatile("st.global.v2.f32 [%0], {%1, %2};" ::"l"(p), "f"(v.x), "f"(v.y) : "memory");
}
__device__ __forceinline__ void stg(double2* p, const double2& v) {
    asm volatile("st.global.v2.f64 [%0], {%1, %2};" ::"l"(p), "d"(v.x), "d"(v.y) : "memory");
}

}  // namespace flb
