// Shared host/device helpers for the B200 path tracer.
//
// The floating-point helpers keep the operand order of the reference's
// vector helpers (Native/renderer.cu:76-96): every sum, product and dot
// product is evaluated left to right with one rounding per operation. The
// library is compiled with --fmad=false (as Native/build.sh:11 compiles the
// reference), so the device and host builds of these functions produce the
// same bits as the reference's device and host builds. Where a fused
// multiply-add is wanted (box tests only) it is written explicitly.
#pragma once
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>

#define RT_HD __host__ __device__ __forceinline__

namespace rt {

constexpr float kPi = 3.14159265358979323846f;

// ---- device allocation ----
// The renderer's device allocations go through deviceAlloc, so a test can
// make the n-th next one fail on the host, as an out-of-memory cudaMalloc
// would, without touching the GPU (RtxDebugFailAllocation).
cudaError_t deviceAllocBytes(void** p, size_t bytes);
template <class T>
inline cudaError_t deviceAlloc(T** p, size_t bytes) {
    return deviceAllocBytes(reinterpret_cast<void**>(p), bytes);
}

// ---- portable bit helpers (device intrinsics, host builtins) ----
RT_HD unsigned popc(unsigned x) {
#ifdef __CUDA_ARCH__
    return __popc(x);
#else
    return (unsigned)__builtin_popcount(x);
#endif
}
// Index of the highest set bit; x must be non-zero.
RT_HD int highestBit(unsigned x) {
#ifdef __CUDA_ARCH__
    return 31 - __clz(x);
#else
    return 31 - __builtin_clz(x);
#endif
}
RT_HD float bitsToFloat(unsigned u) {
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float f; std::memcpy(&f, &u, 4); return f;
#endif
}
RT_HD unsigned floatToBits(float f) {
#ifdef __CUDA_ARCH__
    return __float_as_uint(f);
#else
    unsigned u; std::memcpy(&u, &f, 4); return u;
#endif
}
RT_HD float fmaRn(float a, float b, float c) {
#ifdef __CUDA_ARCH__
    return __fmaf_rn(a, b, c);
#else
    return std::fmaf(a, b, c);
#endif
}
// Correctly rounded reciprocal; identical to 1.0f / x under IEEE division.
RT_HD float recip(float x) {
#ifdef __CUDA_ARCH__
    return __frcp_rn(x);
#else
    return 1.0f / x;
#endif
}

// ---- vector helpers with the reference's operation order ----
RT_HD float3 v3(float x, float y, float z) { return make_float3(x, y, z); }
RT_HD float comp(const float3& v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }
RT_HD float3 add(float3 a, float3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
RT_HD float3 sub(float3 a, float3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
RT_HD float3 scale(float3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
RT_HD float3 mul(float3 a, float3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
RT_HD float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
RT_HD float3 cross(float3 a, float3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
RT_HD float3 normalize(float3 a) { return scale(a, 1.0f / sqrtf(fmaxf(dot(a, a), 1e-20f))); }
RT_HD float3 mirror(float3 d, float3 n) { return sub(d, scale(n, 2.0f * dot(d, n))); }

// sRGB decode applied to input colours (Native/renderer.cu:84,347).
RT_HD float srgbToLinear(float c) { return c <= .04045f ? c / 12.92f : powf((c + .055f) / 1.055f, 2.4f); }
// Exposure tonemap + sRGB encode + 8-bit rounding (Native/renderer.cu:86-90).
RT_HD unsigned char tonemap(float c, float exposure) {
    c = 1.0f - expf(-fmaxf(c, 0.0f) * exposure);
    c = c <= .0031308f ? 12.92f * c : 1.055f * powf(c, 1.0f / 2.4f) - .055f;
    return (unsigned char)(255.0f * fminf(c, 1.0f) + .5f);
}

}  // namespace rt
