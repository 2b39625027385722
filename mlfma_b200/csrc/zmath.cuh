// Complex helpers on double2 (FP64) and float2 (FP32) for the kernels.
#pragma once

#include <cuda_runtime.h>

namespace mlfma {
namespace {

template <class C> __device__ __forceinline__ C zero();
template <> __device__ __forceinline__ double2 zero<double2>() { return make_double2(0.0, 0.0); }
template <> __device__ __forceinline__ float2 zero<float2>() { return make_float2(0.0f, 0.0f); }
__device__ __forceinline__ double2 z0() { return make_double2(0.0, 0.0); }

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a*b + c
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c) {
    return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
__device__ __forceinline__ float2 cfma(float2 a, float2 b, float2 c) {
    return make_float2(fmaf(a.x, b.x, fmaf(-a.y, b.y, c.x)), fmaf(a.x, b.y, fmaf(a.y, b.x, c.y)));
}
// conj(a)*b + c
__device__ __forceinline__ double2 cjfma(double2 a, double2 b, double2 c) {
    return make_double2(fma(a.x, b.x, fma(a.y, b.y, c.x)), fma(a.x, b.y, fma(-a.y, b.x, c.y)));
}
__device__ __forceinline__ float2 cjfma(float2 a, float2 b, float2 c) {
    return make_float2(fmaf(a.x, b.x, fmaf(a.y, b.y, c.x)), fmaf(a.x, b.y, fmaf(-a.y, b.x, c.y)));
}
// s*a + c for real s
__device__ __forceinline__ double2 crfma(double s, double2 a, double2 c) {
    return make_double2(fma(s, a.x, c.x), fma(s, a.y, c.y));
}
__device__ __forceinline__ float2 crfma(float s, float2 a, float2 c) {
    return make_float2(fmaf(s, a.x, c.x), fmaf(s, a.y, c.y));
}
__device__ __forceinline__ double2 cscale(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
__device__ __forceinline__ float2 cscale(float s, float2 a) { return make_float2(s * a.x, s * a.y); }
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }

__device__ __forceinline__ double2 warp_sum(double2 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    return v;
}
__device__ __forceinline__ float2 warp_sum(float2 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    return v;
}
__device__ __forceinline__ void atomic_add_z(double2* p, double2 v) {
    atomicAdd(&p->x, v.x);
    atomicAdd(&p->y, v.y);
}
// Streaming read: data touched once per product (patterns, near-field blocks).
__device__ __forceinline__ double2 ldg_stream(const double2* p) { return __ldcs(p); }
__device__ __forceinline__ float2 ldg_stream(const float2* p) { return __ldcs(p); }

// Conversions between the far-field type and complex double.
template <class C> __device__ __forceinline__ C from_d2(double2 v);
template <> __device__ __forceinline__ double2 from_d2<double2>(double2 v) { return v; }
template <> __device__ __forceinline__ float2 from_d2<float2>(double2 v) {
    return make_float2(static_cast<float>(v.x), static_cast<float>(v.y));
}
__device__ __forceinline__ double2 to_d2(double2 v) { return v; }
__device__ __forceinline__ double2 to_d2(float2 v) { return make_double2(v.x, v.y); }

}  // namespace
}  // namespace mlfma
