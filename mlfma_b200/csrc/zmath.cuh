// Complex FP64 helpers on double2 for the kernels.
#pragma once

#include <cuda_runtime.h>

namespace mlfma {
namespace {

__device__ __forceinline__ double2 z0() { return make_double2(0.0, 0.0); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a*b + c
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c) {
    return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
// conj(a)*b + c
__device__ __forceinline__ double2 cjfma(double2 a, double2 b, double2 c) {
    return make_double2(fma(a.x, b.x, fma(a.y, b.y, c.x)), fma(a.x, b.y, fma(-a.y, b.x, c.y)));
}
__device__ __forceinline__ double2 cscale(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 warp_sum(double2 v) {
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

}  // namespace
}  // namespace mlfma
