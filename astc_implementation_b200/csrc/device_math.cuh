// Device-side arithmetic with the exact float semantics of the search.
//
// The encoder sources are compiled with -fmad=false and IEEE division and
// square root, so every expression below is a sequence of correctly rounded
// single-precision operations.  The WGSL leaves several operations open; the
// choices (identical to the CPU oracle's) are:
//   * min/max return the non-NaN operand; clamp(x,lo,hi) = min(max(x,lo),hi);
//   * normalize(v) = v / sqrt(dot(v,v)) component-wise (a zero vector gives NaN);
//   * dot products sum the component products left to right;
//   * f32 -> u32/i32 saturate, NaN giving the maximum (Tint's conversion rule);
//   * round() is round-half-to-even (rintf);
//   * atan2 follows the Cephes single-precision arctangent (S. L. Moshier,
//     Cephes Math Library), range-reduced at tan(3pi/8) and tan(pi/8).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace astcb200 {
namespace dev {

__device__ __forceinline__ float4 mk(float a) { return make_float4(a, a, a, a); }
__device__ __forceinline__ float4 operator+(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
__device__ __forceinline__ float4 operator-(float4 a, float4 b) { return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
__device__ __forceinline__ float4 operator*(float4 a, float4 b) { return make_float4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w); }
__device__ __forceinline__ float4 operator*(float4 a, float s) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }
__device__ __forceinline__ float4 operator/(float4 a, float4 b) { return make_float4(a.x / b.x, a.y / b.y, a.z / b.z, a.w / b.w); }
__device__ __forceinline__ float dot4(float4 a, float4 b) {
    float r = a.x * b.x;
    r = r + a.y * b.y;
    r = r + a.z * b.z;
    r = r + a.w * b.w;
    return r;
}
__device__ __forceinline__ float dot3(float4 a, float4 b) {
    float r = a.x * b.x;
    r = r + a.y * b.y;
    r = r + a.z * b.z;
    return r;
}
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
__device__ __forceinline__ float4 vmax(float4 a, float4 b) { return make_float4(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z), fmaxf(a.w, b.w)); }
__device__ __forceinline__ float4 vmin(float4 a, float4 b) { return make_float4(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z), fminf(a.w, b.w)); }
__device__ __forceinline__ float4 normalize4(float4 v) {
    const float l = sqrtf(dot4(v, v));
    return make_float4(v.x / l, v.y / l, v.z / l, v.w / l);
}
__device__ __forceinline__ float comp(const float4& v, int c) { return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w; }
__device__ __forceinline__ uint32_t f2u(float v) {
    if (!(v <= 4294967040.0f)) return 4294967295u;
    if (v < 0.0f) return 0u;
    return __float2uint_rz(v);
}
__device__ __forceinline__ int32_t f2i(float v) {
    if (!(v <= 2147483520.0f)) return 2147483647;
    if (v < -2147483648.0f) return (int32_t)0x80000000u;
    return __float2int_rz(v);
}
__device__ __forceinline__ uint32_t fbits(float f) { return __float_as_uint(f); }

__device__ __forceinline__ float atan_pos(float x) {
    float y0;
    if (x > 2.414213562373095f) { y0 = 1.5707963267948966f; x = -1.0f / x; }
    else if (x > 0.4142135623730950f) { y0 = 0.7853981633974483f; x = (x - 1.0f) / (x + 1.0f); }
    else { y0 = 0.0f; }
    const float z = x * x;
    float p = 8.05374449538e-2f * z;
    p = p - 1.38776856032e-1f; p = p * z;
    p = p + 1.99777106478e-1f; p = p * z;
    p = p - 3.33329491539e-1f; p = p * z;
    p = p * x; p = p + x;
    return y0 + p;
}
__device__ __forceinline__ float atan2_search(float y, float x) {
    if (isnan(x) || isnan(y)) return __int_as_float(0x7fc00000);
    const float ax = fabsf(x), ay = fabsf(y);
    if (ax == 0.0f && ay == 0.0f) return 0.0f;
    float r = atan_pos(ay / ax);
    if (x < 0.0f) r = 3.14159265358979323846f - r;
    if (y < 0.0f) r = -r;
    return r;
}

// Colour error weights R, G, B, A (astc.h:60-63).
__device__ __forceinline__ float4 chan_w() { return make_float4(0.30f * 2.25f, 0.59f * 2.25f, 0.11f * 2.25f, 1.0f); }

}  // namespace dev
}  // namespace astcb200
