// ORACLE BUILD SHIM -- test infrastructure, not product code.
// Project-written stand-in for the CUDA Samples' helper_math.h, which the
// reference's device headers include (noor/cuda/path_tracer.cuh:35) and
// which is not present here.  It supplies the float2/float3/float4/int/uint
// vector constructors and component-wise algebra those headers use.  Each
// function is the plain component-wise definition: dot as x*x' + y*y' + z*z'
// left to right, normalize as v * rsqrtf(dot(v, v)), length as
// sqrtf(dot(v, v)), clamp as fmaxf(lo, fminf(v, hi)), lerp as a + t*(b - a).
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#define HM_HD inline __host__ __device__

typedef unsigned int uint;

#ifndef __CUDACC__
inline float fminf(float a, float b) { return a < b ? a : b; }
inline float fmaxf(float a, float b) { return a > b ? a : b; }
inline float rsqrtf(float x) { return 1.0f / sqrtf(x); }
#endif

// ------------------------------------------------------------- constructors
HM_HD float2 make_float2(float s) { return make_float2(s, s); }
HM_HD float2 make_float2(float3 a) { return make_float2(a.x, a.y); }
HM_HD float2 make_float2(int2 a) { return make_float2(float(a.x), float(a.y)); }
HM_HD float2 make_float2(uint2 a) { return make_float2(float(a.x), float(a.y)); }
HM_HD int2 make_int2(int s) { return make_int2(s, s); }
HM_HD int2 make_int2(float2 a) { return make_int2(int(a.x), int(a.y)); }
HM_HD uint2 make_uint2(uint s) { return make_uint2(s, s); }
HM_HD float3 make_float3(float s) { return make_float3(s, s, s); }
HM_HD float3 make_float3(float2 a) { return make_float3(a.x, a.y, 0.0f); }
HM_HD float3 make_float3(float2 a, float s) { return make_float3(a.x, a.y, s); }
HM_HD float3 make_float3(float4 a) { return make_float3(a.x, a.y, a.z); }
HM_HD float3 make_float3(int3 a) { return make_float3(float(a.x), float(a.y), float(a.z)); }
HM_HD float3 make_float3(uint3 a) { return make_float3(float(a.x), float(a.y), float(a.z)); }
HM_HD int3 make_int3(int s) { return make_int3(s, s, s); }
HM_HD int3 make_int3(float3 a) { return make_int3(int(a.x), int(a.y), int(a.z)); }
HM_HD uint3 make_uint3(uint s) { return make_uint3(s, s, s); }
HM_HD float4 make_float4(float s) { return make_float4(s, s, s, s); }
HM_HD float4 make_float4(float3 a) { return make_float4(a.x, a.y, a.z, 0.0f); }
HM_HD float4 make_float4(float3 a, float w) { return make_float4(a.x, a.y, a.z, w); }
HM_HD float4 make_float4(int4 a) { return make_float4(float(a.x), float(a.y), float(a.z), float(a.w)); }
HM_HD int4 make_int4(int s) { return make_int4(s, s, s, s); }
HM_HD uint4 make_uint4(uint s) { return make_uint4(s, s, s, s); }

// ------------------------------------------------------------------ negate
HM_HD float2 operator-(float2 a) { return make_float2(-a.x, -a.y); }
HM_HD float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
HM_HD float4 operator-(float4 a) { return make_float4(-a.x, -a.y, -a.z, -a.w); }
HM_HD int2 operator-(int2 a) { return make_int2(-a.x, -a.y); }
HM_HD int3 operator-(int3 a) { return make_int3(-a.x, -a.y, -a.z); }

// Binary operators for a vector type V with component type S: V op V,
// V op S, S op V, V op= V, V op= S.
#define HM_BIN2(V, S, OP, mk)                                                                       \
    HM_HD V operator OP(V a, V b) { return mk(a.x OP b.x, a.y OP b.y); }                            \
    HM_HD V operator OP(V a, S s) { return mk(a.x OP s, a.y OP s); }                                \
    HM_HD V operator OP(S s, V a) { return mk(s OP a.x, s OP a.y); }                                \
    HM_HD void operator OP##=(V& a, V b) { a.x OP## = b.x; a.y OP## = b.y; }                        \
    HM_HD void operator OP##=(V& a, S s) { a.x OP## = s; a.y OP## = s; }
#define HM_BIN3(V, S, OP, mk)                                                                       \
    HM_HD V operator OP(V a, V b) { return mk(a.x OP b.x, a.y OP b.y, a.z OP b.z); }                \
    HM_HD V operator OP(V a, S s) { return mk(a.x OP s, a.y OP s, a.z OP s); }                      \
    HM_HD V operator OP(S s, V a) { return mk(s OP a.x, s OP a.y, s OP a.z); }                      \
    HM_HD void operator OP##=(V& a, V b) { a.x OP## = b.x; a.y OP## = b.y; a.z OP## = b.z; }        \
    HM_HD void operator OP##=(V& a, S s) { a.x OP## = s; a.y OP## = s; a.z OP## = s; }
#define HM_BIN4(V, S, OP, mk)                                                                       \
    HM_HD V operator OP(V a, V b) { return mk(a.x OP b.x, a.y OP b.y, a.z OP b.z, a.w OP b.w); }    \
    HM_HD V operator OP(V a, S s) { return mk(a.x OP s, a.y OP s, a.z OP s, a.w OP s); }            \
    HM_HD V operator OP(S s, V a) { return mk(s OP a.x, s OP a.y, s OP a.z, s OP a.w); }            \
    HM_HD void operator OP##=(V& a, V b) { a.x OP## = b.x; a.y OP## = b.y; a.z OP## = b.z; a.w OP## = b.w; } \
    HM_HD void operator OP##=(V& a, S s) { a.x OP## = s; a.y OP## = s; a.z OP## = s; a.w OP## = s; }

#define HM_ALL_OPS(BIN, V, S, mk) BIN(V, S, +, mk) BIN(V, S, -, mk) BIN(V, S, *, mk) BIN(V, S, /, mk)
HM_ALL_OPS(HM_BIN2, float2, float, make_float2)
HM_ALL_OPS(HM_BIN3, float3, float, make_float3)
HM_ALL_OPS(HM_BIN4, float4, float, make_float4)
HM_ALL_OPS(HM_BIN2, int2, int, make_int2)
HM_ALL_OPS(HM_BIN3, int3, int, make_int3)
HM_ALL_OPS(HM_BIN2, uint2, uint, make_uint2)
HM_ALL_OPS(HM_BIN3, uint3, uint, make_uint3)
HM_ALL_OPS(HM_BIN4, int4, int, make_int4)
HM_ALL_OPS(HM_BIN4, uint4, uint, make_uint4)
#undef HM_ALL_OPS
#undef HM_BIN2
#undef HM_BIN3
#undef HM_BIN4

// ----------------------------------------------------------- min / max
HM_HD float2 fminf(float2 a, float2 b) { return make_float2(fminf(a.x, b.x), fminf(a.y, b.y)); }
HM_HD float3 fminf(float3 a, float3 b) { return make_float3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
HM_HD float4 fminf(float4 a, float4 b) {
    return make_float4(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z), fminf(a.w, b.w));
}
HM_HD float2 fmaxf(float2 a, float2 b) { return make_float2(fmaxf(a.x, b.x), fmaxf(a.y, b.y)); }
HM_HD float3 fmaxf(float3 a, float3 b) { return make_float3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
HM_HD float4 fmaxf(float4 a, float4 b) {
    return make_float4(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z), fmaxf(a.w, b.w));
}
HM_HD int2 min(int2 a, int2 b) { return make_int2(a.x < b.x ? a.x : b.x, a.y < b.y ? a.y : b.y); }
HM_HD int2 max(int2 a, int2 b) { return make_int2(a.x > b.x ? a.x : b.x, a.y > b.y ? a.y : b.y); }

// -------------------------------------------------------------- lerp/clamp
HM_HD float lerp(float a, float b, float t) { return a + t * (b - a); }
HM_HD float2 lerp(float2 a, float2 b, float t) { return a + t * (b - a); }
HM_HD float3 lerp(float3 a, float3 b, float t) { return a + t * (b - a); }
HM_HD float4 lerp(float4 a, float4 b, float t) { return a + t * (b - a); }
HM_HD float clamp(float f, float a, float b) { return fmaxf(a, fminf(f, b)); }
HM_HD int clamp(int f, int a, int b) { return f < a ? a : (f > b ? b : f); }
HM_HD uint clamp(uint f, uint a, uint b) { return f < a ? a : (f > b ? b : f); }
HM_HD float2 clamp(float2 v, float a, float b) { return make_float2(clamp(v.x, a, b), clamp(v.y, a, b)); }
HM_HD float3 clamp(float3 v, float a, float b) {
    return make_float3(clamp(v.x, a, b), clamp(v.y, a, b), clamp(v.z, a, b));
}
HM_HD float3 clamp(float3 v, float3 a, float3 b) {
    return make_float3(clamp(v.x, a.x, b.x), clamp(v.y, a.y, b.y), clamp(v.z, a.z, b.z));
}
HM_HD float4 clamp(float4 v, float a, float b) {
    return make_float4(clamp(v.x, a, b), clamp(v.y, a, b), clamp(v.z, a, b), clamp(v.w, a, b));
}
HM_HD int2 clamp(int2 v, int a, int b) { return make_int2(clamp(v.x, a, b), clamp(v.y, a, b)); }
HM_HD int2 clamp(int2 v, int2 a, int2 b) { return make_int2(clamp(v.x, a.x, b.x), clamp(v.y, a.y, b.y)); }

// --------------------------------------------------------- dot / length
HM_HD float dot(float2 a, float2 b) { return a.x * b.x + a.y * b.y; }
HM_HD float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
HM_HD float dot(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
HM_HD float length(float2 v) { return sqrtf(dot(v, v)); }
HM_HD float length(float3 v) { return sqrtf(dot(v, v)); }
HM_HD float length(float4 v) { return sqrtf(dot(v, v)); }
HM_HD float2 normalize(float2 v) { return v * rsqrtf(dot(v, v)); }
HM_HD float3 normalize(float3 v) { return v * rsqrtf(dot(v, v)); }
HM_HD float4 normalize(float4 v) { return v * rsqrtf(dot(v, v)); }

// ------------------------------------------------------ floor/frac/fmod/abs
HM_HD float2 floorf(float2 v) { return make_float2(floorf(v.x), floorf(v.y)); }
HM_HD float3 floorf(float3 v) { return make_float3(floorf(v.x), floorf(v.y), floorf(v.z)); }
HM_HD float4 floorf(float4 v) { return make_float4(floorf(v.x), floorf(v.y), floorf(v.z), floorf(v.w)); }
HM_HD float fracf(float v) { return v - floorf(v); }
HM_HD float2 fracf(float2 v) { return make_float2(fracf(v.x), fracf(v.y)); }
HM_HD float3 fracf(float3 v) { return make_float3(fracf(v.x), fracf(v.y), fracf(v.z)); }
HM_HD float2 fmodf(float2 a, float2 b) { return make_float2(fmodf(a.x, b.x), fmodf(a.y, b.y)); }
HM_HD float3 fmodf(float3 a, float3 b) { return make_float3(fmodf(a.x, b.x), fmodf(a.y, b.y), fmodf(a.z, b.z)); }
HM_HD float2 fabs(float2 v) { return make_float2(fabsf(v.x), fabsf(v.y)); }
HM_HD float3 fabs(float3 v) { return make_float3(fabsf(v.x), fabsf(v.y), fabsf(v.z)); }
HM_HD float4 fabs(float4 v) { return make_float4(fabsf(v.x), fabsf(v.y), fabsf(v.z), fabsf(v.w)); }

// ------------------------------------------------------- reflect / cross
HM_HD float3 reflect(float3 i, float3 n) { return i - 2.0f * n * dot(n, i); }
HM_HD float3 cross(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
HM_HD float smoothstep(float a, float b, float x) {
    const float y = clamp((x - a) / (b - a), 0.0f, 1.0f);
    return y * y * (3.0f - 2.0f * y);
}
