// Small float3/float2 algebra for the device path, plus the exactly rounded
// helpers used wherever the result must match a host evaluation bit for bit
// (ray setup, instance transforms, slab test, triangle tests).  nvcc contracts
// a*b+c into one FMA by default; the x* helpers below pin each operation to
// its own IEEE round-to-nearest instruction, which is what a host compiler
// produces with -ffp-contract=off.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define NB_HD __host__ __device__ __forceinline__
#define NB_D __device__ __forceinline__
// code of the BSDF lobes beyond Lambert, conductor and Fresnel specular is
// kept out of line, so that kernels built with it spend no registers on it
// until a scene uses it
#ifndef NB_LOBE_OUTLINE
#define NB_LOBE_OUTLINE 1
#endif
#if NB_LOBE_OUTLINE
#define NB_OUTLINE static __device__ __noinline__
#else
#define NB_OUTLINE NB_D
#endif

namespace nb {

constexpr float kPi = 3.14159265358979323846f;
constexpr float k2Pi = 2.0f * kPi;
constexpr float kInvPi = 1.0f / kPi;
constexpr float kInv2Pi = 1.0f / k2Pi;
constexpr float kPiOver2 = kPi / 2.0f;
constexpr float kPiOver4 = kPi / 4.0f;
constexpr float kOneMinusEps = 1.0f - 1.1920928955078125e-07f;

// ---------------------------------------------------------------- exact ops
NB_D float xmul(float a, float b) { return __fmul_rn(a, b); }
NB_D float xadd(float a, float b) { return __fadd_rn(a, b); }
NB_D float xsub(float a, float b) { return __fsub_rn(a, b); }
NB_D float xdiv(float a, float b) { return __fdiv_rn(a, b); }
// dot product evaluated as ((a.x*b.x + a.y*b.y) + a.z*b.z), no contraction
NB_D float xdot3(float ax, float ay, float az, float bx, float by, float bz) {
    return xadd(xadd(xmul(ax, bx), xmul(ay, by)), xmul(az, bz));
}

// ------------------------------------------------------------------ float3
NB_HD float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
NB_HD float3 f3(float s) { return make_float3(s, s, s); }
NB_HD float3 f3(const float4& v) { return make_float3(v.x, v.y, v.z); }
NB_HD float3 operator+(const float3& a, const float3& b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
NB_HD float3 operator-(const float3& a, const float3& b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
NB_HD float3 operator-(const float3& a) { return f3(-a.x, -a.y, -a.z); }
NB_HD float3 operator*(const float3& a, const float3& b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
NB_HD float3 operator/(const float3& a, const float3& b) { return f3(a.x / b.x, a.y / b.y, a.z / b.z); }
NB_HD float3 operator*(const float3& a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
NB_HD float3 operator*(float s, const float3& a) { return f3(a.x * s, a.y * s, a.z * s); }
NB_HD float3 operator/(const float3& a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
NB_HD float3& operator+=(float3& a, const float3& b) { a = a + b; return a; }
NB_HD float3& operator*=(float3& a, const float3& b) { a = a * b; return a; }
NB_HD float3& operator*=(float3& a, float s) { a = a * s; return a; }
NB_HD float3& operator/=(float3& a, float s) { a = a / s; return a; }
NB_HD float dot(const float3& a, const float3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
NB_HD float3 cross(const float3& a, const float3& b) {
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
NB_HD float length2(const float3& v) { return dot(v, v); }
NB_HD float absdot(const float3& a, const float3& b) { return fabsf(dot(a, b)); }
NB_HD bool is_black(const float3& c) { return c.x == 0.0f && c.y == 0.0f && c.z == 0.0f; }
NB_HD float maxcomp(const float3& c) { return fmaxf(fmaxf(c.x, c.y), c.z); }
NB_HD float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }
NB_HD float3 clamp3(const float3& v, float lo, float hi) {
    return f3(clampf(v.x, lo, hi), clampf(v.y, lo, hi), clampf(v.z, lo, hi));
}
NB_HD float3 fmin3(const float3& a, const float3& b) { return f3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
NB_HD float3 fmax3(const float3& a, const float3& b) { return f3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }

#ifdef __CUDACC__
// unit vector by reciprocal square root (no zero guard), the form the
// reference's plain `normalize` takes
NB_D float3 normalize_fast(const float3& v) { return v * rsqrtf(dot(v, v)); }
// unit vector with a zero-length guard (NOOR::normalize, utils.cuh:545-550)
NB_D float3 normalize_guard(const float3& v) {
    const float l = length2(v);
    if (l == 0.0f) return v;
    return v * rsqrtf(l);
}
NB_D float length3(const float3& v) { return sqrtf(dot(v, v)); }
#endif

NB_HD float2 f2(float x, float y) { return make_float2(x, y); }

// int sign as (0 < v) - (v < 0)
NB_HD float signf_ref(float v) { return (float)((0.0f < v) - (v < 0.0f)); }

NB_HD float3 faceforward(const float3& n, const float3& v) { return dot(v, n) < 0.0f ? -1.0f * n : n; }

// component access by axis index
NB_HD float comp(const float3& v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }

}  // namespace nb
