// ORACLE BUILD SHIM -- test infrastructure.
// The small subset of glm that the reference's host BVH builder
// (noor/source/bvh.cpp, noor/source/splitter.cpp, noor/header/bbox.h,
// splitter.h, spec.h, stat.h) and Wald precomputation (noor/header/triangle.h)
// use, so those files compile unmodified.  glm itself is not shipped with the
// reference (its version is unpinned); the semantics restated here are glm
// 0.9.9's: min(x,y) = (y < x) ? y : x, max(x,y) = (x < y) ? y : x, the
// 3- and 4-argument min/max of gtx/extended_min_max, dot as ((x+y)+z),
// normalize as v * (1/sqrt(dot(v,v))), mat4*vec4 as (c0*x + c1*y) + (c2*z + c3*w).
#pragma once
#include <cmath>
#include <cstdint>
#include <utility>

namespace glm {
typedef uint8_t uint8;
typedef uint16_t uint16;
typedef uint32_t uint32;
typedef int32_t int32;

template <class T> inline T min(T x, T y) { return (y < x) ? y : x; }
template <class T> inline T max(T x, T y) { return (x < y) ? y : x; }
inline bool isinf(float v) { return std::isinf(v); }
inline bool isnan(float v) { return std::isnan(v); }

struct vec4;
struct bvec3 {
    bool x, y, z;
};

struct vec3 {
    float x, y, z;
    vec3() : x(0), y(0), z(0) {}
    explicit vec3(float s) : x(s), y(s), z(s) {}
    vec3(float a, float b, float c) : x(a), y(b), z(c) {}
    vec3(const vec4& v);
    float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    const float& operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
struct vec4 {
    float x, y, z, w;
    vec4() : x(0), y(0), z(0), w(0) {}
    explicit vec4(float s) : x(s), y(s), z(s), w(s) {}
    vec4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
    vec4(const vec3& v, float d) : x(v.x), y(v.y), z(v.z), w(d) {}
    float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
    const float& operator[](int i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
};
inline vec3::vec3(const vec4& v) : x(v.x), y(v.y), z(v.z) {}
struct vec2 {
    float x, y;
};
struct uvec4 {
    uint32 x, y, z, w;
    uvec4() : x(0), y(0), z(0), w(0) {}
    uvec4(uint32 a, uint32 b, uint32 c, uint32 d) : x(a), y(b), z(c), w(d) {}
};

inline vec3 operator+(const vec3& a, const vec3& b) { return vec3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline vec3 operator-(const vec3& a, const vec3& b) { return vec3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline vec3 operator-(const vec3& a) { return vec3(-a.x, -a.y, -a.z); }
inline vec3 operator*(const vec3& a, const vec3& b) { return vec3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline vec3 operator*(const vec3& a, float s) { return vec3(a.x * s, a.y * s, a.z * s); }
inline vec3 operator*(float s, const vec3& a) { return vec3(s * a.x, s * a.y, s * a.z); }
inline vec3 operator/(const vec3& a, float s) { return vec3(a.x / s, a.y / s, a.z / s); }
inline vec4 operator*(const vec4& a, float s) { return vec4(a.x * s, a.y * s, a.z * s, a.w * s); }
inline vec4 operator+(const vec4& a, const vec4& b) { return vec4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }

inline vec3 min(const vec3& a, const vec3& b) { return vec3(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)); }
inline vec3 max(const vec3& a, const vec3& b) { return vec3(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)); }
inline vec3 min(const vec3& a, const vec3& b, const vec3& c) { return min(min(a, b), c); }
inline vec3 max(const vec3& a, const vec3& b, const vec3& c) { return max(max(a, b), c); }
inline vec3 min(const vec3& a, const vec3& b, const vec3& c, const vec3& d) { return min(min(a, b), min(c, d)); }
inline vec3 max(const vec3& a, const vec3& b, const vec3& c, const vec3& d) { return max(max(a, b), max(c, d)); }
inline vec4 min(const vec4& a, const vec4& b) { return vec4(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z), min(a.w, b.w)); }
inline vec4 max(const vec4& a, const vec4& b) { return vec4(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z), max(a.w, b.w)); }
inline vec4 min(const vec4& a, const vec4& b, const vec4& c) { return min(min(a, b), c); }
inline vec4 max(const vec4& a, const vec4& b, const vec4& c) { return max(max(a, b), c); }

inline float dot(const vec3& a, const vec3& b) {
    const vec3 t = a * b;
    return t.x + t.y + t.z;
}
inline vec3 cross(const vec3& x, const vec3& y) {
    return vec3(x.y * y.z - y.y * x.z, x.z * y.x - y.z * x.x, x.x * y.y - y.x * x.y);
}
inline float length(const vec3& v) { return std::sqrt(dot(v, v)); }
inline vec3 normalize(const vec3& v) { return v * (1.0f / std::sqrt(dot(v, v))); }

inline bvec3 greaterThanEqual(const vec3& a, const vec3& b) { return bvec3{a.x >= b.x, a.y >= b.y, a.z >= b.z}; }
inline bvec3 lessThanEqual(const vec3& a, const vec3& b) { return bvec3{a.x <= b.x, a.y <= b.y, a.z <= b.z}; }
inline bvec3 lessThan(const vec3& a, const vec3& b) { return bvec3{a.x < b.x, a.y < b.y, a.z < b.z}; }
inline bool all(const bvec3& b) { return b.x && b.y && b.z; }

// column-major matrices
struct mat4 {
    vec4 c[4];
    mat4() : mat4(1.0f) {}
    explicit mat4(float d) {
        for (int i = 0; i < 4; ++i) c[i] = vec4(0.0f);
        c[0].x = c[1].y = c[2].z = c[3].w = d;
    }
    vec4& operator[](int i) { return c[i]; }
    const vec4& operator[](int i) const { return c[i]; }
};
struct mat3 {
    vec3 c[3];
    mat3() : mat3(1.0f) {}
    explicit mat3(float d) {
        for (int i = 0; i < 3; ++i) c[i] = vec3(0.0f);
        c[0].x = c[1].y = c[2].z = d;
    }
    explicit mat3(const mat4& m) {
        for (int i = 0; i < 3; ++i) c[i] = vec3(m[i].x, m[i].y, m[i].z);
    }
    vec3& operator[](int i) { return c[i]; }
    const vec3& operator[](int i) const { return c[i]; }
};
inline vec4 operator*(const mat4& m, const vec4& v) {
    const vec4 a = m[0] * v.x, b = m[1] * v.y, c = m[2] * v.z, d = m[3] * v.w;
    return (a + b) + (c + d);
}
// cofactor inverse (only needed so WoopTriangle in triangle.h compiles;
// the reference never constructs one)
inline mat4 inverse(const mat4& m) {
    double a[16], inv[16];
    for (int c = 0; c < 4; ++c)
        for (int r = 0; r < 4; ++r) a[4 * c + r] = m[c][r];
    for (int i = 0; i < 16; ++i) inv[i] = 0.0;
    // Gauss-Jordan on a copy
    double w[4][8];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 8; ++c) w[r][c] = c < 4 ? a[4 * c + r] : (c - 4 == r ? 1.0 : 0.0);
    for (int p = 0; p < 4; ++p) {
        int best = p;
        for (int r = p + 1; r < 4; ++r)
            if (std::fabs(w[r][p]) > std::fabs(w[best][p])) best = r;
        for (int c = 0; c < 8; ++c) std::swap(w[p][c], w[best][c]);
        const double d = w[p][p] != 0.0 ? w[p][p] : 1.0;
        for (int c = 0; c < 8; ++c) w[p][c] /= d;
        for (int r = 0; r < 4; ++r)
            if (r != p) {
                const double f = w[r][p];
                for (int c = 0; c < 8; ++c) w[r][c] -= f * w[p][c];
            }
    }
    mat4 o;
    for (int c = 0; c < 4; ++c)
        for (int r = 0; r < 4; ++r) o[c][r] = (float)w[r][4 + c];
    (void)inv;
    return o;
}
// column c of a*b is a times column c of b (the oracle harness compiles the
// CudaCamera constructor, noor/cuda/camera.cuh:66-94, but fills cameras
// field by field)
inline mat4 operator*(const mat4& a, const mat4& b) {
    mat4 o;
    for (int c = 0; c < 4; ++c) o[c] = a * b[c];
    return o;
}
// adjugate over the determinant (the mesh normal transform,
// transpose(inverse(mat3(to_global))), noor/header/assetLoader.h:75-76)
inline mat3 inverse(const mat3& m) {
    const float det = m[0][0] * (m[1][1] * m[2][2] - m[2][1] * m[1][2]) -
                      m[1][0] * (m[0][1] * m[2][2] - m[2][1] * m[0][2]) +
                      m[2][0] * (m[0][1] * m[1][2] - m[1][1] * m[0][2]);
    const float s = 1.0f / det;
    mat3 o;
    o[0][0] = (m[1][1] * m[2][2] - m[2][1] * m[1][2]) * s;
    o[1][0] = -(m[1][0] * m[2][2] - m[2][0] * m[1][2]) * s;
    o[2][0] = (m[1][0] * m[2][1] - m[2][0] * m[1][1]) * s;
    o[0][1] = -(m[0][1] * m[2][2] - m[2][1] * m[0][2]) * s;
    o[1][1] = (m[0][0] * m[2][2] - m[2][0] * m[0][2]) * s;
    o[2][1] = -(m[0][0] * m[2][1] - m[2][0] * m[0][1]) * s;
    o[0][2] = (m[0][1] * m[1][2] - m[1][1] * m[0][2]) * s;
    o[1][2] = -(m[0][0] * m[1][2] - m[1][0] * m[0][2]) * s;
    o[2][2] = (m[0][0] * m[1][1] - m[1][0] * m[0][1]) * s;
    return o;
}
inline mat3 transpose(const mat3& m) {
    mat3 o;
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r) o[c][r] = m[r][c];
    return o;
}
inline vec4 row(const mat4& m, int i) { return vec4(m[0][i], m[1][i], m[2][i], m[3][i]); }
inline vec3 row(const mat3& m, int i) { return vec3(m[0][i], m[1][i], m[2][i]); }
}  // namespace glm
