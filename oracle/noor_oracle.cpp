// ORACLE -- test infrastructure, not product code.
//
// Scalar C++ restatement of Noor's device render routines, used only by the
// tests, __graft_entry__.smoke() and bench.py's CPU baseline as the checker.
// Templated on the scalar type: float is the transcription of the reference
// routines compiled for the host (compiled with -ffp-contract=off, so every
// a*b+c rounds twice as the C source is written), double is the FP64 oracle
// for image RMSE.  Each routine cites the reference file:line it follows
// (paths relative to the reference project root).  It consumes the same
// noor_payload / noor_camera / noor_spec / noor_hosek_sky inputs as the
// CUDA library, reading only the struct layouts from include/noor_b200.h.
//
// Parity status: the reference ships no tests or golden vectors.  The BVH
// builder and Wald precomputation are pinned against the reference's own
// sources compiled under oracle/_ref; the Hosek fit against the reference's
// ArHosekSkyModel.cpp compiled under oracle/_ref; the device routines below
// have no runnable reference (they need an sm_61 GL/CUDA-9 build) and are
// transcriptions -- "parity unpinned" for those routines beyond this file.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

#include "../include/noor_b200.h"

#define OR_API extern "C" __attribute__((visibility("default")))

namespace orc {

template <class T>
struct V {
    T x, y, z;
};
template <class T> inline V<T> mk(T x, T y, T z) { return V<T>{x, y, z}; }
template <class T> inline V<T> operator+(V<T> a, V<T> b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
template <class T> inline V<T> operator-(V<T> a, V<T> b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
template <class T> inline V<T> operator*(V<T> a, V<T> b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
template <class T> inline V<T> operator/(V<T> a, V<T> b) { return mk(a.x / b.x, a.y / b.y, a.z / b.z); }
template <class T> inline V<T> operator*(V<T> a, T s) { return mk(a.x * s, a.y * s, a.z * s); }
template <class T> inline V<T> operator*(T s, V<T> a) { return mk(s * a.x, s * a.y, s * a.z); }
template <class T> inline V<T> operator/(V<T> a, T s) { return mk(a.x / s, a.y / s, a.z / s); }
template <class T> inline T dot(V<T> a, V<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> inline V<T> cross(V<T> a, V<T> b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <class T> inline T len2(V<T> v) { return dot(v, v); }
template <class T> inline T len(V<T> v) { return std::sqrt(dot(v, v)); }
// helper_math normalize: v * rsqrt(dot(v,v)); host rsqrt = 1/sqrt
template <class T> inline V<T> nrm(V<T> v) { return v * (T(1) / std::sqrt(dot(v, v))); }
// NOOR::normalize (utils.cuh:545-550): zero-length guard
template <class T> inline V<T> nrm_g(V<T> v) {
    const T l = len2(v);
    if (l == T(0)) return v;
    return v * (T(1) / std::sqrt(l));
}
template <class T> inline bool black(V<T> c) { return c.x == 0 && c.y == 0 && c.z == 0; }
template <class T> inline T clampv(T v, T lo, T hi) { return std::min(std::max(v, lo), hi); }
template <class T> inline T comp(V<T> v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
template <class T> inline T maxc(V<T> v) { return std::max(std::max(v.x, v.y), v.z); }
template <class T> inline T signv(T v) { return (T)((T(0) < v) - (v < T(0))); }

template <class T> struct K {
    static constexpr T pi = (T)3.14159265358979323846;
    static constexpr T inv_pi = T(1) / pi;
    static constexpr T inv_2pi = T(1) / (T(2) * pi);
    static constexpr T inf = std::numeric_limits<T>::infinity();
};

inline float u2f(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
inline uint32_t f2u(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

// ---------------------------------------------------------------- RNG
// noor/cuda/rng.cuh:37-76
inline uint32_t tea16(uint32_t v0, uint32_t v1) {
    uint32_t s0 = 0;
    for (int n = 0; n < 16; n++) {
        s0 += 0x9e3779b9u;
        v0 += ((v1 << 4) + 0xa341316cu) ^ (v1 + s0) ^ ((v1 >> 5) + 0xc8013ea4u);
        v1 += ((v0 << 4) + 0xad90777du) ^ (v0 + s0) ^ ((v0 >> 5) + 0x7e95761eu);
    }
    return v0;
}
struct Rng {
    uint32_t s;
    float next() {
        s = 1664525u * s + 1013904223u;
        return (float)(s & 0x00FFFFFFu) / (float)0x01000000;
    }
};

// ------------------------------------------------------------ scene view
struct Scene {
    const noor_payload* P;
    const noor_spec* S;
    const noor_hosek_sky* H;
    // env distribution (FP64 build, stored in both precisions)
    int dw = 0, dh = 0;
    std::vector<double> func, cdf, row_int, marg_cdf;
    double marg_int = 0;
    const float* env = nullptr;
    int ew = 0, eh = 0;
    int num_lights = 0;
    bool sky_on = false;
    bool has_bump = false;
    // per-material constants resolved from the 1x1 textures
    struct Mat {
        float diffuse[3], specular[3], transmission[3], emittance[3], ior[3], k[3];
        float rx, ry, coat_ior, emitter_scale, coat_weight, coat_sigma, coat_thickness;
        uint32_t type, dist;
        // slots read per hit: diffuse, specular, emittance, roughness,
        // transmission, ior, k, alpha, bump (texture index, uv scale)
        uint32_t tex_mask;
        uint32_t tex[9];
        float uvs[9][2];
        float bumpfactor;
    };
    std::vector<Mat> mats;
};
enum { TX_DIFFUSE, TX_SPECULAR, TX_EMITTANCE, TX_ROUGHNESS, TX_TRANSMISSION, TX_IOR, TX_K, TX_ALPHA, TX_BUMP };

// A texture fetch as the texture unit computes it (tex2D on an RGBA float
// array, normalised coordinates), the reference's material textures being
// such arrays (noor/cuda/texture.cuh:375-400).  Restated from CUDA's
// documented filtering (linear: the weights are 9-bit fixed point with 8
// fractional bits) and from measurements of the unit: the coordinate's
// fraction x*256 is rounded half up; the four corner weights are integers
// over 256 -- w11 = round_half_up(A*B/256), w10 = A - w11, w01 = B - w11,
// w00 = 256 - A - B + w11 -- and the weighted sum is rounded once.  It
// matches the unit on about 99 % of fetches; the rest differ where the
// unit's fixed-point coordinate rounds the other way (within 1/256 of the
// texel difference).  Point: texel floor(u*W).  Wrap takes the fraction of
// u first; clamp clamps the texel index.
inline void tex_fetch(const noor_texture& t, double u, double v, float out[4]) {
    const int W = t.width, H = t.height;
    if (W == 1 && H == 1) {
        std::memcpy(out, t.rgba, 16);
        return;
    }
    const bool wrap = t.address == NOOR_ADDRESS_WRAP;
    if (wrap) {
        u -= std::floor(u);
        v -= std::floor(v);
    }
    auto idx = [&](long long i, int n) -> long long {
        if (wrap) return ((i % n) + n) % n;
        return std::min<long long>(std::max<long long>(i, 0), n - 1);
    };
    auto texel = [&](long long x, long long y) { return t.rgba + 4 * ((size_t)idx(y, H) * W + (size_t)idx(x, W)); };
    if (t.filter != NOOR_FILTER_LINEAR) {
        const float* q = texel((long long)std::floor(u * W), (long long)std::floor(v * H));
        std::memcpy(out, q, 16);
        return;
    }
    const double x = u * W - 0.5, y = v * H - 0.5;
    long long x0 = (long long)std::floor(x), y0 = (long long)std::floor(y);
    long long A = (long long)std::floor((x - (double)x0) * 256.0 + 0.5);
    long long B = (long long)std::floor((y - (double)y0) * 256.0 + 0.5);
    if (A >= 256) { A = 0; ++x0; }
    if (B >= 256) { B = 0; ++y0; }
    const long long P = A * B;
    const long long w11 = P / 256 + ((P % 256) >= 128 ? 1 : 0);
    const long long w10 = A - w11, w01 = B - w11, w00 = 256 - A - B + w11;
    const float *t00 = texel(x0, y0), *t10 = texel(x0 + 1, y0), *t01 = texel(x0, y0 + 1), *t11 = texel(x0 + 1, y0 + 1);
    for (int c = 0; c < 4; ++c)
        out[c] = (float)(((double)w00 * t00[c] + (double)w10 * t10[c] + (double)w01 * t01[c] + (double)w11 * t11[c]) /
                         256.0);
}
// slot k of material m at uv (uvscale * uv)
template <class T> inline void slot_fetch(const Scene& sc, const Scene::Mat& m, int k, T u, T v, float out[4]) {
    const float su = m.uvs[k][0], sv = m.uvs[k][1];
    tex_fetch(sc.P->textures[m.tex[k]], (double)(float)((T)su * u), (double)(float)((T)sv * v), out);
}

// ------------------------------------------------------------ traversal
template <class T>
struct TRay {
    V<T> o, d, inv;
    int neg[3];
};
template <class T> inline void tray(TRay<T>& r, V<T> o, V<T> d) {
    r.o = o;
    r.d = d;
    r.inv = mk(T(1) / d.x, T(1) / d.y, T(1) / d.z);
    r.neg[0] = d.x > 0 ? 0 : 1;
    r.neg[1] = d.y > 0 ? 0 : 1;
    r.neg[2] = d.z > 0 ? 0 : 1;
}
// CudaRay::transformToObject (ray.cuh:174-180), CudaTransform (transform.cuh:56-63)
template <class T> inline void to_object(TRay<T>& r, const TRay<T>& w, const Scene& sc, uint32_t ins) {
    const noor_payload* P = sc.P;
    V<T> o, d;
    T oo[3], dd[3];
    for (int k = 0; k < 3; ++k) {
        const float* row = P->world_to_object_row[k] + 4 * (size_t)ins;
        const T a = row[0], b = row[1], c = row[2], t = row[3];
        oo[k] = t + ((a * w.o.x + b * w.o.y) + c * w.o.z);
        dd[k] = (a * w.d.x + b * w.d.y) + c * w.d.z;
    }
    o = mk(oo[0], oo[1], oo[2]);
    d = mk(dd[0], dd[1], dd[2]);
    tray(r, o, d);
}
// CudaBBox::intersect (bbox.cuh:62-80)
template <class T> inline bool slab(const TRay<T>& r, const uint32_t* lo, const uint32_t* hi, T tmax) {
    const T mn[3] = {(T)u2f(lo[0]), (T)u2f(lo[1]), (T)u2f(lo[2])};
    const T mx[3] = {(T)u2f(hi[0]), (T)u2f(hi[1]), (T)u2f(hi[2])};
    T tMin = ((r.neg[0] ? mx[0] : mn[0]) - r.o.x) * r.inv.x;
    T tMax = ((r.neg[0] ? mn[0] : mx[0]) - r.o.x) * r.inv.x;
    const T tyMin = ((r.neg[1] ? mx[1] : mn[1]) - r.o.y) * r.inv.y;
    const T tyMax = ((r.neg[1] ? mn[1] : mx[1]) - r.o.y) * r.inv.y;
    if (tMin > tyMax || tyMin > tMax) return false;
    if (tyMin > tMin) tMin = tyMin;
    if (tyMax < tMax) tMax = tyMax;
    const T tzMin = ((r.neg[2] ? mx[2] : mn[2]) - r.o.z) * r.inv.z;
    const T tzMax = ((r.neg[2] ? mn[2] : mx[2]) - r.o.z) * r.inv.z;
    if (tMin > tzMax || tzMin > tMax) return false;
    if (tzMin > tMin) tMin = tzMin;
    if (tzMax < tMax) tMax = tzMax;
    return (tMin < tmax) && (tMax > T(0));
}
// CudaTriangle::intersect (triangle.cuh:82-141)
template <class T> inline bool wald(const TRay<T>& r, const Scene& sc, uint32_t ti, T& tmax, T& bu, T& bv,
                                    uint32_t& mt, uint64_t* ctr) {
    const uint32_t* a = sc.P->wald_ax_nu_nv_nd + 4 * (size_t)ti;
    const uint32_t* c = sc.P->wald_cnu_cnv_deg_mat + 4 * (size_t)ti;
    if (c[2] == 1u) return false;
    const uint32_t k = a[0];
    const uint32_t ku = k == 0 ? 1 : (k == 1 ? 2 : 0), kv = k == 0 ? 2 : (k == 1 ? 0 : 1);
    const T ro_u = comp(r.o, ku), ro_v = comp(r.o, kv), ro_k = comp(r.o, k);
    const T rd_u = comp(r.d, ku), rd_v = comp(r.d, kv), rd_k = comp(r.d, k);
    const T nu = u2f(a[1]), nv = u2f(a[2]), nd = u2f(a[3]);
    const T denom = rd_k + nu * rd_u + nv * rd_v;
    if (denom == T(0)) return false;
    const T t = (nd - ro_k - nu * ro_u - nv * ro_v) / denom;
    if (t < T(0) || t > tmax) return false;
    if (ctr) ctr[2]++;
    const uint32_t* b = sc.P->wald_bnu_bnv_au_av + 4 * (size_t)ti;
    const T hu = ro_u + t * rd_u - (T)u2f(b[2]);
    const T hv = ro_v + t * rd_v - (T)u2f(b[3]);
    const T u = hv * (T)u2f(b[0]) + hu * (T)u2f(b[1]);
    const T v = hu * (T)u2f(c[0]) + hv * (T)u2f(c[1]);
    if (!(u >= T(0) && v >= T(0) && u + v <= T(1))) return false;
    tmax = t;
    bu = u;
    bv = v;
    mt = c[3];
    return true;
}
// Woop, Benthin & Wald 2013 watertight test (JCGT 2(1)), same operation order
// as the device version.
template <class T> struct WtRay {
    int kx, ky, kz;
    T sx, sy, sz;
};
template <class T> inline void wt_setup(WtRay<T>& w, V<T> d) {
    const T ax = std::fabs(d.x), ay = std::fabs(d.y), az = std::fabs(d.z);
    int kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    int kx = kz + 1 == 3 ? 0 : kz + 1;
    int ky = kx + 1 == 3 ? 0 : kx + 1;
    const T dz = comp(d, kz);
    if (dz < T(0)) std::swap(kx, ky);
    w.kx = kx;
    w.ky = ky;
    w.kz = kz;
    w.sx = comp(d, kx) / dz;
    w.sy = comp(d, ky) / dz;
    w.sz = T(1) / dz;
}
template <class T> inline T xorsign(T v, bool neg) { return neg ? -v : v; }
template <class T> inline bool wtt(const TRay<T>& r, const WtRay<T>& w, const Scene& sc, uint32_t ti, T& tmax, T& bu,
                                   T& bv, uint32_t& mt, uint64_t* ctr) {
    const uint32_t* at = sc.P->attribute_indices + 4 * (size_t)ti;
    V<T> p[3];
    for (int k = 0; k < 3; ++k) {
        const float* q = sc.P->vertices + 4 * (size_t)at[k];
        p[k] = mk((T)q[0], (T)q[1], (T)q[2]);
    }
    if (ctr) ctr[2]++;
    const V<T> A = p[0] - r.o, B = p[1] - r.o, C = p[2] - r.o;
    const T Akz = comp(A, w.kz), Bkz = comp(B, w.kz), Ckz = comp(C, w.kz);
    const T Ax = comp(A, w.kx) - w.sx * Akz, Ay = comp(A, w.ky) - w.sy * Akz;
    const T Bx = comp(B, w.kx) - w.sx * Bkz, By = comp(B, w.ky) - w.sy * Bkz;
    const T Cx = comp(C, w.kx) - w.sx * Ckz, Cy = comp(C, w.ky) - w.sy * Ckz;
    T U = Cx * By - Cy * Bx;
    T Vv = Ax * Cy - Ay * Cx;
    T W = Bx * Ay - By * Ax;
    if (U == T(0) || Vv == T(0) || W == T(0)) {
        U = (T)((double)Cx * (double)By - (double)Cy * (double)Bx);
        Vv = (T)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
        W = (T)((double)Bx * (double)Ay - (double)By * (double)Ax);
    }
    if ((U < T(0) || Vv < T(0) || W < T(0)) && (U > T(0) || Vv > T(0) || W > T(0))) return false;
    const T det = U + Vv + W;
    if (det == T(0)) return false;
    const T Az = w.sz * Akz, Bz = w.sz * Bkz, Cz = w.sz * Ckz;
    const T Tt = U * Az + Vv * Bz + W * Cz;
    const bool neg = std::signbit(det);
    const T Ts = xorsign(Tt, neg);
    if (Ts < T(0) || Ts > tmax * xorsign(det, neg)) return false;
    const T rcp = T(1) / det;
    tmax = Tt * rcp;
    bu = Vv * rcp;
    bv = W * rcp;
    mt = sc.P->wald_cnu_cnv_deg_mat[4 * (size_t)ti + 3];
    return true;
}
// intersectQuad (geometry.cuh:105-123)
template <class T> inline bool quad_hit(const noor_area_light& L, V<T> o, V<T> d, T& tmax) {
    const V<T> n = mk((T)L.shape.n[0], (T)L.shape.n[1], (T)L.shape.n[2]);
    const V<T> c = mk((T)L.shape.center[0], (T)L.shape.center[1], (T)L.shape.center[2]);
    const V<T> u = mk((T)L.shape.u[0], (T)L.shape.u[1], (T)L.shape.u[2]);
    const V<T> v = mk((T)L.shape.v[0], (T)L.shape.v[1], (T)L.shape.v[2]);
    const T denom = dot(n, d);
    if (denom == T(0)) return false;
    const T t = -(dot(o, n) - dot(c, n)) / denom;
    if (t > tmax) return false;
    const V<T> p = o + t * d;
    const V<T> ip = p - c;
    const T t0 = dot(ip, u) / dot(u, u);
    if (t0 < T(0) || t0 > T(1)) return false;
    const T t1 = dot(ip, v) / dot(v, v);
    if (t1 < T(0) || t1 > T(1)) return false;
    tmax = t;
    return true;
}
// solveQuadratic (utils.cuh:52-91)
template <class T> inline bool solve_quad(T a, T b, T c, T& x0, T& x1) {
    if (a == T(0)) {
        if (b != T(0)) {
            x0 = x1 = -c / b;
            return true;
        }
        return false;
    }
    const T disc = b * b - T(4) * a * c;
    if (disc < T(0)) return false;
    const T sd = std::sqrt(disc);
    const T q = b < T(0) ? T(-0.5) * (b - sd) : T(-0.5) * (b + sd);
    x0 = q / a;
    x1 = c / q;
    if (x0 > x1) std::swap(x0, x1);
    return true;
}
// intersectSphere / intersectDisk (geometry.cuh:125-163)
template <class T> inline bool sphere_hit(const noor_area_light& L, V<T> o, V<T> d, T& tmax) {
    const V<T> oc = o - mk((T)L.shape.center[0], (T)L.shape.center[1], (T)L.shape.center[2]);
    T t0, t1;
    if (!solve_quad<T>(dot(d, d), T(2) * dot(oc, d), dot(oc, oc) - (T)L.shape.radius2, t0, t1)) return false;
    if (!(t0 <= tmax && t1 >= T(0))) return false;
    if (t0 < T(0)) {
        if (t1 > tmax) return false;
        tmax = t1;
    } else {
        tmax = t0;
    }
    return true;
}
template <class T> inline bool disk_hit(const noor_area_light& L, V<T> o, V<T> d, T& tmax) {
    const V<T> n = mk((T)L.shape.n[0], (T)L.shape.n[1], (T)L.shape.n[2]);
    const V<T> c = mk((T)L.shape.center[0], (T)L.shape.center[1], (T)L.shape.center[2]);
    const T denom = dot(n, d);
    if (denom == T(0)) return false;
    const T t = -(dot(o, n) - dot(c, n)) / denom;
    if (t > tmax) return false;
    const V<T> p = (o + t * d) - c;
    if (dot(p, p) > (T)L.shape.radius2) return false;
    tmax = t;
    return true;
}
// CudaShape::intersect (shapeimp.cuh:73-87)
template <class T> inline bool shape_hit(const noor_area_light& L, V<T> o, V<T> d, T& tmax) {
    if (L.shape.type == NOOR_SHAPE_SPHERE) return sphere_hit<T>(L, o, d, tmax);
    if (L.shape.type == NOOR_SHAPE_DISK) return disk_hit<T>(L, o, d, tmax);
    return quad_hit<T>(L, o, d, tmax);
}

struct Hit {
    double u, v;
    uint32_t tri, ins, mt;
};

// texture coordinates of a vertex as the mesh manager returns them, v
// flipped (mesh.cuh:145-148), and their barycentric interpolation
template <class T> inline void vertex_uv(const Scene& sc, uint32_t i, T& x, T& y) {
    const float* q = sc.P->uvs + 2 * (size_t)i;
    x = q[0];
    y = T(1) - (T)q[1];
}
template <class T> inline void hit_uv(const Scene& sc, const uint32_t* a, T bu, T bv, T& u, T& v) {
    T u0, v0, u1, v1, u2, v2;
    vertex_uv(sc, a[0], u0, v0);
    vertex_uv(sc, a[1], u1, v1);
    vertex_uv(sc, a[2], u2, v2);
    const T w = T(1) - bu - bv;
    u = w * u0 + bu * u1 + bv * u2;
    v = w * v0 + bu * v1 + bv * v2;
}
// the alpha cut of an ALPHA material's triangle (triangle.cuh:124-133)
template <class T> inline bool alpha_cut(const Scene& sc, uint32_t ti, T bu, T bv) {
    const uint32_t* a = sc.P->attribute_indices + 4 * (size_t)ti;
    T u, v;
    hit_uv(sc, a, bu, bv, u, v);
    float c[4];
    slot_fetch<T>(sc, sc.mats[a[3]], TX_ALPHA, u, v, c);
    return c[0] <= 0.0001f;
}

// intersect / intersectP (bvh.cuh:142-234).  ctr (optional): nodes visited,
// triangles tested, triangles whose t fell in range.
template <class T>
bool traverse(const Scene& sc, V<T> o, V<T> d, T& tmax, Hit* rec, bool any, int isect, uint64_t* ctr) {
    const noor_payload* P = sc.P;
    TRay<T> wr, lr;
    tray(wr, o, d);
    lr = wr;
    WtRay<T> wt;
    wt_setup(wt, lr.d);
    T ltmax = tmax;
    uint32_t ins = 0;
    bool hit = false;
    std::vector<uint32_t> stack;
    stack.reserve(64);
    stack.push_back(sc.S->bvh_root_node);
    while (!stack.empty()) {
        const uint32_t ni = stack.back();
        stack.pop_back();
        if (ctr) ctr[0]++;
        const uint32_t* lo = P->bvh_min_right_start + 4 * (size_t)ni;
        const uint32_t* hi = P->bvh_max_axis_count + 4 * (size_t)ni;
        const uint32_t w1 = hi[3];
        if (w1 & NOOR_MESH_NODE_MASK) {
            lr = wr;
            ltmax = tmax;
            wt_setup(wt, lr.d);
        }
        if (!slab(lr, lo, hi, ltmax)) continue;
        if (w1 & NOOR_LIGHT_NODE_MASK) {
            const uint32_t li = w1 & NOOR_LIGHT_MASK;
            if (any) {
                T tm = tmax;
                if (shape_hit(P->area_lights[li], o, d, tm)) return true;
            } else if (shape_hit(P->area_lights[li], o, d, tmax)) {
                hit = true;
                rec->ins = li;
                rec->mt = NOOR_MESHLIGHT | NOOR_EMITTER;
            }
        } else if (w1 & NOOR_MESH_INSTANCE_MASK) {
            ins = w1 & NOOR_TRANS_MASK;
            to_object(lr, wr, sc, ins);
            ltmax = tmax;
            wt_setup(wt, lr.d);
            stack.push_back(lo[3]);
        } else if (w1 & NOOR_MESH_LEAF_MASK) {
            for (uint32_t i = 1; i <= (w1 & NOOR_COUNT_MASK); ++i) stack.push_back(ni + i);
        } else if (w1 & NOOR_TRI_LEAF_MASK) {
            const uint32_t s = lo[3], e = s + (w1 & NOOR_TRI_COUNT_MASK);
            bool lh = false;
            for (uint32_t ti = s; ti < e; ++ti) {
                if (ctr) ctr[1]++;
                T tm = any ? ltmax : ltmax, bu, bv;
                uint32_t mt;
                bool h = isect == NOOR_ISECT_WATERTIGHT ? wtt(lr, wt, sc, ti, tm, bu, bv, mt, ctr)
                                                        : wald(lr, sc, ti, tm, bu, bv, mt, ctr);
                if (h && (mt & NOOR_ALPHA) && alpha_cut<T>(sc, ti, bu, bv)) h = false;
                if (h) {
                    if (any) return true;
                    ltmax = tm;
                    lh = true;
                    rec->u = (double)bu;
                    rec->v = (double)bv;
                    rec->tri = ti;
                    rec->mt = mt;
                }
            }
            if (lh) {
                hit = true;
                tmax = ltmax;
                rec->ins = ins;
            }
        } else {
            const uint32_t axis = w1 & NOOR_AXIS_MASK;
            if (lr.neg[axis]) {
                stack.push_back(ni + 1);
                stack.push_back(lo[3]);
            } else {
                stack.push_back(lo[3]);
                stack.push_back(ni + 1);
            }
        }
    }
    return any ? false : hit;
}

// ------------------------------------------------------------- shading
template <class T> struct Frame {
    V<T> n, s, t, ng;
};
template <class T> inline V<T> to_local(const Frame<T>& F, V<T> v) { return mk(dot(v, F.s), dot(v, F.t), dot(v, F.n)); }
template <class T> inline V<T> to_world(const Frame<T>& F, V<T> v) { return v.x * F.s + v.y * F.t + v.z * F.n; }

// coordinateSystem (utils.cuh:340-347)
template <class T> inline void coord_sys(V<T> v1, V<T>& v2, V<T>& v3) {
    if (std::fabs(v1.x) > std::fabs(v1.y))
        v2 = mk(-v1.z, T(0), v1.x) / std::sqrt(v1.x * v1.x + v1.z * v1.z);
    else
        v2 = mk(T(0), v1.z, -v1.y) / std::sqrt(v1.y * v1.y + v1.z * v1.z);
    v3 = cross(v1, v2);
}

// what computeTangentSpace also keeps for textures and ray differentials
// (intersection.cuh:345-394): uv, dp/du and dp/dv before Gram-Schmidt,
// dn/du and dn/dv
template <class T> struct TOut {
    T u, v;
    V<T> dpdu, dpdv, dndu, dndv;
};

// computeTangentSpace (intersection.cuh:325-394)
template <class T> Frame<T> tangent(const Scene& sc, const Hit& h, TOut<T>* out = nullptr) {
    const noor_payload* P = sc.P;
    const uint32_t* a = P->attribute_indices + 4 * (size_t)h.tri;
    auto vtx = [&](uint32_t i) { const float* q = P->vertices + 4 * (size_t)i; return mk((T)q[0], (T)q[1], (T)q[2]); };
    auto nrmv = [&](uint32_t i) { const float* q = P->normals + 4 * (size_t)i; return mk((T)q[0], (T)q[1], (T)q[2]); };
    auto uv = [&](uint32_t i, T& x, T& y) { const float* q = P->uvs + 2 * (size_t)i; x = q[0]; y = T(1) - (T)q[1]; };
    T u0x, u0y, u1x, u1y, u2x, u2y;
    uv(a[0], u0x, u0y);
    uv(a[1], u1x, u1y);
    uv(a[2], u2x, u2y);
    const V<T> v0 = vtx(a[0]), v1 = vtx(a[1]), v2 = vtx(a[2]);
    const V<T> n0 = nrmv(a[0]), n1 = nrmv(a[1]), n2 = nrmv(a[2]);
    const T bu = (T)h.u, bv = (T)h.v;
    const T w = T(1) - bu - bv;
    const V<T> ni = w * n0 + bu * n1 + bv * n2;
    auto rowmul = [&](const float* const* rows, V<T> x) {
        T r[3];
        for (int k = 0; k < 3; ++k) {
            const float* q = rows[k] + 4 * (size_t)h.ins;
            r[k] = (T)q[0] * x.x + (T)q[1] * x.y + (T)q[2] * x.z;
        }
        return mk(r[0], r[1], r[2]);
    };
    Frame<T> F;
    F.n = nrm_g(nrm(rowmul(P->normal_row, ni)));
    const V<T> dp01 = rowmul(P->object_to_world_row, v1 - v0);
    const V<T> dp02 = rowmul(P->object_to_world_row, v2 - v0);
    F.ng = nrm_g(cross(dp01, dp02));
    const T d1x = u1x - u0x, d1y = u1y - u0y, d2x = u2x - u0x, d2y = u2y - u0y;
    const T det = d1x * d2y - d2x * d1y;
    V<T> dpdu, dpdv;
    if (!(std::fabs(det) < (T)1e-8f)) {
        const T inv = T(1) / det;
        const T a00 = d2y * inv, a01 = -d1y * inv, a10 = -d2x * inv, a11 = d1x * inv;
        dpdu = a00 * dp01 + a01 * dp02;
        dpdv = a10 * dp01 + a11 * dp02;
        if (len2(cross(dpdu, dpdv)) == T(0)) coord_sys(F.ng, dpdu, dpdv);
    } else {
        coord_sys(F.ng, dpdu, dpdv);
    }
    F.s = nrm_g(dpdu - F.n * dot(F.n, dpdu));
    const T sg = dot(cross(F.n, F.s), dpdv) < T(0) ? T(-1) : T(1);
    F.t = nrm_g(sg * cross(F.n, F.s));
    if (out) {
        out->u = w * u0x + bu * u1x + bv * u2x;
        out->v = w * u0y + bu * u1y + bv * u2y;
        out->dpdu = dpdu;
        out->dpdv = dpdv;
        const V<T> dn01 = n1 - n0, dn02 = n2 - n0;
        if (!(std::fabs(det) < (T)1e-8f)) {
            const T inv = T(1) / det;
            const T a00 = d2y * inv, a01 = -d1y * inv, a10 = -d2x * inv, a11 = d1x * inv;
            out->dndu = a00 * dn01 + a01 * dn02;
            out->dndv = a10 * dn01 + a11 * dn02;
        } else {
            const V<T> dn = nrm_g(nrm(rowmul(P->normal_row, cross(dn01, dn02))));
            if (len2(dn) == T(0))
                out->dndu = out->dndv = mk(T(0), T(0), T(0));
            else
                coord_sys(dn, out->dndu, out->dndv);
        }
    }
    return F;
}

// the material's per-hit slots at uv (materialimp.cuh:121-183)
template <class T> inline Scene::Mat textured(const Scene& sc, const Scene::Mat& m0, T u, T v) {
    Scene::Mat m = m0;
    float c[4];
    auto rgb = [&](int k, float* dst) {
        if (!(m.tex_mask & (1u << k))) return;
        slot_fetch<T>(sc, m, k, u, v, c);
        std::memcpy(dst, c, 12);
    };
    rgb(TX_DIFFUSE, m.diffuse);
    rgb(TX_SPECULAR, m.specular);
    rgb(TX_EMITTANCE, m.emittance);
    rgb(TX_TRANSMISSION, m.transmission);
    rgb(TX_IOR, m.ior);
    rgb(TX_K, m.k);
    if (m.tex_mask & (1u << TX_ROUGHNESS)) {
        slot_fetch<T>(sc, m, TX_ROUGHNESS, u, v, c);
        m.rx = c[0];
        m.ry = c[1];
    }
    return m;
}

// ray differentials (CudaRay, ray.cuh:36-200), world space
template <class T> struct RDiff {
    bool on = false;
    V<T> odx, ody, ddx, ddy;
};
template <class T> struct HDiff {
    V<T> dpdx, dpdy, dndu, dndv;
    T dudx = 0, dudy = 0, dvdx = 0, dvdy = 0;
};
// NOOR::solve2x2 (math.cuh:192-207)
template <class T> inline void solve2(T a00, T a01, T a10, T a11, T b0, T b1, T& x0, T& x1) {
    const T det = a00 * a11 - a10 * a01;
    if (std::fabs(det) < (T)1e-10f) {
        x0 = x1 = T(0);
        return;
    }
    const T inv = T(1) / det;
    x0 = (a11 * b0 - a01 * b1) * inv;
    x1 = (a00 * b1 - a10 * b0) * inv;
    if (std::isnan(x0) || std::isnan(x1)) x0 = x1 = T(0);
}
// computeDifferential (intersection.cuh:397-441)
template <class T> HDiff<T> hit_diff(const Frame<T>& F, V<T> p, const TOut<T>& to, const RDiff<T>& rd) {
    HDiff<T> h;
    h.dndu = to.dndu;
    h.dndv = to.dndv;
    h.dpdx = h.dpdy = mk(T(0), T(0), T(0));
    const V<T>& n = F.ng;
    const T dd = dot(n, p);
    const T tx = -(dot(n, rd.odx) - dd) / dot(n, rd.ddx);
    if (std::isinf(tx) || std::isnan(tx)) return h;
    const V<T> px = rd.odx + tx * rd.ddx;
    const T ty = -(dot(n, rd.ody) - dd) / dot(n, rd.ddy);
    if (std::isinf(ty) || std::isnan(ty)) return h;
    const V<T> py = rd.ody + ty * rd.ddy;
    h.dpdx = px - p;
    h.dpdy = py - p;
    int ax, ay;
    if (std::fabs(n.x) > std::fabs(n.y) && std::fabs(n.x) > std::fabs(n.z)) {
        ax = 1;
        ay = 2;
    } else if (std::fabs(n.y) > std::fabs(n.z)) {
        ax = 0;
        ay = 2;
    } else {
        ax = 0;
        ay = 1;
    }
    const T a00 = comp(to.dpdu, ax), a01 = comp(to.dpdv, ax), a10 = comp(to.dpdu, ay), a11 = comp(to.dpdv, ay);
    solve2(a00, a01, a10, a11, comp(h.dpdx, ax), comp(h.dpdx, ay), h.dudx, h.dvdx);
    solve2(a00, a01, a10, a11, comp(h.dpdy, ax), comp(h.dpdy, ay), h.dudy, h.dvdy);
    return h;
}
// bump (accumulate.cuh:47-75)
template <class T> void bump_frame(const Scene& sc, const Scene::Mat& m, T u, T v, const HDiff<T>& h, Frame<T>& F) {
    T du = T(0.5) * (std::fabs(h.dudx) + std::fabs(h.dudy));
    T dv = T(0.5) * (std::fabs(h.dvdx) + std::fabs(h.dvdy));
    du = du == T(0) ? (T)0.001f : du;
    dv = dv == T(0) ? (T)0.001f : dv;
    float c[4];
    slot_fetch<T>(sc, m, TX_BUMP, u, v, c);
    const T disp = c[0];
    const T scale = m.bumpfactor;
    slot_fetch<T>(sc, m, TX_BUMP, u + du, v + T(0), c);
    const T ud = scale * ((T)c[0] - disp) / du;
    slot_fetch<T>(sc, m, TX_BUMP, u + T(0), v + dv, c);
    const T vd = scale * ((T)c[0] - disp) / dv;
    const V<T> sn = F.n;
    V<T> dpdu = F.s + ud * sn;
    const V<T> dpdv = F.t + vd * sn;
    const V<T> n = nrm_g(cross(dpdu, dpdv));
    dpdu = nrm_g(dpdu - n * dot(n, dpdu));
    F.t = nrm_g(cross(n, dpdu));
    F.s = dpdu;
    F.n = dot(F.ng, n) < T(0) ? T(-1) * n : n;
}

// bxdf.cuh:58-96
template <class T> inline T c2t(V<T> w) { return w.z * w.z; }
template <class T> inline T s2t(V<T> w) { return std::max(T(0), T(1) - c2t(w)); }
template <class T> inline T st_(V<T> w) { return std::sqrt(s2t(w)); }
template <class T> inline T tnt(V<T> w) { return st_(w) / w.z; }
template <class T> inline T t2t(V<T> w) { return s2t(w) / c2t(w); }
template <class T> inline T cph(V<T> w) { const T s = st_(w); return s == T(0) ? T(1) : clampv(w.x / s, T(-1), T(1)); }
template <class T> inline T sph(V<T> w) { const T s = st_(w); return s == T(0) ? T(0) : clampv(w.y / s, T(-1), T(1)); }
template <class T> inline T c2p(V<T> w) { return cph(w) * cph(w); }
template <class T> inline T s2p(V<T> w) { return sph(w) * sph(w); }
template <class T> inline bool same(V<T> a, V<T> b) { return a.z * b.z > T(0); }

// fresnel.cuh:58-107
template <class T> T fr_diel(T ci, T ei, T et) {
    ci = clampv(ci, T(-1), T(1));
    if (!(ci > T(0))) {
        std::swap(ei, et);
        ci = std::fabs(ci);
    }
    const T si = std::sqrt(std::max(T(0), T(1) - ci * ci));
    const T st = ei / et * si;
    if (st >= T(1)) return T(1);
    const T ct = std::sqrt(std::max(T(0), T(1) - st * st));
    const T rpa = ((et * ci) - (ei * ct)) / ((et * ci) + (ei * ct));
    const T rpe = ((ei * ci) - (et * ct)) / ((ei * ci) + (et * ct));
    return (rpa * rpa + rpe * rpe) / T(2);
}
template <class T> V<T> sq3(V<T> v) { return mk(std::sqrt(v.x), std::sqrt(v.y), std::sqrt(v.z)); }
template <class T> V<T> fr_cond(T ci, V<T> etaT, V<T> k) {
    ci = clampv(ci, T(-1), T(1));
    const V<T> one = mk(T(1), T(1), T(1));
    const V<T> eta = etaT / one, etak = k / one;
    const T c2 = ci * ci, s2 = T(1) - c2;
    const V<T> eta2 = eta * eta, etak2 = etak * etak;
    const V<T> t0 = eta2 - etak2 - mk(s2, s2, s2);
    const V<T> a2b2 = sq3(t0 * t0 + T(4) * eta2 * etak2);
    const V<T> t1 = a2b2 + mk(c2, c2, c2);
    const V<T> a = sq3(T(0.5) * (a2b2 + t0));
    const V<T> t2 = T(2) * ci * a;
    const V<T> Rs = (t1 - t2) / (t1 + t2);
    const V<T> t3 = c2 * a2b2 + mk(s2 * s2, s2 * s2, s2 * s2);
    const V<T> t4 = t2 * s2;
    const V<T> Rp = Rs * (t3 - t4) / (t3 + t4);
    return T(0.5) * (Rp + Rs);
}

// distribution.cuh:58-342
template <class T> T erf_as(T x) {
    const T a1 = (T)0.254829592f, a2 = (T)-0.284496736f, a3 = (T)1.421413741f, a4 = (T)-1.453152027f,
            a5 = (T)1.061405429f, p = (T)0.3275911f;
    const int sg = x < T(0) ? -1 : 1;
    x = std::fabs(x);
    const T t = T(1) / (T(1) + p * x);
    const T y = T(1) - (((((a5 * t + a4) * t) + a3) * t + a2) * t + a1) * t * std::exp(-x * x);
    return (T)sg * y;
}
template <class T> T erfinv_g(T x) {
    T w, p;
    x = clampv(x, (T)-.99999f, (T).99999f);
    w = -std::log((T(1) - x) * (T(1) + x));
    if (w < T(5)) {
        w = w - (T)2.5f;
        p = (T)2.81022636e-08f;
        p = (T)3.43273939e-07f + p * w;
        p = (T)-3.5233877e-06f + p * w;
        p = (T)-4.39150654e-06f + p * w;
        p = (T)0.00021858087f + p * w;
        p = (T)-0.00125372503f + p * w;
        p = (T)-0.00417768164f + p * w;
        p = (T)0.246640727f + p * w;
        p = (T)1.50140941f + p * w;
    } else {
        w = std::sqrt(w) - T(3);
        p = (T)-0.000200214257f;
        p = (T)0.000100950558f + p * w;
        p = (T)0.00134934322f + p * w;
        p = (T)-0.00367342844f + p * w;
        p = (T)0.00573950773f + p * w;
        p = (T)-0.0076224613f + p * w;
        p = (T)0.00943887047f + p * w;
        p = (T)1.00167406f + p * w;
        p = (T)2.83297682f + p * w;
    }
    return p * x;
}
template <class T> struct Micro {
    T ax, ay;
    uint32_t dist;
    T D(V<T> wh) const {
        const T t2 = t2t(wh);
        if (std::isinf(t2)) return T(0);
        const T c4 = c2t(wh) * c2t(wh);
        if (dist) return std::exp(-t2 * (c2p(wh) / (ax * ax) + s2p(wh) / (ay * ay))) / (K<T>::pi * ax * ay * c4);
        const T e = (c2p(wh) / (ax * ax) + s2p(wh) / (ay * ay)) * t2;
        return T(1) / (K<T>::pi * ax * ay * c4 * (T(1) + e) * (T(1) + e));
    }
    T lambda(V<T> w) const {
        const T at = std::fabs(tnt(w));
        if (std::isinf(at)) return T(0);
        const T alpha = std::sqrt(c2p(w) * ax * ax + s2p(w) * ay * ay);
        if (dist) {
            const T a = T(1) / (alpha * at);
            if (a >= (T)1.6f) return T(0);
            return (T(1) - (T)1.259f * a + (T)0.396f * a * a) / ((T)3.535f * a + (T)2.181f * a * a);
        }
        const T a2t2 = (alpha * at) * (alpha * at);
        return (T(-1) + std::sqrt(T(1) + a2t2)) / T(2);
    }
    T G(V<T> wo, V<T> wi) const { return T(1) / (T(1) + lambda(wo) + lambda(wi)); }
    T G1(V<T> w) const { return T(1) / (T(1) + lambda(w)); }
    T pdf(V<T> wo, V<T> wh) const { return D(wh) * G1(wo) * std::fabs(dot(wo, wh)) / std::fabs(wo.z); }
    void s11_tr(T ct, T U1, T U2, T& sx, T& sy) const {
        if (ct > (T).9999f) {
            const T r = std::sqrt(U1 / (T(1) - U1));
            const T phi = (T)6.28318530718f * U2;
            sx = r * std::cos(phi);
            sy = r * std::sin(phi);
            return;
        }
        const T s = std::sqrt(std::max(T(0), T(1) - ct * ct));
        const T tn = s / ct;
        const T a = T(1) / tn;
        const T G1v = T(2) / (T(1) + std::sqrt(T(1) + T(1) / (a * a)));
        const T A = T(2) * U1 / G1v - T(1);
        T tmp = T(1) / (A * A - T(1));
        if (tmp > (T)1e10f) tmp = (T)1e10f;
        const T B = tn;
        const T Dd = std::sqrt(std::max(B * B * tmp * tmp - (A * A - B * B) * tmp, T(0)));
        const T x1 = B * tmp - Dd, x2 = B * tmp + Dd;
        sx = (A < T(0) || x2 > T(1) / tn) ? x1 : x2;
        T S;
        if (U2 > (T)0.5f) {
            S = T(1);
            U2 = T(2) * (U2 - (T).5f);
        } else {
            S = T(-1);
            U2 = T(2) * ((T).5f - U2);
        }
        const T z = (U2 * (U2 * (U2 * (T)0.27385f - (T)0.73369f) + (T)0.46341f)) /
                    (U2 * (U2 * (U2 * (T)0.093073f + (T)0.309420f) - (T)1.000000f) + (T)0.597999f);
        sy = S * z * std::sqrt(T(1) + sx * sx);
    }
    void s11_bk(T ci, T U1, T U2, T& sx, T& sy) const {
        if (ci > (T).9999f) {
            const T r = std::sqrt(-std::log(T(1) - U1));
            sx = r * std::cos(T(2) * K<T>::pi * U2);
            sy = r * std::sin(T(2) * K<T>::pi * U2);
            return;
        }
        const T si = std::sqrt(std::max(T(0), T(1) - ci * ci));
        const T ti = si / ci, coti = T(1) / ti;
        T a = T(-1), c = erf_as(coti);
        const T sxx = std::max(U1, (T)1e-6f);
        const T th = std::acos(ci);
        const T fit = T(1) + th * ((T)-0.876f + th * ((T)0.4265f - (T)0.0594f * th));
        T b = c - (T(1) + c) * std::pow(T(1) - sxx, fit);
        const T nz = T(1) / (T(1) + c + std::sqrt(K<T>::inv_pi) * ti * std::exp(-coti * coti));
        int it = 0;
        while (++it < 10) {
            if (!(b >= a && b <= c)) b = (T)0.5f * (a + c);
            const T ie = erfinv_g(b);
            const T val = nz * (T(1) + b + std::sqrt(K<T>::inv_pi) * ti * std::exp(-ie * ie)) - sxx;
            const T der = nz * (T(1) - ie * ti);
            if (std::fabs(val) < (T)1e-5f) break;
            if (val > T(0)) c = b; else a = b;
            b -= val / der;
        }
        sx = erfinv_g(b);
        sy = erfinv_g(T(2) * std::max(U2, (T)1e-6f) - T(1));
    }
    V<T> vis(V<T> wi, T U1, T U2) const {
        const V<T> ws = nrm(mk(ax * wi.x, ay * wi.y, wi.z));
        T sx, sy;
        if (dist) s11_bk(ws.z, U1, U2, sx, sy); else s11_tr(ws.z, U1, U2, sx, sy);
        const T tmp = cph(ws) * sx - sph(ws) * sy;
        sy = sph(ws) * sx + cph(ws) * sy;
        sx = tmp;
        sx *= ax;
        sy *= ay;
        return nrm(mk(-sx, -sy, T(1)));
    }
    V<T> sample_wh(V<T> wo, T u1, T u2) const {
        if (dist) {
            const bool flip = wo.z < T(0);
            V<T> wh = vis(flip ? T(-1) * wo : wo, u1, u2);
            return flip ? T(-1) * wh : wh;
        }
        const T s = signv(wo.z);
        return s * vis(s * wo, u1, u2);
    }
};

enum : uint32_t {
    B_REFL = 1u, B_TRANS = 2u, B_DIFF = 4u, B_GLOSSY = 8u, B_SPEC = 16u, B_COND = 32u, B_DIEL = 64u, B_NOOP = 128u,
    B_ALL = 0xFFu
};
// lobe ids, one per BxDF class of bxdf.cuh:119-137 the factory builds
enum : uint32_t {
    kLambert = 1, kCond = 2, kFSpec = 3, kLambertT = 4, kMirror = 5, kMicroDiel = 6, kMicroT = 7, kFBlend = 8,
    kCoat = 9, kCatcher = 10
};
// the BxDF type flags of each lobe (the constructors in bxdf.cuh)
inline uint32_t ltype(uint32_t id) {
    switch (id) {
        case kLambert: return B_REFL | B_DIFF | B_DIEL;
        case kCond: return B_COND | B_REFL | B_GLOSSY;
        case kFSpec: return B_REFL | B_TRANS | B_SPEC | B_DIEL;
        case kLambertT: return B_TRANS | B_DIFF | B_DIEL;
        case kMirror: return B_NOOP | B_REFL | B_SPEC;
        case kMicroDiel: return B_DIEL | B_REFL | B_GLOSSY;
        case kMicroT: return B_TRANS | B_GLOSSY | B_DIEL;
        case kFBlend: return B_REFL | B_GLOSSY | B_DIEL;
        case kCoat: return B_GLOSSY | B_REFL | B_SPEC;
        case kCatcher: return B_REFL | B_TRANS | B_DIFF;
        default: return 0u;
    }
}
const uint32_t kSpecMat = NOOR_MIRROR | NOOR_GLASS | NOOR_CLEARCOAT;
const uint32_t kTranspMat = NOOR_TRANSLUCENT | NOOR_GLASS | NOOR_ROUGHGLASS;
const uint32_t kEmitMat = NOOR_EMITTER | NOOR_MESHLIGHT;

// factoryBSDF (bsdf.cuh:383-461): the lobes in Add order, 8 bits each
inline uint32_t lobe_of(uint32_t mt) {
    const uint32_t t = mt & ~(uint32_t)(NOOR_BUMP | NOOR_ALPHA);
    switch (t) {
        case NOOR_DIFFUSE: return kLambert;
        case NOOR_METAL: return kCond;
        case NOOR_GLASS: return kFSpec;
        case NOOR_MIRROR: return kMirror;
        case NOOR_SUBSTRATE: return kFBlend;
        case NOOR_TRANSLUCENT: return kLambert | kLambertT << 8;
        case NOOR_GLOSSY: return kLambert | kMicroDiel << 8;
        case NOOR_ROUGHGLASS: return kMicroDiel | kMicroT << 8;
        case NOOR_CLEARCOAT: return kCoat;
        case NOOR_SHADOWCATCHER: return kCatcher;
        default: return 0u;
    }
}
inline uint32_t lobe_at(uint32_t lobes, int k) { return (lobes >> (8 * k)) & 0xFFu; }
inline bool matches(uint32_t id, uint32_t flags) {
    const uint32_t t = ltype(id);
    return t && (t & flags) == t;
}
template <class T> V<T> v3f(const float* f) { return mk((T)f[0], (T)f[1], (T)f[2]); }

template <class T> Micro<T> micro(const Scene::Mat& m) {
    Micro<T> mf;
    mf.ax = std::max((T)m.rx * (T)m.rx, (T)1e-3f);
    mf.ay = std::max((T)m.ry * (T)m.ry, (T)1e-3f);
    mf.dist = m.dist;
    return mf;
}
// Refract (bxdf.cuh:103-116)
template <class T> bool refract_r(V<T> wi, V<T> n, T eta, V<T>& wt) {
    const T ci = dot(n, wi);
    const T s2i = std::max(T(0), T(1) - ci * ci);
    const T s2t = eta * eta * s2i;
    if (s2t >= T(1)) return false;
    const T ct = std::sqrt(T(1) - s2t);
    wt = (-eta) * wi + (eta * ci - ct) * n;
    return true;
}
template <class T> T pow5(T v) {
    const T a = v * v;
    return a * a * v;
}
// CudaClearCoat helpers (bxdf.cuh:849-908): absorption, the refraction of
// wo and wi into the substrate (negated; a failed one leaves zero), the
// probability of the coat
template <class T> T coat_abs(const Scene::Mat& m, V<T> wo, V<T> wi) {
    const T sa = (T)m.coat_sigma * (T)m.coat_thickness;
    if (sa != T(0)) return std::exp(-sa * (T(1) / std::fabs(wo.z) + T(1) / std::fabs(wi.z)));
    return T(1);
}
template <class T> void coat_in(const Scene::Mat& m, V<T> wo, V<T> wi, V<T>& wo_c, V<T>& wi_c) {
    const T eta = T(1) / (T)m.coat_ior;
    const V<T> n = mk(T(0), T(0), T(1));
    wo_c = mk(T(0), T(0), T(0));
    wi_c = wo_c;
    refract_r<T>(wo, n, eta, wo_c);
    refract_r<T>(wi, n, eta, wi_c);
    wo_c = T(-1) * wo_c;
    wi_c = T(-1) * wi_c;
}
template <class T> T coat_p(const Scene::Mat& m, T F) {
    const T w = (T)m.coat_weight;
    return F * w / (F * w + (T(1) - F) * (T(1) - w));
}
template <class T> V<T> lobe_eval(uint32_t lobe, const Scene::Mat& m, V<T> wo, V<T> wi);

// BxDF Eval of bxdf.cuh: 252-299 (Lambert), 301-352 (Lambert
// transmission), 472-557 (MicrofacetReflection), 559-656 (Microfacet-
// Transmission), 658-752 (FresnelBlend)
template <class T> V<T> lobe_eval(uint32_t lobe, const Scene::Mat& m, V<T> wo, V<T> wi) {
    const V<T> zero = mk(T(0), T(0), T(0));
    if (lobe == kLambert || lobe == kLambertT) return v3f<T>(m.diffuse) * K<T>::inv_pi;
    if (lobe == kCond || lobe == kMicroDiel) {
        if (!same(wo, wi)) return zero;
        const T cO = std::fabs(wo.z), cI = std::fabs(wi.z);
        if (cI == T(0) || cO == T(0)) return zero;
        V<T> wh = nrm(wi + wo);
        if (black(wh)) return zero;
        wh = wh * signv(wh.z);
        const V<T> F = lobe == kCond ? fr_cond(dot(wo, wh), v3f<T>(m.ior), v3f<T>(m.k))
                                     : mk(T(1), T(1), T(1)) * fr_diel(dot(wo, wh), T(1), (T)m.coat_ior);
        const Micro<T> mf = micro<T>(m);
        return F * v3f<T>(m.specular) * mf.D(wh) * mf.G(wo, wi) / (T(4) * cI * cO);
    }
    if (lobe == kMicroT) {
        if (same(wo, wi)) return zero;
        const T cO = wo.z, cI = wi.z;
        if (cI == T(0) || cO == T(0)) return zero;
        const T ior = (T)m.coat_ior;
        const T eta = wo.z > T(0) ? ior / T(1) : T(1) / ior;
        V<T> wh = nrm_g(wo + wi * eta);
        wh = wh * signv(wh.z);
        const T F = fr_diel(dot(wo, wh), T(1), ior);
        const T sd = dot(wo, wh) + eta * dot(wi, wh);
        const Micro<T> mf = micro<T>(m);
        return (T(1) - F) * v3f<T>(m.transmission) *
               std::fabs(mf.D(wh) * mf.G(wo, wi) * eta * eta * std::fabs(dot(wi, wh)) * std::fabs(dot(wo, wh)) /
                         (cI * cO * sd * sd));
    }
    if (lobe == kFBlend) {
        const V<T> S = v3f<T>(m.specular), one = mk(T(1), T(1), T(1));
        const V<T> diffuse = (T(28) / (T(23) * K<T>::pi)) * v3f<T>(m.diffuse) * (one - S) *
                             (T(1) - pow5(T(1) - T(0.5) * std::fabs(wi.z))) *
                             (T(1) - pow5(T(1) - T(0.5) * std::fabs(wo.z)));
        V<T> wh = wi + wo;
        if (wh.x == T(0) && wh.y == T(0) && wh.z == T(0)) return zero;
        wh = nrm_g(wh);
        const Micro<T> mf = micro<T>(m);
        const T c = dot(wi, wh);
        const V<T> schlick = S + pow5(T(1) - c) * (one - S);
        const V<T> specular =
            mf.D(wh) / (T(4) * std::fabs(dot(wi, wh)) * std::max(std::fabs(wi.z), std::fabs(wo.z))) * schlick;
        return diffuse + specular;
    }
    if (lobe == kCoat) {
        const T F0 = fr_diel(wo.z, T(1), (T)m.coat_ior), F1 = fr_diel(wi.z, T(1), (T)m.coat_ior);
        V<T> wo_c, wi_c;
        coat_in<T>(m, wo, wi, wo_c, wi_c);
        return lobe_eval<T>(kCond, m, wo_c, wi_c) * (T(1) - F0) * (T(1) - F1) * coat_abs<T>(m, wo_c, wi_c);
    }
    // the shadow catcher's 1 / |cos wi|; the caller multiplies in the sky
    if (lobe == kCatcher) return mk(T(1), T(1), T(1)) * (T(1) / std::fabs(wi.z));
    return zero;
}
template <class T> T lobe_pdf(uint32_t lobe, const Scene::Mat& m, V<T> wo, V<T> wi) {
    if (lobe == kLambert) return same(wo, wi) ? std::fabs(wi.z) * K<T>::inv_pi : T(0);
    if (lobe == kLambertT) return !same(wo, wi) ? std::fabs(wi.z) * K<T>::inv_pi : T(0);
    if (lobe == kCond || lobe == kMicroDiel) {
        if (!same(wo, wi)) return T(0);
        const V<T> wh = nrm_g(wo + wi);
        const Micro<T> mf = micro<T>(m);
        return mf.pdf(wo, wh) / (T(4) * dot(wo, wh));
    }
    if (lobe == kMicroT) {
        if (same(wo, wi)) return T(0);
        const T ior = (T)m.coat_ior;
        const T eta = wo.z > T(0) ? ior / T(1) : T(1) / ior;
        const V<T> wh = nrm_g(wo + wi * eta);
        const T sd = dot(wo, wh) + eta * dot(wi, wh);
        const T dwh = std::fabs((eta * eta * dot(wi, wh)) / (sd * sd));
        const Micro<T> mf = micro<T>(m);
        return mf.pdf(wo, wh) * dwh;
    }
    if (lobe == kFBlend) {
        if (!same(wo, wi)) return T(0);
        const V<T> wh = nrm_g(wo + wi);
        const Micro<T> mf = micro<T>(m);
        const T pwh = mf.pdf(wo, wh);
        return T(0.5) * (std::fabs(wi.z) * K<T>::inv_pi + pwh / (T(4) * dot(wo, wh)));
    }
    if (lobe == kCoat) {
        const T F = fr_diel(wo.z, T(1), (T)m.coat_ior);
        V<T> wo_c, wi_c;
        coat_in<T>(m, wo, wi, wo_c, wi_c);
        const T c = coat_p<T>(m, F);
        return lobe_pdf<T>(kCond, m, wo_c, wi_c) * (T(1) - c) + c;
    }
    if (lobe == kCatcher) return T(1);
    return T(0);
}
// concentricSampleDisk / cosineSampleHemisphere (utils.cuh:377-404)
template <class T> void conc_disk(T ux, T uy, T& dx, T& dy) {
    const T ox = T(2) * ux - T(1), oy = T(2) * uy - T(1);
    dx = 0;
    dy = 0;
    if (!(ox == T(0) && oy == T(0))) {
        T th, r;
        if (std::fabs(ox) > std::fabs(oy)) {
            r = ox;
            th = (K<T>::pi / T(4)) * (oy / ox);
        } else {
            r = oy;
            th = (K<T>::pi / T(2)) - (K<T>::pi / T(4)) * (ox / oy);
        }
        dx = r * std::cos(th);
        dy = r * std::sin(th);
    }
}
template <class T> V<T> cos_hemi(T ux, T uy) {
    T dx, dy;
    conc_disk<T>(ux, uy, dx, dy);
    return mk(dx, dy, std::sqrt(std::max(T(0), T(1) - dx * dx - dy * dy)));
}
const float kOneMinusEpsF = 1.0f - std::numeric_limits<float>::epsilon();
// BxDF Sample_f (u already remapped by the BSDF); st = the sampled type
template <class T> V<T> lobe_sample(uint32_t lobe, const Scene::Mat& m, V<T> wo, T ux, T uy, V<T>& wi, T& pdf,
                                    uint32_t& st) {
    st = ltype(lobe);
    const V<T> zero = mk(T(0), T(0), T(0));
    if (lobe == kLambert || lobe == kLambertT) {
        wi = cos_hemi(ux, uy);
        if (lobe == kLambert ? wo.z < T(0) : wo.z > T(0)) wi.z = wi.z * T(-1);
        pdf = lobe_pdf<T>(lobe, m, wo, wi);
        return v3f<T>(m.diffuse) * K<T>::inv_pi;
    }
    if (lobe == kCond || lobe == kMicroDiel) {
        if (wo.z == T(0)) return zero;
        const Micro<T> mf = micro<T>(m);
        const V<T> wh = mf.sample_wh(wo, ux, uy);
        wi = T(-1) * wo + T(2) * dot(wo, wh) * wh;
        if (!same(wo, wi)) {
            pdf = T(0);
            return zero;
        }
        pdf = mf.pdf(wo, wh) / (T(4) * dot(wo, wh));
        return lobe_eval<T>(lobe, m, wo, wi);
    }
    if (lobe == kMirror) {
        // specular reflection with the no-op Fresnel (bxdf.cuh:377-392)
        wi = mk(-wo.x, -wo.y, wo.z);
        pdf = T(1);
        return v3f<T>(m.diffuse) / std::fabs(wi.z);
    }
    if (lobe == kMicroT) {
        if (wo.z == T(0)) return zero;
        const Micro<T> mf = micro<T>(m);
        V<T> wh = mf.sample_wh(wo, ux, uy);
        const T ior = (T)m.coat_ior;
        const T eta = wo.z > T(0) ? T(1) / ior : ior / T(1);
        if (!refract_r(wo, wh, eta, wi)) {
            // helper_math's reflect(i, n) = i - 2 n (n . i), as the reference calls it
            wi = wo - T(2) * wh * dot(wh, wo);
            wh = wh * signv(wh.z);
            const T F = fr_diel(dot(wi, wh), T(1), ior);
            const T cO = wo.z, cI = wi.z;
            const V<T> r = F * v3f<T>(m.specular) * mf.D(wh) * mf.G(wo, wi) / (T(4) * cI * cO);
            pdf = mf.pdf(wo, wh) / (T(4) * dot(wo, wh));
            return r;
        }
        pdf = lobe_pdf<T>(lobe, m, wo, wi);
        return lobe_eval<T>(lobe, m, wo, wi);
    }
    if (lobe == kFBlend) {
        if (ux < T(0.5)) {
            const T lx = (T)std::min((float)(T(2) * ux), kOneMinusEpsF);
            wi = cos_hemi(lx, uy);
            wi.z = wi.z * signv(wi.z);
        } else {
            const T lx = (T)std::min((float)(T(2) * (ux - T(0.5))), kOneMinusEpsF);
            const Micro<T> mf = micro<T>(m);
            const V<T> wh = mf.sample_wh(wo, lx, uy);
            wi = T(-1) * wo + T(2) * dot(wo, wh) * wh;
            if (!same(wo, wi)) return zero;
        }
        pdf = lobe_pdf<T>(lobe, m, wo, wi);
        return lobe_eval<T>(lobe, m, wo, wi);
    }
    if (lobe == kCoat) {
        const T ior = (T)m.coat_ior;
        const T F0 = fr_diel(wo.z, T(1), ior);
        const T ps = coat_p<T>(m, F0);
        if (uy < ps) {
            wi = mk(-wo.x, -wo.y, wo.z);
            pdf = ps;
            st = B_DIEL | B_REFL | B_SPEC;
            return fr_diel(wi.z, T(1), ior) * v3f<T>(m.diffuse) / std::fabs(wi.z);
        }
        const T sy = (uy - ps) / (T(1) - ps);
        const T eta = T(1) / ior;
        V<T> wo_c = zero, wi_c = zero;
        refract_r<T>(wo, mk(T(0), T(0), T(1)), eta, wo_c);
        T p = 0;
        uint32_t st2;
        V<T> r = lobe_sample<T>(kCond, m, T(-1) * wo_c, ux, sy, wi_c, p, st2);
        st = ltype(kCond);
        if (p == T(0)) return zero;
        const T F1 = fr_diel(-wi_c.z, T(1), ior);
        if (!refract_r<T>(T(-1) * wi_c, mk(T(0), T(0), T(-1)), T(1) / eta, wi)) return zero;
        if (F1 == T(1)) return zero;
        r = r * (coat_abs<T>(m, wo_c, wi_c) * (T(1) - F0) * (T(1) - F1));
        r = r / std::fabs(wi_c.z);
        pdf = p * (T(1) - ps);
        return r;
    }
    if (lobe == kCatcher) {
        // uniformSampleHemisphere, left-handed (z = u.x), pdf 1 as in the reference
        const T z = ux;
        const T r = std::sqrt(std::max(T(0), T(1) - z * z));
        const T phi = T(2) * K<T>::pi * uy;
        wi = mk(r * std::cos(phi), r * std::sin(phi), z);
        pdf = T(1);
        return mk(T(1), T(1), T(1)) * (T(1) / std::fabs(wi.z));
    }
    if (lobe == kFSpec) {
        const T ior = (T)m.coat_ior;
        const T F = fr_diel(wo.z, T(1), ior);
        if (ux < F) {
            wi = mk(-wo.x, -wo.y, wo.z);
            pdf = F;
            st = B_REFL | B_SPEC;
            return F * v3f<T>(m.specular) / std::fabs(wi.z);
        }
        const bool entering = wo.z > T(0);
        const T eta = entering ? (T(1) / ior) : (ior / T(1));
        const V<T> n = dot(wo, mk(T(0), T(0), T(1))) < T(0) ? mk(T(0), T(0), T(-1)) : mk(T(0), T(0), T(1));
        const T ci = dot(n, wo);
        const T s2i = std::max(T(0), T(1) - ci * ci);
        const T s2t = eta * eta * s2i;
        if (s2t >= T(1)) return zero;
        const T ct = std::sqrt(T(1) - s2t);
        wi = (-eta) * wo + (eta * ci - ct) * n;
        pdf = T(1) - F;
        st = B_TRANS | B_SPEC;
        return v3f<T>(m.transmission) * eta * eta * (T(1) - F) / std::fabs(wi.z);
    }
    return zero;
}
// CudaBSDF (bsdf.cuh:232-358) over the material's lobes
inline int n_matching(uint32_t lobes, uint32_t flags) {
    return (matches(lobe_at(lobes, 0), flags) ? 1 : 0) + (matches(lobe_at(lobes, 1), flags) ? 1 : 0);
}
inline bool sided(uint32_t id, bool refl) { return (refl && (ltype(id) & B_REFL)) || (!refl && (ltype(id) & B_TRANS)); }
template <class T> V<T> bsdf_eval(uint32_t lobes, const Scene::Mat& m, const Frame<T>& F, V<T> woW, V<T> wiW,
                                  uint32_t flags) {
    const V<T> wo = to_local(F, woW), wi = to_local(F, wiW);
    const bool refl = dot(wiW, F.ng) * dot(woW, F.ng) > T(0);
    V<T> f = mk(T(0), T(0), T(0));
    for (int k = 0; k < 2; ++k) {
        const uint32_t id = lobe_at(lobes, k);
        if (matches(id, flags) && sided(id, refl)) f = f + lobe_eval<T>(id, m, wo, wi);
    }
    return f;
}
template <class T> T bsdf_pdf(uint32_t lobes, const Scene::Mat& m, const Frame<T>& F, V<T> woW, V<T> wiW,
                              uint32_t flags) {
    if (!lobes) return T(0);
    const V<T> wo = to_local(F, woW), wi = to_local(F, wiW);
    if (wo.z == T(0)) return T(0);
    T pdf = T(0);
    int n = 0;
    for (int k = 0; k < 2; ++k) {
        const uint32_t id = lobe_at(lobes, k);
        if (matches(id, flags)) {
            ++n;
            pdf += lobe_pdf<T>(id, m, wo, wi);
        }
    }
    return n > 0 ? pdf / T(n) : T(0);
}
// the BSDF half of Sample_f with its two uniforms given
template <class T> V<T> bsdf_sample_u(uint32_t lobes, const Scene::Mat& m, const Frame<T>& F, V<T> woW,
                                      uint32_t flags, float ux, float uy, V<T>& wiW, T& pdf, uint32_t& st) {
    pdf = T(0);
    st = 0;
    const V<T> zero = mk(T(0), T(0), T(0));
    const int n = n_matching(lobes, flags);
    if (n == 0) return zero;
    const int comp = std::min((int)std::floor(ux * (float)n), n - 1);
    const float uxr = std::min(ux * (float)n - (float)comp, kOneMinusEpsF);
    int chosen = 0;
    for (int k = 0, c = comp; k < 2; ++k)
        if (matches(lobe_at(lobes, k), flags) && c-- == 0) {
            chosen = k;
            break;
        }
    const uint32_t id = lobe_at(lobes, chosen);
    const V<T> wo = to_local(F, woW);
    if (wo.z == T(0)) return zero;
    V<T> wi = zero;
    uint32_t s;
    V<T> f = lobe_sample<T>(id, m, wo, (T)uxr, (T)uy, wi, pdf, s);
    if (pdf == T(0)) return zero;
    st = s;
    wiW = to_world(F, wi);
    const bool spec = (ltype(id) & B_SPEC) != 0;
    const uint32_t other = lobe_at(lobes, 1 - chosen);
    if (!spec && n > 1 && matches(other, flags)) pdf += lobe_pdf<T>(other, m, wo, wi);
    if (n > 1) pdf /= T(n);
    if (!spec) {
        const bool refl = dot(wiW, F.ng) * dot(woW, F.ng) > T(0);
        if (matches(other, flags) && sided(other, refl)) f = f + lobe_eval<T>(other, m, wo, wi);
    }
    return f;
}
template <class T> V<T> bsdf_sample(uint32_t lobes, const Scene::Mat& m, const Frame<T>& F, V<T> woW,
                                    uint32_t flags, Rng& rng, V<T>& wiW, T& pdf, uint32_t& st) {
    if (n_matching(lobes, flags) == 0) {
        pdf = T(0);
        st = 0;
        return mk(T(0), T(0), T(0));
    }
    const float ux = rng.next();
    const float uy = rng.next();
    return bsdf_sample_u<T>(lobes, m, F, woW, flags, ux, uy, wiW, pdf, st);
}

// ----------------------------------------------------------- sky & env
// hosek.cuh:68-101
template <class T> T hosek_int(const float* c, T th, T ga) {
    const T cg = std::cos(ga), cg2 = cg * cg, ct = std::cos(th);
    const T expM = std::exp((T)c[4] * ga);
    const T mieM = (T(1) + cg2) / std::pow(T(1) + (T)c[8] * (T)c[8] - T(2) * (T)c[8] * cg, (T)1.5);
    return (T(1) + (T)c[0] * std::exp((T)c[1] / (ct + (T)0.01f))) *
           ((T)c[2] + (T)c[3] * expM + (T)c[5] * cg2 + (T)c[6] * mieM + (T)c[7] * std::sqrt(ct));
}
template <class T> T inv_gamma(T v) {
    if (v <= (T)0.04045f) return v * T(1) / (T)12.92f;
    return std::pow((v + (T)0.055f) * T(1) / (T)1.055f, (T)2.4f);
}
template <class T> T sph_theta(V<T> v) { return std::acos(clampv(v.y, T(-1), T(1))); }
template <class T> T sph_phi(V<T> v) {
    const T p = std::atan2(v.z, v.x);
    return p < T(0) ? p + T(2) * K<T>::pi : p;
}
template <class T> V<T> hosek(const noor_hosek_sky& H, V<T> v) {
    if (v.y < T(0)) return mk(T(0), T(0), T(0));
    const T th = clampv(sph_theta(v), T(0), K<T>::pi / T(2));
    const V<T> sd = v3f<T>(H.solar_dir);
    const T ga = std::acos(clampv(dot(v, sd), T(-1), T(1)));
    V<T> rgb = mk(hosek_int(H.state[0].configs[0], th, ga) * (T)H.state[0].radiances[0],
                  hosek_int(H.state[1].configs[1], th, ga) * (T)H.state[1].radiances[1],
                  hosek_int(H.state[2].configs[2], th, ga) * (T)H.state[2].radiances[2]);
    if (ga < (T)H.solar_radius) return (T)H.solar_scale * rgb;
    const V<T> s = rgb * (T)0.025f;
    return mk(inv_gamma(s.x), inv_gamma(s.y), inv_gamma(s.z));
}
template <class T> V<T> env_bilinear(const Scene& sc, T u, T v) {
    const int W = sc.ew, H = sc.eh;
    const T x = u * (T)W - (T)0.5, y = v * (T)H - (T)0.5;
    const T fx0 = std::floor(x), fy0 = std::floor(y);
    const T ax = x - fx0, ay = y - fy0;
    int x0 = (int)fx0, y0 = (int)fy0, x1 = x0 + 1, y1 = y0 + 1;
    x0 = std::min(std::max(x0, 0), W - 1);
    x1 = std::min(std::max(x1, 0), W - 1);
    y0 = std::min(std::max(y0, 0), H - 1);
    y1 = std::min(std::max(y1, 0), H - 1);
    auto tx = [&](int xx, int yy) { return v3f<T>(sc.env + 4 * ((size_t)yy * W + xx)); };
    return ((T(1) - ax) * (T(1) - ay)) * tx(x0, y0) + (ax * (T(1) - ay)) * tx(x1, y0) +
           ((T(1) - ax) * ay) * tx(x0, y1) + (ax * ay) * tx(x1, y1);
}
template <class T> V<T> env_eval(const Scene& sc, V<T> dir) {
    if (sc.S->skydome_type == NOOR_SKY_PHYSICAL) return hosek<T>(*sc.H, dir);
    return env_bilinear<T>(sc, sph_phi(dir) * K<T>::inv_2pi, sph_theta(dir) * K<T>::inv_pi);
}
inline double lum(double r, double g, double b) { return (double)(0.2126f) * r + (double)(0.7152f) * g + (double)(0.0722f) * b; }

// env distribution: PBRT-v3 Distribution2D over luminance x sin(theta)
// (the build's definition; the reference's is noor/cuda/distribution2d.cuh)
void build_dist(Scene& sc) {
    const bool sky = sc.S->skydome_type == NOOR_SKY_PHYSICAL;
    const int w = sky ? 2048 : sc.ew, h = sky ? 1024 : sc.eh;
    sc.dw = w;
    sc.dh = h;
    sc.func.assign((size_t)w * h, 0.0);
    // the sky's cells: luminance x sin(theta) over 4 x 4 sub-samples in
    // FP64, rounded once to FP32 (rows split over the host threads)
    auto rows = [&](int j0, int j1) {
        for (int j = j0; j < j1; ++j)
            for (int i = 0; i < w; ++i) {
                double f = 0;
                if (sky) {
                    double acc = 0.0;
                    for (int b = 0; b < 4; ++b) {
                        const double th = ((double)j + ((double)b + 0.5) * 0.25) / (double)h * K<double>::pi;
                        const double st = std::sin(th), ct = std::cos(th);
                        for (int a = 0; a < 4; ++a) {
                            const double ph = ((double)i + ((double)a + 0.5) * 0.25) / (double)w * (2.0 * K<double>::pi);
                            const V<double> d = nrm(mk(st * std::cos(ph), ct, st * std::sin(ph)));
                            const V<double> c = hosek<double>(*sc.H, d);
                            acc += std::max(0.0, lum(c.x, c.y, c.z)) * st;
                        }
                    }
                    f = (float)(acc / 16.0);
                } else {
                    const float* t = sc.env + 4 * ((size_t)j * w + i);
                    const float st = std::sin(((float)j + 0.5f) / (float)h * K<float>::pi);
                    const float y = 0.2126f * t[0] + 0.7152f * t[1] + 0.0722f * t[2];
                    f = std::max(0.0f, y) * st;
                }
                sc.func[(size_t)j * w + i] = (double)(float)f;
            }
    };
    if (sky) {
        const int T = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
        std::vector<std::thread> th;
        for (int t = 0; t < T; ++t) th.emplace_back(rows, h * t / T, h * (t + 1) / T);
        for (auto& x : th) x.join();
    } else {
        rows(0, h);
    }
    sc.cdf.assign((size_t)h * (w + 1), 0.0);
    sc.row_int.assign(h, 0.0);
    for (int j = 0; j < h; ++j) {
        double* c = sc.cdf.data() + (size_t)j * (w + 1);
        for (int i = 0; i < w; ++i) c[i + 1] = c[i] + sc.func[(size_t)j * w + i] / w;
        const double tot = c[w];
        sc.row_int[j] = tot;
        for (int i = 0; i <= w; ++i) c[i] = tot > 0 ? c[i] / tot : (double)i / w;
    }
    sc.marg_cdf.assign(h + 1, 0.0);
    for (int j = 0; j < h; ++j) sc.marg_cdf[j + 1] = sc.marg_cdf[j] + sc.row_int[j] / h;
    sc.marg_int = sc.marg_cdf[h];
    for (int j = 0; j <= h; ++j) sc.marg_cdf[j] = sc.marg_int > 0 ? sc.marg_cdf[j] / sc.marg_int : (double)j / h;
}
template <class T> T sample1d(const double* func, const double* cdf, int n, double integral, T u, T& pdf, int& off) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if ((T)cdf[mid] <= u) lo = mid; else hi = mid - 1;
    }
    off = std::min(lo, n - 1);
    const T c0 = (T)cdf[off], c1 = (T)cdf[off + 1];
    T du = u - c0;
    if (c1 - c0 > T(0)) du /= (c1 - c0);
    pdf = integral > 0 ? (T)func[off] / (T)integral : T(0);
    return ((T)off + du) / (T)n;
}
template <class T> void dist_sample(const Scene& sc, T u0, T u1, T& x, T& y, T& pdf) {
    T pv, pu;
    int row, col;
    y = sample1d<T>(sc.row_int.data(), sc.marg_cdf.data(), sc.dh, sc.marg_int, u1, pv, row);
    x = sample1d<T>(sc.func.data() + (size_t)row * sc.dw, sc.cdf.data() + (size_t)row * (sc.dw + 1), sc.dw,
                    sc.row_int[row], u0, pu, col);
    pdf = pu * pv;
}
template <class T> T dist_pdf(const Scene& sc, T x, T y) {
    const int iu = std::min(std::max((int)(x * sc.dw), 0), sc.dw - 1);
    const int iv = std::min(std::max((int)(y * sc.dh), 0), sc.dh - 1);
    return sc.marg_int > 0 ? (T)sc.func[(size_t)iv * sc.dw + iu] / (T)sc.marg_int : T(0);
}
template <class T> V<T> env_sample_dir(const Scene& sc, Rng& rng, T& pdf) {
    const T u0 = rng.next(), u1 = rng.next();
    T x, y, mp;
    dist_sample<T>(sc, u0, u1, x, y, mp);
    const T ph = x * T(2) * K<T>::pi, th = y * K<T>::pi;
    const T ct = std::cos(th), st = std::sin(th);
    const V<T> d = nrm(mk(st * std::cos(ph), ct, st * std::sin(ph)));
    pdf = st == T(0) ? T(0) : mp / (T(2) * K<T>::pi * K<T>::pi * st);
    return d;
}
template <class T> T env_pdf(const Scene& sc, V<T> wi) {
    if (!sc.sky_on) return T(0);
    const T th = sph_theta(wi), ph = sph_phi(wi), st = std::sin(th);
    if (st == T(0)) return T(0);
    return dist_pdf<T>(sc, ph * K<T>::inv_2pi, th * K<T>::inv_pi) / (T(2) * K<T>::pi * K<T>::pi * st);
}

// ----------------------------------------------------------- integrator
template <class T> struct Is {
    V<T> p, wo;
    Frame<T> F;
    uint32_t mt, lobe, mat;
};
constexpr uint32_t kGlossyMat =
    NOOR_MIRROR | NOOR_GLASS | NOOR_CLEARCOAT | NOOR_ROUGHGLASS | NOOR_METAL | NOOR_SUBSTRATE | NOOR_GLOSSY;
constexpr uint32_t kDielMat = NOOR_GLASS | NOOR_ROUGHGLASS | NOOR_GLOSSY | NOOR_SUBSTRATE | NOOR_CLEARCOAT;
template <class T> V<T> spawn(const Is<T>& I, V<T> dir, T bias) {
    return dot(dir, I.F.ng) >= T(0) ? I.p + bias * I.F.ng : I.p - bias * I.F.ng;
}
// the scattered ray's differentials (spawnRay, intersection.cuh:111-186)
template <class T> RDiff<T> spawn_diff(const Is<T>& I, const HDiff<T>& h, const RDiff<T>& in, V<T> o, V<T> wi,
                                       T eta_in) {
    RDiff<T> r;
    r.on = true;
    r.odx = o + h.dpdx;
    r.ody = o + h.dpdy;
    const V<T>& sn = I.F.n;
    const V<T>& wo = I.wo;
    const V<T> dwodx = T(-1) * (in.ddx + wo), dwody = T(-1) * (in.ddy + wo);
    if (dot(wi, I.F.ng) >= T(0)) {
        const V<T> dndx = h.dndu * h.dudx + h.dndv * h.dvdx;
        const V<T> dndy = h.dndu * h.dudy + h.dndv * h.dvdy;
        const T dDNdx = dot(dwodx, sn) + dot(wo, dndx), dDNdy = dot(dwody, sn) + dot(wo, dndy);
        r.ddx = wi - dwodx + T(2) * (dot(wo, sn) * dndx + dDNdx * sn);
        r.ddy = wi - dwody + T(2) * (dot(wo, sn) * dndy + dDNdy * sn);
    } else {
        const V<T> w = T(-1) * wo;
        const T eta = dot(wo, sn) > T(0) ? T(1) / eta_in : eta_in;
        const V<T> dndx = h.dndu * h.dudx + h.dndv * h.dvdx;
        const V<T> dndy = h.dndv * h.dudy + h.dndv * h.dvdy;   // as the reference pairs them
        const T dDNdx = dot(dwodx, sn) + dot(wo, dndx), dDNdy = dot(dwody, sn) + dot(wo, dndy);
        const T mu = eta * dot(w, sn) - dot(wi, sn);
        const T dmudx = (eta - (eta * eta * dot(w, sn)) / dot(wi, sn)) * dDNdx;
        const T dmudy = (eta - (eta * eta * dot(w, sn)) / dot(wi, sn)) * dDNdy;
        r.ddx = wi + eta * dwodx - (mu * dndx + dmudx * sn);
        r.ddy = wi + eta * dwody - (mu * dndy + dmudy * sn);
    }
    const T sc = (T)0.25f;
    r.odx = (T(1) - sc) * o + sc * r.odx;
    r.ody = (T(1) - sc) * o + sc * r.ody;
    r.ddx = (T(1) - sc) * wi + sc * r.ddx;
    r.ddy = (T(1) - sc) * wi + sc * r.ddy;
    return r;
}
template <class T> V<T> area_p(const noor_area_light& A, int which) {
    return which == 0 ? v3f<T>(A.shape.center) : (which == 1 ? v3f<T>(A.shape.u) : (which == 2 ? v3f<T>(A.shape.v) : v3f<T>(A.shape.n)));
}

// CudaAreaLight::Le (lightimp.cuh:29-36): w is the direction of the ray
// arriving at the light
template <class T> V<T> area_le(const noor_area_light& A, V<T> w) {
    if (A.shape.type == NOOR_SHAPE_SPHERE) return v3f<T>(A.ke);
    return (A.two_sided || dot(w, area_p<T>(A, 3)) < T(0)) ? v3f<T>(A.ke) : mk(T(0), T(0), T(0));
}
// sampleQuad / sampleSphere / sampleDisk (geometry.cuh:27-103); the quad
// and disk pdf divide by |n . w| with w = P - p unnormalised, as there
template <class T> V<T> area_sample(const Scene& sc, const noor_area_light& A, V<T> P, Rng& rng, T& pdf) {
    const T bias = (T)sc.S->reflection_bias;
    const V<T> c = area_p<T>(A, 0), n = area_p<T>(A, 3);
    const T rad = (T)A.shape.radius, rad2 = (T)A.shape.radius2;
    if (A.shape.type == NOOR_SHAPE_SPHERE) {
        const float r1 = rng.next();
        const float r2 = rng.next();
        const V<T> w = nrm(c - P);
        V<T> u, v;
        coord_sys<T>(w, u, v);
        const T sin2max = rad2 / len2(P - c);
        const T cosmax = std::sqrt(std::max(T(0), T(1) - sin2max));
        const T ct = (T(1) - (T)r1) + (T)r1 * cosmax;
        const T st = std::sqrt(std::max(T(0), T(1) - ct * ct));
        const T phi = (T)r2 * (T(2) * K<T>::pi);
        const T dc = len(P - c);
        const T ds = dc * ct - std::sqrt(std::max(T(0), rad2 - dc * dc * st * st));
        const T ca = (dc * dc + rad2 - ds * ds) / (T(2) * dc * rad);
        const T sa = std::sqrt(std::max(T(0), T(1) - ca * ca));
        const V<T> N = sa * std::cos(phi) * (T(-1) * u) + sa * std::sin(phi) * (T(-1) * v) + ca * (T(-1) * w);
        V<T> p = c + rad * N;
        p = p * (rad / len(p - c));
        p = p + bias * N;
        pdf = (T(1) / (T(2) * K<T>::pi)) / (T(1) - cosmax);
        return p;
    }
    V<T> p;
    if (A.shape.type == NOOR_SHAPE_DISK) {
        const float ux = rng.next();
        const float uy = rng.next();
        T dx, dy;
        conc_disk<T>((T)ux, (T)uy, dx, dy);
        V<T> u, v;
        coord_sys<T>(n, u, v);
        p = (dx * rad) * u + (dy * rad) * v + T(0) * n + c + bias * n;
    } else {
        const float r1 = rng.next();
        const float r2 = rng.next();
        p = c + area_p<T>(A, 1) * (T)r1 + area_p<T>(A, 2) * (T)r2 + bias * n;
    }
    const V<T> w = P - p;
    pdf = len2(w) / (std::fabs(dot(n, T(-1) * w)) * (T)A.shape.area);
    if (std::isinf(pdf)) pdf = 0;
    return p;
}
// CudaShape::pdf (shapeimp.cuh:28-52)
template <class T> T area_pdf(const noor_area_light& A, V<T> P, V<T> wi) {
    T lp = 0;
    if (A.shape.type == NOOR_SHAPE_SPHERE) {
        const T sin2max = (T)A.shape.radius2 / len2(P - area_p<T>(A, 0));
        const T cosmax = std::sqrt(std::max(T(0), T(1) - sin2max));
        lp = (T(1) / (T(2) * K<T>::pi)) / (T(1) - cosmax);
    } else {
        T tm = K<T>::inf;
        if (shape_hit<T>(A, P, wi, tm)) {
            const V<T> p = P + tm * wi;
            lp = len2(p - P) / (std::fabs(dot(area_p<T>(A, 3), T(-1) * wi)) * (T)A.shape.area);
        }
    }
    if (std::isinf(lp)) lp = 0;
    return lp;
}
// point / spot / distant sample_Li (lightimp.cuh:191-241); k counts from
// the first point light
template <class T> V<T> delta_sample(const Scene& sc, int k, V<T> P, V<T>& to, T& pdf) {
    const noor_payload* Pl = sc.P;
    const V<T> zero = mk(T(0), T(0), T(0));
    pdf = 1;
    if (k >= Pl->num_point_lights + Pl->num_spot_lights) {
        const noor_distant_light& L = Pl->distant_lights[k - Pl->num_point_lights - Pl->num_spot_lights];
        to = P + T(2) * (T)sc.S->world_radius * v3f<T>(L.direction);
        return v3f<T>(L.ke);
    }
    const bool spot = k >= Pl->num_point_lights;
    const float* pos = spot ? Pl->spot_lights[k - Pl->num_point_lights].position : Pl->point_lights[k].position;
    const float* ke = spot ? Pl->spot_lights[k - Pl->num_point_lights].ke : Pl->point_lights[k].ke;
    to = v3f<T>(pos);
    const T dist2 = len2(to - P);
    if (dist2 == T(0)) {
        pdf = 0;
        return zero;
    }
    if (!spot) return v3f<T>(ke) / dist2;
    // CudaSpotLight::falloff (light.cuh:198-206)
    const noor_spot_light& L = Pl->spot_lights[k - Pl->num_point_lights];
    const V<T> v = to - P;
    const T c = dot(v3f<T>(L.direction), v / len(v));
    T fo = 1;
    if (c < (T)L.cos_outer) {
        fo = 0;
    } else if (c < (T)L.cos_inner) {
        const T dl = (c - (T)L.cos_outer) / ((T)L.cos_inner - (T)L.cos_outer);
        fo = (dl * dl) * (dl * dl);
    }
    if (fo == T(0)) {
        pdf = 0;
        return zero;
    }
    return v3f<T>(ke) * fo / dist2;
}

// traversal work: rays, nodes popped, triangles tested, triangles whose t
// passed the range test (all rays), and the same three for shadow rays alone
struct Counters {
    uint64_t ext = 0, shadow = 0, nodes = 0, tris = 0, tri_in_range = 0;
    uint64_t sh_nodes = 0, sh_tris = 0, sh_in_range = 0;
};

template <class T> bool occl(const Scene& sc, V<T> o, V<T> d, T tmax, int isect, Counters* c) {
    uint64_t ctr[3] = {0, 0, 0};
    if (c) c->shadow++;
    const bool r = traverse<T>(sc, o, d, tmax, nullptr, true, isect, c ? ctr : nullptr);
    if (c) {
        c->nodes += ctr[0];
        c->tris += ctr[1];
        c->tri_in_range += ctr[2];
        c->sh_nodes += ctr[0];
        c->sh_tris += ctr[1];
        c->sh_in_range += ctr[2];
    }
    return r;
}

// the shadow catcher's sky factor (bxdf.cuh:213-218)
template <class T> V<T> catcher_sky(const Scene& sc, const Is<T>& I) {
    return env_eval<T>(sc, T(-1) * to_world(I.F, to_local(I.F, I.wo)));
}

// sampleLight / sampleBSDF (direct.cuh:32-110) with the build's stated
// choices for the unpicked-light case (no BSDF half, no draws)
template <class T>
V<T> direct(const Scene& sc, const Scene::Mat& m, const Is<T>& I, Rng& rng, int isect, Counters* c) {
    const V<T> zero = mk(T(0), T(0), T(0));
    if (I.mt & kSpecMat) return zero;
    const int nl = sc.sky_on ? sc.num_lights : sc.num_lights - 1;
    if (nl == 0) return zero;
    const T bias = (T)sc.S->reflection_bias;
    const bool mis = sc.S->mis != 0;
    const int li = (int)((float)nl * rng.next());
    const int na = sc.P->num_area_lights;
    const int nd = sc.P->num_point_lights + sc.P->num_spot_lights + sc.P->num_distant_lights;
    const bool delta = li >= na && li < na + nd;
    const bool catcher = I.lobe == kCatcher;
    const uint32_t nonspec = B_ALL & ~B_SPEC;
    V<T> Ld = zero;
    {
        V<T> Li = zero, wi = zero, to = zero;
        T lpdf = 0;
        if (li < na) {
            const noor_area_light& A = sc.P->area_lights[li];
            const V<T> p = area_sample<T>(sc, A, I.p, rng, lpdf);
            if (lpdf != T(0)) {
                to = p;
                const V<T> v = to - I.p;
                wi = v / len(v);
                Li = area_le<T>(A, wi);
            }
        } else if (delta) {
            Li = delta_sample<T>(sc, li - na, I.p, to, lpdf);
            const V<T> v = to - I.p;
            wi = v / len(v);
        } else {
            const V<T> dir = env_sample_dir<T>(sc, rng, lpdf);
            if (std::isinf(lpdf) || std::isnan(lpdf)) lpdf = 0;
            to = I.p + T(2) * (T)sc.S->world_radius * dir;
            const V<T> v = to - I.p;
            wi = v / len(v);
            Li = sc.sky_on ? env_eval<T>(sc, wi) : zero;
        }
        Li = Li * (T)nl;
        if (lpdf != T(0) && !black(Li)) {
            V<T> f = bsdf_eval<T>(I.lobe, m, I.F, I.wo, wi, nonspec);
            if (catcher) f = f * catcher_sky<T>(sc, I);
            if (!black(f)) {
                f = f * std::fabs(dot(wi, I.F.n));
                const V<T> so = spawn(I, wi, bias);
                if (!occl<T>(sc, so, wi, len(so - to), isect, c)) {
                    if (catcher) {
                        Ld = f;   // direct.cuh:51
                    } else if (!mis || delta) {
                        Ld = Li * f / lpdf;
                    } else {
                        const T sp = bsdf_pdf<T>(I.lobe, m, I.F, I.wo, wi, nonspec);
                        Ld = Li * f * ((lpdf * lpdf) / (lpdf * lpdf + sp * sp)) / lpdf;
                    }
                }
            }
        }
    }
    if (!mis) return Ld;
    // sampleBSDF: nothing (and no draw) for a delta light or a shadow
    // catcher (direct.cuh:77, 129)
    if (delta || catcher) return Ld;
    rng.next();
    rng.next();
    V<T> wi;
    T sp;
    uint32_t st;
    V<T> f = bsdf_sample<T>(I.lobe, m, I.F, I.wo, nonspec, rng, wi, sp, st);
    if (black(f) || sp == T(0)) return Ld;
    f = f * std::fabs(dot(wi, I.F.n));
    T w = T(1);
    if (!(st & B_SPEC)) {
        T lp = 0;
        if (li < na) {
            lp = area_pdf<T>(sc.P->area_lights[li], I.p, wi);
        } else {
            lp = env_pdf<T>(sc, wi);
        }
        if (std::isinf(lp)) lp = 0;
        if (lp == T(0)) return Ld;
        w = (sp * sp) / (sp * sp + lp * lp);
    }
    const V<T> so = spawn(I, wi, bias);
    T tm = T(2) * (T)sc.S->world_radius;
    bool lh;
    V<T> Le;
    if (li < na) {
        const noor_area_light& A = sc.P->area_lights[li];
        lh = shape_hit<T>(A, so, wi, tm);
        Le = area_le<T>(A, wi);
    } else {
        lh = sc.sky_on;
        Le = sc.sky_on ? env_eval<T>(sc, wi) : zero;
    }
    if (!lh) return Ld;
    const V<T> cc = Le * f * w / sp;
    if (black(cc)) return Ld;
    const V<T> to = so + tm * wi;
    const V<T> v = to - I.p;
    const V<T> vwi = v / len(v);
    const V<T> so2 = spawn(I, vwi, bias);
    if (!occl<T>(sc, so2, vwi, len(so2 - to), isect, c)) Ld = Ld + cc;
    return Ld;
}

// pathtracer() (path_tracer.cu:26-75)
template <class T> V<T> radiance(const Scene& sc, V<T> o, V<T> d, Rng& rng, int isect, Counters* c,
                                 RDiff<T> rd = RDiff<T>{}) {
    V<T> L = mk(T(0), T(0), T(0)), beta = mk(T(1), T(1), T(1));
    bool specb = false;
    const T bias = (T)sc.S->reflection_bias;
    for (uint32_t b = 0; b < sc.S->bounces; ++b) {
        T tmax = K<T>::inf;
        Hit h{0, 0, 0, 0, 0};
        uint64_t ctr[3] = {0, 0, 0};
        if (c) c->ext++;
        const bool hit = traverse<T>(sc, o, d, tmax, &h, false, isect, c ? ctr : nullptr);
        if (c) {
            c->nodes += ctr[0];
            c->tris += ctr[1];
            c->tri_in_range += ctr[2];
        }
        if (!hit) {
            if (sc.sky_on && (b == 0 || specb)) L = L + beta * env_eval<T>(sc, nrm(d));
            break;
        }
        Is<T> I;
        I.p = o + tmax * d;
        I.wo = nrm(T(-1) * d);
        I.mt = h.mt;
        I.lobe = lobe_of(h.mt);
        I.mat = sc.P->attribute_indices[4 * (size_t)h.tri + 3];
        if (I.mt & kEmitMat) {
            if (b == 0 || specb) {
                if (I.mt & NOOR_MESHLIGHT) {
                    L = L + beta * area_le<T>(sc.P->area_lights[h.ins], d);
                } else {
                    // an emitter's texture is read at the barycentrics
                    const Scene::Mat em = textured<T>(sc, sc.mats[I.mat], (T)h.u, (T)h.v);
                    L = L + beta * ((T)em.emitter_scale * v3f<T>(em.emittance));
                }
            }
            break;
        }
        TOut<T> to;
        I.F = tangent<T>(sc, h, &to);
        const Scene::Mat m = textured<T>(sc, sc.mats[I.mat], to.u, to.v);
        HDiff<T> hd;
        if (rd.on) {
            hd = hit_diff<T>(I.F, I.p, to, rd);
            if (I.mt & NOOR_BUMP) bump_frame<T>(sc, m, to.u, to.v, hd, I.F);
        }
        L = L + beta * direct<T>(sc, m, I, rng, isect, c);
        rng.next();
        rng.next();
        V<T> wi;
        T pdf;
        uint32_t st;
        V<T> f = bsdf_sample<T>(I.lobe, m, I.F, I.wo, B_ALL, rng, wi, pdf, st);
        if (pdf == T(0)) break;
        if (I.lobe == kCatcher) f = f * catcher_sky<T>(sc, I);
        beta = beta * (f * std::fabs(dot(wi, I.F.n)) / pdf);
        if (!(I.mt & kTranspMat) && dot(wi, I.F.ng) < T(0)) break;
        if (b >= sc.S->rr) {
            const T q = std::max((T)0.05f, T(1) - maxc(beta));
            if ((T)rng.next() < q) break;
            beta = beta / (T(1) - q);
        }
        specb = (I.mt & kSpecMat) != 0;
        o = spawn(I, wi, bias);
        if (rd.on && (I.mt & kGlossyMat))
            rd = spawn_diff<T>(I, hd, rd, o, wi, (I.mt & kDielMat) ? (T)m.coat_ior : T(1));
        else
            rd.on = false;
        d = wi;
    }
    return mk(clampv(L.x, T(0), T(100)), clampv(L.y, T(0), T(100)), clampv(L.z, T(0), T(100)));
}

// generateRay, pinhole (cameraimp.cuh:182-228)
// generateRay of CudaPerspCamera (pinhole and thin lens), CudaOrthoCamera
// and CudaEnvCamera (cameraimp.cuh:51-230), then CudaRay::transform
// With rd, also the ray's differentials (each camera type's, then
// transformDifferentials: origins as points, directions as vectors).
template <class T> void cam_ray(const noor_camera& C, uint32_t x, uint32_t y, Rng& rng, V<T>& o, V<T>& d,
                                RDiff<T>* rd = nullptr) {
    const float rxf = (float)x + rng.next() - 0.5f;
    const float ryf = (float)y + rng.next() - 0.5f;
    const T rx = rxf, ry = ryf;
    const V<T> zero = mk(T(0), T(0), T(0));
    V<T> dc, oc = zero, odx = zero, ody = zero, ddx = zero, ddy = zero;
    const V<T> dxc = mk((T)C.raster_to_camera[0][0], (T)C.raster_to_camera[1][0], (T)C.raster_to_camera[2][0]);
    const V<T> dyc = mk((T)C.raster_to_camera[0][1], (T)C.raster_to_camera[1][1], (T)C.raster_to_camera[2][1]);
    bool at_origin = true;
    auto env_dir = [&](T px, T py) {
        const T theta = K<T>::pi * py / (T)C.h + K<T>::pi;
        const T phi = (T(2) * K<T>::pi) * px / (T)C.w - K<T>::pi / T(2);
        const T st = std::sin(theta), ct = std::cos(theta);
        return nrm(nrm(mk(st * std::cos(phi), ct, st * std::sin(phi))));
    };
    if (C.type == NOOR_CAMERA_ENV) {
        dc = env_dir(rx, ry);
        ddx = env_dir(rx + T(1), ry);
        ddy = env_dir(rx, ry + T(1));
    } else {
        T pc[3];
        for (int r = 0; r < 3; ++r)
            pc[r] = (T)C.raster_to_camera[r][3] + ((T)C.raster_to_camera[r][0] * rx +
                                                   (T)C.raster_to_camera[r][1] * ry + (T)C.raster_to_camera[r][2] * T(0));
        const V<T> pcv = mk(pc[0], pc[1], pc[2]);
        if (C.type == NOOR_CAMERA_ORTHO) {
            oc = pcv;
            dc = mk(T(0), T(0), T(-1));
            at_origin = false;
            odx = oc + dxc;
            ody = oc + dyc;
            ddx = ddy = dc;
        } else {
            dc = nrm(pcv);
            if (C.lens_radius > 0.0f) {
                const float u1 = rng.next();
                const float u2 = rng.next();
                T lx, ly;
                conc_disk<T>((T)u1, (T)u2, lx, ly);
                const T plx = (T)C.lens_radius * lx, ply = (T)C.lens_radius * ly;
                T ft = -(T)C.focal_length / dc.z;
                const V<T> pf = zero + ft * dc;
                oc = mk(plx, ply, T(0));
                dc = nrm(pf - oc);
                at_origin = false;
                const V<T> dx = nrm(pcv + dxc);
                ft = -(T)C.focal_length / dx.z;
                odx = mk(plx, ply, T(0));
                ddx = nrm(zero + ft * dx - odx);
                const V<T> dy = nrm(pcv + dyc);
                ft = -(T)C.focal_length / dy.z;
                ody = mk(plx, ply, T(0));
                ddy = nrm(zero + ft * dy - ody);
            } else {
                ddx = nrm(pcv + dxc);
                ddy = nrm(pcv + dyc);
            }
        }
    }
    if (rd) {
        auto point = [&](V<T> q) {
            T r3[3];
            for (int r = 0; r < 3; ++r)
                r3[r] = (T)C.camera_to_world[r][3] + ((T)C.camera_to_world[r][0] * q.x +
                                                      (T)C.camera_to_world[r][1] * q.y + (T)C.camera_to_world[r][2] * q.z);
            return mk(r3[0], r3[1], r3[2]);
        };
        auto vec = [&](V<T> q) {
            T r3[3];
            for (int r = 0; r < 3; ++r)
                r3[r] = (T)C.camera_to_world[r][0] * q.x + (T)C.camera_to_world[r][1] * q.y +
                        (T)C.camera_to_world[r][2] * q.z;
            return mk(r3[0], r3[1], r3[2]);
        };
        rd->on = true;
        rd->odx = point(odx);
        rd->ody = point(ody);
        rd->ddx = vec(ddx);
        rd->ddy = vec(ddy);
    }
    if (at_origin) {
        o = mk((T)C.camera_to_world[0][3], (T)C.camera_to_world[1][3], (T)C.camera_to_world[2][3]);
    } else {
        T ow[3];
        for (int r = 0; r < 3; ++r)
            ow[r] = (T)C.camera_to_world[r][3] + ((T)C.camera_to_world[r][0] * oc.x + (T)C.camera_to_world[r][1] * oc.y +
                                                  (T)C.camera_to_world[r][2] * oc.z);
        o = mk(ow[0], ow[1], ow[2]);
    }
    T dw[3];
    for (int r = 0; r < 3; ++r)
        dw[r] = (T)C.camera_to_world[r][0] * dc.x + (T)C.camera_to_world[r][1] * dc.y + (T)C.camera_to_world[r][2] * dc.z;
    d = nrm(mk(dw[0], dw[1], dw[2]));
}

struct Ctx {
    Scene sc;
};

// ------------------------------------------------ adjoint reference (FP64)
// The library's differentiable estimator: sampling detached (directions,
// light picks, MIS weights, pdfs and every early exit from the scene as
// loaded), BSDF values and environment radiance from parameter arrays
// (albedo M x 3 -- Lambert reflectance or conductor tint --, roughness M,
// env texels H x W x 3).  Its gradient is taken here by the product rule
// over the stored path (L = sum_t B_k(t) * v_t, B_k the product of the
// scatter factors before vertex k), with the roughness derivative of f by
// an FP64 central difference -- an independent restatement of what the
// library computes by path replay with analytic derivatives.
struct AdjPar {
    const float* alb;
    const float* rough;
    const float* env;
    uint32_t bounces;
};
struct BW {
    size_t idx[4];
    double w[4];
};
// texel weights of env_bilinear for direction dir
inline BW env_weights_d(const Scene& sc, V<double> dir) {
    const double u = sph_phi(dir) * K<double>::inv_2pi, v = sph_theta(dir) * K<double>::inv_pi;
    const int W = sc.ew, H = sc.eh;
    const double x = u * W - 0.5, y = v * H - 0.5;
    const double fx0 = std::floor(x), fy0 = std::floor(y);
    const double ax = x - fx0, ay = y - fy0;
    int x0 = (int)fx0, y0 = (int)fy0, x1 = x0 + 1, y1 = y0 + 1;
    x0 = std::min(std::max(x0, 0), W - 1);
    x1 = std::min(std::max(x1, 0), W - 1);
    y0 = std::min(std::max(y0, 0), H - 1);
    y1 = std::min(std::max(y1, 0), H - 1);
    BW b;
    b.idx[0] = (size_t)y0 * W + x0;
    b.idx[1] = (size_t)y0 * W + x1;
    b.idx[2] = (size_t)y1 * W + x0;
    b.idx[3] = (size_t)y1 * W + x1;
    b.w[0] = (1 - ax) * (1 - ay);
    b.w[1] = ax * (1 - ay);
    b.w[2] = (1 - ax) * ay;
    b.w[3] = ax * ay;
    return b;
}
inline V<double> env_param(const AdjPar& P, const BW& b) {
    V<double> c = mk(0.0, 0.0, 0.0);
    for (int k = 0; k < 4; ++k) c = c + b.w[k] * v3f<double>(P.env + 3 * b.idx[k]);
    return c;
}
// conductor value without tint, alpha = max(r^2, 1e-3) on both axes
inline V<double> cond_untinted(const Scene::Mat& m, V<double> wo, V<double> wi, double r) {
    const V<double> z = mk(0.0, 0.0, 0.0);
    if (!same(wo, wi)) return z;
    const double cO = std::fabs(wo.z), cI = std::fabs(wi.z);
    if (cI == 0 || cO == 0) return z;
    V<double> wh = nrm(wi + wo);
    if (black(wh)) return z;
    wh = wh * signv(wh.z);
    const V<double> F = fr_cond(dot(wo, wh), v3f<double>(m.ior), v3f<double>(m.k));
    Micro<double> mf;
    mf.ax = mf.ay = std::max(r * r, (double)1e-3f);
    mf.dist = m.dist;
    return F * mf.D(wh) * mf.G(wo, wi) / (4.0 * cI * cO);
}
// f with the parameters, df/dalbedo (per channel) and df/droughness
struct FVal {
    V<double> f, f_alb, f_r;
    bool has;
};
inline FVal eval_f(uint32_t lobe, const Scene::Mat& m0, const AdjPar& P, uint32_t mi, const Frame<double>& F,
                   V<double> woW, V<double> wiW) {
    const V<double> z = mk(0.0, 0.0, 0.0);
    FVal r{z, z, z, false};
    const V<double> wo = to_local(F, woW), wi = to_local(F, wiW);
    if (!(dot(wiW, F.ng) * dot(woW, F.ng) > 0)) return r;
    const V<double> a = v3f<double>(P.alb + 3 * mi);
    if (lobe == kLambert) {
        r.f_alb = mk(K<double>::inv_pi, K<double>::inv_pi, K<double>::inv_pi);
        r.f = a * K<double>::inv_pi;
        r.has = true;
    } else if (lobe == kCond) {
        const double rr = P.rough[mi];
        const V<double> fu = cond_untinted(m0, wo, wi, rr);
        r.f_alb = fu;
        r.f = fu * a;
        const double h = 1e-6;
        if (rr * rr > (double)1e-3f && (rr - h) * (rr - h) > (double)1e-3f)
            r.f_r = (cond_untinted(m0, wo, wi, rr + h) - cond_untinted(m0, wo, wi, rr - h)) * a / (2 * h);
        r.has = true;
    }
    return r;
}
struct ATerm {
    size_t k;             // scatter factors before this term
    V<double> val, d_alb, d_r, fs;
    uint32_t mat;
    bool has_mat, env;
    BW bw;
    double xscale;
};
struct AVtx {
    V<double> s, ds_alb, ds_r;
    uint32_t mat;
    bool has_mat;
};
inline void add_term(std::vector<ATerm>& ts, size_t k, V<double> X, const FVal& fv, double s, uint32_t mat, bool env,
                     const BW& bw, double xscale) {
    ATerm t;
    t.k = k;
    t.val = X * fv.f * s;
    t.d_alb = X * fv.f_alb * s;
    t.d_r = X * fv.f_r * s;
    t.fs = fv.f * s;
    t.mat = mat;
    t.has_mat = fv.has;
    t.env = env;
    t.bw = bw;
    t.xscale = xscale;
    ts.push_back(t);
}
// one path of the detached estimator (pathtracer() with the parameter
// substitution, Russian roulette off)
inline void adj_path(const Scene& sc, const AdjPar& P, V<double> o, V<double> d, Rng& rng, int isect,
                     std::vector<AVtx>& vs, std::vector<ATerm>& ts) {
    vs.clear();
    ts.clear();
    const V<double> zero = mk(0.0, 0.0, 0.0);
    const double bias = sc.S->reflection_bias;
    const bool hdr = sc.S->skydome_type == NOOR_SKY_HDR;
    const bool mis = sc.S->mis != 0;
    const uint32_t nonspec = B_ALL & ~B_SPEC;
    const int na = sc.P->num_area_lights;
    bool specb = false;
    for (uint32_t b = 0; b < P.bounces; ++b) {
        double tmax = K<double>::inf;
        Hit h{0, 0, 0, 0, 0};
        if (!traverse<double>(sc, o, d, tmax, &h, false, isect, nullptr)) {
            if (sc.sky_on && (b == 0 || specb)) {
                const V<double> dir = nrm(d);
                FVal one{mk(1.0, 1.0, 1.0), zero, zero, false};
                BW bw{};
                if (hdr) {
                    bw = env_weights_d(sc, dir);
                    add_term(ts, vs.size(), env_param(P, bw), one, 1.0, 0, true, bw, 1.0);
                } else {
                    add_term(ts, vs.size(), env_eval<double>(sc, dir), one, 1.0, 0, false, bw, 1.0);
                }
            }
            break;
        }
        Is<double> I;
        I.p = o + tmax * d;
        I.wo = nrm(-1.0 * d);
        I.mt = h.mt;
        I.lobe = lobe_of(h.mt);
        I.mat = sc.P->attribute_indices[4 * (size_t)h.tri + 3];
        if (I.mt & kEmitMat) {
            if (b == 0 || specb) {
                V<double> Le;
                if (I.mt & NOOR_MESHLIGHT) {
                    const noor_area_light& A = sc.P->area_lights[h.ins];
                    Le = (A.two_sided || dot(d, area_p<double>(A, 3)) < 0) ? v3f<double>(A.ke) : zero;
                } else {
                    const Scene::Mat& em = sc.mats[I.mat];
                    Le = (double)em.emitter_scale * v3f<double>(em.emittance);
                }
                FVal one{mk(1.0, 1.0, 1.0), zero, zero, false};
                add_term(ts, vs.size(), Le, one, 1.0, 0, false, BW{}, 1.0);
            }
            break;
        }
        I.F = tangent<double>(sc, h);
        const Scene::Mat& m0 = sc.mats[I.mat];
        const size_t k = vs.size();
        // direct lighting (direct<T> with the substitution)
        const int nl = sc.sky_on ? sc.num_lights : sc.num_lights - 1;
        if (!(I.mt & kSpecMat) && nl > 0) {
            const int li = (int)((float)nl * rng.next());
            V<double> Li = zero, wi = zero, to = zero;
            double lpdf = 0;
            if (li < na) {
                const noor_area_light& A = sc.P->area_lights[li];
                const float r1 = rng.next();
                const float r2 = rng.next();
                const V<double> n = area_p<double>(A, 3);
                const V<double> p = area_p<double>(A, 0) + area_p<double>(A, 1) * (double)r1 +
                                    area_p<double>(A, 2) * (double)r2 + bias * n;
                const V<double> w = I.p - p;
                lpdf = len2(w) / (std::fabs(dot(n, -1.0 * w)) * (double)A.shape.area);
                if (std::isinf(lpdf)) lpdf = 0;
                if (lpdf != 0) {
                    to = p;
                    const V<double> v = to - I.p;
                    wi = v / len(v);
                    Li = (A.two_sided || dot(wi, n) < 0) ? v3f<double>(A.ke) : zero;
                }
            } else {
                const V<double> dir = env_sample_dir<double>(sc, rng, lpdf);
                if (std::isinf(lpdf) || std::isnan(lpdf)) lpdf = 0;
                to = I.p + 2.0 * (double)sc.S->world_radius * dir;
                const V<double> v = to - I.p;
                wi = v / len(v);
                Li = sc.sky_on ? env_eval<double>(sc, wi) : zero;
            }
            Li = Li * (double)nl;
            if (lpdf != 0 && !black(Li)) {
                const V<double> f0 = bsdf_eval<double>(I.lobe, m0, I.F, I.wo, wi, nonspec);
                if (!black(f0)) {
                    const V<double> so = spawn(I, wi, bias);
                    if (!occl<double>(sc, so, wi, len(so - to), isect, nullptr)) {
                        const FVal fv = eval_f(I.lobe, m0, P, I.mat, I.F, I.wo, wi);
                        double w = 1;
                        if (mis) {
                            const double sp = bsdf_pdf<double>(I.lobe, m0, I.F, I.wo, wi, nonspec);
                            w = (lpdf * lpdf) / (lpdf * lpdf + sp * sp);
                        }
                        const double s = std::fabs(dot(wi, I.F.n)) * w / lpdf;
                        const bool env = li >= na && hdr;
                        BW bw{};
                        V<double> X = Li;
                        if (env) {
                            bw = env_weights_d(sc, wi);
                            X = env_param(P, bw) * (double)nl;
                        }
                        add_term(ts, k, X, fv, s, I.mat, env, bw, (double)nl);
                    }
                }
            }
            if (mis) {
                rng.next();
                rng.next();
                double sp;
                uint32_t st;
                const V<double> f0 = bsdf_sample<double>(I.lobe, m0, I.F, I.wo, nonspec, rng, wi, sp, st);
                bool go = !black(f0) && sp != 0;
                double w = 1;
                if (go && !(st & B_SPEC)) {
                    double lp = 0;
                    if (li < na) {
                        const noor_area_light& A = sc.P->area_lights[li];
                        double tm = K<double>::inf;
                        if (quad_hit<double>(A, I.p, wi, tm)) {
                            const V<double> p = I.p + tm * wi;
                            lp = len2(p - I.p) / (std::fabs(dot(area_p<double>(A, 3), -1.0 * wi)) * (double)A.shape.area);
                            if (std::isinf(lp)) lp = 0;
                        }
                    } else {
                        lp = env_pdf<double>(sc, wi);
                    }
                    if (std::isinf(lp)) lp = 0;
                    if (lp == 0) go = false;
                    else w = (sp * sp) / (sp * sp + lp * lp);
                }
                if (go) {
                    const V<double> so = spawn(I, wi, bias);
                    double tm = 2.0 * (double)sc.S->world_radius;
                    bool lh;
                    V<double> Le;
                    if (li < na) {
                        const noor_area_light& A = sc.P->area_lights[li];
                        lh = quad_hit<double>(A, so, wi, tm);
                        Le = (A.two_sided || dot(wi, area_p<double>(A, 3)) < 0) ? v3f<double>(A.ke) : zero;
                    } else {
                        lh = sc.sky_on;
                        Le = sc.sky_on ? env_eval<double>(sc, wi) : zero;
                    }
                    if (lh && !black(Le)) {
                        const V<double> to2 = so + tm * wi;
                        const V<double> v = to2 - I.p;
                        const V<double> vwi = v / len(v);
                        const V<double> so2 = spawn(I, vwi, bias);
                        if (!occl<double>(sc, so2, vwi, len(so2 - to2), isect, nullptr)) {
                            const FVal fv = eval_f(I.lobe, m0, P, I.mat, I.F, I.wo, wi);
                            const double s = std::fabs(dot(wi, I.F.n)) * w / sp;
                            const bool env = li >= na && hdr;
                            BW bw{};
                            V<double> X = Le;
                            if (env) {
                                bw = env_weights_d(sc, wi);
                                X = env_param(P, bw);
                            }
                            add_term(ts, k, X, fv, s, I.mat, env, bw, 1.0);
                        }
                    }
                }
            }
        }
        // scatter
        rng.next();
        rng.next();
        V<double> wi;
        double pdf;
        uint32_t st;
        const V<double> f0 = bsdf_sample<double>(I.lobe, m0, I.F, I.wo, B_ALL, rng, wi, pdf, st);
        if (pdf == 0) break;
        const double cs = std::fabs(dot(wi, I.F.n)) / pdf;
        AVtx v{zero, zero, zero, I.mat, false};
        if (st & B_SPEC) {
            v.s = f0 * cs;
        } else {
            const FVal fv = eval_f(I.lobe, m0, P, I.mat, I.F, I.wo, wi);
            v.s = fv.f * cs;
            v.ds_alb = fv.f_alb * cs;
            v.ds_r = fv.f_r * cs;
            v.has_mat = fv.has;
        }
        vs.push_back(v);
        if (!(I.mt & kTranspMat) && dot(wi, I.F.ng) < 0) break;
        specb = (I.mt & kSpecMat) != 0;
        o = spawn(I, wi, bias);
        d = wi;
    }
}

}  // namespace orc

using namespace orc;

// --------------------------------------------------------------- C API
OR_API void* oracle_create(const noor_payload* P, const noor_spec* S, const noor_hosek_sky* H) {
    Ctx* c = new Ctx();
    Scene& sc = c->sc;
    sc.P = P;
    sc.S = S;
    sc.H = H;
    const noor_texture& env = P->textures[P->num_textures - 1];
    sc.env = env.rgba;
    sc.ew = env.width;
    sc.eh = env.height;
    sc.num_lights = P->num_area_lights + P->num_point_lights + P->num_spot_lights + P->num_distant_lights +
                    P->num_infinite_lights;
    sc.sky_on = (S->lighting_type & NOOR_LIGHT_SKY_MASK) != 0;
    sc.mats.resize(P->num_materials);
    for (uint32_t i = 0; i < P->num_materials; ++i) {
        const noor_material& m = P->materials[i];
        Scene::Mat& d = sc.mats[i];
        auto t = [&](uint32_t idx, float* o) { std::memcpy(o, P->textures[idx].rgba, 12); };
        t(m.diffuse_tex_idx, d.diffuse);
        t(m.specular_tex_idx, d.specular);
        t(m.transmission_tex_idx, d.transmission);
        t(m.emittance_tex_idx, d.emittance);
        t(m.ior_tex_idx, d.ior);
        t(m.k_tex_idx, d.k);
        d.rx = P->textures[m.roughness_tex_idx].rgba[0];
        d.ry = P->textures[m.roughness_tex_idx].rgba[1];
        d.coat_ior = m.coat_ior;
        d.coat_weight = m.coat_weight;
        d.coat_sigma = m.coat_sigma;
        d.coat_thickness = m.coat_thickness;
        d.emitter_scale = m.emitter_scale;
        d.type = m.type;
        d.dist = m.distribution;
        // the slots read per hit: image textures, and the alpha and bump
        // maps of ALPHA and BUMP materials
        d.tex_mask = 0;
        auto image = [&](uint32_t idx) { return P->textures[idx].width != 1 || P->textures[idx].height != 1; };
        auto slot = [&](int k, uint32_t idx, const float* uvs) {
            d.tex[k] = idx;
            d.uvs[k][0] = uvs ? uvs[0] : 1.0f;
            d.uvs[k][1] = uvs ? uvs[1] : 1.0f;
            d.tex_mask |= 1u << k;
        };
        if (image(m.diffuse_tex_idx)) slot(TX_DIFFUSE, m.diffuse_tex_idx, m.diffuse_uvscale);
        if (image(m.specular_tex_idx)) slot(TX_SPECULAR, m.specular_tex_idx, m.specular_uvscale);
        if (image(m.emittance_tex_idx)) slot(TX_EMITTANCE, m.emittance_tex_idx, m.emittance_uvscale);
        if (image(m.roughness_tex_idx)) slot(TX_ROUGHNESS, m.roughness_tex_idx, m.roughness_uvscale);
        if (image(m.transmission_tex_idx)) slot(TX_TRANSMISSION, m.transmission_tex_idx, nullptr);
        if (image(m.ior_tex_idx)) slot(TX_IOR, m.ior_tex_idx, nullptr);
        if (image(m.k_tex_idx)) slot(TX_K, m.k_tex_idx, nullptr);
        if (m.type & NOOR_ALPHA) slot(TX_ALPHA, m.transparency_tex_idx, m.transparency_uvscale);
        if (m.type & NOOR_BUMP) slot(TX_BUMP, m.bump_tex_idx, m.bump_uvscale);
        d.bumpfactor = m.bumpfactor;
        if (m.type & NOOR_BUMP) sc.has_bump = true;
    }
    build_dist(sc);
    return c;
}
OR_API void oracle_destroy(void* h) { delete (Ctx*)h; }

// closest hit for a ray batch (same struct as the library's noor_ray/noor_hit)
OR_API void oracle_trace_closest(void* h, const noor_ray* rays, noor_hit* hits, size_t n, int isect, int threads) {
    const Scene& sc = ((Ctx*)h)->sc;
    auto work = [&](size_t b, size_t e) {
        for (size_t i = b; i < e; ++i) {
            const noor_ray& r = rays[i];
            float tmax = r.tmax;
            Hit rec{0, 0, 0, 0, 0};
            const bool hh = traverse<float>(sc, mk(r.org[0], r.org[1], r.org[2]), mk(r.dir[0], r.dir[1], r.dir[2]),
                                            tmax, &rec, false, isect, nullptr);
            noor_hit& o = hits[i];
            o.t = tmax;
            o.tri_idx = rec.tri;
            o.ins_idx = rec.ins;
            o.material_type = rec.mt;
            o.u = (float)rec.u;
            o.v = (float)rec.v;
            o.hit = hh ? 1u : 0u;
            o.pad = 0;
        }
    };
    const int T = std::max(1, threads);
    std::vector<std::thread> th;
    for (int t = 0; t < T; ++t) th.emplace_back(work, n * t / T, n * (t + 1) / T);
    for (auto& x : th) x.join();
}

OR_API void oracle_trace_any(void* h, const noor_ray* rays, uint32_t* occ, size_t n, int isect) {
    const Scene& sc = ((Ctx*)h)->sc;
    for (size_t i = 0; i < n; ++i) {
        const noor_ray& r = rays[i];
        float tmax = r.tmax;
        occ[i] = traverse<float>(sc, mk(r.org[0], r.org[1], r.org[2]), mk(r.dir[0], r.dir[1], r.dir[2]), tmax, nullptr,
                                 true, isect, nullptr)
                     ? 1u
                     : 0u;
    }
}

// camera rays of frame `frame` for pixels [0, w*h)
OR_API void oracle_camera_rays(const noor_camera* C, uint32_t frame, noor_ray* rays) {
    const uint32_t n = C->w * C->h;
    for (uint32_t p = 0; p < n; ++p) {
        Rng rng{tea16(p, frame)};
        V<float> o, d;
        cam_ray<float>(*C, p % C->w, p / C->w, rng, o, d);
        noor_ray& r = rays[p];
        r.org[0] = o.x; r.org[1] = o.y; r.org[2] = o.z;
        r.dir[0] = d.x; r.dir[1] = d.y; r.dir[2] = d.z;
        r.tmax = std::numeric_limits<float>::infinity();
        r.pad = 0;
    }
}

// Render pixels [p0, p1) x frames [f0, f0+nf): out = per-pixel mean rgb
// (sequential Kahan sum in FP32 mode, plain sum in FP64), counters
// (optional, 8 x uint64: ext rays, shadow rays, nodes, triangles, triangles
// in range, then nodes, triangles, triangles in range of the shadow rays alone).
OR_API void oracle_render(void* h, uint32_t f0, uint32_t nf, uint32_t p0, uint32_t p1, const noor_camera* C,
                          int fp64, int isect, int threads, float* out_rgb, uint64_t* counters) {
    const Scene& sc = ((Ctx*)h)->sc;
    const int T = std::max(1, threads);
    std::atomic<uint32_t> next{p0};
    std::vector<Counters> cs(T);
    auto work = [&](int tid) {
        Counters* c = counters ? &cs[tid] : nullptr;
        for (;;) {
            const uint32_t b = next.fetch_add(64);
            if (b >= p1) break;
            const uint32_t e = std::min(b + 64, p1);
            for (uint32_t p = b; p < e; ++p) {
                const uint32_t x = p % C->w, y = p / C->w;
                double sd[3] = {0, 0, 0};
                float sf[3] = {0, 0, 0}, cf[3] = {0, 0, 0};
                for (uint32_t f = 0; f < nf; ++f) {
                    Rng rng{tea16(p, f0 + f)};
                    // camera rays carry differentials where bump maps read them
                    if (fp64) {
                        V<double> o, d;
                        RDiff<double> rd;
                        cam_ray<double>(*C, x, y, rng, o, d, sc.has_bump ? &rd : nullptr);
                        const V<double> L = radiance<double>(sc, o, d, rng, isect, c, rd);
                        sd[0] += L.x; sd[1] += L.y; sd[2] += L.z;
                    } else {
                        V<float> o, d;
                        RDiff<float> rd;
                        cam_ray<float>(*C, x, y, rng, o, d, sc.has_bump ? &rd : nullptr);
                        const V<float> L = radiance<float>(sc, o, d, rng, isect, c, rd);
                        const float l[3] = {L.x, L.y, L.z};
                        for (int k = 0; k < 3; ++k) {
                            const float yk = l[k] - cf[k];
                            const float t = sf[k] + yk;
                            cf[k] = (t - sf[k]) - yk;
                            sf[k] = t;
                        }
                    }
                }
                float* q = out_rgb + 3 * (size_t)(p - p0);
                for (int k = 0; k < 3; ++k) q[k] = fp64 ? (float)(sd[k] / nf) : sf[k] / (float)nf;
            }
        }
    };
    std::vector<std::thread> th;
    for (int t = 0; t < T; ++t) th.emplace_back(work, t);
    for (auto& x : th) x.join();
    if (counters) {
        for (int k = 0; k < 8; ++k) counters[k] = 0;
        for (auto& c : cs) {
            counters[0] += c.ext;
            counters[1] += c.shadow;
            counters[2] += c.nodes;
            counters[3] += c.tris;
            counters[4] += c.tri_in_range;
            counters[5] += c.sh_nodes;
            counters[6] += c.sh_tris;
            counters[7] += c.sh_in_range;
        }
    }
}

// BSDF batch in the local frame (same record layout as noor_eval_bsdf)
OR_API void oracle_eval_bsdf(void* h, int kind, const float* in, float* out, size_t n, int fp64) {
    const Scene& sc = ((Ctx*)h)->sc;
    for (size_t i = 0; i < n; ++i) {
        const float* p = in + 16 * i;
        const Scene::Mat& m = sc.mats[(uint32_t)p[8]];
        const uint32_t lobe = lobe_of(m.type);
        float* q = out + 8 * i;
        auto run = [&](auto zero) {
            using T = decltype(zero);
            Frame<T> F;
            F.n = F.ng = mk(T(0), T(0), T(1));
            F.s = mk(T(1), T(0), T(0));
            F.t = mk(T(0), T(1), T(0));
            const V<T> wo = mk((T)p[0], (T)p[1], (T)p[2]), wi = mk((T)p[3], (T)p[4], (T)p[5]);
            V<T> f = mk(T(0), T(0), T(0)), ws = f;
            T pdf = 0;
            uint32_t st = 0;
            if (kind == 0) f = bsdf_eval<T>(lobe, m, F, wo, wi, B_ALL);
            else if (kind == 1) pdf = bsdf_pdf<T>(lobe, m, F, wo, wi, B_ALL);
            else {
                V<T> w = f;
                f = bsdf_sample_u<T>(lobe, m, F, wo, B_ALL, p[6], p[7], w, pdf, st);
                if (pdf != T(0)) ws = w;
            }
            q[0] = (float)f.x; q[1] = (float)f.y; q[2] = (float)f.z; q[3] = (float)pdf;
            q[4] = (float)ws.x; q[5] = (float)ws.y; q[6] = (float)ws.z; q[7] = (float)st;
        };
        if (fp64) run(0.0); else run(0.0f);
    }
}

// Stand-alone routines, the record layouts of noor_eval_routines
// (include/noor_b200.h): 0 / 1 Trowbridge-Reitz / Beckmann
// (distribution.cuh:58-342), 2 Fresnel (fresnel.cuh:58-107), 3 warps
// (utils.cuh:377-404,470-486,487-539).
template <class T> void routine(int kind, const float* p, float* q) {
    if (kind <= 1) {
        Micro<T> m;
        m.ax = std::max((T)p[0] * (T)p[0], (T)1e-3f);
        m.ay = std::max((T)p[1] * (T)p[1], (T)1e-3f);
        m.dist = (uint32_t)kind;
        const V<T> wo = v3f<T>(p + 2), wh = v3f<T>(p + 5);
        const V<T> s = m.sample_wh(wo, (T)p[8], (T)p[9]);
        const T r[12] = {m.D(wh), m.G(wo, wh), m.pdf(wo, wh), s.x, s.y, s.z, T(0), m.ax, T(0), T(0), T(0), T(0)};
        for (int k = 0; k < 12; ++k) q[k] = (float)r[k];
    } else if (kind == 2) {
        q[0] = (float)fr_diel<T>((T)p[0], (T)p[1], (T)p[2]);
        const V<T> c = fr_cond<T>((T)p[0], v3f<T>(p + 3), v3f<T>(p + 6));
        q[1] = (float)c.x;
        q[2] = (float)c.y;
        q[3] = (float)c.z;
    } else {
        const T ux = (T)p[0], uy = (T)p[1];
        T dx, dy;
        conc_disk<T>(ux, uy, dx, dy);
        const V<T> c = cos_hemi<T>(ux, uy);
        const T hz = ux, hr = std::sqrt(std::max(T(0), T(1) - hz * hz)), hp = T(2) * K<T>::pi * uy;
        const V<T> hh = mk(hr * std::cos(hp), hr * std::sin(hp), hz);
        const T ph = ux * T(2) * K<T>::pi, th = uy * K<T>::pi;
        const T ct = std::cos(th), st = std::sin(th);
        const V<T> d = nrm(mk(st * std::cos(ph), ct, st * std::sin(ph)));
        const T ph2 = (ux * ux) / (ux * ux + uy * uy);
        const T r[16] = {dx, dy, c.x, c.y, c.z, hh.x, hh.y, hh.z, d.x, d.y, d.z, st, ph2,
                         erf_as<T>((T)p[2]), erfinv_g<T>((T)p[2]), T(0)};
        for (int k = 0; k < 16; ++k) q[k] = (float)r[k];
    }
}
OR_API void oracle_routines(int kind, const float* in, float* out, size_t n, int fp64) {
    const int ni = kind <= 1 ? 12 : (kind == 2 ? 9 : 3), no = kind <= 1 ? 12 : (kind == 2 ? 4 : 16);
    for (size_t i = 0; i < n; ++i) {
        if (fp64) routine<double>(kind, in + ni * i, out + no * i);
        else routine<float>(kind, in + ni * i, out + no * i);
    }
}

OR_API void oracle_eval_sky(void* h, const float* dirs, float* rgb, size_t n, int fp64) {
    const Scene& sc = ((Ctx*)h)->sc;
    for (size_t i = 0; i < n; ++i) {
        if (fp64) {
            const V<double> c = env_eval<double>(sc, mk((double)dirs[3 * i], (double)dirs[3 * i + 1], (double)dirs[3 * i + 2]));
            rgb[3 * i] = (float)c.x; rgb[3 * i + 1] = (float)c.y; rgb[3 * i + 2] = (float)c.z;
        } else {
            const V<float> c = env_eval<float>(sc, mk(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]));
            rgb[3 * i] = c.x; rgb[3 * i + 1] = c.y; rgb[3 * i + 2] = c.z;
        }
    }
}

// FP64 env distribution: sizes, func (h*w), normalised cdf (h*(w+1)),
// row integrals (h), marginal cdf (h+1), marginal integral
OR_API void oracle_env_distribution(void* h, int* w, int* hh, double* func, double* cdf, double* row_int,
                                    double* marg_cdf, double* marg_int) {
    const Scene& sc = ((Ctx*)h)->sc;
    if (w) *w = sc.dw;
    if (hh) *hh = sc.dh;
    if (func) std::memcpy(func, sc.func.data(), sc.func.size() * 8);
    if (cdf) std::memcpy(cdf, sc.cdf.data(), sc.cdf.size() * 8);
    if (row_int) std::memcpy(row_int, sc.row_int.data(), sc.row_int.size() * 8);
    if (marg_cdf) std::memcpy(marg_cdf, sc.marg_cdf.data(), sc.marg_cdf.size() * 8);
    if (marg_int) *marg_int = sc.marg_int;
}

// u -> {x, y, pdf_sample, pdf_eval} in FP64
OR_API void oracle_env_sample(void* h, const float* u, double* out, size_t n) {
    const Scene& sc = ((Ctx*)h)->sc;
    for (size_t i = 0; i < n; ++i) {
        double x, y, pdf;
        dist_sample<double>(sc, (double)u[2 * i], (double)u[2 * i + 1], x, y, pdf);
        out[4 * i] = x;
        out[4 * i + 1] = y;
        out[4 * i + 2] = pdf;
        out[4 * i + 3] = dist_pdf<double>(sc, x, y);
    }
}

// The reference's CudaDistribution2D sampling (distribution2d.cuh:230-336)
// on its own tables (func, cdf: h*(w+2)+1 floats, row r at r*(w+1), the
// marginal at h*(w+1)): u (2 floats) -> {x, y, pdf of the sample, Pdf(x, y)}
struct RefDist {
    const float *func, *cdf;
    int w, h;
    float c(int row, int col) const { return cdf[(size_t)row * (w + 1) + col]; }
    float f(int row, int col) const { return func[(size_t)row * (w + 1) + col]; }
    float fi(int row) const { return f(row, row == h ? h : w); }
    float sample1d(int row, int n, float u, float& pdf, int& off) const {
        int l = 0, r = n, interval = -1;
        while (l <= r) {
            const int m = l + (r - l) / 2;
            if (c(row, m) <= u) {
                l = m + 1;
                interval = m;
            } else {
                r = m - 1;
            }
        }
        off = std::min(std::max(interval, 0), n - 1);
        const float fv = f(row, off), c0 = c(row, off), c1 = c(row, off + 1), fint = fi(row);
        float du = u - c0;
        if (c1 - c0 > 0.0f) du /= (c1 - c0);
        pdf = fint > 0.0f ? fv / fint : 0.0f;
        return ((float)off + du) / (float)n;
    }
};
OR_API void oracle_ref_dist_sample(const float* func, const float* cdf, int w, int h, const float* u, float* out,
                                   size_t n) {
    const RefDist D{func, cdf, w, h};
    for (size_t i = 0; i < n; ++i) {
        float py, px;
        int v, cc;
        const float y = D.sample1d(h, h + 1, u[2 * i + 1], py, v);
        const float x = D.sample1d(v, w + 1, u[2 * i], px, cc);
        out[4 * i] = x;
        out[4 * i + 1] = y;
        out[4 * i + 2] = px * py;
        const int iu = std::min(std::max((int)(x * w), 0), w - 1), iv = std::min(std::max((int)(y * h), 0), h - 1);
        out[4 * i + 3] = D.f(iv, iu) / D.fi(h);
    }
}

OR_API uint32_t oracle_tea16(uint32_t a, uint32_t b) { return tea16(a, b); }
// CudaRNG(id, frame) (rng.cuh:37-76) for (id, frame) pairs: the seed word and
// `draws` floats each
OR_API void oracle_rng(const uint32_t* pairs, size_t n, int draws, uint32_t* seed, float* out) {
    for (size_t i = 0; i < n; ++i) {
        Rng r{tea16(pairs[2 * i], pairs[2 * i + 1])};
        seed[i] = r.s;
        for (int k = 0; k < draws; ++k) out[i * draws + k] = r.next();
    }
}

// Env-texel footprint of the forward paths: replays the paths the adjoint's
// forward traces (frames [f0, f0 + spp) per pixel) and counts, per env
// texel, the radiance lookups that reach the image -- an env term of the
// path with a non-zero throughput before it, a non-zero factor and a
// non-zero bilinear weight on that texel.  Forward only: it reads no
// gradient, so a texel the adjoint leaves at zero is still counted when a
// path reaches it.  counts: env_h x env_w.
OR_API void oracle_env_footprint(void* h, const noor_camera* C, uint32_t f0, uint32_t spp, uint32_t bounces,
                                 const float* alb, const float* rough, const float* env3, int isect, int threads,
                                 uint32_t* counts) {
    const Scene& sc = ((Ctx*)h)->sc;
    const AdjPar P{alb, rough, env3, bounces};
    const size_t NT = (size_t)sc.ew * sc.eh;
    const uint32_t npix = C->w * C->h;
    const int T = std::max(1, threads);
    std::atomic<uint32_t> next{0};
    std::vector<std::vector<uint32_t>> acc(T, std::vector<uint32_t>(NT, 0u));
    auto work = [&](int tid) {
        std::vector<uint32_t>& A = acc[tid];
        std::vector<AVtx> vs;
        std::vector<ATerm> ts;
        for (;;) {
            const uint32_t b0 = next.fetch_add(16);
            if (b0 >= npix) break;
            for (uint32_t p = b0; p < std::min(b0 + 16, npix); ++p)
                for (uint32_t f = 0; f < spp; ++f) {
                    Rng rng{tea16(p, f0 + f)};
                    V<double> o, d;
                    cam_ray<double>(*C, p % C->w, p / C->w, rng, o, d);
                    adj_path(sc, P, o, d, rng, isect, vs, ts);
                    for (const ATerm& t : ts) {
                        if (!t.env) continue;
                        V<double> B = mk(1.0, 1.0, 1.0);
                        for (size_t k = 0; k < t.k; ++k) B = B * vs[k].s;
                        if (black(B * t.fs * t.xscale)) continue;
                        for (int q = 0; q < 4; ++q)
                            if (t.bw.w[q] > 0.0) ++A[t.bw.idx[q]];
                    }
                }
        }
    };
    std::vector<std::thread> th;
    for (int t = 0; t < T; ++t) th.emplace_back(work, t);
    for (auto& x : th) x.join();
    for (size_t i = 0; i < NT; ++i) {
        uint32_t c = 0;
        for (auto& a : acc) c += a[i];
        counts[i] = c;
    }
}

// FP64 reference of the library's adjoint (noor_adjoint_forward/backward):
// img = per-pixel mean of clamp(L, 0, 100) over frames [f0, f0 + spp);
// gradients of sum(grad_img * img) with respect to albedo (M x 3),
// roughness (M) and env texels (env_h x env_w x 3), accumulated in FP64.
// grad_img may be null (forward only).
OR_API void oracle_adjoint(void* h, const noor_camera* C, uint32_t f0, uint32_t spp, uint32_t bounces,
                           const float* alb, const float* rough, const float* env3, const float* grad_img, int isect,
                           int threads, double* img, double* g_alb, double* g_rough, double* g_env) {
    const Scene& sc = ((Ctx*)h)->sc;
    const AdjPar P{alb, rough, env3, bounces};
    const uint32_t M = sc.P->num_materials;
    const size_t NE = (size_t)sc.ew * sc.eh * 3;
    const uint32_t npix = C->w * C->h;
    const int T = std::max(1, threads);
    std::atomic<uint32_t> next{0};
    struct Acc {
        std::vector<double> alb, rough, env;
    };
    std::vector<Acc> acc(T);
    auto work = [&](int tid) {
        Acc& A = acc[tid];
        if (grad_img) {
            A.alb.assign((size_t)M * 3, 0.0);
            A.rough.assign(M, 0.0);
            A.env.assign(NE, 0.0);
        }
        std::vector<AVtx> vs;
        std::vector<ATerm> ts;
        std::vector<V<double>> B;
        for (;;) {
            const uint32_t b0 = next.fetch_add(16);
            if (b0 >= npix) break;
            const uint32_t e0 = std::min(b0 + 16, npix);
            for (uint32_t p = b0; p < e0; ++p) {
                V<double> sum = mk(0.0, 0.0, 0.0);
                const V<double> gi = grad_img ? v3f<double>(grad_img + 3 * (size_t)p) * (1.0 / spp) : mk(0.0, 0.0, 0.0);
                for (uint32_t f = 0; f < spp; ++f) {
                    Rng rng{tea16(p, f0 + f)};
                    V<double> o, d;
                    cam_ray<double>(*C, p % C->w, p / C->w, rng, o, d);
                    adj_path(sc, P, o, d, rng, isect, vs, ts);
                    B.assign(vs.size() + 1, mk(1.0, 1.0, 1.0));
                    for (size_t j = 0; j < vs.size(); ++j) B[j + 1] = B[j] * vs[j].s;
                    V<double> L = mk(0.0, 0.0, 0.0);
                    for (const ATerm& t : ts) L = L + B[t.k] * t.val;
                    sum = sum + mk(clampv(L.x, 0.0, 100.0), clampv(L.y, 0.0, 100.0), clampv(L.z, 0.0, 100.0));
                    if (!grad_img) continue;
                    // derivative of the final clamp
                    const V<double> g = mk(L.x > 0 && L.x < 100 ? gi.x : 0.0, L.y > 0 && L.y < 100 ? gi.y : 0.0,
                                           L.z > 0 && L.z < 100 ? gi.z : 0.0);
                    if (black(g)) continue;
                    for (const ATerm& t : ts) {
                        const V<double> gB = g * B[t.k];
                        if (t.has_mat) {
                            const V<double> da = gB * t.d_alb;
                            A.alb[3 * t.mat] += da.x;
                            A.alb[3 * t.mat + 1] += da.y;
                            A.alb[3 * t.mat + 2] += da.z;
                            const V<double> dr = gB * t.d_r;
                            A.rough[t.mat] += dr.x + dr.y + dr.z;
                        }
                        if (t.env) {
                            const V<double> ge = gB * t.fs * t.xscale;
                            for (int q = 0; q < 4; ++q) {
                                double* e = &A.env[3 * t.bw.idx[q]];
                                e[0] += ge.x * t.bw.w[q];
                                e[1] += ge.y * t.bw.w[q];
                                e[2] += ge.z * t.bw.w[q];
                            }
                        }
                        // scatter factors before the term
                        for (size_t j = 0; j < t.k; ++j) {
                            if (!vs[j].has_mat) continue;
                            V<double> pj = mk(1.0, 1.0, 1.0);
                            for (size_t i = 0; i < t.k; ++i)
                                if (i != j) pj = pj * vs[i].s;
                            const V<double> base = g * pj * t.val;
                            const V<double> da = base * vs[j].ds_alb;
                            A.alb[3 * vs[j].mat] += da.x;
                            A.alb[3 * vs[j].mat + 1] += da.y;
                            A.alb[3 * vs[j].mat + 2] += da.z;
                            const V<double> dr = base * vs[j].ds_r;
                            A.rough[vs[j].mat] += dr.x + dr.y + dr.z;
                        }
                    }
                }
                if (img) {
                    img[3 * (size_t)p] = sum.x / spp;
                    img[3 * (size_t)p + 1] = sum.y / spp;
                    img[3 * (size_t)p + 2] = sum.z / spp;
                }
            }
        }
    };
    std::vector<std::thread> th;
    for (int t = 0; t < T; ++t) th.emplace_back(work, t);
    for (auto& x : th) x.join();
    if (!grad_img) return;
    for (size_t i = 0; i < (size_t)M * 3; ++i) {
        g_alb[i] = 0;
        for (auto& a : acc) g_alb[i] += a.alb[i];
    }
    for (size_t i = 0; i < M; ++i) {
        g_rough[i] = 0;
        for (auto& a : acc) g_rough[i] += a.rough[i];
    }
    if (g_env)
        for (size_t i = 0; i < NE; ++i) {
            g_env[i] = 0;
            for (auto& a : acc) g_env[i] += a.env[i];
        }
}
