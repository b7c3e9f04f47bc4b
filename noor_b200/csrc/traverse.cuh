// Two-level BVH traversal (closest hit and any hit) with a per-thread stack
// in shared memory, and the two ray/triangle tests:
//   * NOOR_ISECT_REF_WALD: the reference's Wald projection test
//     (noor/cuda/triangle.cuh:82-198), evaluated with exactly rounded
//     operations in the order the source writes them;
//   * NOOR_ISECT_WATERTIGHT: Woop, Benthin & Wald 2013, "Watertight
//     Ray/Triangle Intersection" (JCGT 2(1)), with its double-precision
//     fallback on zero edge functions.
// The traversal order reproduces noor/cuda/bvh.cuh:142-234: pop, slab test,
// then by node kind; an inner node pushes the far child first so the near
// child (chosen by the ray's direction sign on the split axis) pops next.
#pragma once
#include "scene_dev.cuh"
#include "wide_bvh.h"

namespace nb {

// ray in the space of the BVH level being traversed
struct TRay {
    float3 o, d, inv;
    uint32_t neg;  // bit a set when d[a] <= 0 (noor/cuda/ray.cuh:200-206)
};

NB_D void tray_setup(TRay& r, const float3& o, const float3& d) {
    r.o = o;
    r.d = d;
    r.inv = f3(xdiv(1.0f, d.x), xdiv(1.0f, d.y), xdiv(1.0f, d.z));
    r.neg = (d.x > 0.0f ? 0u : 1u) | (d.y > 0.0f ? 0u : 2u) | (d.z > 0.0f ? 0u : 4u);
}

// world -> object: origin as translation + M*o, direction as M*d, no
// renormalisation, so t is shared by both levels (noor/cuda/ray.cuh:174-180)
NB_D void tray_to_object(TRay& r, const TRay& w, const DevXform* xf) {
    const float4 r0 = __ldg(&xf->w2o[0]);
    const float4 r1 = __ldg(&xf->w2o[1]);
    const float4 r2 = __ldg(&xf->w2o[2]);
    const float3 o = f3(xadd(r0.w, xdot3(r0.x, r0.y, r0.z, w.o.x, w.o.y, w.o.z)),
                        xadd(r1.w, xdot3(r1.x, r1.y, r1.z, w.o.x, w.o.y, w.o.z)),
                        xadd(r2.w, xdot3(r2.x, r2.y, r2.z, w.o.x, w.o.y, w.o.z)));
    const float3 d = f3(xdot3(r0.x, r0.y, r0.z, w.d.x, w.d.y, w.d.z),
                        xdot3(r1.x, r1.y, r1.z, w.d.x, w.d.y, w.d.z),
                        xdot3(r2.x, r2.y, r2.z, w.d.x, w.d.y, w.d.z));
    tray_setup(r, o, d);
}

// A ray whose origin and direction components are all finite and non-zero:
// an identity transform maps it onto itself bit for bit (1 x = x, 0 y = +-0,
// x +- 0 = x), which a zero or non-finite component would not guarantee
// (-0 turns into +0, 0 inf into NaN).
NB_D bool ray_plain(const float3& o, const float3& d) {
    const float m = 3.40282347e38f;
    const float ao[3] = {fabsf(o.x), fabsf(o.y), fabsf(o.z)}, ad[3] = {fabsf(d.x), fabsf(d.y), fabsf(d.z)};
    bool ok = true;
#pragma unroll
    for (int i = 0; i < 3; ++i) ok = ok && ao[i] > 0.0f && ao[i] <= m && ad[i] > 0.0f && ad[i] <= m;
    return ok;
}

// The level's ray moved into instance `ins`'s object space
// (noor/cuda/ray.cuh:174-180).  An instance whose world-to-object rows are
// exactly the identity (DevScene::xf_ident, set at upload) leaves a plain
// ray as it is, so the world ray is kept.  Returns whether the level's ray
// is the world ray.
NB_D bool enter_instance(TRay& lr, const TRay& wr, const DevScene& S, uint32_t ins, bool plain) {
    if (plain && ((__ldg(&S.xf_ident[ins >> 5]) >> (ins & 31u)) & 1u)) {
        lr = wr;
        return true;
    }
    tray_to_object(lr, wr, S.xforms + ins);
    return false;
}

// slab test of noor/cuda/bbox.cuh:62-80
NB_D bool slab_hit_f(const TRay& r, float mnx, float mny, float mnz, float mxx, float mxy, float mxz, float tmax) {
    const bool nx = r.neg & 1u, ny = r.neg & 2u, nz = r.neg & 4u;
    float tMin = xmul(xsub(nx ? mxx : mnx, r.o.x), r.inv.x);
    float tMax = xmul(xsub(nx ? mnx : mxx, r.o.x), r.inv.x);
    const float tyMin = xmul(xsub(ny ? mxy : mny, r.o.y), r.inv.y);
    const float tyMax = xmul(xsub(ny ? mny : mxy, r.o.y), r.inv.y);
    if (tMin > tyMax || tyMin > tMax) return false;
    if (tyMin > tMin) tMin = tyMin;
    if (tyMax < tMax) tMax = tyMax;
    const float tzMin = xmul(xsub(nz ? mxz : mnz, r.o.z), r.inv.z);
    const float tzMax = xmul(xsub(nz ? mnz : mxz, r.o.z), r.inv.z);
    if (tMin > tzMax || tzMin > tMax) return false;
    if (tzMin > tMin) tMin = tzMin;
    if (tzMax < tMax) tMax = tzMax;
    return (tMin < tmax) && (tMax > 0.0f);
}
NB_D bool slab_hit(const TRay& r, const uint4& lo, const uint4& hi, float tmax) {
    return slab_hit_f(r, __uint_as_float(lo.x), __uint_as_float(lo.y), __uint_as_float(lo.z), __uint_as_float(hi.x),
                      __uint_as_float(hi.y), __uint_as_float(hi.z), tmax);
}

// Wald projection test (noor/cuda/triangle.cuh:82-141); on success writes
// t into tmax and the barycentrics (u weights v1, v weights v2).
NB_D bool wald_test(const TRay& r, const DevWaldTri* tri, float& tmax, float& bu, float& bv,
                    uint32_t& mtype) {
    const uint4 a = __ldg(&tri->ax_nu_nv_nd);
    const uint4 c = __ldg(&tri->cnu_cnv_deg_mat);
    if (c.z == 1u) return false;
    const uint32_t k = a.x;
    const uint32_t ku = (k == 0u) ? 1u : (k == 1u ? 2u : 0u);
    const uint32_t kv = (k == 0u) ? 2u : (k == 1u ? 0u : 1u);
    const float ro_u = comp(r.o, ku), ro_v = comp(r.o, kv), ro_k = comp(r.o, k);
    const float rd_u = comp(r.d, ku), rd_v = comp(r.d, kv), rd_k = comp(r.d, k);
    const float nu = __uint_as_float(a.y), nv = __uint_as_float(a.z), nd = __uint_as_float(a.w);
    const float denom = xadd(xadd(rd_k, xmul(nu, rd_u)), xmul(nv, rd_v));
    if (denom == 0.0f) return false;
    const float t = xdiv(xsub(xsub(xsub(nd, ro_k), xmul(nu, ro_u)), xmul(nv, ro_v)), denom);
    if (t < 0.0f || t > tmax) return false;
    const uint4 b = __ldg(&tri->bnu_bnv_au_av);
    const float hu = xsub(xadd(ro_u, xmul(t, rd_u)), __uint_as_float(b.z));
    const float hv = xsub(xadd(ro_v, xmul(t, rd_v)), __uint_as_float(b.w));
    const float u = xadd(xmul(hv, __uint_as_float(b.x)), xmul(hu, __uint_as_float(b.y)));
    const float v = xadd(xmul(hu, __uint_as_float(c.x)), xmul(hv, __uint_as_float(c.y)));
    if (!(u >= 0.0f && v >= 0.0f && xadd(u, v) <= 1.0f)) return false;
    tmax = t;
    bu = u;
    bv = v;
    mtype = c.w;
    return true;
}

// per-ray constants of the watertight test
struct WtRay {
    int kx, ky, kz;
    float sx, sy, sz;
};

NB_D void wt_setup(WtRay& w, const float3& d) {
    const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    int kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    int kx = kz + 1 == 3 ? 0 : kz + 1;
    int ky = kx + 1 == 3 ? 0 : kx + 1;
    const float dz = comp(d, kz);
    if (dz < 0.0f) {
        const int t = kx;
        kx = ky;
        ky = t;
    }
    w.kx = kx;
    w.ky = ky;
    w.kz = kz;
    w.sx = xdiv(comp(d, kx), dz);
    w.sy = xdiv(comp(d, ky), dz);
    w.sz = xdiv(1.0f, dz);
}

NB_D float xorsign(float v, uint32_t signbit) { return __uint_as_float(__float_as_uint(v) ^ signbit); }

NB_D bool wt_test(const TRay& r, const WtRay& w, const DevWtTri* tri, float& tmax, float& bu,
                  float& bv, uint32_t& mtype) {
    const float4 p0 = __ldg(&tri->v0);
    const float4 p1 = __ldg(&tri->v1);
    const float4 p2 = __ldg(&tri->v2);
    const float3 A = f3(xsub(p0.x, r.o.x), xsub(p0.y, r.o.y), xsub(p0.z, r.o.z));
    const float3 B = f3(xsub(p1.x, r.o.x), xsub(p1.y, r.o.y), xsub(p1.z, r.o.z));
    const float3 C = f3(xsub(p2.x, r.o.x), xsub(p2.y, r.o.y), xsub(p2.z, r.o.z));
    const float Akz = comp(A, w.kz), Bkz = comp(B, w.kz), Ckz = comp(C, w.kz);
    const float Ax = xsub(comp(A, w.kx), xmul(w.sx, Akz));
    const float Ay = xsub(comp(A, w.ky), xmul(w.sy, Akz));
    const float Bx = xsub(comp(B, w.kx), xmul(w.sx, Bkz));
    const float By = xsub(comp(B, w.ky), xmul(w.sy, Bkz));
    const float Cx = xsub(comp(C, w.kx), xmul(w.sx, Ckz));
    const float Cy = xsub(comp(C, w.ky), xmul(w.sy, Ckz));
    float U = xsub(xmul(Cx, By), xmul(Cy, Bx));
    float V = xsub(xmul(Ax, Cy), xmul(Ay, Cx));
    float W = xsub(xmul(Bx, Ay), xmul(By, Ax));
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        // products of two floats are exact in double; one rounding each
        U = (float)__dsub_rn(__dmul_rn((double)Cx, (double)By), __dmul_rn((double)Cy, (double)Bx));
        V = (float)__dsub_rn(__dmul_rn((double)Ax, (double)Cy), __dmul_rn((double)Ay, (double)Cx));
        W = (float)__dsub_rn(__dmul_rn((double)Bx, (double)Ay), __dmul_rn((double)By, (double)Ax));
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    const float det = xadd(xadd(U, V), W);
    if (det == 0.0f) return false;
    const float Az = xmul(w.sz, Akz), Bz = xmul(w.sz, Bkz), Cz = xmul(w.sz, Ckz);
    const float T = xadd(xadd(xmul(U, Az), xmul(V, Bz)), xmul(W, Cz));
    const uint32_t sgn = __float_as_uint(det) & 0x80000000u;
    const float Ts = xorsign(T, sgn);
    if (Ts < 0.0f || Ts > xmul(tmax, xorsign(det, sgn))) return false;
    const float rcp = xdiv(1.0f, det);
    tmax = xmul(T, rcp);
    bu = xmul(V, rcp);
    bv = xmul(W, rcp);
    mtype = __float_as_uint(p0.w);
    return true;
}

// The alpha cut of an ALPHA material's triangle (noor/cuda/triangle.cuh:
// 124-133): the transparency map at the hit's interpolated uv; a texel of
// 1e-4 or less lets the ray through.
template <int ISECT>
NB_OUTLINE bool alpha_cut(const DevScene& S, uint32_t ti, float bu, float bv) {
    const uint4 a = ISECT == NOOR_ISECT_WATERTIGHT ? __ldg(&S.wtri[ti].attr) : __ldg(&S.wald[ti].attr);
    const float2 uv = lerp_uv(vertex_uv(S, a.x), vertex_uv(S, a.y), vertex_uv(S, a.z), bu, bv);
    return slot_tex(S.mat_tex[a.w], kTexAlpha, uv).x <= 0.0001f;
}

// Arithmetic of the light-shape tests: with X (the reference's Wald mode,
// whose hit distances are the reference's to the bit) each operation rounds
// on its own; otherwise the compiler may contract multiply-adds.
template <bool X> NB_D float smul(float a, float b) { return X ? __fmul_rn(a, b) : a * b; }
template <bool X> NB_D float sadd(float a, float b) { return X ? __fadd_rn(a, b) : a + b; }
template <bool X> NB_D float ssub(float a, float b) { return X ? __fsub_rn(a, b) : a - b; }
template <bool X> NB_D float sdot(float ax, float ay, float az, float bx, float by, float bz) {
    return sadd<X>(sadd<X>(smul<X>(ax, bx), smul<X>(ay, by)), smul<X>(az, bz));
}

// quad of an area light (noor/cuda/geometry.cuh:105-123); note the
// reference accepts negative t (no lower bound), kept as is.
template <bool X = false>
NB_D bool quad_hit(const DevAreaLight& q, const float3& o, const float3& d, float& tmax) {
    const float denom = sdot<X>(q.n.x, q.n.y, q.n.z, d.x, d.y, d.z);
    if (denom == 0.0f) return false;
    const float t = -ssub<X>(sdot<X>(o.x, o.y, o.z, q.n.x, q.n.y, q.n.z),
                             sdot<X>(q.center.x, q.center.y, q.center.z, q.n.x, q.n.y, q.n.z)) /
                    denom;
    if (t > tmax) return false;
    // pointAtParameter(t) - center
    const float ix = ssub<X>(sadd<X>(o.x, smul<X>(t, d.x)), q.center.x);
    const float iy = ssub<X>(sadd<X>(o.y, smul<X>(t, d.y)), q.center.y);
    const float iz = ssub<X>(sadd<X>(o.z, smul<X>(t, d.z)), q.center.z);
    const float t0 = sdot<X>(ix, iy, iz, q.u.x, q.u.y, q.u.z) / sdot<X>(q.u.x, q.u.y, q.u.z, q.u.x, q.u.y, q.u.z);
    if (t0 < 0.0f || t0 > 1.0f) return false;
    const float t1 = sdot<X>(ix, iy, iz, q.v.x, q.v.y, q.v.z) / sdot<X>(q.v.x, q.v.y, q.v.z, q.v.x, q.v.y, q.v.z);
    if (t1 < 0.0f || t1 > 1.0f) return false;
    tmax = t;
    return true;
}

// solveQuadratic (noor/cuda/utils.cuh:52-91): the root of larger magnitude
// first, the other from x0 * x1 = c / a; returns x0 <= x1
template <bool X = false>
NB_D bool solve_quadratic(float a, float b, float c, float& x0, float& x1) {
    if (a == 0.0f) {
        if (b != 0.0f) {
            x0 = x1 = -c / b;
            return true;
        }
        return false;
    }
    const float disc = ssub<X>(smul<X>(b, b), smul<X>(smul<X>(4.0f, a), c));
    if (disc < 0.0f) return false;
    const float sd = sqrtf(disc);
    const float q = b < 0.0f ? smul<X>(-0.5f, ssub<X>(b, sd)) : smul<X>(-0.5f, sadd<X>(b, sd));
    x0 = q / a;
    x1 = c / q;
    if (x0 > x1) {
        const float t = x0;
        x0 = x1;
        x1 = t;
    }
    return true;
}

// sphere of an area light (noor/cuda/geometry.cuh:125-150): nearest root in
// [0, tmax], else the far root when the near one is behind the origin
template <bool X = false>
NB_D bool sphere_hit(const DevAreaLight& s, const float3& o, const float3& d, float& tmax) {
    const float ox = ssub<X>(o.x, s.center.x), oy = ssub<X>(o.y, s.center.y), oz = ssub<X>(o.z, s.center.z);
    float t0, t1;
    if (!solve_quadratic<X>(sdot<X>(d.x, d.y, d.z, d.x, d.y, d.z), smul<X>(2.0f, sdot<X>(ox, oy, oz, d.x, d.y, d.z)),
                            ssub<X>(sdot<X>(ox, oy, oz, ox, oy, oz), s.radius2), t0, t1))
        return false;
    if (!(t0 <= tmax && t1 >= 0.0f)) return false;
    if (t0 < 0.0f) {
        if (t1 > tmax) return false;
        tmax = t1;
    } else {
        tmax = t0;
    }
    return true;
}

// disk of an area light (noor/cuda/geometry.cuh:152-163); like the quad, no
// lower bound on t
template <bool X = false>
NB_D bool disk_hit(const DevAreaLight& q, const float3& o, const float3& d, float& tmax) {
    const float denom = sdot<X>(q.n.x, q.n.y, q.n.z, d.x, d.y, d.z);
    if (denom == 0.0f) return false;
    const float t = -ssub<X>(sdot<X>(o.x, o.y, o.z, q.n.x, q.n.y, q.n.z),
                             sdot<X>(q.center.x, q.center.y, q.center.z, q.n.x, q.n.y, q.n.z)) /
                    denom;
    if (t > tmax) return false;
    const float px = ssub<X>(sadd<X>(o.x, smul<X>(t, d.x)), q.center.x);
    const float py = ssub<X>(sadd<X>(o.y, smul<X>(t, d.y)), q.center.y);
    const float pz = ssub<X>(sadd<X>(o.z, smul<X>(t, d.z)), q.center.z);
    if (sdot<X>(px, py, pz, px, py, pz) > q.radius2) return false;
    tmax = t;
    return true;
}

// CudaShape::intersect (noor/cuda/shapeimp.cuh:73-87).  EXT false: the
// scene's area lights are all quads (kernels for such scenes leave the
// other shapes' code out)
template <bool EXT = true, bool X = false>
NB_D bool shape_hit(const DevAreaLight& a, const float3& o, const float3& d, float& tmax) {
    if (!EXT || a.type == NOOR_SHAPE_QUAD) return quad_hit<X>(a, o, d, tmax);
    if (a.type == NOOR_SHAPE_SPHERE) return sphere_hit<X>(a, o, d, tmax);
    return disk_hit<X>(a, o, d, tmax);
}

struct HitRec {
    float u, v;
    uint32_t tri;
    uint32_t ins;
    uint32_t mtype;
};

// Shared-memory stack: entry i of this thread lives at stk[i * stride].
struct SmemStack {
    uint32_t* base;
    int stride;
    int cap;
};

// Node kinds that are not inner nodes (an inner node has none of these bits)
constexpr uint32_t kNodeKindMask =
    NOOR_LIGHT_NODE_MASK | NOOR_MESH_INSTANCE_MASK | NOOR_MESH_LEAF_MASK | NOOR_TRI_LEAF_MASK;
constexpr uint32_t kNoNode = 0xFFFFFFFFu;

// Closest hit.  tmax in: ray extent, out: hit distance.  Returns hit flag;
// on stack overflow sets *status and returns what was found so far.
// The visit order is that of the reference's stack loop: the node the
// reference would pop next (the near child of an inner node, the last child
// of a mesh leaf, the root of an instance) is kept in a register instead of
// being pushed and popped at once, and inner nodes are dispatched first.
template <int ISECT, bool EXT = true>
NB_D bool trace_closest(const DevScene& S, const float3& o, const float3& d, float& tmax,
                        HitRec& rec, const SmemStack& st, uint32_t* status) {
    TRay wr;
    tray_setup(wr, o, d);
    TRay lr = wr;
    WtRay wt;
    if (ISECT == NOOR_ISECT_WATERTIGHT) wt_setup(wt, lr.d);
    bool wtw = true;  // wt holds the world ray's constants
    const bool plain = ray_plain(o, d);
    float ltmax = tmax;
    uint32_t ins = 0;
    bool hit = false;
    int top = 0;
    uint32_t ni = S.root;
    for (;;) {
        const DevNode* nd = S.nodes + ni;
        const uint4 lo = __ldg(&nd->lo);
        const uint4 hi = __ldg(&nd->hi);
        uint32_t next = kNoNode;
        if (hi.w & NOOR_MESH_NODE_MASK) {
            lr = wr;
            ltmax = tmax;
            if (ISECT == NOOR_ISECT_WATERTIGHT && !wtw) {
                wt_setup(wt, wr.d);
                wtw = true;
            }
        }
        if (slab_hit(lr, lo, hi, ltmax)) {
            if (!(hi.w & kNodeKindMask)) {
                // inner: the near child (by the ray's sign on the split axis) next, the far one pushed
                if (top + 1 > st.cap) { atomicOr(status, NOOR_DEV_STACK_OVERFLOW); break; }
                const uint32_t axis = hi.w & NOOR_AXIS_MASK;
                const bool neg = (lr.neg >> axis) & 1u;
                st.base[top * st.stride] = neg ? ni + 1 : lo.w;
                ++top;
                next = neg ? lo.w : ni + 1;
            } else if (hi.w & NOOR_LIGHT_NODE_MASK) {
                const uint32_t li = hi.w & NOOR_LIGHT_MASK;
                if ((int)li < S.num_area_lights &&
                    shape_hit<EXT, ISECT == NOOR_ISECT_REF_WALD>(S.area_lights[li], o, d, tmax)) {
                    hit = true;
                    rec.ins = li;
                    rec.mtype = NOOR_MESHLIGHT | NOOR_EMITTER;
                }
            } else if (hi.w & NOOR_MESH_INSTANCE_MASK) {
                ins = hi.w & NOOR_TRANS_MASK;
                const bool same = enter_instance(lr, wr, S, ins, plain);
                ltmax = tmax;
                if (ISECT == NOOR_ISECT_WATERTIGHT && !(same && wtw)) {
                    wt_setup(wt, lr.d);
                    wtw = same;
                }
                next = lo.w;
            } else if (hi.w & NOOR_MESH_LEAF_MASK) {
                const uint32_t cnt = hi.w & NOOR_COUNT_MASK;
                if (top + (int)cnt > st.cap + 1) { atomicOr(status, NOOR_DEV_STACK_OVERFLOW); break; }
                for (uint32_t i = 1; i < cnt; ++i) {
                    st.base[top * st.stride] = ni + i;
                    ++top;
                }
                if (cnt) next = ni + cnt;
            } else {
                const uint32_t start = lo.w;
                const uint32_t end = start + (hi.w & NOOR_TRI_COUNT_MASK);
                bool leaf_hit = false;
                for (uint32_t ti = start; ti < end; ++ti) {
                    float bu, bv;
                    uint32_t mt;
                    bool h;
                    if (EXT && S.has_alpha) {
                        // the hit distance is kept only past the alpha cut
                        float tc = ltmax;
                        if (ISECT == NOOR_ISECT_WATERTIGHT)
                            h = wt_test(lr, wt, S.wtri + ti, tc, bu, bv, mt);
                        else
                            h = wald_test(lr, S.wald + ti, tc, bu, bv, mt);
                        if (h && (mt & NOOR_ALPHA) && alpha_cut<ISECT>(S, ti, bu, bv)) h = false;
                        if (h) ltmax = tc;
                    } else if (ISECT == NOOR_ISECT_WATERTIGHT) {
                        h = wt_test(lr, wt, S.wtri + ti, ltmax, bu, bv, mt);
                    } else {
                        h = wald_test(lr, S.wald + ti, ltmax, bu, bv, mt);
                    }
                    if (h) {
                        leaf_hit = true;
                        rec.u = bu;
                        rec.v = bv;
                        rec.tri = ti;
                        rec.mtype = mt;
                    }
                }
                if (leaf_hit) {
                    hit = true;
                    tmax = ltmax;
                    rec.ins = ins;
                }
            }
        }
        if (next == kNoNode) {
            if (top == 0) break;
            --top;
            next = st.base[top * st.stride];
        }
        ni = next;
    }
    return hit;
}

// Any hit within (0, tmax]; light nodes count as occluders.  Same visit
// order and register-held next node as trace_closest.
template <int ISECT, bool EXT = true>
NB_D bool trace_any(const DevScene& S, const float3& o, const float3& d, float tmax,
                    const SmemStack& st, uint32_t* status) {
    TRay wr;
    tray_setup(wr, o, d);
    TRay lr = wr;
    WtRay wt;
    if (ISECT == NOOR_ISECT_WATERTIGHT) wt_setup(wt, lr.d);
    bool wtw = true;  // wt holds the world ray's constants
    const bool plain = ray_plain(o, d);
    float ltmax = tmax;
    int top = 0;
    uint32_t ni = S.root;
    for (;;) {
        const DevNode* nd = S.nodes + ni;
        const uint4 lo = __ldg(&nd->lo);
        const uint4 hi = __ldg(&nd->hi);
        uint32_t next = kNoNode;
        if (hi.w & NOOR_MESH_NODE_MASK) {
            lr = wr;
            ltmax = tmax;
            if (ISECT == NOOR_ISECT_WATERTIGHT && !wtw) {
                wt_setup(wt, wr.d);
                wtw = true;
            }
        }
        if (slab_hit(lr, lo, hi, ltmax)) {
            if (!(hi.w & kNodeKindMask)) {
                if (top + 1 > st.cap) { atomicOr(status, NOOR_DEV_STACK_OVERFLOW); return false; }
                const uint32_t axis = hi.w & NOOR_AXIS_MASK;
                const bool neg = (lr.neg >> axis) & 1u;
                st.base[top * st.stride] = neg ? ni + 1 : lo.w;
                ++top;
                next = neg ? lo.w : ni + 1;
            } else if (hi.w & NOOR_LIGHT_NODE_MASK) {
                const uint32_t li = hi.w & NOOR_LIGHT_MASK;
                float tm = tmax;
                if ((int)li < S.num_area_lights && shape_hit<EXT, ISECT == NOOR_ISECT_REF_WALD>(S.area_lights[li], o, d, tm))
                    return true;
            } else if (hi.w & NOOR_MESH_INSTANCE_MASK) {
                const bool same = enter_instance(lr, wr, S, hi.w & NOOR_TRANS_MASK, plain);
                ltmax = tmax;
                if (ISECT == NOOR_ISECT_WATERTIGHT && !(same && wtw)) {
                    wt_setup(wt, lr.d);
                    wtw = same;
                }
                next = lo.w;
            } else if (hi.w & NOOR_MESH_LEAF_MASK) {
                const uint32_t cnt = hi.w & NOOR_COUNT_MASK;
                if (top + (int)cnt > st.cap + 1) { atomicOr(status, NOOR_DEV_STACK_OVERFLOW); return false; }
                for (uint32_t i = 1; i < cnt; ++i) {
                    st.base[top * st.stride] = ni + i;
                    ++top;
                }
                if (cnt) next = ni + cnt;
            } else {
                const uint32_t start = lo.w;
                const uint32_t end = start + (hi.w & NOOR_TRI_COUNT_MASK);
                for (uint32_t ti = start; ti < end; ++ti) {
                    float tm = ltmax, bu, bv;
                    uint32_t mt;
                    bool h;
                    if (ISECT == NOOR_ISECT_WATERTIGHT)
                        h = wt_test(lr, wt, S.wtri + ti, tm, bu, bv, mt);
                    else
                        h = wald_test(lr, S.wald + ti, tm, bu, bv, mt);
                    if (h && EXT && S.has_alpha && (mt & NOOR_ALPHA) && alpha_cut<ISECT>(S, ti, bu, bv)) h = false;
                    if (h) return true;
                }
            }
        }
        if (next == kNoNode) {
            if (top == 0) break;
            --top;
            next = st.base[top * st.stride];
        }
        ni = next;
    }
    return false;
}

// A ray below which the four-wide tree's boxes may not stand in for the
// binary tree's: a direction component that is zero, subnormal or NaN (its
// slab reciprocal is infinite, and the per-axis intervals stop being
// monotone in the box), or an origin that is not finite.  Such rays walk the
// binary tree node by node.
NB_D bool wide_degenerate(const float3& o, const float3& d) {
    const float m = 1.17549435e-38f;  // FLT_MIN
    return !(fabsf(d.x) >= m && fabsf(d.y) >= m && fabsf(d.z) >= m && fabsf(o.x) <= 3.40282347e38f &&
             fabsf(o.y) <= 3.40282347e38f && fabsf(o.z) <= 3.40282347e38f);
}

NB_D uint32_t word_of(const uint4& v, uint32_t s) { return s == 0 ? v.x : (s == 1 ? v.y : (s == 2 ? v.z : v.w)); }
NB_D float comp4(const float4& v, uint32_t s) { return s == 0 ? v.x : (s == 1 ? v.y : (s == 2 ? v.z : v.w)); }

// The slab test of noor/cuda/bbox.cuh:62-80 on a wide node's four entry
// boxes at once, axis by axis: the same operations and comparisons as
// slab_hit_f for each box, the near and far bounds of an axis picked by
// address (the ray's sign) instead of per box.  Bit s set when box s passes.
NB_D uint32_t slab4(const TRay& r, const DevNode4* nd, float tmax) {
    const float4* b = &nd->lox;  // lox, loy, loz, hix, hiy, hiz
    float t0[4], t1[4];
    uint32_t ok = 0xFu;
    {
        const uint32_t n = (r.neg & 1u) ? 3u : 0u;
        const float4 a = __ldg(b + n), c = __ldg(b + (3u - n));
#pragma unroll
        for (uint32_t s = 0; s < 4; ++s) {
            t0[s] = xmul(xsub(comp4(a, s), r.o.x), r.inv.x);
            t1[s] = xmul(xsub(comp4(c, s), r.o.x), r.inv.x);
        }
    }
    {
        const uint32_t n = (r.neg & 2u) ? 3u : 0u;
        const float4 a = __ldg(b + 1 + n), c = __ldg(b + 1 + (3u - n));
#pragma unroll
        for (uint32_t s = 0; s < 4; ++s) {
            const float u0 = xmul(xsub(comp4(a, s), r.o.y), r.inv.y);
            const float u1 = xmul(xsub(comp4(c, s), r.o.y), r.inv.y);
            if (t0[s] > u1 || u0 > t1[s]) ok &= ~(1u << s);
            if (u0 > t0[s]) t0[s] = u0;
            if (u1 < t1[s]) t1[s] = u1;
        }
    }
    {
        const uint32_t n = (r.neg & 4u) ? 3u : 0u;
        const float4 a = __ldg(b + 2 + n), c = __ldg(b + 2 + (3u - n));
#pragma unroll
        for (uint32_t s = 0; s < 4; ++s) {
            const float u0 = xmul(xsub(comp4(a, s), r.o.z), r.inv.z);
            const float u1 = xmul(xsub(comp4(c, s), r.o.z), r.inv.z);
            if (t0[s] > u1 || u0 > t1[s]) ok &= ~(1u << s);
            if (u0 > t0[s]) t0[s] = u0;
            if (u1 < t1[s]) t1[s] = u1;
        }
    }
#pragma unroll
    for (uint32_t s = 0; s < 4; ++s)
        if (!(t0[s] < tmax && t1[s] > 0.0f)) ok &= ~(1u << s);
    return ok;
}

// A wide node's visit: its entries that pass the slab test (and its
// deferred ones) in the binary traversal's order for the ray's octant (the
// node's order table), the first into `next`, the rest pushed so that they
// come off the stack in order.  False on a stack overflow.
NB_D bool wide_visit(const DevNode4* nd, const uint4& meta, const TRay& r, float tmax, const SmemStack& st, int cap,
                     int& top, uint32_t& next, uint32_t* status) {
    const uint4 cw = __ldg(&nd->child);
    uint32_t inc = slab4(r, nd, tmax);
#pragma unroll
    for (uint32_t s = 0; s < 4; ++s) {
        const uint32_t w = word_of(cw, s);
        if (w == kWNone) inc &= ~(1u << s);
        else if ((w & (kWRef | kWUntested)) == (kWRef | kWUntested)) inc |= 1u << s;
    }
    if (!inc) return true;
    const uint32_t oct = r.neg & 7u;
    const uint32_t order = ((oct & 4u) ? meta.z : meta.y) >> (8u * (oct & 3u));
    // last in order first: each taken word pushes the one held before it
#pragma unroll
    for (int j = 3; j >= 0; --j) {
        const uint32_t s = (order >> (2 * j)) & 3u;
        if (!((inc >> s) & 1u)) continue;
        if (next != kWNone) {
            if (top + 1 > cap) {
                atomicOr(status, NOOR_DEV_STACK_OVERFLOW);
                return false;
            }
            st.base[top * st.stride] = next;
            ++top;
        }
        next = word_of(cw, s);
    }
    return true;
}

// An inner node taken from the stack or a ref once its box passed: its wide
// node, or for a ray below which boxes may not be skipped one binary step
// (the far child pushed, the near one next, as trace_closest takes them).
// False on a stack overflow or a missing wide node.
NB_D bool inner_step(const DevScene& S, uint32_t ni, const uint4& lo, const uint4& hi, const TRay& r, bool deg,
                     const SmemStack& st, int cap, int& top, uint32_t& next, uint32_t* status) {
    if (deg) {
        if (top + 1 > cap) {
            atomicOr(status, NOOR_DEV_STACK_OVERFLOW);
            return false;
        }
        const bool neg = (r.neg >> (hi.w & NOOR_AXIS_MASK)) & 1u;
        st.base[top * st.stride] = kWRef | kWUntested | (neg ? ni + 1 : lo.w);
        ++top;
        next = kWRef | kWUntested | (neg ? lo.w : ni + 1);
        return true;
    }
    next = __ldg(&S.map4[ni]);
    if (next == kWNone) {
        atomicOr(status, NOOR_DEV_BAD_INDEX);
        return false;
    }
    return true;
}

// Any hit over the four-wide tree (S.nodes4, layout in wide_bvh.h): the same
// answer as trace_any on the binary tree.  Binary nodes (leaves, mesh
// leaves, instances, light nodes and deferred entries) are taken as the
// binary traversal takes them; a ref carries kWUntested when its box has not
// been tested yet.  The stack holds S.stack_cap4 words, the deepest this
// tree can need.  The walk is kept in an Any4 so that a kernel can advance
// many rays a step at a time (any4_step) and start a new ray on a lane as
// soon as its last one ends.
struct Any4 {
    TRay wr, lr;        // the world ray, the ray of the level being walked
    WtRay wt;           // watertight constants of wt_ray's level
    float tmax;
    uint32_t next;      // the word taken next
    int top;
    bool wdeg, ldeg;    // wide_degenerate of the world / level ray
    bool wtw;           // wt holds the world ray's constants
    bool plain;         // ray_plain of the world ray
};

template <int ISECT>
NB_D void any4_init(Any4& a, const DevScene& S, const float3& o, const float3& d, float tmax) {
    tray_setup(a.wr, o, d);
    a.lr = a.wr;
    a.wdeg = a.ldeg = wide_degenerate(o, d);
    if (ISECT == NOOR_ISECT_WATERTIGHT) wt_setup(a.wt, d);
    a.wtw = true;
    a.plain = ray_plain(o, d);
    a.tmax = tmax;
    a.top = 0;
    a.next = kWRef | kWUntested | S.root;
}

enum : int { kAnyRunning = 0, kAnyHit = 1, kAnyMiss = 2, kAnyFailed = 3 };

// One step of the walk: a wide node's visit or one binary node.
template <int ISECT, bool EXT>
NB_D int any4_step(Any4& a, const DevScene& S, const SmemStack& st, uint32_t* status) {
    const int cap = S.stack_cap4;
    const uint32_t cur = a.next;
    a.next = kWNone;
    if (!(cur & kWRef)) {
        const DevNode4* nd = S.nodes4 + cur;
        const uint4 meta = __ldg(&nd->meta);
        if (meta.x & kW4World) {
            a.lr = a.wr;
            a.ldeg = a.wdeg;
            if (ISECT == NOOR_ISECT_WATERTIGHT && !a.wtw) {
                wt_setup(a.wt, a.wr.d);
                a.wtw = true;
            }
        }
        if (!wide_visit(nd, meta, a.lr, a.tmax, st, cap, a.top, a.next, status)) return kAnyFailed;
    } else {
        const uint32_t ni = cur & kWIndex;
        const DevNode* nd = S.nodes + ni;
        const uint4 lo = __ldg(&nd->lo);
        const uint4 hi = __ldg(&nd->hi);
        if (hi.w & NOOR_MESH_NODE_MASK) {
            a.lr = a.wr;
            a.ldeg = a.wdeg;
            if (ISECT == NOOR_ISECT_WATERTIGHT && !a.wtw) {
                wt_setup(a.wt, a.wr.d);
                a.wtw = true;
            }
        }
        if (!(cur & kWUntested) || slab_hit(a.lr, lo, hi, a.tmax)) {
            if (!(hi.w & kNodeKindMask)) {
                if (!inner_step(S, ni, lo, hi, a.lr, a.ldeg, st, cap, a.top, a.next, status)) return kAnyFailed;
            } else if (hi.w & NOOR_LIGHT_NODE_MASK) {
                const uint32_t li = hi.w & NOOR_LIGHT_MASK;
                float tm = a.tmax;
                if ((int)li < S.num_area_lights &&
                    shape_hit<EXT, ISECT == NOOR_ISECT_REF_WALD>(S.area_lights[li], a.wr.o, a.wr.d, tm))
                    return kAnyHit;
            } else if (hi.w & NOOR_MESH_INSTANCE_MASK) {
                const bool same = enter_instance(a.lr, a.wr, S, hi.w & NOOR_TRANS_MASK, a.plain);
                a.ldeg = same ? a.wdeg : wide_degenerate(a.lr.o, a.lr.d);
                if (ISECT == NOOR_ISECT_WATERTIGHT && !(same && a.wtw)) {
                    wt_setup(a.wt, a.lr.d);
                    a.wtw = same;
                }
                a.next = kWRef | kWUntested | lo.w;
            } else if (hi.w & NOOR_MESH_LEAF_MASK) {
                const uint32_t cnt = hi.w & NOOR_COUNT_MASK;
                if (a.top + (int)cnt > cap + 1) {
                    atomicOr(status, NOOR_DEV_STACK_OVERFLOW);
                    return kAnyFailed;
                }
                for (uint32_t i = 1; i < cnt; ++i) {
                    st.base[a.top * st.stride] = kWRef | kWUntested | (ni + i);
                    ++a.top;
                }
                if (cnt) a.next = kWRef | kWUntested | (ni + cnt);
            } else {
                const uint32_t start = lo.w;
                const uint32_t end = start + (hi.w & NOOR_TRI_COUNT_MASK);
                for (uint32_t ti = start; ti < end; ++ti) {
                    float tm = a.tmax, bu, bv;
                    uint32_t mt;
                    bool h;
                    if (ISECT == NOOR_ISECT_WATERTIGHT)
                        h = wt_test(a.lr, a.wt, S.wtri + ti, tm, bu, bv, mt);
                    else
                        h = wald_test(a.lr, S.wald + ti, tm, bu, bv, mt);
                    if (h && EXT && S.has_alpha && (mt & NOOR_ALPHA) && alpha_cut<ISECT>(S, ti, bu, bv)) h = false;
                    if (h) return kAnyHit;
                }
            }
        }
    }
    if (a.next == kWNone) {
        if (a.top == 0) return kAnyMiss;
        --a.top;
        a.next = st.base[a.top * st.stride];
    }
    return kAnyRunning;
}

template <int ISECT, bool EXT = true>
NB_D bool trace_any4(const DevScene& S, const float3& o, const float3& d, float tmax, const SmemStack& st,
                     uint32_t* status) {
    Any4 a;
    any4_init<ISECT>(a, S, o, d, tmax);
    for (;;) {
        const int r = any4_step<ISECT, EXT>(a, S, st, status);
        if (r != kAnyRunning) return r == kAnyHit;
    }
}

// Closest hit over the four-wide tree: the same hit, to the bit, as
// trace_closest.  Leaves are taken in the binary traversal's order, and
// every binary node (leaf, mesh leaf, instance, light) is slab-tested when it
// is taken, against the hit distance of that moment, as the binary traversal
// tests it; a wide node's tests only skip entries that the binary traversal
// would find missed later (its hit distance only shrinks, and a box inside a
// missed box is missed).  The stack holds S.stack_cap4 words.
template <int ISECT, bool EXT = true>
NB_D bool trace_closest4(const DevScene& S, const float3& o, const float3& d, float& tmax, HitRec& rec,
                         const SmemStack& st, uint32_t* status) {
    TRay wr;
    tray_setup(wr, o, d);
    const bool wdeg = wide_degenerate(o, d);
    TRay lr = wr;
    bool ldeg = wdeg;
    WtRay wt;
    if (ISECT == NOOR_ISECT_WATERTIGHT) wt_setup(wt, lr.d);
    bool wtw = true;  // wt holds the world ray's constants
    const bool plain = ray_plain(o, d);
    float ltmax = tmax;
    uint32_t ins = 0;
    bool hit = false;
    const int cap = S.stack_cap4;
    int top = 0;
    uint32_t next = kWRef | S.root;
    for (;;) {
        const uint32_t cur = next;
        next = kWNone;
        if (!(cur & kWRef)) {
            const DevNode4* nd = S.nodes4 + cur;
            const uint4 meta = __ldg(&nd->meta);
            if (meta.x & kW4World) {
                lr = wr;
                ltmax = tmax;
                ldeg = wdeg;
                if (ISECT == NOOR_ISECT_WATERTIGHT && !wtw) {
                    wt_setup(wt, wr.d);
                    wtw = true;
                }
            }
            if (!wide_visit(nd, meta, lr, ltmax, st, cap, top, next, status)) return hit;
        } else {
            const uint32_t ni = cur & kWIndex;
            const DevNode* nd = S.nodes + ni;
            const uint4 lo = __ldg(&nd->lo);
            const uint4 hi = __ldg(&nd->hi);
            if (hi.w & NOOR_MESH_NODE_MASK) {
                lr = wr;
                ltmax = tmax;
                ldeg = wdeg;
                if (ISECT == NOOR_ISECT_WATERTIGHT && !wtw) {
                    wt_setup(wt, wr.d);
                    wtw = true;
                }
            }
            if (slab_hit(lr, lo, hi, ltmax)) {
                if (!(hi.w & kNodeKindMask)) {
                    if (!inner_step(S, ni, lo, hi, lr, ldeg, st, cap, top, next, status)) return hit;
                } else if (hi.w & NOOR_LIGHT_NODE_MASK) {
                    const uint32_t li = hi.w & NOOR_LIGHT_MASK;
                    if ((int)li < S.num_area_lights &&
                        shape_hit<EXT, ISECT == NOOR_ISECT_REF_WALD>(S.area_lights[li], o, d, tmax)) {
                        hit = true;
                        rec.ins = li;
                        rec.mtype = NOOR_MESHLIGHT | NOOR_EMITTER;
                    }
                } else if (hi.w & NOOR_MESH_INSTANCE_MASK) {
                    ins = hi.w & NOOR_TRANS_MASK;
                    const bool same = enter_instance(lr, wr, S, ins, plain);
                    ltmax = tmax;
                    ldeg = same ? wdeg : wide_degenerate(lr.o, lr.d);
                    if (ISECT == NOOR_ISECT_WATERTIGHT && !(same && wtw)) {
                        wt_setup(wt, lr.d);
                        wtw = same;
                    }
                    next = kWRef | lo.w;
                } else if (hi.w & NOOR_MESH_LEAF_MASK) {
                    const uint32_t cnt = hi.w & NOOR_COUNT_MASK;
                    if (top + (int)cnt > cap + 1) {
                        atomicOr(status, NOOR_DEV_STACK_OVERFLOW);
                        return hit;
                    }
                    for (uint32_t i = 1; i < cnt; ++i) {
                        st.base[top * st.stride] = kWRef | (ni + i);
                        ++top;
                    }
                    if (cnt) next = kWRef | (ni + cnt);
                } else {
                    const uint32_t start = lo.w;
                    const uint32_t end = start + (hi.w & NOOR_TRI_COUNT_MASK);
                    bool leaf_hit = false;
                    for (uint32_t ti = start; ti < end; ++ti) {
                        float bu, bv;
                        uint32_t mt;
                        bool h;
                        if (EXT && S.has_alpha) {
                            float tc = ltmax;
                            if (ISECT == NOOR_ISECT_WATERTIGHT)
                                h = wt_test(lr, wt, S.wtri + ti, tc, bu, bv, mt);
                            else
                                h = wald_test(lr, S.wald + ti, tc, bu, bv, mt);
                            if (h && (mt & NOOR_ALPHA) && alpha_cut<ISECT>(S, ti, bu, bv)) h = false;
                            if (h) ltmax = tc;
                        } else if (ISECT == NOOR_ISECT_WATERTIGHT) {
                            h = wt_test(lr, wt, S.wtri + ti, ltmax, bu, bv, mt);
                        } else {
                            h = wald_test(lr, S.wald + ti, ltmax, bu, bv, mt);
                        }
                        if (h) {
                            leaf_hit = true;
                            rec.u = bu;
                            rec.v = bv;
                            rec.tri = ti;
                            rec.mtype = mt;
                        }
                    }
                    if (leaf_hit) {
                        hit = true;
                        tmax = ltmax;
                        rec.ins = ins;
                    }
                }
            }
        }
        if (next == kWNone) {
            if (top == 0) break;
            --top;
            next = st.base[top * st.stride];
        }
    }
    return hit;
}

// Closest hit on the four-wide tree (WIDE: the kernel is launched only for
// scenes with S.closest4 set) or on the binary one
template <int ISECT, bool EXT, bool WIDE>
NB_D bool trace_primary(const DevScene& S, const float3& o, const float3& d, float& tmax, HitRec& rec,
                        const SmemStack& st, uint32_t* status) {
    if (WIDE) return trace_closest4<ISECT, EXT>(S, o, d, tmax, rec, st, status);
    return trace_closest<ISECT, EXT>(S, o, d, tmax, rec, st, status);
}

// Any hit on the four-wide tree (WIDE: launched only for scenes with
// S.nodes4 set) or on the binary one
template <int ISECT, bool EXT, bool WIDE>
NB_D bool trace_shadow(const DevScene& S, const float3& o, const float3& d, float tmax, const SmemStack& st,
                       uint32_t* status) {
    if (WIDE) return trace_any4<ISECT, EXT>(S, o, d, tmax, st, status);
    return trace_any<ISECT, EXT>(S, o, d, tmax, st, status);
}

}  // namespace nb
