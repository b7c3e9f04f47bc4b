// Path integrator of noor/cuda/path_tracer.cu:26-75 with the direct-lighting,
// scattering and Russian-roulette steps of noor/cuda/direct.cuh,
// scatter.cuh and accumulate.cuh.  Random numbers are drawn in the
// reference's order; where C++ leaves the order unspecified
// (make_float2(rng(), rng()), a + u*rng() + v*rng()) the first operand draws
// first.  Deliberate differences, each stated where it is made:
//   * a path whose BSDF sample has pdf 0 ends there (the reference walks on
//     along a zero direction that can add nothing but a NaN, which its final
//     clamp turns into 0);
//   * the BSDF half of MIS runs against the light the light-sampling half
//     picked; when no light was picked (specular material or no light) it
//     adds nothing and draws nothing (the reference reads an uninitialised
//     index there);
//   * shadow rays whose contribution is already zero are not traced.
#pragma once
#include "shading.cuh"

namespace nb {

struct Isect {
    float3 p;
    float3 wo;
    Frame F;
    uint32_t mtype;
    uint32_t lobe;
    uint32_t mat;
};

struct RayStats {
    uint32_t ext;
    uint32_t shadow;
};

constexpr uint32_t kNonSpecular = BSDF_ALL & ~BSDF_SPECULAR;

NB_D float3 spawn_origin(const Isect& I, const float3& dir, float bias) {
    return dot(dir, I.F.ng) >= 0.0f ? I.p + bias * I.F.ng : I.p - bias * I.F.ng;
}

// Visibility(from, to) of noor/cuda/intersection.cuh:27-44
NB_D void visibility(const float3& from, const float3& to, float3& wi) {
    const float3 v = to - from;
    const float dist = length3(v);
    wi = v / dist;
}

// light pick + sample_Li (noor/cuda/lightimp.cuh:412-453, 97-108, 175-187)
NB_D float3 sample_li(const DevScene& S, const Isect& I, Rng& rng, int nl, int li, float3& wi, float3& to,
                      float& pdf) {
    float3 Li = f3(0.0f);
    pdf = 0.0f;
    if (li < S.num_area_lights) {
        const DevAreaLight& A = S.area_lights[li];
        const float r1 = rng.next();
        const float r2 = rng.next();
        const float3 p = A.center + A.u * r1 + A.v * r2 + S.bias * A.n;
        const float3 w = I.p - p;
        const float dist2 = length2(w);
        pdf = dist2 / (absdot(A.n, -1.0f * w) * A.area);
        if (isinf(pdf)) pdf = 0.0f;
        if (pdf == 0.0f) return f3(0.0f);
        to = p;
        visibility(I.p, to, wi);
        Li = (A.two_sided || dot(wi, A.n) < 0.0f) ? A.ke : f3(0.0f);
    } else {
        const float3 dir = env_sample_dir(S, rng, pdf);
        if (isinf(pdf) || isnan(pdf)) pdf = 0.0f;
        to = I.p + 2.0f * S.world_radius * dir;
        visibility(I.p, to, wi);
        Li = S.sky_on ? env_eval(S, wi) : f3(0.0f);
    }
    if (isinf(pdf)) pdf = 0.0f;
    return Li * (float)nl;
}

// pdf_Li of light li for direction wi (lightimp.cuh:89-95,161-173; shapeimp.cuh:28-52)
NB_D float light_pdf(const DevScene& S, const Isect& I, int li, const float3& wi) {
    float pdf = 0.0f;
    if (li < S.num_area_lights) {
        const DevAreaLight& A = S.area_lights[li];
        float tm = kInf;
        if (!quad_hit(A, I.p, wi, tm)) return 0.0f;
        const float3 p = I.p + tm * wi;
        pdf = length2(p - I.p) / (absdot(A.n, -1.0f * wi) * A.area);
        if (isinf(pdf)) pdf = 0.0f;
    } else {
        pdf = env_pdf(S, wi);
    }
    return isinf(pdf) ? 0.0f : pdf;
}

// A shadow ray whose contribution counts only if nothing blocks it.
struct ShadowRay {
    float3 o;
    float3 d;
    float tmax;
};

// sampleLight (noor/cuda/direct.cuh:32-67) up to the occlusion test: returns
// the contribution it adds when the shadow ray `sr` is unblocked (zero, with
// no ray needed, on every early exit).  The MIS weight is applied here; the
// reference evaluates it after the occlusion test, which draws no random
// numbers, so the order does not change the result.
template <bool EXT = true>
NB_D float3 light_sample_contrib(const DevScene& S, const DevMaterial& m, const Isect& I, Rng& rng, bool mis,
                                 int& light_idx, bool& picked, ShadowRay& sr) {
    picked = false;
    if (I.mtype & kSpecularMat) return f3(0.0f);
    const int nl = S.sky_on ? S.num_lights : S.num_lights - 1;
    if (nl == 0) return f3(0.0f);
    const int li = (int)((float)nl * rng.next());
    light_idx = li;
    picked = true;
    float3 wi, to;
    float lpdf;
    const float3 Li = sample_li(S, I, rng, nl, li, wi, to, lpdf);
    if (lpdf == 0.0f || is_black(Li)) return f3(0.0f);
    float3 f = bsdf_eval<EXT>(I.lobe, m, I.F, I.wo, wi, kNonSpecular);
    if (is_black(f)) return f3(0.0f);
    f *= absdot(wi, I.F.n);
    sr.o = spawn_origin(I, wi, S.bias);
    sr.d = wi;
    sr.tmax = length3(sr.o - to);
    if (!mis) return Li * f / lpdf;
    const float spdf = bsdf_pdf<EXT>(I.lobe, m, I.F, I.wo, wi, kNonSpecular);
    const float w = power_heuristic(lpdf, spdf);
    return Li * f * w / lpdf;
}

// sampleBSDF (noor/cuda/direct.cuh:69-110) up to the occlusion test
template <bool EXT = true>
NB_D float3 bsdf_mis_contrib(const DevScene& S, const DevMaterial& m, const Isect& I, Rng& rng, int li,
                             ShadowRay& sr) {
    const uint32_t flags = (I.mtype & kSpecularMat) ? BSDF_ALL : kNonSpecular;
    rng.next();  // two draws the reference makes and never reads (direct.cuh:79)
    rng.next();
    float3 wi;
    float spdf;
    uint32_t stype;
    float3 f = bsdf_sample<EXT>(I.lobe, m, I.F, I.wo, flags, rng, wi, spdf, stype);
    if (is_black(f) || spdf == 0.0f) return f3(0.0f);
    f *= absdot(wi, I.F.n);
    float w = 1.0f;
    if (!(stype & BSDF_SPECULAR)) {
        const float lp = light_pdf(S, I, li, wi);
        if (lp == 0.0f) return f3(0.0f);
        w = power_heuristic(spdf, lp);
    }
    const float3 so = spawn_origin(I, wi, S.bias);
    float tm = 2.0f * S.world_radius;
    bool lh;
    float3 Le;
    if (li < S.num_area_lights) {
        const DevAreaLight& A = S.area_lights[li];
        lh = quad_hit(A, so, wi, tm);
        Le = (A.two_sided || dot(wi, A.n) < 0.0f) ? A.ke : f3(0.0f);
    } else {
        lh = S.sky_on != 0;
        Le = S.sky_on ? env_eval(S, wi) : f3(0.0f);
    }
    if (!lh) return f3(0.0f);
    const float3 c = Le * f * w / spdf;
    if (is_black(c)) return f3(0.0f);
    const float3 to = so + tm * wi;
    float3 vwi;
    visibility(I.p, to, vwi);
    sr.o = spawn_origin(I, vwi, S.bias);
    sr.d = vwi;
    sr.tmax = length3(sr.o - to);
    return c;
}

// Builds the hit record of CudaIntersection (intersection.cuh:319-377).
template <int ISECT, bool EXT = true>
NB_D void make_isect(const DevScene& S, const float3& o, const float3& d, float t, const HitRec& rec, Isect& I) {
    I.p = o + t * d;
    I.wo = normalize_fast(-1.0f * d);
    I.mtype = rec.mtype;
    I.lobe = lobe_of<EXT>(rec.mtype);
    if (ISECT == NOOR_ISECT_WATERTIGHT) {
        const DevWtTri* T = S.wtri + rec.tri;
        const uint4 attr = __ldg(&T->attr);
        I.mat = attr.w;
        if (rec.mtype & kEmitterMat) return;
        float4 vv[3];
        vv[0] = __ldg(&T->v0);
        vv[1] = __ldg(&T->v1);
        vv[2] = __ldg(&T->v2);
        I.F = tangent_frame(S, attr, rec.ins, rec.u, rec.v, vv);
    } else {
        const uint4 attr = __ldg(&S.wald[rec.tri].attr);
        I.mat = attr.w;
        if (rec.mtype & kEmitterMat) return;
        I.F = tangent_frame(S, attr, rec.ins, rec.u, rec.v, nullptr);
    }
}

// pathtracer() of noor/cuda/path_tracer.cu:26-75; returns clamp(L, 0, 100)
// EXT false: the specialisation for scenes whose materials use only the
// Lambert, conductor and Fresnel-specular lobes
template <int ISECT, bool EXT = true>
NB_D float3 path_radiance(const DevScene& S, float3 o, float3 d, Rng& rng, const SmemStack& st, uint32_t* status,
                          RayStats& rs, float3* first_hit, bool* first_hit_valid) {
    float3 L = f3(0.0f);
    float3 beta = f3(1.0f);
    bool spec_bounce = false;
    for (uint32_t bounce = 0; bounce < S.bounces; ++bounce) {
        float tmax = kInf;
        HitRec rec;
        rs.ext++;
        if (!trace_closest<ISECT>(S, o, d, tmax, rec, st, status)) {
            if (S.sky_on && (bounce == 0 || spec_bounce)) L += beta * env_eval(S, normalize_fast(d));
            break;
        }
        Isect I;
        make_isect<ISECT, EXT>(S, o, d, tmax, rec, I);
        if (bounce == 0 && first_hit) {
            *first_hit = I.p;
            *first_hit_valid = true;
        }
        if (I.mtype & kEmitterMat) {
            if (bounce == 0 || spec_bounce) {
                if (I.mtype & NOOR_MESHLIGHT) {
                    const DevAreaLight& A = S.area_lights[rec.ins];
                    L += beta * ((A.two_sided || dot(d, A.n) < 0.0f) ? A.ke : f3(0.0f));
                } else {
                    const DevMaterial& em = S.materials[I.mat];
                    L += beta * (em.emitter_scale * em.emittance);
                }
            }
            // an emitter has no BSDF lobe: nothing more can be added
            break;
        }
        const DevMaterial m = S.materials[I.mat];
        // accumulate (accumulate.cuh:83-99): direct lighting, then scatter
        int li = 0;
        bool picked;
        ShadowRay sr;
        float3 Ld = light_sample_contrib<EXT>(S, m, I, rng, S.mis != 0, li, picked, sr);
        if (!is_black(Ld)) {
            rs.shadow++;
            if (trace_any<ISECT>(S, sr.o, sr.d, sr.tmax, st, status)) Ld = f3(0.0f);
        }
        if (S.mis && picked) {
            float3 c = bsdf_mis_contrib<EXT>(S, m, I, rng, li, sr);
            if (!is_black(c)) {
                rs.shadow++;
                if (trace_any<ISECT>(S, sr.o, sr.d, sr.tmax, st, status)) c = f3(0.0f);
            }
            Ld += c;
        }
        L += beta * Ld;
        // scatter (scatter.cuh:27-41)
        rng.next();  // two draws the reference makes and never reads (scatter.cuh:34)
        rng.next();
        float3 wi;
        float pdf;
        uint32_t stype;
        const float3 f = bsdf_sample<EXT>(I.lobe, m, I.F, I.wo, BSDF_ALL, rng, wi, pdf, stype);
        if (pdf == 0.0f) break;
        beta *= f * absdot(wi, I.F.n) / pdf;
        // correct_sidedness (accumulate.cuh:40-45)
        if (!(I.mtype & kTransparentMat) && dot(wi, I.F.ng) < 0.0f) break;
        // rr_terminate (accumulate.cuh:27-38)
        if (bounce >= S.rr) {
            const float q = fmaxf(0.05f, 1.0f - maxcomp(beta));
            if (rng.next() < q) break;
            beta /= 1.0f - q;
        }
        spec_bounce = (I.mtype & kSpecularMat) != 0;
        o = spawn_origin(I, wi, S.bias);
        d = wi;
    }
    return clamp3(L, 0.0f, 100.0f);
}

}  // namespace nb
