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

// CudaAreaLight::Le (noor/cuda/lightimp.cuh:29-36): a sphere emits on
// both sides, a quad or disk towards -n unless two-sided; w is the
// direction of the ray arriving at the light
template <bool EXT = true>
NB_D float3 area_le(const DevAreaLight& A, const float3& w) {
    if (EXT && A.type == NOOR_SHAPE_SPHERE) return A.ke;
    return (A.two_sided || dot(w, A.n) < 0.0f) ? A.ke : f3(0.0f);
}

template <bool EXT = true>
NB_D bool is_delta_light(const DevScene& S, int li) {
    return EXT && li >= S.num_area_lights && li < S.num_area_lights + S.num_delta_lights;
}

// sampleQuad / sampleSphere / sampleDisk (noor/cuda/geometry.cuh:27-103):
// a point p on the shape (offset by the reflection bias along its normal)
// and the pdf of reaching it from I.p.  For quads and disks that pdf is the
// reference's dist^2 / (|n . w| area) with w = P - p NOT normalised
// (geometry.cuh:37-38, 98-100), i.e. the solid-angle pdf divided by the
// distance: those lights come out brighter by the distance to them.  Kept
// as is, since the point is the reference's image; the MIS pdf of the same
// lights (light_pdf) uses the unit direction, as the reference's does.
NB_D float3 curved_sample(const DevAreaLight& A, float bias, const float3& P, Rng& rng, float& pdf) {
    if (A.type == NOOR_SHAPE_SPHERE) {
        // uniform cone of directions towards the sphere (pbrt's method);
        // the sampled point is rescaled as the reference does (p, not
        // p - center, scaled by radius / |p - center|)
        const float r1 = rng.next();
        const float r2 = rng.next();
        const float3 w = normalize_fast(A.center - P);
        float3 u, v;
        coordinate_system(w, u, v);
        const float sin2max = A.radius2 / length2(P - A.center);
        const float cosmax = sqrtf(fmaxf(0.0f, 1.0f - sin2max));
        const float ct = (1.0f - r1) + r1 * cosmax;
        const float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
        const float phi = r2 * k2Pi;
        const float dc = length3(P - A.center);
        const float ds = dc * ct - sqrtf(fmaxf(0.0f, A.radius2 - dc * dc * st * st));
        const float ca = (dc * dc + A.radius2 - ds * ds) / (2.0f * dc * A.radius);
        const float sa = sqrtf(fmaxf(0.0f, 1.0f - ca * ca));
        const float3 N = sa * cosf(phi) * (-1.0f * u) + sa * sinf(phi) * (-1.0f * v) + ca * (-1.0f * w);
        float3 p = A.center + A.radius * N;
        p *= A.radius / length3(p - A.center);
        p += bias * N;
        pdf = kInv2Pi / (1.0f - cosmax);
        return p;
    }
    const float ux = rng.next();
    const float uy = rng.next();
    const float2 cd = concentric_disk(ux, uy);
    const float px = cd.x * A.radius, py = cd.y * A.radius;
    float3 u, v;
    coordinate_system(A.n, u, v);
    const float3 p = px * u + py * v + 0.0f * A.n + A.center + bias * A.n;
    const float3 w = P - p;
    pdf = length2(w) / (absdot(A.n, -1.0f * w) * A.area);
    if (isinf(pdf)) pdf = 0.0f;
    return p;
}
template <bool EXT = true>
NB_D float3 area_sample(const DevScene& S, const DevAreaLight& A, const float3& P, Rng& rng, float& pdf) {
    if (EXT && A.type != NOOR_SHAPE_QUAD) return curved_sample(A, S.bias, P, rng, pdf);
    const float r1 = rng.next();
    const float r2 = rng.next();
    const float3 p = A.center + A.u * r1 + A.v * r2 + S.bias * A.n;
    const float3 w = P - p;
    pdf = length2(w) / (absdot(A.n, -1.0f * w) * A.area);
    if (isinf(pdf)) pdf = 0.0f;
    return p;
}

// point / spot / distant sample_Li (lightimp.cuh:191-241): pdf 1, or 0
// when the light gives nothing
NB_D float3 delta_sample(const DevDeltaLight& D, float world_radius, const float3& P, float3& to, float3& wi,
                               float& pdf) {
    pdf = 1.0f;
    if (D.kind == kDeltaDistant) {
        to = P + 2.0f * world_radius * D.dir;
        visibility(P, to, wi);
        return D.ke;
    }
    to = D.pos;
    visibility(P, to, wi);
    const float dist2 = length2(to - P);
    if (dist2 == 0.0f) {
        pdf = 0.0f;
        return f3(0.0f);
    }
    if (D.kind != kDeltaSpot) return D.ke / dist2;
    // CudaSpotLight::falloff (light.cuh:198-206)
    const float c = dot(D.dir, wi);
    float fo = 1.0f;
    if (c < D.cos_outer) {
        fo = 0.0f;
    } else if (c < D.cos_inner) {
        const float dl = (c - D.cos_outer) / (D.cos_inner - D.cos_outer);
        fo = (dl * dl) * (dl * dl);
    }
    if (fo == 0.0f) {
        pdf = 0.0f;
        return f3(0.0f);
    }
    return D.ke * fo / dist2;
}

// light pick + sample_Li (noor/cuda/lightimp.cuh:412-453; area 97-108,
// infinite 175-187).  EXT false: quad area lights and the infinite light only
template <bool EXT = true>
NB_D float3 sample_li(const DevScene& S, const Isect& I, Rng& rng, int nl, int li, float3& wi, float3& to,
                      float& pdf) {
    float3 Li = f3(0.0f);
    pdf = 0.0f;
    if (li < S.num_area_lights) {
        const DevAreaLight& A = S.area_lights[li];
        const float3 p = area_sample<EXT>(S, A, I.p, rng, pdf);
        if (pdf == 0.0f) return f3(0.0f);
        to = p;
        visibility(I.p, to, wi);
        Li = area_le<EXT>(A, wi);
    } else if (is_delta_light<EXT>(S, li)) {
        Li = delta_sample(S.delta_lights[li - S.num_area_lights], S.world_radius, I.p, to, wi, pdf);
        if (pdf == 0.0f) return f3(0.0f);
    } else {
        const float3 dir = env_sample_dir<EXT>(S, rng, pdf);
        if (isinf(pdf) || isnan(pdf)) pdf = 0.0f;
        to = I.p + 2.0f * S.world_radius * dir;
        visibility(I.p, to, wi);
        Li = S.sky_on ? env_eval<EXT>(S, wi) : f3(0.0f);
    }
    if (isinf(pdf)) pdf = 0.0f;
    return Li * (float)nl;
}

NB_D float curved_pdf(const DevAreaLight& A, const float3& P, const float3& wi) {
    if (A.type == NOOR_SHAPE_SPHERE) {
        const float sin2max = A.radius2 / length2(P - A.center);
        const float cosmax = sqrtf(fmaxf(0.0f, 1.0f - sin2max));
        return kInv2Pi / (1.0f - cosmax);
    }
    float tm = kInf;
    if (!disk_hit(A, P, wi, tm)) return 0.0f;
    const float3 p = P + tm * wi;
    return length2(p - P) / (absdot(A.n, -1.0f * wi) * A.area);
}

// pdf_Li of light li for direction wi (lightimp.cuh:89-95,161-173;
// shapeimp.cuh:28-52); delta lights are never asked
template <bool EXT = true>
NB_D float light_pdf(const DevScene& S, const Isect& I, int li, const float3& wi) {
    float pdf = 0.0f;
    if (li < S.num_area_lights) {
        const DevAreaLight& A = S.area_lights[li];
        if (EXT && A.type != NOOR_SHAPE_QUAD) {
            pdf = curved_pdf(A, I.p, wi);
        } else {
            float tm = kInf;
            if (!quad_hit(A, I.p, wi, tm)) return 0.0f;
            const float3 p = I.p + tm * wi;
            pdf = length2(p - I.p) / (absdot(A.n, -1.0f * wi) * A.area);
        }
        if (isinf(pdf)) pdf = 0.0f;
    } else if (is_delta_light<EXT>(S, li)) {
        pdf = 0.0f;
    } else {
        pdf = env_pdf<EXT>(S, wi);
    }
    return isinf(pdf) ? 0.0f : pdf;
}

// The shadow catcher's sky factor: the sky along -toWorld(wo)
// (noor/cuda/bxdf.cuh:213-218, the local wo taken back to world space)
template <bool EXT>
NB_D bool is_catcher(const Isect& I) {
    return EXT && I.lobe == kLobeCatcher;
}
template <bool EXT>
NB_D float3 catcher_sky(const DevScene& S, const Isect& I) {
    return env_eval<EXT>(S, -1.0f * to_world(I.F, to_local(I.F, I.wo)));
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
    const float3 Li = sample_li<EXT>(S, I, rng, nl, li, wi, to, lpdf);
    if (lpdf == 0.0f || is_black(Li)) return f3(0.0f);
    float3 f = bsdf_eval<EXT>(I.lobe, m, I.F, I.wo, wi, kNonSpecular);
    if (is_catcher<EXT>(I)) f *= catcher_sky<EXT>(S, I);
    if (is_black(f)) return f3(0.0f);
    f *= absdot(wi, I.F.n);
    sr.o = spawn_origin(I, wi, S.bias);
    sr.d = wi;
    sr.tmax = length3(sr.o - to);
    // a shadow catcher adds its value wherever the light is unblocked
    // (direct.cuh:51)
    if (is_catcher<EXT>(I)) return f;
    if (!mis || is_delta_light<EXT>(S, li)) return Li * f / lpdf;
    const float spdf = bsdf_pdf<EXT>(I.lobe, m, I.F, I.wo, wi, kNonSpecular);
    const float w = power_heuristic(lpdf, spdf);
    return Li * f * w / lpdf;
}

// sampleBSDF (noor/cuda/direct.cuh:69-110) up to the occlusion test
template <bool EXT = true>
NB_D float3 bsdf_mis_contrib(const DevScene& S, const DevMaterial& m, const Isect& I, Rng& rng, int li,
                             ShadowRay& sr) {
    const uint32_t flags = (I.mtype & kSpecularMat) ? BSDF_ALL : kNonSpecular;
    if (is_delta_light<EXT>(S, li)) return f3(0.0f);  // before any draw (direct.cuh:77)
    if (is_catcher<EXT>(I)) return f3(0.0f);         // directMIS skips it (direct.cuh:129)
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
        const float lp = light_pdf<EXT>(S, I, li, wi);
        if (lp == 0.0f) return f3(0.0f);
        w = power_heuristic(spdf, lp);
    }
    const float3 so = spawn_origin(I, wi, S.bias);
    float tm = 2.0f * S.world_radius;
    bool lh;
    float3 Le;
    if (li < S.num_area_lights) {
        const DevAreaLight& A = S.area_lights[li];
        lh = shape_hit<EXT>(A, so, wi, tm);
        Le = area_le<EXT>(A, wi);
    } else {
        lh = S.sky_on != 0;
        Le = S.sky_on ? env_eval<EXT>(S, wi) : f3(0.0f);
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
        if (!trace_closest<ISECT, EXT>(S, o, d, tmax, rec, st, status)) {
            if (S.sky_on && (bounce == 0 || spec_bounce)) L += beta * env_eval<EXT>(S, normalize_fast(d));
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
                    L += beta * area_le<EXT>(S.area_lights[rec.ins], d);
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
            if (trace_any<ISECT, EXT>(S, sr.o, sr.d, sr.tmax, st, status)) Ld = f3(0.0f);
        }
        if (S.mis && picked) {
            float3 c = bsdf_mis_contrib<EXT>(S, m, I, rng, li, sr);
            if (!is_black(c)) {
                rs.shadow++;
                if (trace_any<ISECT, EXT>(S, sr.o, sr.d, sr.tmax, st, status)) c = f3(0.0f);
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
        beta *= (is_catcher<EXT>(I) ? f * catcher_sky<EXT>(S, I) : f) * absdot(wi, I.F.n) / pdf;
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
