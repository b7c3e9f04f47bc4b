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
    float2 uv;      // the hit's texture coordinates (barycentrics on emitters); set where textures are read
};

// material types whose scattered ray keeps differentials
// (CudaIntersection::isGlossy, NOOR_GLOSSY of path_tracer.cuh:121-124)
constexpr uint32_t kGlossyMat =
    NOOR_MIRROR | NOOR_GLASS | NOOR_CLEARCOAT | NOOR_ROUGHGLASS | NOOR_METAL | NOOR_SUBSTRATE | NOOR_GLOSSY;
// material types with a dielectric Fresnel lobe, which set the intersection's
// eta (CudaBxDF::factoryFresnel, bxdf.cuh:190-200)
constexpr uint32_t kDielectricMat = NOOR_GLASS | NOOR_ROUGHGLASS | NOOR_GLOSSY | NOOR_SUBSTRATE | NOOR_CLEARCOAT;

// the texture-read slots of a material at uv (materialimp.cuh:121-183):
// colours and roughness replace the load-time constants
NB_D void apply_textures(const DevScene& S, uint32_t mi, float2 uv, DevMaterial& m) {
    const DevMatTex& T = S.mat_tex[mi];
    const uint32_t k = m.tex_mask;
    if (k & (1u << kTexDiffuse)) m.diffuse = f3(slot_tex(T, kTexDiffuse, uv));
    if (k & (1u << kTexSpecular)) m.specular = f3(slot_tex(T, kTexSpecular, uv));
    if (k & (1u << kTexEmittance)) m.emittance = f3(slot_tex(T, kTexEmittance, uv));
    if (k & (1u << kTexTransmission)) m.transmission = f3(slot_tex(T, kTexTransmission, uv));
    if (k & (1u << kTexIor)) m.ior = f3(slot_tex(T, kTexIor, uv));
    if (k & (1u << kTexK)) m.k = f3(slot_tex(T, kTexK, uv));
    if (k & (1u << kTexRoughness)) {
        const float4 r = slot_tex(T, kTexRoughness, uv);
        m.rough_x = r.x;
        m.rough_y = r.y;
    }
}

// The hit's differentials (CudaIntersection::computeDifferential,
// intersection.cuh:397-441): where the offset rays meet the tangent plane,
// and the uv steps solving dp = dpdu du + dpdv dv on the two largest axes of
// the geometric normal.  All zero where an offset ray misses the plane.
struct HitDiff {
    float3 dpdx, dpdy, dndu, dndv;
    float dudx, dudy, dvdx, dvdy;
};
NB_D void solve2x2(float a00, float a01, float a10, float a11, float b0, float b1, float& x0, float& x1) {
    const float det = a00 * a11 - a10 * a01;
    if (fabsf(det) < 1e-10f) {
        x0 = x1 = 0.0f;
        return;
    }
    const float inv = 1.0f / det;
    x0 = (a11 * b0 - a01 * b1) * inv;
    x1 = (a00 * b1 - a10 * b0) * inv;
    if (isnan(x0) || isnan(x1)) x0 = x1 = 0.0f;
}
NB_D HitDiff hit_differential(const Isect& I, const TangentOut& to, const RayDiff& rd) {
    HitDiff h;
    h.dndu = to.dndu;
    h.dndv = to.dndv;
    h.dpdx = h.dpdy = f3(0.0f);
    h.dudx = h.dudy = h.dvdx = h.dvdy = 0.0f;
    const float3& n = I.F.ng;
    const float dd = dot(n, I.p);
    const float tx = -(dot(n, rd.odx) - dd) / dot(n, rd.ddx);
    if (isinf(tx) || isnan(tx)) return h;
    const float3 px = rd.odx + tx * rd.ddx;
    const float ty = -(dot(n, rd.ody) - dd) / dot(n, rd.ddy);
    if (isinf(ty) || isnan(ty)) return h;
    const float3 py = rd.ody + ty * rd.ddy;
    h.dpdx = px - I.p;
    h.dpdy = py - I.p;
    int ax, ay;
    if (fabsf(n.x) > fabsf(n.y) && fabsf(n.x) > fabsf(n.z)) {
        ax = 1;
        ay = 2;
    } else if (fabsf(n.y) > fabsf(n.z)) {
        ax = 0;
        ay = 2;
    } else {
        ax = 0;
        ay = 1;
    }
    const float a00 = comp(to.dpdu, ax), a01 = comp(to.dpdv, ax), a10 = comp(to.dpdu, ay), a11 = comp(to.dpdv, ay);
    solve2x2(a00, a01, a10, a11, comp(h.dpdx, ax), comp(h.dpdx, ay), h.dudx, h.dvdx);
    solve2x2(a00, a01, a10, a11, comp(h.dpdy, ax), comp(h.dpdy, ay), h.dudy, h.dvdy);
    return h;
}

// Bump mapping (accumulate.cuh:47-75, after PBRT): the bump map's slopes
// over a uv step of half the pixel's footprint (0.001 where it is zero)
// tilt dp/du and dp/dv along the shading normal; the frame is rebuilt from
// them and the normal turned to the geometric normal's side.
NB_D void bump(const DevScene& S, uint32_t mi, float2 uv, const HitDiff& h, Frame& F) {
    const DevMatTex& T = S.mat_tex[mi];
    float du = 0.5f * (fabsf(h.dudx) + fabsf(h.dudy));
    float dv = 0.5f * (fabsf(h.dvdx) + fabsf(h.dvdy));
    du = du == 0.0f ? 0.001f : du;
    dv = dv == 0.0f ? 0.001f : dv;
    const float disp = slot_tex(T, kTexBump, uv).x;
    const float scale = T.bumpfactor;
    const float ud = scale * (slot_tex(T, kTexBump, f2(uv.x + du, uv.y + 0.0f)).x - disp) / du;
    const float vd = scale * (slot_tex(T, kTexBump, f2(uv.x + 0.0f, uv.y + dv)).x - disp) / dv;
    const float3 sn = F.n;
    float3 dpdu = F.s + ud * sn;
    const float3 dpdv = F.t + vd * sn;
    float3 n = normalize_guard(cross(dpdu, dpdv));
    dpdu = normalize_guard(dpdu - n * dot(n, dpdu));
    F.t = normalize_guard(cross(n, dpdu));
    F.s = dpdu;
    F.n = dot(F.ng, n) < 0.0f ? -1.0f * n : n;   // NOOR::faceforward
}

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

// The differentials of the scattered ray (CudaIntersection::spawnRay,
// intersection.cuh:111-186): mirror or refraction offsets from the normal's
// derivatives, pulled a quarter of the way back to the ray itself.  `o` is
// the scattered ray's origin; eta the intersection's (1 unless a
// dielectric lobe set it).
NB_D RayDiff spawn_diff(const Isect& I, const HitDiff& h, const RayDiff& in, const float3& o, const float3& wi,
                        float eta_in) {
    RayDiff r;
    r.on = true;
    r.odx = o + h.dpdx;
    r.ody = o + h.dpdy;
    const float3& sn = I.F.n;
    const float3& wo = I.wo;
    const float3 dwodx = -1.0f * (in.ddx + wo);
    const float3 dwody = -1.0f * (in.ddy + wo);
    if (dot(wi, I.F.ng) >= 0.0f) {
        const float3 dndx = h.dndu * h.dudx + h.dndv * h.dvdx;
        const float3 dndy = h.dndu * h.dudy + h.dndv * h.dvdy;
        const float dDNdx = dot(dwodx, sn) + dot(wo, dndx);
        const float dDNdy = dot(dwody, sn) + dot(wo, dndy);
        r.ddx = wi - dwodx + 2.0f * (dot(wo, sn) * dndx + dDNdx * sn);
        r.ddy = wi - dwody + 2.0f * (dot(wo, sn) * dndy + dDNdy * sn);
    } else {
        const float3 w = -1.0f * wo;
        const float eta = dot(wo, sn) > 0.0f ? 1.0f / eta_in : eta_in;
        const float3 dndx = h.dndu * h.dudx + h.dndv * h.dvdx;
        // the reference's dn/dy pairs dn/dv with both du/dy and dv/dy
        const float3 dndy = h.dndv * h.dudy + h.dndv * h.dvdy;
        const float dDNdx = dot(dwodx, sn) + dot(wo, dndx);
        const float dDNdy = dot(dwody, sn) + dot(wo, dndy);
        const float mu = eta * dot(w, sn) - dot(wi, sn);
        const float dmudx = (eta - (eta * eta * dot(w, sn)) / dot(wi, sn)) * dDNdx;
        const float dmudy = (eta - (eta * eta * dot(w, sn)) / dot(wi, sn)) * dDNdy;
        r.ddx = wi + eta * dwodx - (mu * dndx + dmudx * sn);
        r.ddy = wi + eta * dwody - (mu * dndy + dmudy * sn);
    }
    // scaleDifferentials(.25f) (ray.cuh:182-189)
    const float s = 0.25f;
    r.odx = (1.0f - s) * o + s * r.odx;
    r.ody = (1.0f - s) * o + s * r.ody;
    r.ddx = (1.0f - s) * wi + s * r.ddx;
    r.ddy = (1.0f - s) * wi + s * r.ddy;
    return r;
}

// Builds the hit record of CudaIntersection (intersection.cuh:319-377).
// With `to`, also the texture coordinates and derivatives of TangentOut
// (I.uv: the barycentrics on an emitter, whose record stops before them).
template <int ISECT, bool EXT = true>
NB_D void make_isect(const DevScene& S, const float3& o, const float3& d, float t, const HitRec& rec, Isect& I,
                     TangentOut* to = nullptr) {
    I.p = o + t * d;
    I.wo = normalize_fast(-1.0f * d);
    I.mtype = rec.mtype;
    I.lobe = lobe_of<EXT>(rec.mtype);
    if (to) I.uv = f2(rec.u, rec.v);
    if (ISECT == NOOR_ISECT_WATERTIGHT) {
        const DevWtTri* T = S.wtri + rec.tri;
        const uint4 attr = __ldg(&T->attr);
        I.mat = attr.w;
        if (rec.mtype & kEmitterMat) return;
        float4 vv[3];
        vv[0] = __ldg(&T->v0);
        vv[1] = __ldg(&T->v1);
        vv[2] = __ldg(&T->v2);
        I.F = tangent_frame(S, attr, rec.ins, rec.u, rec.v, vv, to);
    } else {
        const uint4 attr = __ldg(&S.wald[rec.tri].attr);
        I.mat = attr.w;
        if (rec.mtype & kEmitterMat) return;
        I.F = tangent_frame(S, attr, rec.ins, rec.u, rec.v, nullptr, to);
    }
    if (to) I.uv = to->uv;
}

// pathtracer() of noor/cuda/path_tracer.cu:26-75; returns clamp(L, 0, 100)
// EXT false: the specialisation for scenes whose materials use only the
// Lambert, conductor and Fresnel-specular lobes
// DIFF: the specialisation for scenes with bump maps, whose rays carry
// differentials (rd: the camera ray's) -- the reference bumps only where a
// differential ray arrives (accumulate.cuh:90-92)
template <int ISECT, bool EXT = true, bool DIFF = false>
NB_D float3 path_radiance(const DevScene& S, float3 o, float3 d, Rng& rng, const SmemStack& st, uint32_t* status,
                          RayStats& rs, float3* first_hit, bool* first_hit_valid, RayDiff rd = RayDiff{}) {
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
        TangentOut to;
        const bool tex = EXT && S.has_tex;
        make_isect<ISECT, EXT>(S, o, d, tmax, rec, I, tex ? &to : nullptr);
        if (bounce == 0 && first_hit) {
            *first_hit = I.p;
            *first_hit_valid = true;
        }
        if (I.mtype & kEmitterMat) {
            if (bounce == 0 || spec_bounce) {
                if (I.mtype & NOOR_MESHLIGHT) {
                    L += beta * area_le<EXT>(S.area_lights[rec.ins], d);
                } else {
                    DevMaterial em = S.materials[I.mat];
                    if (tex && em.tex_mask) apply_textures(S, I.mat, I.uv, em);
                    L += beta * (em.emitter_scale * em.emittance);
                }
            }
            // an emitter has no BSDF lobe: nothing more can be added
            break;
        }
        DevMaterial m = S.materials[I.mat];
        HitDiff hd;
        if (DIFF && rd.on) {
            hd = hit_differential(I, to, rd);
            if (I.mtype & NOOR_BUMP) bump(S, I.mat, I.uv, hd, I.F);
        }
        if (tex && m.tex_mask) apply_textures(S, I.mat, I.uv, m);
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
        if (DIFF) {
            if (rd.on && (I.mtype & kGlossyMat))
                rd = spawn_diff(I, hd, rd, o, wi, (I.mtype & kDielectricMat) ? m.coat_ior : 1.0f);
            else
                rd.on = false;
        }
        d = wi;
    }
    return clamp3(L, 0.0f, 100.0f);
}

}  // namespace nb
