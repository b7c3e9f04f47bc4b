// Device shading routines of the render path: RNG, camera, local shading
// frame, BxDF lobes, Fresnel, microfacet distributions, Hosek-Wilkie sky,
// environment texture and its piecewise-constant 2D distribution.
// Each routine states the reference routine it follows.
#pragma once
#include "traverse.cuh"

namespace nb {

constexpr float kInf = __builtin_huge_valf();

// ------------------------------------------------------------------- RNG
// TEA<16> seed of (pixel, frame) and the 24-bit LCG of noor/cuda/rng.cuh:37-76
NB_HD uint32_t tea16(uint32_t v0, uint32_t v1) {
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
    NB_HD float next() {
        s = 1664525u * s + 1013904223u;
        return (float)(s & 0x00FFFFFFu) / (float)0x01000000;
    }
};

// ---------------------------------------------------------------- camera
// CudaPerspCamera::generateRay (noor/cuda/cameraimp.cuh:182-228), pinhole
NB_D float2 concentric_disk(float ux, float uy);

// EXT false: a kernel for pinhole cameras only
template <bool EXT = true>
NB_D void camera_ray(const DevCamera& C, uint32_t x, uint32_t y, Rng& rng, float3& o, float3& d) {
    const float rx = (float)x + rng.next() - 0.5f;
    const float ry = (float)y + rng.next() - 0.5f;
    float3 dc, oc = f3(0.0f);
    bool at_origin = true;
    if (EXT && C.type == NOOR_CAMERA_ENV) {
        // CudaEnvCamera::genDir (cameraimp.cuh:54-60): sphericalDirection
        // (utils.cuh:457-468, right-handed: y up), normalised twice
        const float theta = kPi * ry / (float)C.h + kPi;
        const float phi = k2Pi * rx / (float)C.w - kPiOver2;
        const float st = sinf(theta), ct = cosf(theta);
        dc = normalize_fast(normalize_fast(f3(st * cosf(phi), ct, st * sinf(phi))));
    } else {
        const float3 pc = f3(C.r2c[0].w + (C.r2c[0].x * rx + C.r2c[0].y * ry + C.r2c[0].z * 0.0f),
                             C.r2c[1].w + (C.r2c[1].x * rx + C.r2c[1].y * ry + C.r2c[1].z * 0.0f),
                             C.r2c[2].w + (C.r2c[2].x * rx + C.r2c[2].y * ry + C.r2c[2].z * 0.0f));
        if (EXT && C.type == NOOR_CAMERA_ORTHO) {
            // CudaOrthoCamera (cameraimp.cuh:231-252): from the raster point, along -z
            oc = pc;
            dc = f3(0.0f, 0.0f, -1.0f);
            at_origin = false;
        } else {
            dc = normalize_fast(pc);
            if (EXT && C.lens_radius > 0.0f) {
                // thin lens (cameraimp.cuh:191-202): a point on the lens, through
                // the point of the pinhole ray on the plane of focus
                const float u1 = rng.next();
                const float u2 = rng.next();
                const float2 l = concentric_disk(u1, u2);
                const float ft = -C.focal_length / dc.z;
                const float3 pf = f3(0.0f) + ft * dc;
                oc = f3(C.lens_radius * l.x, C.lens_radius * l.y, 0.0f);
                dc = normalize_fast(pf - oc);
                at_origin = false;
            }
        }
    }
    // CudaRay::transform: the origin as a point, the direction as a vector
    if (at_origin)
        o = f3(C.c2w[0].w, C.c2w[1].w, C.c2w[2].w);
    else
        o = f3(C.c2w[0].w + (C.c2w[0].x * oc.x + C.c2w[0].y * oc.y + C.c2w[0].z * oc.z),
               C.c2w[1].w + (C.c2w[1].x * oc.x + C.c2w[1].y * oc.y + C.c2w[1].z * oc.z),
               C.c2w[2].w + (C.c2w[2].x * oc.x + C.c2w[2].y * oc.y + C.c2w[2].z * oc.z));
    const float3 dw = f3(C.c2w[0].x * dc.x + C.c2w[0].y * dc.y + C.c2w[0].z * dc.z,
                         C.c2w[1].x * dc.x + C.c2w[1].y * dc.y + C.c2w[1].z * dc.z,
                         C.c2w[2].x * dc.x + C.c2w[2].y * dc.y + C.c2w[2].z * dc.z);
    d = normalize_fast(dw);
}

// Ray differentials of CudaRay (noor/cuda/ray.cuh:36-200): the offset rays
// one pixel right (dx) and down (dy); world space.
struct RayDiff {
    bool on;
    float3 odx, ody, ddx, ddy;
};

// generateRay with the differentials every camera type gives its ray
// (cameraimp.cuh:71-89, 183-228, 236-252), then CudaRay::transform
// (ray.cuh:160-174): the origins as points, the directions as vectors (the
// offset directions are not renormalised).  Draws the same numbers as
// camera_ray.
NB_D void camera_ray_diff(const DevCamera& C, uint32_t x, uint32_t y, Rng& rng, float3& o, float3& d, RayDiff& rd) {
    const float rx = (float)x + rng.next() - 0.5f;
    const float ry = (float)y + rng.next() - 0.5f;
    float3 dc, oc = f3(0.0f), odx = f3(0.0f), ody = f3(0.0f), ddx, ddy;
    const float3 dxc = f3(C.r2c[0].x, C.r2c[1].x, C.r2c[2].x);   // _dxCamera
    const float3 dyc = f3(C.r2c[0].y, C.r2c[1].y, C.r2c[2].y);   // _dyCamera
    auto env_dir = [&](float px, float py) {
        const float theta = kPi * py / (float)C.h + kPi;
        const float phi = k2Pi * px / (float)C.w - kPiOver2;
        const float st = sinf(theta), ct = cosf(theta);
        return normalize_fast(normalize_fast(f3(st * cosf(phi), ct, st * sinf(phi))));
    };
    if (C.type == NOOR_CAMERA_ENV) {
        dc = env_dir(rx, ry);
        ddx = env_dir(rx + 1.0f, ry);
        ddy = env_dir(rx, ry + 1.0f);
    } else {
        const float3 pc = f3(C.r2c[0].w + (C.r2c[0].x * rx + C.r2c[0].y * ry + C.r2c[0].z * 0.0f),
                             C.r2c[1].w + (C.r2c[1].x * rx + C.r2c[1].y * ry + C.r2c[1].z * 0.0f),
                             C.r2c[2].w + (C.r2c[2].x * rx + C.r2c[2].y * ry + C.r2c[2].z * 0.0f));
        if (C.type == NOOR_CAMERA_ORTHO) {
            oc = pc;
            dc = f3(0.0f, 0.0f, -1.0f);
            odx = oc + dxc;
            ody = oc + dyc;
            ddx = ddy = dc;
        } else {
            dc = normalize_fast(pc);
            if (C.lens_radius > 0.0f) {
                const float u1 = rng.next();
                const float u2 = rng.next();
                const float2 l = concentric_disk(u1, u2);
                const float2 pl = f2(C.lens_radius * l.x, C.lens_radius * l.y);
                float ft = -C.focal_length / dc.z;
                const float3 pf = f3(0.0f) + ft * dc;
                oc = f3(pl.x, pl.y, 0.0f);
                dc = normalize_fast(pf - oc);
                const float3 dx = normalize_fast(pc + dxc);
                ft = -C.focal_length / dx.z;
                odx = f3(pl.x, pl.y, 0.0f);
                ddx = normalize_fast(f3(0.0f) + ft * dx - odx);
                const float3 dy = normalize_fast(pc + dyc);
                ft = -C.focal_length / dy.z;
                ody = f3(pl.x, pl.y, 0.0f);
                ddy = normalize_fast(f3(0.0f) + ft * dy - ody);
            } else {
                ddx = normalize_fast(pc + dxc);
                ddy = normalize_fast(pc + dyc);
            }
        }
    }
    auto point = [&](const float3& p) {
        return f3(C.c2w[0].w + (C.c2w[0].x * p.x + C.c2w[0].y * p.y + C.c2w[0].z * p.z),
                  C.c2w[1].w + (C.c2w[1].x * p.x + C.c2w[1].y * p.y + C.c2w[1].z * p.z),
                  C.c2w[2].w + (C.c2w[2].x * p.x + C.c2w[2].y * p.y + C.c2w[2].z * p.z));
    };
    auto vec = [&](const float3& v) {
        return f3(C.c2w[0].x * v.x + C.c2w[0].y * v.y + C.c2w[0].z * v.z,
                  C.c2w[1].x * v.x + C.c2w[1].y * v.y + C.c2w[1].z * v.z,
                  C.c2w[2].x * v.x + C.c2w[2].y * v.y + C.c2w[2].z * v.z);
    };
    o = point(oc);
    d = normalize_fast(vec(dc));
    rd.on = true;
    rd.odx = point(odx);
    rd.ody = point(ody);
    rd.ddx = vec(ddx);
    rd.ddy = vec(ddy);
}

// ------------------------------------------------------------ utilities
NB_D float rgb2y(const float3& c) { return dot(c, f3(0.2126f, 0.7152f, 0.0722f)); }
NB_D float power_heuristic(float f, float g) { return (f * f) / (f * f + g * g); }
NB_D bool isinf_f(float v) { return isinf(v); }

// coordinateSystem, noor/cuda/utils.cuh:340-347
NB_D void coordinate_system(const float3& v1, float3& v2, float3& v3) {
    if (fabsf(v1.x) > fabsf(v1.y))
        v2 = f3(-v1.z, 0.0f, v1.x) / sqrtf(v1.x * v1.x + v1.z * v1.z);
    else
        v2 = f3(0.0f, v1.z, -v1.y) / sqrtf(v1.y * v1.y + v1.z * v1.z);
    v3 = cross(v1, v2);
}

// concentricSampleDisk / cosineSampleHemisphere (utils.cuh:377-404)
NB_D float2 concentric_disk(float ux, float uy) {
    const float ox = 2.0f * ux - 1.0f, oy = 2.0f * uy - 1.0f;
    if (ox == 0.0f && oy == 0.0f) return f2(0.0f, 0.0f);
    float theta, r;
    if (fabsf(ox) > fabsf(oy)) {
        r = ox;
        theta = kPiOver4 * (oy / ox);
    } else {
        r = oy;
        theta = kPiOver2 - kPiOver4 * (ox / oy);
    }
    return f2(r * cosf(theta), r * sinf(theta));
}
NB_D float3 cosine_hemisphere(float ux, float uy) {
    const float2 d = concentric_disk(ux, uy);
    const float z = sqrtf(fmaxf(0.0f, 1.0f - d.x * d.x - d.y * d.y));
    return f3(d.x, d.y, z);
}

// uniformSampleHemisphere, left handed (utils.cuh:364-372): z = u.x
NB_D float3 uniform_hemisphere(float ux, float uy) {
    const float z = ux;
    const float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
    const float phi = 2.0f * kPi * uy;
    return f3(r * cosf(phi), r * sinf(phi), z);
}

NB_D float spherical_phi(const float3& v) {
    const float p = atan2f(v.z, v.x);
    return (p < 0.0f) ? (p + k2Pi) : p;
}
NB_D float spherical_theta(const float3& v) { return acosf(clampf(v.y, -1.0f, 1.0f)); }
// sphericalDirection(u, sinTheta) (utils.cuh:470-476): phi = 2 pi u.x,
// theta = pi u.y, y up, normalised
NB_D float3 spherical_direction(float ux, float uy, float& sin_theta) {
    const float phi = ux * k2Pi;
    const float theta = uy * kPi;
    const float ct = cosf(theta);
    sin_theta = sinf(theta);
    return normalize_fast(f3(sin_theta * cosf(phi), ct, sin_theta * sinf(phi)));
}

// ----------------------------------------------------------- shading frame
struct Frame {
    float3 n;   // shading normal
    float3 s;   // dpdu after Gram-Schmidt
    float3 t;   // dpdv
    float3 ng;  // geometric normal
};
NB_D float3 to_local(const Frame& F, const float3& v) { return f3(dot(v, F.s), dot(v, F.t), dot(v, F.n)); }
NB_D float3 to_world(const Frame& F, const float3& v) { return v.x * F.s + v.y * F.t + v.z * F.n; }

// What computeTangentSpace also derives for textures and ray differentials:
// the interpolated texture coordinates, dp/du and dp/dv before the frame's
// Gram-Schmidt step, and the normal's derivatives dn/du, dn/dv
// (intersection.cuh:345-394).
struct TangentOut {
    float2 uv;
    float3 dpdu, dpdv;
    float3 dndu, dndv;
};

// CudaIntersection::computeTangentSpace (noor/cuda/intersection.cuh:325-394);
// with `out` also the uv and the derivatives above.
NB_D Frame tangent_frame(const DevScene& S, const uint4& attr, uint32_t ins, float bu, float bv,
                         const float4* tri_verts /* 3 object-space vertices or null */,
                         TangentOut* out = nullptr) {
    const DevXform* X = S.xforms + ins;
    float2 uv0 = __ldg(&S.uvs[attr.x]), uv1 = __ldg(&S.uvs[attr.y]), uv2 = __ldg(&S.uvs[attr.z]);
    uv0.y = 1.0f - uv0.y;
    uv1.y = 1.0f - uv1.y;
    uv2.y = 1.0f - uv2.y;
    float3 v0, v1, v2;
    if (tri_verts) {
        v0 = f3(tri_verts[0]);
        v1 = f3(tri_verts[1]);
        v2 = f3(tri_verts[2]);
    } else {
        v0 = f3(__ldg(&S.vertices[attr.x]));
        v1 = f3(__ldg(&S.vertices[attr.y]));
        v2 = f3(__ldg(&S.vertices[attr.z]));
    }
    const float3 n0 = f3(__ldg(&S.normals[attr.x]));
    const float3 n1 = f3(__ldg(&S.normals[attr.y]));
    const float3 n2 = f3(__ldg(&S.normals[attr.z]));
    const float4 N0 = __ldg(&X->nrm[0]), N1 = __ldg(&X->nrm[1]), N2 = __ldg(&X->nrm[2]);
    const float w = 1.0f - bu - bv;
    const float3 ni = w * n0 + bu * n1 + bv * n2;
    const float3 nt = f3(N0.x * ni.x + N0.y * ni.y + N0.z * ni.z, N1.x * ni.x + N1.y * ni.y + N1.z * ni.z,
                         N2.x * ni.x + N2.y * ni.y + N2.z * ni.z);
    Frame F;
    F.n = normalize_guard(normalize_fast(nt));
    const float4 S0 = __ldg(&X->o2w[0]), S1 = __ldg(&X->o2w[1]), S2 = __ldg(&X->o2w[2]);
    const float3 e1 = v1 - v0, e2 = v2 - v0;
    const float3 dp01 = f3(S0.x * e1.x + S0.y * e1.y + S0.z * e1.z, S1.x * e1.x + S1.y * e1.y + S1.z * e1.z,
                           S2.x * e1.x + S2.y * e1.y + S2.z * e1.z);
    const float3 dp02 = f3(S0.x * e2.x + S0.y * e2.y + S0.z * e2.z, S1.x * e2.x + S1.y * e2.y + S1.z * e2.z,
                           S2.x * e2.x + S2.y * e2.y + S2.z * e2.z);
    F.ng = normalize_guard(cross(dp01, dp02));
    const float2 d1 = f2(uv1.x - uv0.x, uv1.y - uv0.y);
    const float2 d2 = f2(uv2.x - uv0.x, uv2.y - uv0.y);
    const float det = d1.x * d2.y - d2.x * d1.y;
    float3 dpdu, dpdv;
    if (!(fabsf(det) < 1e-8f)) {
        const float inv = 1.0f / det;
        const float a00 = d2.y * inv, a01 = -d1.y * inv, a10 = -d2.x * inv, a11 = d1.x * inv;
        dpdu = a00 * dp01 + a01 * dp02;
        dpdv = a10 * dp01 + a11 * dp02;
        if (length2(cross(dpdu, dpdv)) == 0.0f) coordinate_system(F.ng, dpdu, dpdv);
    } else {
        coordinate_system(F.ng, dpdu, dpdv);
    }
    F.s = normalize_guard(dpdu - F.n * dot(F.n, dpdu));
    const float sign = dot(cross(F.n, F.s), dpdv) < 0.0f ? -1.0f : 1.0f;
    F.t = normalize_guard(sign * cross(F.n, F.s));
    if (out) {
        out->uv = lerp_uv(uv0, uv1, uv2, bu, bv);
        out->dpdu = dpdu;
        out->dpdv = dpdv;
        // normal derivatives from the object-space vertex normals
        const float3 dn01 = n1 - n0, dn02 = n2 - n0;
        if (!(fabsf(det) < 1e-8f)) {
            const float inv = 1.0f / det;
            const float a00 = d2.y * inv, a01 = -d1.y * inv, a10 = -d2.x * inv, a11 = d1.x * inv;
            out->dndu = a00 * dn01 + a01 * dn02;
            out->dndv = a10 * dn01 + a11 * dn02;
        } else {
            const float3 c = cross(dn01, dn02);
            const float3 ct = f3(N0.x * c.x + N0.y * c.y + N0.z * c.z, N1.x * c.x + N1.y * c.y + N1.z * c.z,
                                 N2.x * c.x + N2.y * c.y + N2.z * c.z);
            const float3 dn = normalize_guard(normalize_fast(ct));
            if (length2(dn) == 0.0f) {
                out->dndu = out->dndv = f3(0.0f);
            } else {
                coordinate_system(dn, out->dndu, out->dndv);
            }
        }
    }
    return F;
}

// -------------------------------------------------- spherical trig helpers
// (noor/cuda/bxdf.cuh:58-96), on local-frame vectors
NB_D float cos2t(const float3& w) { return w.z * w.z; }
NB_D float sin2t(const float3& w) { return fmaxf(0.0f, 1.0f - cos2t(w)); }
NB_D float sint(const float3& w) { return sqrtf(sin2t(w)); }
NB_D float tant(const float3& w) { return sint(w) / w.z; }
NB_D float tan2t(const float3& w) { return sin2t(w) / cos2t(w); }
NB_D float cosphi(const float3& w) {
    const float s = sint(w);
    return (s == 0.0f) ? 1.0f : clampf(w.x / s, -1.0f, 1.0f);
}
NB_D float sinphi(const float3& w) {
    const float s = sint(w);
    return (s == 0.0f) ? 0.0f : clampf(w.y / s, -1.0f, 1.0f);
}
NB_D float cos2phi(const float3& w) { return cosphi(w) * cosphi(w); }
NB_D float sin2phi(const float3& w) { return sinphi(w) * sinphi(w); }
NB_D bool same_hemi(const float3& a, const float3& b) { return a.z * b.z > 0.0f; }

// ---------------------------------------------------------------- Fresnel
// fresnelDielectric (noor/cuda/fresnel.cuh:58-80).  Every operation rounds
// on its own (no FMA contraction), the arithmetic of the reference built for
// the host: near the critical angle the cosine of refraction cancels, and
// a contracted 1 - sin^2 moves the result by up to 1e-4.
NB_D float fresnel_dielectric(float cosI, float etaI, float etaT) {
    cosI = clampf(cosI, -1.0f, 1.0f);
    if (!(cosI > 0.0f)) {
        const float tmp = etaI;
        etaI = etaT;
        etaT = tmp;
        cosI = fabsf(cosI);
    }
    const float sinI = sqrtf(fmaxf(0.0f, xsub(1.0f, xmul(cosI, cosI))));
    const float sinT = xmul(xdiv(etaI, etaT), sinI);
    if (sinT >= 1.0f) return 1.0f;
    const float cosT = sqrtf(fmaxf(0.0f, xsub(1.0f, xmul(sinT, sinT))));
    const float a = xmul(etaT, cosI), b = xmul(etaI, cosT), c = xmul(etaI, cosI), d = xmul(etaT, cosT);
    const float rpar = xdiv(xsub(a, b), xadd(a, b));
    const float rper = xdiv(xsub(c, d), xadd(c, d));
    return xdiv(xadd(xmul(rpar, rpar), xmul(rper, rper)), 2.0f);
}
NB_D float3 sqrt3(const float3& v) { return f3(sqrtf(v.x), sqrtf(v.y), sqrtf(v.z)); }
// fresnelConductor with etaI = 1 (noor/cuda/fresnel.cuh:81-107), per
// channel, each operation rounded on its own as above
NB_D float fresnel_conductor1(float cosI, float c2, float s2, float eta, float k) {
    const float eta2 = xmul(eta, eta), etak2 = xmul(k, k);
    const float t0 = xsub(xsub(eta2, etak2), s2);
    const float a2b2 = sqrtf(xadd(xmul(t0, t0), xmul(xmul(4.0f, eta2), etak2)));
    const float t1 = xadd(a2b2, c2);
    const float a = sqrtf(xmul(0.5f, xadd(a2b2, t0)));
    const float t2 = xmul(xmul(2.0f, cosI), a);
    const float Rs = xdiv(xsub(t1, t2), xadd(t1, t2));
    const float t3 = xadd(xmul(c2, a2b2), xmul(s2, s2));
    const float t4 = xmul(t2, s2);
    const float Rp = xdiv(xmul(Rs, xsub(t3, t4)), xadd(t3, t4));
    return xmul(0.5f, xadd(Rp, Rs));
}
NB_D float3 fresnel_conductor(float cosI, const float3& etaT, const float3& k) {
    cosI = clampf(cosI, -1.0f, 1.0f);
    const float c2 = xmul(cosI, cosI);
    const float s2 = xsub(1.0f, c2);
    return f3(fresnel_conductor1(cosI, c2, s2, etaT.x, k.x), fresnel_conductor1(cosI, c2, s2, etaT.y, k.y),
              fresnel_conductor1(cosI, c2, s2, etaT.z, k.z));
}

// ---------------------------------------------- Trowbridge-Reitz (GGX)
// CudaTrowbridgeReitz (noor/cuda/distribution.cuh:58-183)
NB_D float ggx_D(const float3& wh, float ax, float ay) {
    const float t2 = tan2t(wh);
    if (isinf(t2)) return 0.0f;
    const float c4 = cos2t(wh) * cos2t(wh);
    const float e = (cos2phi(wh) / (ax * ax) + sin2phi(wh) / (ay * ay)) * t2;
    return 1.0f / (kPi * ax * ay * c4 * (1.0f + e) * (1.0f + e));
}
NB_D float ggx_lambda(const float3& w, float ax, float ay) {
    const float at = fabsf(tant(w));
    if (isinf(at)) return 0.0f;
    const float alpha = sqrtf(cos2phi(w) * ax * ax + sin2phi(w) * ay * ay);
    const float a2t2 = (alpha * at) * (alpha * at);
    return (-1.0f + sqrtf(1.0f + a2t2)) / 2.0f;
}
NB_D void ggx_sample11(float cosT, float U1, float U2, float& sx, float& sy) {
    if (cosT > .9999f) {
        const float r = sqrtf(U1 / (1.0f - U1));
        const float phi = 6.28318530718f * U2;
        sx = r * cosf(phi);
        sy = r * sinf(phi);
        return;
    }
    const float sinT = sqrtf(fmaxf(0.0f, 1.0f - cosT * cosT));
    const float tanT = sinT / cosT;
    const float a = 1.0f / tanT;
    const float G1 = 2.0f / (1.0f + sqrtf(1.0f + 1.0f / (a * a)));
    const float A = 2.0f * U1 / G1 - 1.0f;
    float tmp = 1.0f / (A * A - 1.0f);
    if (tmp > 1e10f) tmp = 1e10f;
    const float B = tanT;
    const float D = sqrtf(fmaxf(B * B * tmp * tmp - (A * A - B * B) * tmp, 0.0f));
    const float sx1 = B * tmp - D;
    const float sx2 = B * tmp + D;
    sx = (A < 0.0f || sx2 > 1.0f / tanT) ? sx1 : sx2;
    float S;
    if (U2 > 0.5f) {
        S = 1.0f;
        U2 = 2.0f * (U2 - .5f);
    } else {
        S = -1.0f;
        U2 = 2.0f * (.5f - U2);
    }
    const float z = (U2 * (U2 * (U2 * 0.27385f - 0.73369f) + 0.46341f)) /
                    (U2 * (U2 * (U2 * 0.093073f + 0.309420f) - 1.000000f) + 0.597999f);
    sy = S * z * sqrtf(1.0f + sx * sx);
}

// ------------------------------------------------------------- Beckmann
// Erf (Abramowitz & Stegun 7.1.26) and ErfInv (Giles 2010 single-precision
// polynomial), the two approximations noor/cuda/utils.cuh:487-539 uses
NB_D float erf_as(float x) {
    const float a1 = 0.254829592f, a2 = -0.284496736f, a3 = 1.421413741f, a4 = -1.453152027f,
                a5 = 1.061405429f, p = 0.3275911f;
    const int sign = x < 0.0f ? -1 : 1;
    x = fabsf(x);
    const float t = 1.0f / (1.0f + p * x);
    const float y = 1.0f - (((((a5 * t + a4) * t) + a3) * t + a2) * t + a1) * t * expf(-x * x);
    return sign * y;
}
NB_D float erfinv_giles(float x) {
    float w, p;
    x = clampf(x, -.99999f, .99999f);
    w = -logf((1.0f - x) * (1.0f + x));
    if (w < 5.0f) {
        w = w - 2.5f;
        p = 2.81022636e-08f;
        p = 3.43273939e-07f + p * w;
        p = -3.5233877e-06f + p * w;
        p = -4.39150654e-06f + p * w;
        p = 0.00021858087f + p * w;
        p = -0.00125372503f + p * w;
        p = -0.00417768164f + p * w;
        p = 0.246640727f + p * w;
        p = 1.50140941f + p * w;
    } else {
        w = sqrtf(w) - 3.0f;
        p = -0.000200214257f;
        p = 0.000100950558f + p * w;
        p = 0.00134934322f + p * w;
        p = -0.00367342844f + p * w;
        p = 0.00573950773f + p * w;
        p = -0.0076224613f + p * w;
        p = 0.00943887047f + p * w;
        p = 1.00167406f + p * w;
        p = 2.83297682f + p * w;
    }
    return p * x;
}
// CudaBeckmannDistribution (noor/cuda/distribution.cuh:185-342)
NB_D float beck_D(const float3& wh, float ax, float ay) {
    const float t2 = tan2t(wh);
    if (isinf(t2)) return 0.0f;
    const float c4 = cos2t(wh) * cos2t(wh);
    return expf(-t2 * (cos2phi(wh) / (ax * ax) + sin2phi(wh) / (ay * ay))) / (kPi * ax * ay * c4);
}
NB_D float beck_lambda(const float3& w, float ax, float ay) {
    const float at = fabsf(tant(w));
    if (isinf(at)) return 0.0f;
    const float alpha = sqrtf(cos2phi(w) * ax * ax + sin2phi(w) * ay * ay);
    const float a = 1.0f / (alpha * at);
    if (a >= 1.6f) return 0.0f;
    return (1.0f - 1.259f * a + 0.396f * a * a) / (3.535f * a + 2.181f * a * a);
}
NB_D void beck_sample11(float cosI, float U1, float U2, float& sx, float& sy) {
    if (cosI > .9999f) {
        const float r = sqrtf(-logf(1.0f - U1));
        const float sp = sinf(2.0f * kPi * U2);
        const float cp = cosf(2.0f * kPi * U2);
        sx = r * cp;
        sy = r * sp;
        return;
    }
    const float sinI = sqrtf(fmaxf(0.0f, 1.0f - cosI * cosI));
    const float tanI = sinI / cosI;
    const float cotI = 1.0f / tanI;
    float a = -1.0f;
    float c = erf_as(cotI);
    const float sample_x = fmaxf(U1, 1e-6f);
    const float thetaI = acosf(cosI);
    const float fit = 1.0f + thetaI * (-0.876f + thetaI * (0.4265f - 0.0594f * thetaI));
    float b = c - (1.0f + c) * powf(1.0f - sample_x, fit);
    const float norm = 1.0f / (1.0f + c + sqrtf(kInvPi) * tanI * expf(-cotI * cotI));
    int it = 0;
    while (++it < 10) {
        if (!(b >= a && b <= c)) b = 0.5f * (a + c);
        const float ie = erfinv_giles(b);
        const float value = norm * (1.0f + b + sqrtf(kInvPi) * tanI * expf(-ie * ie)) - sample_x;
        const float deriv = norm * (1.0f - ie * tanI);
        if (fabsf(value) < 1e-5f) break;
        if (value > 0.0f)
            c = b;
        else
            a = b;
        b -= value / deriv;
    }
    sx = erfinv_giles(b);
    sy = erfinv_giles(2.0f * fmaxf(U2, 1e-6f) - 1.0f);
}

// microfacet distribution dispatch: dist 0 = Trowbridge-Reitz, 1 = Beckmann
struct Micro {
    float ax, ay;
    uint32_t dist;
    NB_D float D(const float3& wh) const { return dist ? beck_D(wh, ax, ay) : ggx_D(wh, ax, ay); }
    NB_D float lambda(const float3& w) const { return dist ? beck_lambda(w, ax, ay) : ggx_lambda(w, ax, ay); }
    NB_D float G(const float3& wo, const float3& wi) const { return 1.0f / (1.0f + lambda(wo) + lambda(wi)); }
    NB_D float G1(const float3& w) const { return 1.0f / (1.0f + lambda(w)); }
    NB_D float pdf(const float3& wo, const float3& wh) const { return D(wh) * G1(wo) * absdot(wo, wh) / fabsf(wo.z); }
    NB_D float3 sample_visible(const float3& wi, float U1, float U2) const {
        const float3 ws = normalize_fast(f3(ax * wi.x, ay * wi.y, wi.z));
        float sx, sy;
        if (dist)
            beck_sample11(ws.z, U1, U2, sx, sy);
        else
            ggx_sample11(ws.z, U1, U2, sx, sy);
        const float tmp = cosphi(ws) * sx - sinphi(ws) * sy;
        sy = sinphi(ws) * sx + cosphi(ws) * sy;
        sx = tmp;
        sx *= ax;
        sy *= ay;
        return normalize_fast(f3(-sx, -sy, 1.0f));
    }
    // Sample_wh: TR flips by sign(wo.z) (distribution.cuh:104-107), Beckmann by
    // wo.z < 0 (distribution.cuh:222-229)
    NB_D float3 sample_wh(const float3& wo, float u1, float u2) const {
        if (dist) {
            const bool flip = wo.z < 0.0f;
            float3 wh = sample_visible(flip ? -1.0f * wo : wo, u1, u2);
            return flip ? -1.0f * wh : wh;
        }
        const float s = signf_ref(wo.z);
        return s * sample_visible(s * wo, u1, u2);
    }
};

NB_D Micro make_micro(const DevMaterial& m) {
    Micro mf;
    mf.ax = fmaxf(m.rough_x * m.rough_x, 1e-3f);
    mf.ay = fmaxf(m.rough_y * m.rough_y, 1e-3f);
    mf.dist = m.distribution;
    return mf;
}

// -------------------------------------------------------------- lobes
// BxDF type bits (noor/cuda/path_tracer.cuh:106-119)
enum : uint32_t {
    BSDF_REFLECTION = 1u << 0,
    BSDF_TRANSMISSION = 1u << 1,
    BSDF_DIFFUSE = 1u << 2,
    BSDF_GLOSSY = 1u << 3,
    BSDF_SPECULAR = 1u << 4,
    BSDF_CONDUCTOR = 1u << 5,
    BSDF_DIELECTRIC = 1u << 6,
    BSDF_NOOP = 1u << 7,
    BSDF_ALL = 0xFFu
};


// Lobe ids, one per BxDF class the material factory builds
// (noor/cuda/bxdf.cuh:119-137): the low 8 bits are the class's BxDF type
// flags (its constructor's), bits 8-15 tell apart classes with equal flags.
enum : uint32_t {
    kLobeNone = 0,
    // CudaLambertianReflection (bxdf.cuh:252-299)
    kLobeLambert = BSDF_REFLECTION | BSDF_DIFFUSE | BSDF_DIELECTRIC,
    // CudaMicrofacetReflection with the conductor Fresnel (bxdf.cuh:472-557)
    kLobeConductor = BSDF_CONDUCTOR | BSDF_REFLECTION | BSDF_GLOSSY,
    // CudaFresnelSpecular (bxdf.cuh:754-839)
    kLobeFresnelSpec = BSDF_REFLECTION | BSDF_TRANSMISSION | BSDF_SPECULAR | BSDF_DIELECTRIC,
    // CudaLambertianTransmission (bxdf.cuh:301-352)
    kLobeLambertT = BSDF_TRANSMISSION | BSDF_DIFFUSE | BSDF_DIELECTRIC,
    // CudaSpecularReflection with the no-op Fresnel (bxdf.cuh:354-404)
    kLobeMirror = BSDF_NOOP | BSDF_REFLECTION | BSDF_SPECULAR,
    // CudaMicrofacetReflection with the dielectric Fresnel
    kLobeMicroDiel = (BSDF_DIELECTRIC | BSDF_REFLECTION | BSDF_GLOSSY) | 1u << 8,
    // CudaMicrofacetTransmission (bxdf.cuh:559-656)
    kLobeMicroT = BSDF_TRANSMISSION | BSDF_GLOSSY | BSDF_DIELECTRIC,
    // CudaFresnelBlend (bxdf.cuh:658-752)
    kLobeFresnelBlend = (BSDF_REFLECTION | BSDF_GLOSSY | BSDF_DIELECTRIC) | 2u << 8,
    // CudaClearCoat (bxdf.cuh:842-992): a conductor microfacet substrate
    // under a dielectric specular coat
    kLobeClearCoat = (BSDF_GLOSSY | BSDF_REFLECTION | BSDF_SPECULAR) | 3u << 8,
    // CudaShadowCatcher (bxdf.cuh:203-250).  Its value is the sky seen
    // along the incoming ray over |cos wi|; the lobe functions return the
    // 1 / |cos wi| part and the integrator multiplies in the sky
    kLobeCatcher = (BSDF_REFLECTION | BSDF_TRANSMISSION | BSDF_DIFFUSE) | 4u << 8,
};
NB_HD uint32_t lobe_type(uint32_t id) { return id & 0xFFu; }

constexpr uint32_t kSpecularMat = NOOR_MIRROR | NOOR_GLASS | NOOR_CLEARCOAT;      // NOOR_SPECULAR
constexpr uint32_t kTransparentMat = NOOR_TRANSLUCENT | NOOR_GLASS | NOOR_ROUGHGLASS;
constexpr uint32_t kEmitterMat = NOOR_EMITTER | NOOR_MESHLIGHT;

// The lobes factoryBSDF builds for a material (noor/cuda/bsdf.cuh:383-461),
// in the order it adds them: lobe k in bits 16k..16k+15; 0 = none (an
// Oren-Nayar material or a mix of type bits builds none there either).
NB_HD uint32_t lobe_of(uint32_t mtype) {
    const uint32_t t = mtype & ~(uint32_t)(NOOR_BUMP | NOOR_ALPHA);
    switch (t) {
        case NOOR_DIFFUSE: return kLobeLambert;
        case NOOR_METAL: return kLobeConductor;
        case NOOR_GLASS: return kLobeFresnelSpec;
        case NOOR_MIRROR: return kLobeMirror;
        case NOOR_SUBSTRATE: return kLobeFresnelBlend;
        case NOOR_TRANSLUCENT: return kLobeLambert | kLobeLambertT << 16;
        case NOOR_GLOSSY: return kLobeLambert | kLobeMicroDiel << 16;
        case NOOR_ROUGHGLASS: return kLobeMicroDiel | kLobeMicroT << 16;
        case NOOR_CLEARCOAT: return kLobeClearCoat;
        case NOOR_SHADOWCATCHER: return kLobeCatcher;
        default: return 0u;
    }
}
// the wavefront's shading queue of a surface hit: Lambert, conductor, the rest
NB_HD uint32_t shade_kind(uint32_t lobes) {
    return lobes == kLobeLambert ? 0u : (lobes == kLobeConductor ? 1u : 2u);
}
// EXT false: only the three lobes a specialised kernel handles
template <bool EXT>
NB_D uint32_t lobe_of(uint32_t mtype) {
    if (EXT) return lobe_of(mtype);
    const uint32_t t = mtype & ~(uint32_t)(NOOR_BUMP | NOOR_ALPHA);
    if (t == NOOR_DIFFUSE) return kLobeLambert;
    if (t == NOOR_METAL) return kLobeConductor;
    if (t == NOOR_GLASS) return kLobeFresnelSpec;
    return 0u;
}
NB_D uint32_t lobe_at(uint32_t lobes, int k) { return (lobes >> (16 * k)) & 0xFFFFu; }
// EXT false: the id is one of the three lobes whose ids are their flags
template <bool EXT = true>
NB_D bool lobe_matches(uint32_t id, uint32_t flags) {
    const uint32_t t = EXT ? lobe_type(id) : id;
    return t != 0u && (t & flags) == t;
}

// Refract (bxdf.cuh:103-116)
NB_D bool refract_ref(const float3& wi, const float3& n, float eta, float3& wt) {
    const float cosThetaI = dot(n, wi);
    const float sin2ThetaI = fmaxf(0.0f, 1.0f - cosThetaI * cosThetaI);
    const float sin2ThetaT = eta * eta * sin2ThetaI;
    if (sin2ThetaT >= 1.0f) return false;
    const float cosThetaT = sqrtf(1.0f - sin2ThetaT);
    wt = -eta * wi + (eta * cosThetaI - cosThetaT) * n;
    return true;
}
NB_D float pow5(float v) {
    const float a = v * v;
    return a * a * v;
}
NB_D float3 schlick(const DevMaterial& m, float c) { return m.specular + pow5(1.0f - c) * (f3(1.0f) - m.specular); }

NB_D float3 lobe_eval(uint32_t lobe, const DevMaterial& m, const float3& wo, const float3& wi);
NB_D float lobe_pdf(uint32_t lobe, const DevMaterial& m, const float3& wo, const float3& wi);

// CudaMicrofacetReflection (bxdf.cuh:472-557) with the conductor or the
// dielectric Fresnel
NB_D float3 micro_refl_eval(const DevMaterial& m, const float3& wo, const float3& wi, bool conductor) {
    // CudaMicrofacetReflection::Eval (bxdf.cuh:482-506)
    if (!same_hemi(wo, wi)) return f3(0.0f);
    const float cO = fabsf(wo.z), cI = fabsf(wi.z);
    if (cI == 0.0f || cO == 0.0f) return f3(0.0f);
    float3 wh = normalize_fast(wi + wo);
    if (is_black(wh)) return f3(0.0f);
    wh *= signf_ref(wh.z);
    const float3 F = conductor ? fresnel_conductor(dot(wo, wh), m.ior, m.k)
                                            : f3(fresnel_dielectric(dot(wo, wh), 1.0f, m.coat_ior));
    const Micro mf = make_micro(m);
    return F * m.specular * mf.D(wh) * mf.G(wo, wi) / (4.0f * cI * cO);
}
NB_D float micro_refl_pdf(const DevMaterial& m, const float3& wo, const float3& wi) {
    if (!same_hemi(wo, wi)) return 0.0f;
    const float3 wh = normalize_guard(wo + wi);
    const Micro mf = make_micro(m);
    return mf.pdf(wo, wh) / (4.0f * dot(wo, wh));
}
NB_D float3 micro_refl_sample(const DevMaterial& m, const float3& wo, float ux, float uy, float3& wi, float& pdf,
                              bool conductor) {
    // CudaMicrofacetReflection::Sample_f (bxdf.cuh:520-539)
    if (wo.z == 0.0f) return f3(0.0f);
    const Micro mf = make_micro(m);
    const float3 wh = mf.sample_wh(wo, ux, uy);
    wi = -1.0f * wo + 2.0f * dot(wo, wh) * wh;
    if (!same_hemi(wo, wi)) {
        pdf = 0.0f;
        return f3(0.0f);
    }
    pdf = mf.pdf(wo, wh) / (4.0f * dot(wo, wh));
    return micro_refl_eval(m, wo, wi, conductor);
}

// CudaClearCoat::absorption (bxdf.cuh:849-860)
NB_D float coat_absorption(const DevMaterial& m, const float3& wo, const float3& wi) {
    const float sa = m.coat_sigma * m.coat_thickness;
    if (sa != 0.0f) return expf(-sa * (1.0f / fabsf(wo.z) + 1.0f / fabsf(wi.z)));
    return 1.0f;
}
// the coat's Refract of wo and wi into the substrate, negated
// (bxdf.cuh:869-874); a failed refraction leaves the zero vector (the
// reference leaves the vector unset; with coat_ior > 1 it cannot fail)
NB_D void coat_refract(const DevMaterial& m, const float3& wo, const float3& wi, float3& wo_c, float3& wi_c) {
    const float eta = 1.0f / m.coat_ior;
    const float3 n = f3(0.0f, 0.0f, 1.0f);
    wo_c = f3(0.0f);
    wi_c = f3(0.0f);
    refract_ref(wo, n, eta, wo_c);
    refract_ref(wi, n, eta, wi_c);
    wo_c *= -1.0f;
    wi_c *= -1.0f;
}
// probability of sampling the coat (bxdf.cuh:891, 908)
NB_D float coat_prob(const DevMaterial& m, float F) {
    const float w = m.coat_weight;
    return F * w / (F * w + (1.0f - F) * (1.0f - w));
}

// BxDF::Eval of a lobe, local frame (every lobe)
NB_D float3 lobe_eval_all(uint32_t lobe, const DevMaterial& m, const float3& wo, const float3& wi) {
    if (lobe == kLobeLambert || lobe == kLobeLambertT) return m.diffuse * kInvPi;
    if (lobe == kLobeConductor || lobe == kLobeMicroDiel) return micro_refl_eval(m, wo, wi, lobe == kLobeConductor);
    if (lobe == kLobeMicroT) {
        // CudaMicrofacetTransmission::Eval (bxdf.cuh:567-590); etaI = 1, etaT = coat_ior
        if (same_hemi(wo, wi)) return f3(0.0f);
        const float cO = wo.z, cI = wi.z;
        if (cI == 0.0f || cO == 0.0f) return f3(0.0f);
        const float eta = wo.z > 0.0f ? m.coat_ior / 1.0f : 1.0f / m.coat_ior;
        float3 wh = normalize_guard(wo + wi * eta);
        wh *= signf_ref(wh.z);
        const float F = fresnel_dielectric(dot(wo, wh), 1.0f, m.coat_ior);
        const float sd = dot(wo, wh) + eta * dot(wi, wh);
        const Micro mf = make_micro(m);
        return (1.0f - F) * m.transmission *
               fabsf(mf.D(wh) * mf.G(wo, wi) * eta * eta * absdot(wi, wh) * absdot(wo, wh) / (cI * cO * sd * sd));
    }
    if (lobe == kLobeFresnelBlend) {
        // CudaFresnelBlend::Eval (bxdf.cuh:670-688)
        const float3 diffuse = (28.0f / (23.0f * kPi)) * m.diffuse * (f3(1.0f) - m.specular) *
                               (1.0f - pow5(1.0f - 0.5f * fabsf(wi.z))) * (1.0f - pow5(1.0f - 0.5f * fabsf(wo.z)));
        float3 wh = wi + wo;
        if (wh.x == 0.0f && wh.y == 0.0f && wh.z == 0.0f) return f3(0.0f);
        wh = normalize_guard(wh);
        const Micro mf = make_micro(m);
        const float3 specular =
            mf.D(wh) / (4.0f * absdot(wi, wh) * fmaxf(fabsf(wi.z), fabsf(wo.z))) * schlick(m, dot(wi, wh));
        return diffuse + specular;
    }
    if (lobe == kLobeClearCoat) {
        // CudaClearCoat::Eval (bxdf.cuh:862-880)
        const float F0 = fresnel_dielectric(wo.z, 1.0f, m.coat_ior);
        const float F1 = fresnel_dielectric(wi.z, 1.0f, m.coat_ior);
        float3 wo_c, wi_c;
        coat_refract(m, wo, wi, wo_c, wi_c);
        const float3 r = micro_refl_eval(m, wo_c, wi_c, true) * (1.0f - F0) * (1.0f - F1);
        return r * coat_absorption(m, wo_c, wi_c);
    }
    if (lobe == kLobeCatcher) return f3(1.0f / fabsf(wi.z));  // times the sky (bxdf.cuh:213-218)
    return f3(0.0f);  // specular lobes: delta
}
NB_D float lobe_pdf_all(uint32_t lobe, const DevMaterial& m, const float3& wo, const float3& wi) {
    if (lobe == kLobeLambert) return same_hemi(wo, wi) ? fabsf(wi.z) * kInvPi : 0.0f;
    if (lobe == kLobeLambertT) return !same_hemi(wo, wi) ? fabsf(wi.z) * kInvPi : 0.0f;
    if (lobe == kLobeConductor || lobe == kLobeMicroDiel) return micro_refl_pdf(m, wo, wi);
    if (lobe == kLobeMicroT) {
        // CudaMicrofacetTransmission::Pdf (bxdf.cuh:592-606)
        if (same_hemi(wo, wi)) return 0.0f;
        const float eta = wo.z > 0.0f ? m.coat_ior / 1.0f : 1.0f / m.coat_ior;
        const float3 wh = normalize_guard(wo + wi * eta);
        const float sd = dot(wo, wh) + eta * dot(wi, wh);
        const float dwh_dwi = fabsf((eta * eta * dot(wi, wh)) / (sd * sd));
        const Micro mf = make_micro(m);
        return mf.pdf(wo, wh) * dwh_dwi;
    }
    if (lobe == kLobeFresnelBlend) {
        // CudaFresnelBlend::Pdf (bxdf.cuh:690-699)
        if (!same_hemi(wo, wi)) return 0.0f;
        const float3 wh = normalize_guard(wo + wi);
        const Micro mf = make_micro(m);
        const float pdf_wh = mf.pdf(wo, wh);
        return 0.5f * (fabsf(wi.z) * kInvPi + pdf_wh / (4.0f * dot(wo, wh)));
    }
    if (lobe == kLobeClearCoat) {
        // CudaClearCoat::Pdf (bxdf.cuh:882-902): the substrate's density
        // plus the coat's probability
        const float F = fresnel_dielectric(wo.z, 1.0f, m.coat_ior);
        float3 wo_c, wi_c;
        coat_refract(m, wo, wi, wo_c, wi_c);
        const float c = coat_prob(m, F);
        return micro_refl_pdf(m, wo_c, wi_c) * (1.0f - c) + c;
    }
    if (lobe == kLobeCatcher) return 1.0f;
    return 0.0f;
}
// BxDF::Sample_f of a lobe (u already remapped by the BSDF); pdf stays 0 on
// failure; stype = the sampled BxDF type
NB_D float3 lobe_sample_all(uint32_t lobe, const DevMaterial& m, const float3& wo, float ux, float uy, float3& wi,
                            float& pdf, uint32_t& stype) {
    stype = lobe_type(lobe);
    if (lobe == kLobeLambert || lobe == kLobeLambertT) {
        // CudaLambertianReflection / Transmission::Sample_f (bxdf.cuh:270-285, 321-336)
        wi = cosine_hemisphere(ux, uy);
        if (lobe == kLobeLambert ? wo.z < 0.0f : wo.z > 0.0f) wi.z *= -1.0f;
        pdf = lobe_pdf(lobe, m, wo, wi);
        return m.diffuse * kInvPi;
    }
    if (lobe == kLobeConductor || lobe == kLobeMicroDiel)
        return micro_refl_sample(m, wo, ux, uy, wi, pdf, lobe == kLobeConductor);
    if (lobe == kLobeMirror) {
        // CudaSpecularReflection::Sample_f (bxdf.cuh:377-392), no-op Fresnel
        wi = f3(-wo.x, -wo.y, wo.z);
        pdf = 1.0f;
        return m.diffuse / fabsf(wi.z);
    }
    if (lobe == kLobeMicroT) {
        // CudaMicrofacetTransmission::Sample_f (bxdf.cuh:609-637)
        if (wo.z == 0.0f) return f3(0.0f);
        const Micro mf = make_micro(m);
        float3 wh = mf.sample_wh(wo, ux, uy);
        const float eta = wo.z > 0.0f ? 1.0f / m.coat_ior : m.coat_ior / 1.0f;
        if (!refract_ref(wo, wh, eta, wi)) {
            // total internal reflection: the reference reflects with
            // helper_math's reflect(i, n) = i - 2 n (n . i)
            wi = wo - 2.0f * wh * dot(wh, wo);
            wh *= signf_ref(wh.z);
            const float F = fresnel_dielectric(dot(wi, wh), 1.0f, m.coat_ior);
            const float cO = wo.z, cI = wi.z;
            const float3 r = F * m.specular * mf.D(wh) * mf.G(wo, wi) / (4.0f * cI * cO);
            pdf = mf.pdf(wo, wh) / (4.0f * dot(wo, wh));
            return r;
        }
        pdf = lobe_pdf(lobe, m, wo, wi);
        return lobe_eval(lobe, m, wo, wi);
    }
    if (lobe == kLobeFresnelBlend) {
        // CudaFresnelBlend::Sample_f (bxdf.cuh:701-727)
        if (ux < 0.5f) {
            const float lx = fminf(2.0f * ux, kOneMinusEps);
            wi = cosine_hemisphere(lx, uy);
            wi.z *= signf_ref(wi.z);
        } else {
            const float lx = fminf(2.0f * (ux - 0.5f), kOneMinusEps);
            const Micro mf = make_micro(m);
            const float3 wh = mf.sample_wh(wo, lx, uy);
            wi = -1.0f * wo + 2.0f * dot(wo, wh) * wh;
            if (!same_hemi(wo, wi)) return f3(0.0f);
        }
        pdf = lobe_pdf(lobe, m, wo, wi);
        return lobe_eval(lobe, m, wo, wi);
    }
    if (lobe == kLobeClearCoat) {
        // CudaClearCoat::Sample_f (bxdf.cuh:904-950): the second number
        // chooses coat or substrate and is rescaled for the choice
        const float F0 = fresnel_dielectric(wo.z, 1.0f, m.coat_ior);
        const float ps = coat_prob(m, F0);
        if (uy < ps) {
            // CudaSpecularReflection::Sample_f with the dielectric Fresnel
            wi = f3(-wo.x, -wo.y, wo.z);
            pdf = ps;
            stype = BSDF_DIELECTRIC | BSDF_REFLECTION | BSDF_SPECULAR;
            return fresnel_dielectric(wi.z, 1.0f, m.coat_ior) * m.diffuse / fabsf(wi.z);
        }
        const float sy = (uy - ps) / (1.0f - ps);
        const float eta = 1.0f / m.coat_ior;
        float3 wo_c = f3(0.0f), wi_c;
        refract_ref(wo, f3(0.0f, 0.0f, 1.0f), eta, wo_c);
        float p = 0.0f;
        float3 r = micro_refl_sample(m, -1.0f * wo_c, ux, sy, wi_c, p, true);
        stype = kLobeConductor;
        if (p == 0.0f) return f3(0.0f);
        const float F1 = fresnel_dielectric(-wi_c.z, 1.0f, m.coat_ior);
        // refract out; under total internal reflection the reference
        // leaves wi unset, here the sample fails
        if (!refract_ref(-1.0f * wi_c, f3(0.0f, 0.0f, -1.0f), 1.0f / eta, wi)) return f3(0.0f);
        if (F1 == 1.0f) return f3(0.0f);
        r *= coat_absorption(m, wo_c, wi_c) * (1.0f - F0) * (1.0f - F1);
        r /= fabsf(wi_c.z);
        pdf = p * (1.0f - ps);
        return r;
    }
    if (lobe == kLobeCatcher) {
        // CudaShadowCatcher::Sample_f: uniformSampleHemisphere with pdf 1,
        // as the reference has it
        wi = uniform_hemisphere(ux, uy);
        pdf = 1.0f;
        return f3(1.0f / fabsf(wi.z));
    }
    if (lobe == kLobeFresnelSpec) {
        // CudaFresnelSpecular::Sample_f (bxdf.cuh:775-809), IOR = coat_ior
        const float ior = m.coat_ior;
        const float F = fresnel_dielectric(wo.z, 1.0f, ior);
        if (ux < F) {
            wi = f3(-wo.x, -wo.y, wo.z);
            pdf = F;
            stype = BSDF_REFLECTION | BSDF_SPECULAR;
            return F * m.specular / fabsf(wi.z);
        }
        const bool entering = wo.z > 0.0f;
        const float eta = entering ? (1.0f / ior) : (ior / 1.0f);
        const float3 n = faceforward(f3(0.0f, 0.0f, 1.0f), wo);
        const float cI = dot(n, wo);
        const float s2I = fmaxf(0.0f, 1.0f - cI * cI);
        const float s2T = eta * eta * s2I;
        if (s2T >= 1.0f) return f3(0.0f);
        const float cT = sqrtf(1.0f - s2T);
        wi = -eta * wo + (eta * cI - cT) * n;
        pdf = 1.0f - F;
        stype = BSDF_TRANSMISSION | BSDF_SPECULAR;
        return m.transmission * eta * eta * (1.0f - F) / fabsf(wi.z);
    }
    return f3(0.0f);
}

// The lobes the configurations use (Lambert, conductor, Fresnel specular)
// are expanded inline; the others are one shared out-of-line copy, so that
// their code does not grow the registers and spills of the integrators'
// hot loops.
NB_OUTLINE float3 lobe_eval_extra(uint32_t lobe, const DevMaterial& m, float3 wo, float3 wi) {
    return lobe_eval_all(lobe, m, wo, wi);
}
NB_OUTLINE float lobe_pdf_extra(uint32_t lobe, const DevMaterial& m, float3 wo, float3 wi) {
    return lobe_pdf_all(lobe, m, wo, wi);
}
NB_OUTLINE float3 lobe_sample_extra(uint32_t lobe, const DevMaterial& m, float3 wo, float ux, float uy,
                                                 float3& wi, float& pdf, uint32_t& stype) {
    return lobe_sample_all(lobe, m, wo, ux, uy, wi, pdf, stype);
}
NB_HD bool lobe_common(uint32_t lobe) {
    return lobe == kLobeNone || lobe == kLobeLambert || lobe == kLobeConductor || lobe == kLobeFresnelSpec;
}
// EXT false: a kernel specialised for scenes whose materials use only the
// lobes above (the other lobes' code is left out)
template <bool EXT>
NB_D float3 lobe_eval(uint32_t lobe, const DevMaterial& m, const float3& wo, const float3& wi) {
    if (lobe == kLobeLambert) return m.diffuse * kInvPi;
    if (lobe == kLobeConductor) return lobe_eval_all(kLobeConductor, m, wo, wi);
    if (!EXT || lobe_common(lobe)) return f3(0.0f);
    return lobe_eval_extra(lobe, m, wo, wi);
}
NB_D float3 lobe_eval(uint32_t lobe, const DevMaterial& m, const float3& wo, const float3& wi) {
    return lobe_eval<true>(lobe, m, wo, wi);
}
template <bool EXT>
NB_D float lobe_pdf(uint32_t lobe, const DevMaterial& m, const float3& wo, const float3& wi) {
    if (lobe == kLobeLambert) return same_hemi(wo, wi) ? fabsf(wi.z) * kInvPi : 0.0f;
    if (lobe == kLobeConductor) return lobe_pdf_all(kLobeConductor, m, wo, wi);
    if (!EXT || lobe_common(lobe)) return 0.0f;
    return lobe_pdf_extra(lobe, m, wo, wi);
}
NB_D float lobe_pdf(uint32_t lobe, const DevMaterial& m, const float3& wo, const float3& wi) {
    return lobe_pdf<true>(lobe, m, wo, wi);
}
template <bool EXT = true>
NB_D float3 lobe_sample(uint32_t lobe, const DevMaterial& m, const float3& wo, float ux, float uy, float3& wi,
                        float& pdf, uint32_t& stype) {
    if (lobe == kLobeLambert) return lobe_sample_all(kLobeLambert, m, wo, ux, uy, wi, pdf, stype);
    if (lobe == kLobeConductor) return lobe_sample_all(kLobeConductor, m, wo, ux, uy, wi, pdf, stype);
    if (lobe == kLobeFresnelSpec) return lobe_sample_all(kLobeFresnelSpec, m, wo, ux, uy, wi, pdf, stype);
    if (!EXT || lobe_common(lobe)) {
        stype = 0u;
        return f3(0.0f);
    }
    return lobe_sample_extra(lobe, m, wo, ux, uy, wi, pdf, stype);
}

// CudaBSDF (noor/cuda/bsdf.cuh:232-358) over a material's lobes.  A
// one-lobe material (every material the configurations use) takes the
// inline path; two-lobe materials go through one shared out-of-line copy of
// the general aggregation, which keeps the integrators' hot loops as lean
// as for one lobe.
NB_D int lobes_matching(uint32_t lobes, uint32_t flags) {
    return (lobe_matches(lobe_at(lobes, 0), flags) ? 1 : 0) + (lobe_matches(lobe_at(lobes, 1), flags) ? 1 : 0);
}
template <bool EXT = true>
NB_D bool lobe_sided(uint32_t id, bool reflect) {
    const uint32_t t = EXT ? lobe_type(id) : id;
    return (reflect && (t & BSDF_REFLECTION)) || (!reflect && (t & BSDF_TRANSMISSION));
}
NB_D float3 bsdf_eval_n(uint32_t lobes, const DevMaterial& m, const Frame& F, const float3& woW, const float3& wiW,
                        uint32_t flags) {
    const float3 wo = to_local(F, woW), wi = to_local(F, wiW);
    const bool reflect = dot(wiW, F.ng) * dot(woW, F.ng) > 0.0f;
    float3 f = f3(0.0f);
    for (int k = 0; k < 2; ++k) {
        const uint32_t id = lobe_at(lobes, k);
        if (lobe_matches(id, flags) && lobe_sided(id, reflect)) f += lobe_eval(id, m, wo, wi);
    }
    return f;
}
NB_D float bsdf_pdf_n(uint32_t lobes, const DevMaterial& m, const Frame& F, const float3& woW, const float3& wiW,
                      uint32_t flags) {
    if (lobes == 0u) return 0.0f;
    const float3 wo = to_local(F, woW), wi = to_local(F, wiW);
    if (wo.z == 0.0f) return 0.0f;
    float pdf = 0.0f;
    int n = 0;
    for (int k = 0; k < 2; ++k) {
        const uint32_t id = lobe_at(lobes, k);
        if (lobe_matches(id, flags)) {
            ++n;
            pdf += lobe_pdf(id, m, wo, wi);
        }
    }
    return n > 0 ? pdf / (float)n : 0.0f;
}
// one lobe chosen uniformly among the matching ones by ux (remapped for the
// lobe), with the other matching lobes' pdf and value added unless the
// chosen lobe is specular; pdf 0 = no sample
NB_D float3 bsdf_sample_n(uint32_t lobes, const DevMaterial& m, const Frame& F, const float3& woW, uint32_t flags,
                          float ux, float uy, float3& wiW, float& pdf, uint32_t& stype) {
    pdf = 0.0f;
    stype = 0u;
    const int n = lobes_matching(lobes, flags);
    if (n == 0) return f3(0.0f);
    const int comp = min((int)floorf(ux * (float)n), n - 1);
    const float uxr = fminf(ux * (float)n - (float)comp, kOneMinusEps);
    int chosen = -1;
    for (int k = 0, c = comp; k < 2; ++k)
        if (lobe_matches(lobe_at(lobes, k), flags) && c-- == 0) {
            chosen = k;
            break;
        }
    const uint32_t id = lobe_at(lobes, chosen);
    const float3 wo = to_local(F, woW);
    if (wo.z == 0.0f) return f3(0.0f);
    float3 wi = f3(0.0f);
    uint32_t st;
    float3 f = lobe_sample(id, m, wo, uxr, uy, wi, pdf, st);
    if (pdf == 0.0f) return f3(0.0f);
    stype = st;
    wiW = to_world(F, wi);
    const bool specular = (lobe_type(id) & BSDF_SPECULAR) != 0u;
    const uint32_t other = lobe_at(lobes, 1 - chosen);
    if (!specular && n > 1 && lobe_matches(other, flags)) pdf += lobe_pdf(other, m, wo, wi);
    if (n > 1) pdf /= (float)n;
    if (!specular) {
        const bool reflect = dot(wiW, F.ng) * dot(woW, F.ng) > 0.0f;
        if (lobe_matches(other, flags) && lobe_sided(other, reflect)) f += lobe_eval(other, m, wo, wi);
    }
    return f;
}
NB_OUTLINE float3 bsdf_eval_two(uint32_t lobes, const DevMaterial& m, const Frame& F, float3 woW,
                                                    float3 wiW, uint32_t flags) {
    return bsdf_eval_n(lobes, m, F, woW, wiW, flags);
}
NB_OUTLINE float bsdf_pdf_two(uint32_t lobes, const DevMaterial& m, const Frame& F, float3 woW,
                                                  float3 wiW, uint32_t flags) {
    return bsdf_pdf_n(lobes, m, F, woW, wiW, flags);
}
NB_OUTLINE float3 bsdf_sample_two(uint32_t lobes, const DevMaterial& m, const Frame& F,
                                                      float3 woW, uint32_t flags, float ux, float uy, float3& wiW,
                                                      float& pdf, uint32_t& stype) {
    return bsdf_sample_n(lobes, m, F, woW, flags, ux, uy, wiW, pdf, stype);
}

// one lobe: the aggregation above with n <= 1, written out
template <bool EXT = true>
NB_D float3 bsdf_eval(uint32_t lobes, const DevMaterial& m, const Frame& F, const float3& woW, const float3& wiW,
                      uint32_t flags) {
    if (EXT && lobes > 0xFFFFu) return bsdf_eval_two(lobes, m, F, woW, wiW, flags);
    const float3 wo = to_local(F, woW), wi = to_local(F, wiW);
    const bool reflect = dot(wiW, F.ng) * dot(woW, F.ng) > 0.0f;
    if (lobe_matches<EXT>(lobes, flags) && lobe_sided<EXT>(lobes, reflect)) return lobe_eval<EXT>(lobes, m, wo, wi);
    return f3(0.0f);
}
template <bool EXT = true>
NB_D float bsdf_pdf(uint32_t lobes, const DevMaterial& m, const Frame& F, const float3& woW, const float3& wiW,
                    uint32_t flags) {
    if (EXT && lobes > 0xFFFFu) return bsdf_pdf_two(lobes, m, F, woW, wiW, flags);
    if (lobes == 0u) return 0.0f;
    const float3 wo = to_local(F, woW), wi = to_local(F, wiW);
    if (wo.z == 0.0f) return 0.0f;
    return lobe_matches<EXT>(lobes, flags) ? lobe_pdf<EXT>(lobes, m, wo, wi) : 0.0f;
}
template <bool EXT = true>
NB_D float3 bsdf_sample_u(uint32_t lobes, const DevMaterial& m, const Frame& F, const float3& woW, uint32_t flags,
                          float ux, float uy, float3& wiW, float& pdf, uint32_t& stype) {
    if (EXT && lobes > 0xFFFFu) return bsdf_sample_two(lobes, m, F, woW, flags, ux, uy, wiW, pdf, stype);
    pdf = 0.0f;
    stype = 0u;
    if (!lobe_matches<EXT>(lobes, flags)) return f3(0.0f);
    const float uxr = fminf(ux * 1.0f - 0.0f, kOneMinusEps);
    const float3 wo = to_local(F, woW);
    if (wo.z == 0.0f) return f3(0.0f);
    float3 wi = f3(0.0f);
    uint32_t st;
    const float3 f = lobe_sample<EXT>(lobes, m, wo, uxr, uy, wi, pdf, st);
    if (pdf == 0.0f) return f3(0.0f);
    stype = st;
    wiW = to_world(F, wi);
    return f;
}
// draws two random numbers when a lobe matches
template <bool EXT = true>
NB_D float3 bsdf_sample(uint32_t lobes, const DevMaterial& m, const Frame& F, const float3& woW, uint32_t flags,
                        Rng& rng, float3& wiW, float& pdf, uint32_t& stype) {
    if (EXT ? lobes_matching(lobes, flags) == 0 : !lobe_matches<false>(lobes, flags)) {
        pdf = 0.0f;
        stype = 0u;
        return f3(0.0f);
    }
    const float ux = rng.next();
    const float uy = rng.next();
    return bsdf_sample_u<EXT>(lobes, m, F, woW, flags, ux, uy, wiW, pdf, stype);
}

// ------------------------------------------------------------ sky & env
NB_D float hosek_radiance_internal(const float* c, float theta, float gamma) {
    const float cg = cosf(gamma);
    const float cg2 = cg * cg;
    const float ct = cosf(theta);
    const float expM = expf(c[4] * gamma);
    const float rayM = cg2;
    const float mieM = (1.0f + cg2) / powf((1.0f + c[8] * c[8] - 2.0f * c[8] * cg), 1.5f);
    const float zenith = sqrtf(ct);
    return (1.0f + c[0] * expf(c[1] / (ct + 0.01f))) *
           (c[2] + c[3] * expM + c[5] * rayM + c[6] * mieM + c[7] * zenith);
}
NB_D float inverse_gamma(float v) {
    if (v <= 0.04045f) return v * 1.0f / 12.92f;
    return powf((v + 0.055f) * 1.0f / 1.055f, 2.4f);
}
// CudaHosekSky::querySkyModel (noor/cuda/hosek.cuh:86-101)
NB_D float3 hosek_query(const DevHosek& H, const float3& v) {
    if (v.y < 0.0f) return f3(0.0f);
    const float theta = clampf(spherical_theta(v), 0.0f, kPiOver2);
    const float gamma = acosf(clampf(dot(v, H.solar_dir), -1.0f, 1.0f));
    float3 rgb;
    rgb.x = hosek_radiance_internal(H.configs[0], theta, gamma) * H.radiance[0];
    rgb.y = hosek_radiance_internal(H.configs[1], theta, gamma) * H.radiance[1];
    rgb.z = hosek_radiance_internal(H.configs[2], theta, gamma) * H.radiance[2];
    if (gamma < H.solar_radius) return H.solar_scale * rgb;
    const float3 s = rgb * 0.025f;
    return f3(inverse_gamma(s.x), inverse_gamma(s.y), inverse_gamma(s.z));
}

// bilinear lookup at normalized (u,v) with clamp addressing, exact weights
// (the reference filters in hardware: tex2D with cudaFilterModeLinear)
NB_D float3 env_bilinear(const DevScene& S, float u, float v) {
    const int W = S.env_w, H = S.env_h;
    const float x = u * (float)W - 0.5f, y = v * (float)H - 0.5f;
    const float fx0 = floorf(x), fy0 = floorf(y);
    const float ax = x - fx0, ay = y - fy0;
    int x0 = (int)fx0, y0 = (int)fy0;
    int x1 = x0 + 1, y1 = y0 + 1;
    x0 = min(max(x0, 0), W - 1);
    x1 = min(max(x1, 0), W - 1);
    y0 = min(max(y0, 0), H - 1);
    y1 = min(max(y1, 0), H - 1);
    const float4 t00 = __ldg(&S.env[y0 * W + x0]), t10 = __ldg(&S.env[y0 * W + x1]);
    const float4 t01 = __ldg(&S.env[y1 * W + x0]), t11 = __ldg(&S.env[y1 * W + x1]);
    const float w00 = (1.0f - ax) * (1.0f - ay), w10 = ax * (1.0f - ay), w01 = (1.0f - ax) * ay, w11 = ax * ay;
    return w00 * f3(t00) + w10 * f3(t10) + w01 * f3(t01) + w11 * f3(t11);
}

NB_OUTLINE float3 env_texture(const DevScene& S, float u, float v) { return f3(tex2D<float4>(S.env_tex, u, v)); }

// CudaSkyDomeManager::evaluate(dir) (noor/cuda/skydome.cuh:93-101); with
// NOOR_ENV_REFERENCE maps are read through the texture unit as there.  The
// mode's code is compiled only where REF is true (the kernels' extended
// builds, which scenes using the mode select): the default builds carry none.
template <bool REF = true>
NB_D float3 env_eval(const DevScene& S, const float3& dir) {
    if (S.sky_type == NOOR_SKY_PHYSICAL) return hosek_query(S.hosek, dir);
    const float phi = spherical_phi(dir) * kInv2Pi;
    const float theta = spherical_theta(dir) * kInvPi;
    if (REF && S.env_ref) return env_texture(S, phi, theta);
    return env_bilinear(S, phi, theta);
}

// The reference's CudaDistribution2D sampling (noor/cuda/distribution2d.cuh:
// 230-336) on its own tables, NOOR_ENV_REFERENCE.  As there, the marginal
// search runs over h + 1 CDF entries and the conditional over w + 1 (the
// row integral and the next row's first entry included) and the sample is
// divided by that count; the entries past a CDF's end are never selected
// for u < 1 (the last real entry is 1).
NB_D float rdist_cdf(const DevScene& S, int row, int col) { return __ldg(&S.rcdf[(size_t)row * (S.rw + 1) + col]); }
NB_D float rdist_func(const DevScene& S, int row, int col) { return __ldg(&S.rfunc[(size_t)row * (S.rw + 1) + col]); }
NB_D float rdist_func_int(const DevScene& S, int row) { return rdist_func(S, row, row == S.rh ? S.rh : S.rw); }
NB_D float rdist_sample1d(const DevScene& S, int row, int n, float u, float& pdf, int& off) {
    int l = 0, r = n, interval = -1;
    while (l <= r) {
        const int m = l + (r - l) / 2;
        if (rdist_cdf(S, row, m) <= u) {
            l = m + 1;
            interval = m;
        } else {
            r = m - 1;
        }
    }
    off = min(max(interval, 0), n - 1);
    const float func = rdist_func(S, row, off);
    const float c0 = rdist_cdf(S, row, off), c1 = rdist_cdf(S, row, off + 1);
    const float fi = rdist_func_int(S, row);
    float du = u - c0;
    if (c1 - c0 > 0.0f) du /= (c1 - c0);
    pdf = fi > 0.0f ? func / fi : 0.0f;
    return ((float)off + du) / (float)n;
}
// out of line (like the extra lobes): kernels that never meet the mode
// spend no instruction cache or registers on it
NB_OUTLINE float2 rdist_sample(const DevScene& S, float u0, float u1, float& pdf) {
    float py, px;
    int v, c;
    const float y = rdist_sample1d(S, S.rh, S.rh + 1, u1, py, v);
    const float x = rdist_sample1d(S, v, S.rw + 1, u0, px, c);
    pdf = px * py;
    return f2(x, y);
}
NB_OUTLINE float rdist_pdf(const DevScene& S, float x, float y) {
    const int iu = min(max((int)(x * S.rw), 0), S.rw - 1);
    const int iv = min(max((int)(y * S.rh), 0), S.rh - 1);
    return rdist_func(S, iv, iu) / rdist_func_int(S, S.rh);
}

// piecewise-constant 1D sampling over one CDF (PBRT-v3 Distribution1D)
NB_D float sample_1d(const float* func, const float* cdf, int n, float integral, float u, float& pdf, int& off,
                     const int* guide = nullptr) {
    int lo = 0, hi = n;  // largest i in [0, n] with cdf[i] <= u, clamped to [0, n-1]
    if (guide) {
        // that index lies between the guide entries one bin either side of
        // u's (the bin of u * kDistGuide may be off by one in rounding)
        const int k = min((int)(u * (float)kDistGuide), kDistGuide - 1);
        lo = __ldg(&guide[max(k - 1, 0)]);
        hi = __ldg(&guide[min(k + 2, kDistGuide)]);
    }
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&cdf[mid]) <= u)
            lo = mid;
        else
            hi = mid - 1;
    }
    off = min(lo, n - 1);
    const float c0 = __ldg(&cdf[off]), c1 = __ldg(&cdf[off + 1]);
    float du = u - c0;
    if (c1 - c0 > 0.0f) du /= (c1 - c0);
    pdf = integral > 0.0f ? __ldg(&func[off]) / integral : 0.0f;
    return ((float)off + du) / (float)n;
}

NB_D float2 dist_sample(const DevDist2D& D, float u0, float u1, float& pdf) {
    float pv, pu;
    int row;
    const float y = sample_1d(D.row_int, D.marg_cdf, D.h, D.marg_int, u1, pv, row, D.mguide);
    int col;
    const float x = sample_1d(D.func + (size_t)row * D.w, D.cdf + (size_t)row * (D.w + 1), D.w,
                              __ldg(&D.row_int[row]), u0, pu, col,
                              D.guide ? D.guide + (size_t)row * (kDistGuide + 1) : nullptr);
    pdf = pu * pv;
    return f2(x, y);
}
NB_D float dist_pdf(const DevDist2D& D, float x, float y) {
    const int iu = min(max((int)(x * D.w), 0), D.w - 1);
    const int iv = min(max((int)(y * D.h), 0), D.h - 1);
    return D.marg_int > 0.0f ? __ldg(&D.func[(size_t)iv * D.w + iu]) / D.marg_int : 0.0f;
}

// importance_sample_dir (noor/cuda/skydome.cuh:130-140) on the build's
// distribution; draws two random numbers
template <bool REF = true>
NB_D float3 env_sample_dir(const DevScene& S, Rng& rng, float& pdf) {
    const float u0 = rng.next();
    const float u1 = rng.next();
    float mp;
    const float2 uv = (REF && S.env_ref) ? rdist_sample(S, u0, u1, mp) : dist_sample(S.dist, u0, u1, mp);
    float st;
    const float3 dir = spherical_direction(uv.x, uv.y, st);
    pdf = (st == 0.0f) ? 0.0f : mp / (2.0f * kPi * kPi * st);
    return dir;
}
// CudaInfiniteLight::pdf_Li (noor/cuda/lightimp.cuh:161-173)
template <bool REF = true>
NB_D float env_pdf(const DevScene& S, const float3& wi) {
    if (!S.sky_on) return 0.0f;
    const float theta = spherical_theta(wi);
    const float phi = spherical_phi(wi);
    const float st = sinf(theta);
    if (st == 0.0f) return 0.0f;
    const float x = phi * kInv2Pi, y = theta * kInvPi;
    return ((REF && S.env_ref) ? rdist_pdf(S, x, y) : dist_pdf(S.dist, x, y)) / (2.0f * kPi * kPi * st);
}

}  // namespace nb
