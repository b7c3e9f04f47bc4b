// Path-replay backpropagation (Vicini, Speierer & Jakob 2021, "Path Replay
// Backpropagation", ACM TOG 40(4)) for the megakernel's estimator, with
// respect to per-material albedo (Lambert reflectance, conductor specular
// tint), conductor roughness and the environment texels.
//
// The estimator is differentiated with its sampling detached: directions,
// light picks, MIS weights and pdfs come from the scene as loaded (the
// parameters at the start of an optimisation step), while BSDF values and
// environment radiance come from the parameter buffers.  The forward pass
// renders that estimator; the backward pass replays every path from its
// seed (no path storage: memory stays O(pixels)), first to total its
// radiance, then again to push dLoss/dpixel through each vertex:
//   d(beta * direct)/dparams at the vertex, and
//   L_remaining * dlog f / dparams for the scattering factor, where
//   L_remaining is the radiance the path collects after the vertex.
// Russian roulette must be off (rr >= bounces): its decision depends on
// the throughput and would make the estimator discontinuous.
#include <algorithm>
#include <cstring>

#include "host_common.h"
#include "integrator.cuh"
#include "runtime.h"

namespace nb {

struct AdjParams {
    const float* albedo;     // M x 3
    const float* rough;      // M
    const float* env;        // H x W x 3 (radiance texels for evaluation)
    int env_w, env_h;
    float* g_albedo;         // M x 3
    float* g_rough;          // M
    float* g_env;            // H x W x 3
    const float* grad_img;   // npix x 3
    float* image;            // npix x 3
    uint32_t num_mats;
    uint32_t spp;
    uint32_t frame0;
    uint32_t* status;
};

// material with the evaluation parameters substituted
NB_D DevMaterial eval_material(const DevMaterial& m0, const AdjParams& P, uint32_t mi) {
    DevMaterial m = m0;
    const float3 a = f3(P.albedo[3 * mi], P.albedo[3 * mi + 1], P.albedo[3 * mi + 2]);
    if (lobe_of(m.type) == kLobeLambert) m.diffuse = a;
    if (lobe_of(m.type) == kLobeConductor) {
        m.specular = a;
        m.rough_x = m.rough_y = P.rough[mi];
    }
    return m;
}

// f, the value without the tint (conductor), and dlog f / droughness
struct FDeriv {
    float3 f;
    float3 f_untinted;
    float dlogf_dr;
};

NB_D float ggx_dlogD_dalpha(const float3& wh, float a) {
    const float t2 = tan2t(wh);
    if (isinf(t2)) return 0.0f;
    const float a2 = a * a;
    return 2.0f * (t2 - a2) / (a * (a2 + t2));
}
NB_D float ggx_dlambda_dalpha(const float3& w, float a) {
    const float at = fabsf(tant(w));
    if (isinf(at)) return 0.0f;
    const float t2 = at * at;
    return a * t2 / (2.0f * sqrtf(1.0f + a * a * t2));
}
// Beckmann: D = exp(-tan^2/a^2) / (pi a^2 cos^4); Lambda is the rational fit
// in x = 1 / (a |tan|), zero for x >= 1.6
NB_D float beck_dlogD_dalpha(const float3& wh, float a) {
    const float t2 = tan2t(wh);
    if (isinf(t2)) return 0.0f;
    return 2.0f * t2 / (a * a * a) - 2.0f / a;
}
NB_D float beck_dlambda_dalpha(const float3& w, float a) {
    const float at = fabsf(tant(w));
    if (isinf(at)) return 0.0f;
    const float x = 1.0f / (a * at);
    if (x >= 1.6f) return 0.0f;
    const float n = 1.0f - 1.259f * x + 0.396f * x * x, dn = -1.259f + 0.792f * x;
    const float q = 3.535f * x + 2.181f * x * x, dq = 3.535f + 4.362f * x;
    const float dlam_dx = (dn * q - n * dq) / (q * q);
    return dlam_dx * (-x / a);
}

// BSDF value at (wo, wi) in the local frame with the evaluation material
NB_D FDeriv lobe_value(uint32_t lobe, const DevMaterial& m, const Frame& F, const float3& woW, const float3& wiW) {
    FDeriv r{f3(0.0f), f3(0.0f), 0.0f};
    const float3 wo = to_local(F, woW), wi = to_local(F, wiW);
    const bool reflect = dot(wiW, F.ng) * dot(woW, F.ng) > 0.0f;
    if (!reflect) return r;
    if (lobe == kLobeLambert) {
        r.f = m.diffuse * kInvPi;
        r.f_untinted = f3(kInvPi);
        return r;
    }
    if (lobe == kLobeConductor) {
        if (!same_hemi(wo, wi)) return r;
        const float cO = fabsf(wo.z), cI = fabsf(wi.z);
        if (cI == 0.0f || cO == 0.0f) return r;
        float3 wh = normalize_fast(wi + wo);
        if (is_black(wh)) return r;
        wh *= signf_ref(wh.z);
        const float3 Fr = fresnel_conductor(dot(wo, wh), m.ior, m.k);
        const Micro mf = make_micro(m);
        const float D = mf.D(wh), G = mf.G(wo, wi);
        r.f_untinted = Fr * D * G / (4.0f * cI * cO);
        r.f = r.f_untinted * m.specular;
        const float a = mf.ax;
        const float r2 = m.rough_x * m.rough_x;
        // alpha = max(r^2, 1e-3): dalpha/dr = 2r above the floor, 0 on it
        if (r2 > 1e-3f) {
            const float dla = mf.dist == 0u ? ggx_dlogD_dalpha(wh, a) -
                                                  (ggx_dlambda_dalpha(wo, a) + ggx_dlambda_dalpha(wi, a)) * G
                                            : beck_dlogD_dalpha(wh, a) -
                                                  (beck_dlambda_dalpha(wo, a) + beck_dlambda_dalpha(wi, a)) * G;
            r.dlogf_dr = dla * 2.0f * m.rough_x;
        }
    }
    return r;
}

// bilinear texel weights of direction `dir` in the evaluation env map
struct Bilerp {
    int idx[4];
    float w[4];
};
NB_D Bilerp env_weights(const AdjParams& P, const float3& dir) {
    const float u = spherical_phi(dir) * kInv2Pi, v = spherical_theta(dir) * kInvPi;
    const int W = P.env_w, H = P.env_h;
    const float x = u * (float)W - 0.5f, y = v * (float)H - 0.5f;
    const float fx0 = floorf(x), fy0 = floorf(y);
    const float ax = x - fx0, ay = y - fy0;
    int x0 = (int)fx0, y0 = (int)fy0, x1 = x0 + 1, y1 = y0 + 1;
    x0 = min(max(x0, 0), W - 1);
    x1 = min(max(x1, 0), W - 1);
    y0 = min(max(y0, 0), H - 1);
    y1 = min(max(y1, 0), H - 1);
    Bilerp b;
    b.idx[0] = y0 * W + x0;
    b.idx[1] = y0 * W + x1;
    b.idx[2] = y1 * W + x0;
    b.idx[3] = y1 * W + x1;
    b.w[0] = (1.0f - ax) * (1.0f - ay);
    b.w[1] = ax * (1.0f - ay);
    b.w[2] = (1.0f - ax) * ay;
    b.w[3] = ax * ay;
    return b;
}
NB_D float3 env_radiance(const AdjParams& P, const Bilerp& b) {
    float3 c = f3(0.0f);
    for (int k = 0; k < 4; ++k)
        c += b.w[k] * f3(P.env[3 * b.idx[k]], P.env[3 * b.idx[k] + 1], P.env[3 * b.idx[k] + 2]);
    return c;
}

// One term X (.) f * s of the estimator: X is light radiance (env texels
// when `env`), f the BSDF value at the vertex.
struct Term {
    float3 X;
    FDeriv f;
    float s;
    bool env;
    Bilerp bl;
    float xscale;   // light-count factor multiplying the env radiance
};

struct PathCtx {
    const DevScene& S;
    const AdjParams& P;
    const SmemStack& st;
    uint32_t* status;
};

// direct lighting at a vertex (sampleLight + sampleBSDF), occlusion traced;
// returns up to two terms
template <int ISECT>
NB_D int direct_terms(const PathCtx& C, const DevMaterial& m0, const DevMaterial& me, const Isect& I, Rng& rng,
                      Term* T) {
    const DevScene& S = C.S;
    int nt = 0;
    if (I.mtype & kSpecularMat) return 0;
    const int nl = S.sky_on ? S.num_lights : S.num_lights - 1;
    if (nl == 0) return 0;
    const int li = (int)((float)nl * rng.next());
    {
        float3 wi, to;
        float lpdf;
        // radiance from the sampling scene first (decides the early exits as
        // the primal does), evaluation radiance below
        const float3 Li0 = sample_li(S, I, rng, nl, li, wi, to, lpdf);
        if (lpdf != 0.0f && !is_black(Li0)) {
            const float3 f0 = bsdf_eval<false>(I.lobe, m0, I.F, I.wo, wi, kNonSpecular);
            if (!is_black(f0)) {
                const ShadowRay sr{spawn_origin(I, wi, S.bias), wi, 0.0f};
                const float tmax = length3(sr.o - to);
                if (!trace_any<ISECT, false>(S, sr.o, sr.d, tmax, C.st, C.status)) {
                    Term& t = T[nt++];
                    t.f = lobe_value(I.lobe, me, I.F, I.wo, wi);
                    float w = 1.0f;
                    if (S.mis) w = power_heuristic(lpdf, bsdf_pdf<false>(I.lobe, m0, I.F, I.wo, wi, kNonSpecular));
                    t.s = absdot(wi, I.F.n) * w / lpdf;
                    t.env = li >= S.num_area_lights && S.sky_type == NOOR_SKY_HDR;
                    t.xscale = (float)nl;
                    if (t.env) {
                        t.bl = env_weights(C.P, wi);
                        t.X = env_radiance(C.P, t.bl) * (float)nl;
                    } else {
                        t.X = Li0;
                    }
                }
            }
        }
    }
    if (!S.mis) return nt;
    rng.next();
    rng.next();
    float3 wi;
    float spdf;
    uint32_t stype;
    const float3 f0 = bsdf_sample<false>(I.lobe, m0, I.F, I.wo, kNonSpecular, rng, wi, spdf, stype);
    if (is_black(f0) || spdf == 0.0f) return nt;
    float w = 1.0f;
    if (!(stype & BSDF_SPECULAR)) {
        const float lp = light_pdf(S, I, li, wi);
        if (lp == 0.0f) return nt;
        w = power_heuristic(spdf, lp);
    }
    const float3 so = spawn_origin(I, wi, S.bias);
    float tm = 2.0f * S.world_radius;
    bool lh;
    float3 Le;
    const bool env = li >= S.num_area_lights;
    if (!env) {
        const DevAreaLight& A = S.area_lights[li];
        lh = quad_hit(A, so, wi, tm);
        Le = (A.two_sided || dot(wi, A.n) < 0.0f) ? A.ke : f3(0.0f);
    } else {
        lh = S.sky_on != 0;
        Le = S.sky_on ? env_eval<false>(S, wi) : f3(0.0f);
    }
    if (!lh || is_black(Le)) return nt;
    const float3 to = so + tm * wi;
    float3 vwi;
    visibility(I.p, to, vwi);
    const float3 so2 = spawn_origin(I, vwi, S.bias);
    if (trace_any<ISECT, false>(S, so2, vwi, length3(so2 - to), C.st, C.status)) return nt;
    Term& t = T[nt++];
    t.f = lobe_value(I.lobe, me, I.F, I.wo, wi);
    t.s = absdot(wi, I.F.n) * w / spdf;
    t.env = env && S.sky_type == NOOR_SKY_HDR;
    t.xscale = 1.0f;
    if (t.env) {
        t.bl = env_weights(C.P, wi);
        t.X = env_radiance(C.P, t.bl);
    } else {
        t.X = Le;
    }
    return nt;
}

NB_D float3 term_value(const Term& t) { return t.X * t.f.f * t.s; }

// gradient of beta (.) t with beta held fixed
NB_D void term_grad(const PathCtx& C, const Term& t, const float3& beta, const float3& dl, uint32_t mi, uint32_t lobe,
                    float* sm_alb, float* sm_rough) {
    const float3 g = dl * beta;  // dLoss/d(term) per channel
    const float3 xs = t.X * t.s;
    if (lobe == kLobeLambert || lobe == kLobeConductor) {
        const float3 da = g * xs * t.f.f_untinted;  // d/d albedo_c
        atomicAdd(&sm_alb[3 * mi + 0], da.x);
        atomicAdd(&sm_alb[3 * mi + 1], da.y);
        atomicAdd(&sm_alb[3 * mi + 2], da.z);
        if (lobe == kLobeConductor && t.f.dlogf_dr != 0.0f) {
            const float3 v = g * xs * t.f.f;
            atomicAdd(&sm_rough[mi], (v.x + v.y + v.z) * t.f.dlogf_dr);
        }
    }
    if (t.env) {
        const float3 ge = g * t.f.f * (t.s * t.xscale);
        for (int k = 0; k < 4; ++k) {
            if (t.bl.w[k] == 0.0f) continue;
            float* e = C.P.g_env + 3 * t.bl.idx[k];
            atomicAdd(e + 0, ge.x * t.bl.w[k]);
            atomicAdd(e + 1, ge.y * t.bl.w[k]);
            atomicAdd(e + 2, ge.z * t.bl.w[k]);
        }
    }
}

// One replay of a path.  MODE 0: return its radiance.  MODE 1: push
// dl (dLoss/dL) through the path, with Ltot its radiance from MODE 0.
template <int ISECT, int MODE>
NB_D float3 replay(const PathCtx& C, uint32_t pix, uint32_t frame, const DevCamera& cam, const float3& dl,
                   float3 Ltot, float* sm_alb, float* sm_rough) {
    const DevScene& S = C.S;
    Rng rng{tea16(pix, frame)};
    float3 o, d;
    camera_ray<false>(cam, pix % cam.w, pix / cam.w, rng, o, d);
    float3 L = f3(0.0f), beta = f3(1.0f);
    float3 Lrem = Ltot;
    bool spec = false;
    for (uint32_t bounce = 0; bounce < S.bounces; ++bounce) {
        float tmax = kInf;
        HitRec rec;
        if (!trace_closest<ISECT, false>(S, o, d, tmax, rec, C.st, C.status)) {
            if (S.sky_on && (bounce == 0 || spec)) {
                const float3 dir = normalize_fast(d);
                float3 Le;
                Bilerp bl;
                const bool env = S.sky_type == NOOR_SKY_HDR;
                if (env) {
                    bl = env_weights(C.P, dir);
                    Le = env_radiance(C.P, bl);
                } else {
                    Le = env_eval<false>(S, dir);
                }
                L += beta * Le;
                if (MODE == 1 && env) {
                    const float3 ge = dl * beta;
                    for (int k = 0; k < 4; ++k) {
                        if (bl.w[k] == 0.0f) continue;
                        float* e = C.P.g_env + 3 * bl.idx[k];
                        atomicAdd(e + 0, ge.x * bl.w[k]);
                        atomicAdd(e + 1, ge.y * bl.w[k]);
                        atomicAdd(e + 2, ge.z * bl.w[k]);
                    }
                }
            }
            break;
        }
        Isect I;
        make_isect<ISECT, false>(S, o, d, tmax, rec, I);
        if (I.mtype & kEmitterMat) {
            if (bounce == 0 || spec) {
                if (I.mtype & NOOR_MESHLIGHT) {
                    const DevAreaLight& A = S.area_lights[rec.ins];
                    L += beta * ((A.two_sided || dot(d, A.n) < 0.0f) ? A.ke : f3(0.0f));
                } else {
                    const DevMaterial& em = S.materials[I.mat];
                    L += beta * (em.emitter_scale * em.emittance);
                }
            }
            break;
        }
        const DevMaterial m0 = S.materials[I.mat];
        const DevMaterial me = eval_material(m0, C.P, I.mat);
        Term T[2];
        const int nt = direct_terms<ISECT>(C, m0, me, I, rng, T);
        float3 Ld = f3(0.0f);
        for (int k = 0; k < nt; ++k) Ld += term_value(T[k]);
        const float3 contrib = beta * Ld;
        L += contrib;
        if (MODE == 1) {
            for (int k = 0; k < nt; ++k) term_grad(C, T[k], beta, dl, I.mat, I.lobe, sm_alb, sm_rough);
            Lrem = Lrem - contrib;
        }
        rng.next();
        rng.next();
        float3 wi;
        float pdf;
        uint32_t stype;
        const float3 f0 = bsdf_sample<false>(I.lobe, m0, I.F, I.wo, BSDF_ALL, rng, wi, pdf, stype);
        if (pdf == 0.0f) break;
        float3 fe;
        FDeriv fd{f3(0.0f), f3(0.0f), 0.0f};
        if (stype & BSDF_SPECULAR) {
            fe = f0;  // specular lobes carry no differentiable parameter here
        } else {
            fd = lobe_value(I.lobe, me, I.F, I.wo, wi);
            fe = fd.f;
        }
        if (MODE == 1 && !(stype & BSDF_SPECULAR)) {
            // Lrem scales with f at this vertex
            const float3 g = dl * Lrem;
            if (I.lobe == kLobeLambert || I.lobe == kLobeConductor) {
                const float3 da = f3(fe.x != 0.0f ? g.x * fd.f_untinted.x / fe.x : 0.0f,
                                     fe.y != 0.0f ? g.y * fd.f_untinted.y / fe.y : 0.0f,
                                     fe.z != 0.0f ? g.z * fd.f_untinted.z / fe.z : 0.0f);
                atomicAdd(&sm_alb[3 * I.mat + 0], da.x);
                atomicAdd(&sm_alb[3 * I.mat + 1], da.y);
                atomicAdd(&sm_alb[3 * I.mat + 2], da.z);
                if (I.lobe == kLobeConductor && fd.dlogf_dr != 0.0f)
                    atomicAdd(&sm_rough[I.mat], (g.x + g.y + g.z) * fd.dlogf_dr);
            }
        }
        beta *= fe * absdot(wi, I.F.n) / pdf;
        if (!(I.mtype & kTransparentMat) && dot(wi, I.F.ng) < 0.0f) break;
        spec = (I.mtype & kSpecularMat) != 0;
        o = spawn_origin(I, wi, S.bias);
        d = wi;
    }
    return L;
}

constexpr int kAdjBlock = 128;
constexpr int kAdjMaxMats = 256;
// samples per pass: the per-sample radiance of a chunk (npix x kAdjChunk
// float4) is the only buffer that grows with the sample count
constexpr uint32_t kAdjChunk = 4;

// Work items of a chunk: item i = (sample c0 + i / npix, pixel i % npix), so
// the lanes of a warp trace neighbouring pixels of one sample.

// Radiance of every path of a chunk (the MODE 0 replay), unclamped
template <int ISECT>
__global__ void __launch_bounds__(kAdjBlock) adj_radiance(DevScene S, DevCamera cam, AdjParams P, uint32_t c0,
                                                          uint32_t nc, float4* Lbuf) {
    extern __shared__ uint32_t smem[];
    const uint32_t npix = cam.w * cam.h;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npix * nc) return;
    const uint32_t pix = i % npix, s = c0 + i / npix;
    SmemStack st{smem + threadIdx.x, (int)blockDim.x, S.stack_cap};
    const PathCtx ctx{S, P, st, P.status};
    const float3 L = replay<ISECT, 0>(ctx, pix, P.frame0 + s, cam, f3(0.0f), f3(0.0f), nullptr, nullptr);
    Lbuf[i] = make_float4(L.x, L.y, L.z, 0.0f);
}

// Forward: each pixel's clamped samples added in sample order with Kahan's
// compensation (the state carried across chunks); the last chunk writes the
// mean
__global__ void adj_accumulate(uint32_t npix, uint32_t nc, const float4* Lbuf, float4* kahan, int first, int last,
                               float inv_spp, float* image) {
    const uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x;
    if (pix >= npix) return;
    float3 sum = f3(0.0f), comp = f3(0.0f);
    if (!first) {
        sum = f3(kahan[2 * pix]);
        comp = f3(kahan[2 * pix + 1]);
    }
    for (uint32_t c = 0; c < nc; ++c) {
        const float3 Lc = clamp3(f3(Lbuf[(size_t)c * npix + pix]), 0.0f, 100.0f);
        const float3 y = Lc - comp;
        const float3 t = sum + y;
        comp = (t - sum) - y;
        sum = t;
    }
    if (last) {
        image[3 * pix + 0] = sum.x * inv_spp;
        image[3 * pix + 1] = sum.y * inv_spp;
        image[3 * pix + 2] = sum.z * inv_spp;
    } else {
        kahan[2 * pix] = make_float4(sum.x, sum.y, sum.z, 0.0f);
        kahan[2 * pix + 1] = make_float4(comp.x, comp.y, comp.z, 0.0f);
    }
}

// Backward: for every path of a chunk, dLoss/dL through the final clamp,
// then the MODE 1 replay pushes it to the parameters.  Resident blocks loop
// over the items, so each block adds its material gradients (accumulated in
// shared memory) to the global ones once.
template <int ISECT>
__global__ void __launch_bounds__(kAdjBlock) adj_gradient(DevScene S, DevCamera cam, AdjParams P, uint32_t c0,
                                                          uint32_t nc, const float4* Lbuf) {
    extern __shared__ uint32_t smem[];
    __shared__ float sm_alb[3 * kAdjMaxMats];
    __shared__ float sm_rough[kAdjMaxMats];
    for (int i = threadIdx.x; i < 3 * kAdjMaxMats; i += blockDim.x) sm_alb[i] = 0.0f;
    for (int i = threadIdx.x; i < kAdjMaxMats; i += blockDim.x) sm_rough[i] = 0.0f;
    __syncthreads();
    const uint32_t npix = cam.w * cam.h;
    SmemStack st{smem + threadIdx.x, (int)blockDim.x, S.stack_cap};
    const PathCtx ctx{S, P, st, P.status};
    const float inv_spp = 1.0f / (float)P.spp;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npix * nc; i += gridDim.x * blockDim.x) {
        const uint32_t pix = i % npix, s = c0 + i / npix;
        const float3 gi = f3(P.grad_img[3 * pix], P.grad_img[3 * pix + 1], P.grad_img[3 * pix + 2]) * inv_spp;
        const float3 L = f3(Lbuf[i]);
        // derivative of the final clamp to [0, 100]
        const float3 dl = f3(L.x > 0.0f && L.x < 100.0f ? gi.x : 0.0f, L.y > 0.0f && L.y < 100.0f ? gi.y : 0.0f,
                             L.z > 0.0f && L.z < 100.0f ? gi.z : 0.0f);
        if (is_black(dl)) continue;
        replay<ISECT, 1>(ctx, pix, P.frame0 + s, cam, dl, L, sm_alb, sm_rough);
    }
    __syncthreads();
    const uint32_t nm = min(P.num_mats, (uint32_t)kAdjMaxMats);
    for (uint32_t i = threadIdx.x; i < 3 * nm; i += blockDim.x)
        if (sm_alb[i] != 0.0f) atomicAdd(&P.g_albedo[i], sm_alb[i]);
    for (uint32_t i = threadIdx.x; i < nm; i += blockDim.x)
        if (sm_rough[i] != 0.0f) atomicAdd(&P.g_rough[i], sm_rough[i]);
}

static int adjoint_run(const noor_adjoint_desc* desc, int mode, float* image, const float* grad_img, float* g_alb,
                       float* g_rough, float* g_env) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    if (!desc || !desc->d_albedo || !desc->d_roughness) return set_error(NOOR_ERR_INVALID, "adjoint: null buffer");
    if (desc->spp == 0) return set_error(NOOR_ERR_INVALID, "adjoint: spp must be positive");
    SceneState& st = *C->scenes[0];
    DevScene S = st.dev;
    if (desc->bounces) S.bounces = desc->bounces;
    if (S.rr < S.bounces)
        return set_error(NOOR_ERR_INVALID, "adjoint: Russian roulette must be off (spec.rr >= bounces)");
    if (st.materials_host.size() > (size_t)kAdjMaxMats)
        return set_error(NOOR_ERR_CAPACITY, "adjoint: at most 256 materials");
    // the estimator is differentiated for Lambert and conductor lobes; glass
    // (specular, no parameter) and emitters pass through
    for (const auto& m : st.materials_host) {
        const uint32_t l = lobe_of(m.type);
        if (!(m.type & (NOOR_EMITTER | NOOR_MESHLIGHT)) && l != kLobeLambert && l != kLobeConductor &&
            l != kLobeFresnelSpec)
            return set_error(NOOR_ERR_UNSUPPORTED, "adjoint: materials other than diffuse, metal and glass");
        if (m.tex_mask)
            return set_error(NOOR_ERR_UNSUPPORTED, "adjoint: textured, alpha-cut or bump-mapped materials");
    }
    if (C->cam.type != NOOR_CAMERA_PERSP || C->cam.lens_radius > 0.0f)
        return set_error(NOOR_ERR_UNSUPPORTED, "adjoint: cameras other than the pinhole");
    if (!st.quad_lights_only || S.num_delta_lights > 0)
        return set_error(NOOR_ERR_UNSUPPORTED, "adjoint: lights other than quad area lights and the sky");
    if (st.dev.env_ref)
        return set_error(NOOR_ERR_UNSUPPORTED, "adjoint: the reference's environment sampling (NOOR_ENV_REFERENCE)");
    if (S.sky_type == NOOR_SKY_HDR && (!desc->d_env || (mode == 1 && !g_env)))
        return set_error(NOOR_ERR_INVALID, "adjoint: env buffer missing");
    if (desc->width != C->cam.w || desc->height != C->cam.h)
        return set_error(NOOR_ERR_INVALID, "adjoint: image size differs from the camera's");
    AdjParams P{};
    P.albedo = desc->d_albedo;
    P.rough = desc->d_roughness;
    P.env = desc->d_env;
    P.env_w = S.env_w;
    P.env_h = S.env_h;
    P.image = image;
    P.grad_img = grad_img;
    P.g_albedo = g_alb;
    P.g_rough = g_rough;
    P.g_env = g_env;
    P.num_mats = (uint32_t)st.materials_host.size();
    P.spp = desc->spp;
    P.frame0 = desc->first_frame ? desc->first_frame : 1;
    P.status = C->status;
    const uint32_t npix = C->cam.w * C->cam.h;
    const size_t sm = (size_t)S.stack_cap * kAdjBlock * 4;
    // buffers: per-sample radiance of one chunk, and (forward) the Kahan
    // state per pixel across chunks; kept in the context between calls
    const uint32_t chunk = std::min<uint32_t>(P.spp, kAdjChunk);
    const size_t need = ((size_t)chunk + 2) * npix * sizeof(float4);
    cudaError_t e = cudaSuccess;
    if (C->adj_bytes < need) {
        if (C->adj_buf) cudaFree(C->adj_buf);
        C->adj_buf = nullptr;
        C->adj_bytes = 0;
        e = cudaMalloc(&C->adj_buf, need);
        if (e != cudaSuccess) return cuda_fail(e, "adjoint buffers");
        C->adj_bytes = need;
    }
    float4* Lbuf = static_cast<float4*>(C->adj_buf);
    float4* kahan = Lbuf + (size_t)chunk * npix;
    using RadKernel = void (*)(DevScene, DevCamera, AdjParams, uint32_t, uint32_t, float4*);
    using GradKernel = void (*)(DevScene, DevCamera, AdjParams, uint32_t, uint32_t, const float4*);
    const bool wt = S.isect == NOOR_ISECT_WATERTIGHT;
    const RadKernel kr = wt ? adj_radiance<NOOR_ISECT_WATERTIGHT> : adj_radiance<NOOR_ISECT_REF_WALD>;
    const GradKernel kg = wt ? adj_gradient<NOOR_ISECT_WATERTIGHT> : adj_gradient<NOOR_ISECT_REF_WALD>;
    e = cudaFuncSetAttribute(kr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(kg, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    int per_sm = 1;
    if (e == cudaSuccess && mode == 1) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kg, kAdjBlock, sm);
    if (e != cudaSuccess) return cuda_fail(e, "adjoint setup");
    const uint32_t grid_g = (uint32_t)std::max(1, per_sm) * (uint32_t)std::max(1, C->sm_count);
    for (uint32_t c0 = 0; c0 < P.spp && e == cudaSuccess; c0 += chunk) {
        const uint32_t nc = std::min(chunk, P.spp - c0);
        kr<<<(npix * nc + kAdjBlock - 1) / kAdjBlock, kAdjBlock, sm, C->stream>>>(S, C->cam, P, c0, nc, Lbuf);
        if (mode == 0)
            adj_accumulate<<<(npix + 255) / 256, 256, 0, C->stream>>>(npix, nc, Lbuf, kahan, c0 == 0,
                                                                      c0 + nc >= P.spp, 1.0f / (float)P.spp, image);
        else
            kg<<<grid_g, kAdjBlock, sm, C->stream>>>(S, C->cam, P, c0, nc, Lbuf);
        e = cudaGetLastError();
        C->launches += 2;
    }
    if (e != cudaSuccess) return cuda_fail(e, "adjoint");
    return sync_and_check(*C, "adjoint");
}

}  // namespace nb

using namespace nb;

extern "C" int noor_adjoint_forward(const noor_adjoint_desc* desc, float* d_image) {
    if (!d_image) return set_error(NOOR_ERR_INVALID, "adjoint: null image");
    return adjoint_run(desc, 0, d_image, nullptr, nullptr, nullptr, nullptr);
}

extern "C" int noor_adjoint_backward(const noor_adjoint_desc* desc, const float* d_grad_image, float* d_grad_albedo,
                                     float* d_grad_roughness, float* d_grad_env) {
    if (!d_grad_image || !d_grad_albedo || !d_grad_roughness)
        return set_error(NOOR_ERR_INVALID, "adjoint: null gradient buffer");
    return adjoint_run(desc, 1, nullptr, d_grad_image, d_grad_albedo, d_grad_roughness, d_grad_env);
}
