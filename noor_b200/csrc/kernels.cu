// Render and parity kernels: the plain megakernel (one path per
// (pixel, frame), noor/cuda/path_tracer.cu:77-100), the film fold, ray-batch
// traversal and the device-routine evaluators used by the parity tests.
#include "kernels.h"
#include "integrator.cuh"

namespace nb {

// warp-aggregated add of per-lane counts into a 64-bit device counter
NB_D void warp_count(unsigned long long* ctr, uint32_t v) {
    const uint32_t mask = __activemask();
    const uint32_t s = __reduce_add_sync(mask, v);
    const int leader = __ffs(mask) - 1;
    if ((int)(threadIdx.x & 31) == leader && s) atomicAdd(ctr, (unsigned long long)s);
}

NB_D void kahan_add(float3& sum, float3& c, const float3& x) {
    const float3 y = x - c;
    const float3 t = sum + y;
    c = (t - sum) - y;
    sum = t;
}

// minimum resident blocks per SM the megakernel is compiled for: 7 caps its
// registers at 65536 / (128 * 7) = 73, i.e. 28 warps per SM instead of 12
// at its natural ~155 registers; the traversal is latency-bound, so the
// occupancy is worth the spilled values (measured faster on the sky-lit
// 2.6M-triangle scene than 5 or 6)
#ifndef NB_MEGA_MIN_BLOCKS
#define NB_MEGA_MIN_BLOCKS 7
#endif

template <int ISECT, int FILM, bool EXT, bool DIFF = false>
__global__ void __launch_bounds__(kMegaBlock, NB_MEGA_MIN_BLOCKS) megakernel(DevScene S, DevCamera C, MegaArgs a) {
    extern __shared__ uint32_t smem[];
    const uint32_t npix = C.w * C.h;
    const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t pix = idx % npix;
    const uint32_t chunk = idx / npix;
    RayStats rs{0u, 0u};
    uint32_t paths = 0;
    if (chunk < a.chunks) {
        const uint32_t per = (a.nframes + a.chunks - 1) / a.chunks;
        const uint32_t fb = chunk * per;
        const uint32_t fe = min(fb + per, a.nframes);
        SmemStack st{smem + threadIdx.x, (int)blockDim.x, S.stack_cap};
        const uint32_t x = pix % C.w, y = pix / C.w;
        float3 sum = f3(0.0f), comp = f3(0.0f);
        float4 mean = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
        if (a.chunks == 1u && !a.fresh) {
            if (FILM == NOOR_FILM_KAHAN) {
                sum = f3(a.film_sum[pix]);
                comp = f3(a.film_comp[pix]);
            } else {
                mean = a.film_sum[pix];
            }
        }
        float3 hitp = f3(0.0f);
        bool hit_valid = false;
        const bool want_hit = (pix == C.center) && (chunk == a.chunks - 1u);
        for (uint32_t f = fb; f < fe; ++f) {
            const uint32_t frame = a.frame0 + f;
            Rng rng{tea16(pix, frame)};
            float3 o, d;
            RayDiff rd{};
            if (DIFF)
                camera_ray_diff(C, x, y, rng, o, d, rd);
            else
                camera_ray<EXT>(C, x, y, rng, o, d);
            hit_valid = false;
            const float3 L = path_radiance<ISECT, EXT, DIFF>(S, o, d, rng, st, a.status, rs,
                                                             want_hit ? &hitp : nullptr, &hit_valid, rd);
            ++paths;
            if (FILM == NOOR_FILM_KAHAN) {
                kahan_add(sum, comp, L);
            } else {
                // framebuffer.set: lerp(old, new, 1/frame) (framebuffer.cuh:72-76)
                const float4 old = frame > 1u ? mean : make_float4(0.0f, 0.0f, 0.0f, 1.0f);
                const float t = 1.0f / (float)frame;
                mean = make_float4(old.x + t * (L.x - old.x), old.y + t * (L.y - old.y), old.z + t * (L.z - old.z),
                                   old.w + t * (1.0f - old.w));
            }
        }
        if (a.chunks == 1u) {
            if (FILM == NOOR_FILM_KAHAN) {
                a.film_sum[pix] = make_float4(sum.x, sum.y, sum.z, 1.0f);
                a.film_comp[pix] = make_float4(comp.x, comp.y, comp.z, 0.0f);
            } else {
                a.film_sum[pix] = mean;
            }
        } else {
            const size_t o = (size_t)chunk * npix + pix;
            a.part_sum[o] = make_float4(sum.x, sum.y, sum.z, 0.0f);
            a.part_comp[o] = make_float4(comp.x, comp.y, comp.z, 0.0f);
        }
        if (want_hit) *a.lookat = make_float4(hitp.x, hitp.y, hitp.z, hit_valid ? 1.0f : 0.0f);
    }
    warp_count(a.counters + 0, rs.ext);
    warp_count(a.counters + 1, rs.shadow);
    warp_count(a.counters + 2, paths);
}

// folds the per-chunk partial sums into the Kahan film in chunk order
__global__ void fold_partials(uint32_t npix, uint32_t chunks, uint32_t fresh, float4* film_sum, float4* film_comp,
                              const float4* part_sum, const float4* part_comp) {
    const uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x;
    if (pix >= npix) return;
    float3 sum = f3(0.0f), comp = f3(0.0f);
    if (!fresh) {
        sum = f3(film_sum[pix]);
        comp = f3(film_comp[pix]);
    }
    for (uint32_t c = 0; c < chunks; ++c) {
        const size_t o = (size_t)c * npix + pix;
        kahan_add(sum, comp, f3(part_sum[o]));
        kahan_add(sum, comp, -1.0f * f3(part_comp[o]));
    }
    film_sum[pix] = make_float4(sum.x, sum.y, sum.z, 1.0f);
    film_comp[pix] = make_float4(comp.x, comp.y, comp.z, 0.0f);
}

// film -> mean rgba
__global__ void film_resolve(uint32_t npix, int mode, float inv_count, const float4* film_sum, float4* out) {
    const uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x;
    if (pix >= npix) return;
    const float4 s = film_sum[pix];
    out[pix] = mode == NOOR_FILM_KAHAN ? make_float4(s.x * inv_count, s.y * inv_count, s.z * inv_count, 1.0f) : s;
}

template <int ISECT, bool WIDE>
__global__ void __launch_bounds__(kTraceBlock) k_trace_closest(DevScene S, const noor_ray* rays, noor_hit* hits,
                                                               size_t n, uint32_t* status) {
    extern __shared__ uint32_t smem[];
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    SmemStack st{smem + threadIdx.x, (int)blockDim.x, S.stack_cap};
    const noor_ray r = rays[i];
    float tmax = r.tmax;
    HitRec rec{0.0f, 0.0f, 0u, 0u, 0u};
    const bool h = trace_primary<ISECT, true, WIDE>(S, f3(r.org[0], r.org[1], r.org[2]), f3(r.dir[0], r.dir[1], r.dir[2]),
                                        tmax, rec, st, status);
    noor_hit o;
    o.t = tmax;
    o.tri_idx = rec.tri;
    o.ins_idx = rec.ins;
    o.material_type = rec.mtype;
    o.u = rec.u;
    o.v = rec.v;
    o.hit = h ? 1u : 0u;
    o.pad = 0u;
    hits[i] = o;
}

template <int ISECT, bool WIDE>
__global__ void __launch_bounds__(kTraceBlock) k_trace_any(DevScene S, const noor_ray* rays, uint32_t* occ,
                                                           size_t n, uint32_t* status) {
    extern __shared__ uint32_t smem[];
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    SmemStack st{smem + threadIdx.x, (int)blockDim.x, S.stack_cap};
    const noor_ray r = rays[i];
    occ[i] = trace_shadow<ISECT, true, WIDE>(S, f3(r.org[0], r.org[1], r.org[2]), f3(r.dir[0], r.dir[1], r.dir[2]),
                                             r.tmax, st, status)
                 ? 1u
                 : 0u;
}

__global__ void k_camera_rays(DevCamera C, uint32_t frame, noor_ray* rays) {
    const uint32_t npix = C.w * C.h;
    const uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x;
    if (pix >= npix) return;
    Rng rng{tea16(pix, frame)};
    float3 o, d;
    camera_ray(C, pix % C.w, pix / C.w, rng, o, d);
    noor_ray r;
    r.org[0] = o.x;
    r.org[1] = o.y;
    r.org[2] = o.z;
    r.tmax = kInf;
    r.dir[0] = d.x;
    r.dir[1] = d.y;
    r.dir[2] = d.z;
    r.pad = 0.0f;
    rays[pix] = r;
}

// in: {wo[3], wi[3], u[2], mat, 0..} (16 floats) in the local frame whose
// geometric and shading normals are +z; out: {f[3], pdf, wi[3], type}
__global__ void k_eval_bsdf(DevScene S, int kind, const float* in, float* out, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* p = in + 16 * i;
    const float3 wo = f3(p[0], p[1], p[2]);
    const float3 wi = f3(p[3], p[4], p[5]);
    const uint32_t mi = (uint32_t)p[8];
    const DevMaterial m = S.materials[mi];
    Frame F;
    F.n = f3(0.0f, 0.0f, 1.0f);
    F.ng = F.n;
    F.s = f3(1.0f, 0.0f, 0.0f);
    F.t = f3(0.0f, 1.0f, 0.0f);
    const uint32_t lobe = lobe_of(m.type);
    float* q = out + 8 * i;
    float3 f = f3(0.0f), wo_s = f3(0.0f);
    float pdf = 0.0f;
    uint32_t st = 0;
    if (kind == 0) {
        f = bsdf_eval(lobe, m, F, wo, wi, BSDF_ALL);
    } else if (kind == 1) {
        pdf = bsdf_pdf(lobe, m, F, wo, wi, BSDF_ALL);
    } else {
        // the BSDF's Sample_f with its two uniforms given (no RNG)
        float3 w = f3(0.0f);
        f = bsdf_sample_u(lobe, m, F, wo, BSDF_ALL, p[6], p[7], w, pdf, st);
        if (pdf != 0.0f) wo_s = w;
    }
    q[0] = f.x;
    q[1] = f.y;
    q[2] = f.z;
    q[3] = pdf;
    q[4] = wo_s.x;
    q[5] = wo_s.y;
    q[6] = wo_s.z;
    q[7] = (float)st;
}

// Stand-alone shading routines for parity tests; record layouts in
// include/noor_b200.h (noor_eval_routines).
__global__ void k_eval_routines(int kind, const float* in, float* out, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (kind <= 1) {
        const float* p = in + 12 * i;
        float* q = out + 12 * i;
        Micro m;
        m.ax = fmaxf(p[0] * p[0], 1e-3f);
        m.ay = fmaxf(p[1] * p[1], 1e-3f);
        m.dist = (uint32_t)kind;
        const float3 wo = f3(p[2], p[3], p[4]), wh = f3(p[5], p[6], p[7]);
        const float3 s = m.sample_wh(wo, p[8], p[9]);
        const float r[12] = {m.D(wh), m.G(wo, wh), m.pdf(wo, wh), s.x, s.y, s.z, 0.0f, m.ax, 0.0f, 0.0f, 0.0f, 0.0f};
        for (int k = 0; k < 12; ++k) q[k] = r[k];
    } else if (kind == 2) {
        const float* p = in + 9 * i;
        float* q = out + 4 * i;
        q[0] = fresnel_dielectric(p[0], p[1], p[2]);
        const float3 c = fresnel_conductor(p[0], f3(p[3], p[4], p[5]), f3(p[6], p[7], p[8]));
        q[1] = c.x;
        q[2] = c.y;
        q[3] = c.z;
    } else {
        const float* p = in + 3 * i;
        float* q = out + 16 * i;
        const float2 d = concentric_disk(p[0], p[1]);
        const float3 c = cosine_hemisphere(p[0], p[1]);
        float st;
        const float3 sd = spherical_direction(p[0], p[1], st);
        const float3 h = uniform_hemisphere(p[0], p[1]);
        const float r[16] = {d.x, d.y, c.x, c.y, c.z, h.x, h.y, h.z, sd.x, sd.y, sd.z, st,
                             power_heuristic(p[0], p[1]), erf_as(p[2]), erfinv_giles(p[2]), 0.0f};
        for (int k = 0; k < 16; ++k) q[k] = r[k];
    }
}

__global__ void k_eval_sky(DevScene S, const float* dirs, float* rgb, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float3 c = env_eval<true>(S, f3(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]));
    rgb[3 * i] = c.x;
    rgb[3 * i + 1] = c.y;
    rgb[3 * i + 2] = c.z;
}

// u -> {x, y, pdf_sample, pdf_eval}
__global__ void k_env_sample(DevScene S, const float* u, float* out, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float pdf;
    const float2 xy = S.env_ref ? rdist_sample(S, u[2 * i], u[2 * i + 1], pdf) : dist_sample(S.dist, u[2 * i], u[2 * i + 1], pdf);
    out[4 * i] = xy.x;
    out[4 * i + 1] = xy.y;
    out[4 * i + 2] = pdf;
    out[4 * i + 3] = S.env_ref ? rdist_pdf(S, xy.x, xy.y) : dist_pdf(S.dist, xy.x, xy.y);
}

// debug_skydome_kernel (noor/cuda/path_tracer.cu:102-122)
__global__ void k_debug_skydome(DevScene S, DevCamera C, uint32_t frame, float4* film, int mis) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= C.w || y >= C.h) return;
    const uint32_t id = y * C.w + x;
    const float u = x / (float)C.w, v = y / (float)C.h;
    float3 c;
    if (S.sky_type == NOOR_SKY_PHYSICAL) {
        float3 dir = f3(sinf(v * kPi) * cosf(u * k2Pi), cosf(v * kPi), sinf(v * kPi) * sinf(u * k2Pi));
        c = sinf(v * kPi) * hosek_query(S.hosek, normalize_fast(dir));
    } else {
        c = env_bilinear(S, u, v);
    }
    film[id] = make_float4(c.x, c.y, c.z, 1.0f);
    if (mis) {
        Rng rng{tea16(id, frame)};
        const float a = rng.next();
        const float b = rng.next();
        float pdf;
        const float2 s = dist_sample(S.dist, a, b, pdf);
        const uint32_t px = min((uint32_t)(s.x * C.w), C.w - 1), py = min((uint32_t)(s.y * C.h), C.h - 1);
        film[py * C.w + px] = make_float4(1.0f, 0.0f, 0.0f, 1.0f);
    }
}

// ------------------------------------------------------------ launchers
static size_t stack_bytes(const DevScene& S, int block) { return (size_t)S.stack_cap * block * sizeof(uint32_t); }

cudaError_t launch_megakernel(const DevScene& S, const DevCamera& C, const MegaArgs& a, cudaStream_t s) {
    const uint32_t npix = C.w * C.h;
    const uint64_t threads = (uint64_t)npix * a.chunks;
    const uint32_t grid = (uint32_t)((threads + kMegaBlock - 1) / kMegaBlock);
    const size_t sm = stack_bytes(S, kMegaBlock);
    cudaError_t e;
    // scenes without the extra lobes and lights, seen through a pinhole, run
    // a specialisation without the other code (the kernel's registers are
    // capped, so unused branches cost spills)
    const bool ext_cam = C.type != NOOR_CAMERA_PERSP || C.lens_radius > 0.0f;
#define NB_MK2(I, F, X, D)                                                                      \
    do {                                                                                        \
        e = cudaFuncSetAttribute(megakernel<I, F, X, D>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm); \
        if (e != cudaSuccess) return e;                                                         \
        megakernel<I, F, X, D><<<grid, kMegaBlock, sm, s>>>(S, C, a);                           \
    } while (0)
#define NB_MK(I, F)                     \
    do {                                \
        if (S.has_bump) NB_MK2(I, F, true, true); \
        else if (S.ext_lobes || S.ext_lights || S.env_ref || S.has_tex || ext_cam) NB_MK2(I, F, true, false); \
        else NB_MK2(I, F, false, false); \
    } while (0)
    if (S.isect == NOOR_ISECT_WATERTIGHT) {
        if (S.film_mode == NOOR_FILM_KAHAN) NB_MK(NOOR_ISECT_WATERTIGHT, NOOR_FILM_KAHAN);
        else NB_MK(NOOR_ISECT_WATERTIGHT, NOOR_FILM_REF_LERP);
    } else {
        if (S.film_mode == NOOR_FILM_KAHAN) NB_MK(NOOR_ISECT_REF_WALD, NOOR_FILM_KAHAN);
        else NB_MK(NOOR_ISECT_REF_WALD, NOOR_FILM_REF_LERP);
    }
#undef NB_MK
#undef NB_MK2
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (a.chunks > 1u) {
        fold_partials<<<(npix + 255) / 256, 256, 0, s>>>(npix, a.chunks, a.fresh, a.film_sum, a.film_comp,
                                                          a.part_sum, a.part_comp);
        e = cudaGetLastError();
    }
    return e;
}

cudaError_t launch_resolve(uint32_t npix, int mode, float inv_count, const float4* film_sum, float4* out,
                           cudaStream_t s) {
    film_resolve<<<(npix + 255) / 256, 256, 0, s>>>(npix, mode, inv_count, film_sum, out);
    return cudaGetLastError();
}

// one launch of a ray-batch kernel: the four-wide or the binary traversal,
// per intersector
template <template <int, bool> class K, class T>
static cudaError_t launch_trace(const DevScene& S, bool wide, const noor_ray* rays, T* out, size_t n,
                                uint32_t* status, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    // room for the four-wide tree's stacks as well as the binary one's
    const size_t sm = (size_t)S.stack_words * kTraceBlock * sizeof(uint32_t);
    const uint32_t grid = (uint32_t)((n + kTraceBlock - 1) / kTraceBlock);
    auto go = [&](auto kern) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        kern<<<grid, kTraceBlock, sm, s>>>(S, rays, out, n, status);
        return cudaGetLastError();
    };
    if (S.isect == NOOR_ISECT_WATERTIGHT)
        return wide ? go(K<NOOR_ISECT_WATERTIGHT, true>::fn) : go(K<NOOR_ISECT_WATERTIGHT, false>::fn);
    return wide ? go(K<NOOR_ISECT_REF_WALD, true>::fn) : go(K<NOOR_ISECT_REF_WALD, false>::fn);
}
template <int I, bool W>
struct ClosestK {
    static constexpr auto fn = k_trace_closest<I, W>;
};
template <int I, bool W>
struct AnyK {
    static constexpr auto fn = k_trace_any<I, W>;
};

cudaError_t launch_trace_closest(const DevScene& S, const noor_ray* rays, noor_hit* hits, size_t n, uint32_t* status,
                                 cudaStream_t s) {
    return launch_trace<ClosestK>(S, S.closest4 != 0u, rays, hits, n, status, s);
}

cudaError_t launch_trace_any(const DevScene& S, const noor_ray* rays, uint32_t* occ, size_t n, uint32_t* status,
                             cudaStream_t s) {
    return launch_trace<AnyK>(S, S.nodes4 != nullptr, rays, occ, n, status, s);
}

cudaError_t launch_camera_rays(const DevCamera& C, uint32_t frame, noor_ray* rays, cudaStream_t s) {
    const uint32_t npix = C.w * C.h;
    k_camera_rays<<<(npix + 255) / 256, 256, 0, s>>>(C, frame, rays);
    return cudaGetLastError();
}

cudaError_t launch_eval_bsdf(const DevScene& S, int kind, const float* in, float* out, size_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_eval_bsdf<<<(uint32_t)((n + 255) / 256), 256, 0, s>>>(S, kind, in, out, n);
    return cudaGetLastError();
}

cudaError_t launch_eval_routines(int kind, const float* in, float* out, size_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_eval_routines<<<(uint32_t)((n + 255) / 256), 256, 0, s>>>(kind, in, out, n);
    return cudaGetLastError();
}

cudaError_t launch_eval_sky(const DevScene& S, const float* dirs, float* rgb, size_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_eval_sky<<<(uint32_t)((n + 255) / 256), 256, 0, s>>>(S, dirs, rgb, n);
    return cudaGetLastError();
}

cudaError_t launch_env_sample(const DevScene& S, const float* u, float* out, size_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_env_sample<<<(uint32_t)((n + 255) / 256), 256, 0, s>>>(S, u, out, n);
    return cudaGetLastError();
}

cudaError_t launch_debug_skydome(const DevScene& S, const DevCamera& C, uint32_t frame, float4* film, int mis,
                                 cudaStream_t s) {
    dim3 b(16, 16), g((C.w + 15) / 16, (C.h + 15) / 16);
    k_debug_skydome<<<g, b, 0, s>>>(S, C, frame, film, mis);
    return cudaGetLastError();
}

}  // namespace nb
