// ORACLE -- test infrastructure, not product code.
//
// The reference's own device routines (noor/cuda/*.cuh), compiled UNMODIFIED
// from the reference tree by nvcc for sm_100a into oracle/_ref/libnoor_refdev.so
// (oracle/Makefile, target `refdev`), behind C entry points that the tests and
// tests/golden/make_refdev_golden.py call.  Only tests/ and the fixture
// script use it; it is the checker, never the thing measured.
//
// What is the reference's code and what is the harness's:
//   * every routine evaluated below -- CudaRNG, the microfacet distributions,
//     Fresnel terms, the sampling warps, querySkyModel, the BVH traversal and
//     Wald triangle test, generateRay, CudaIntersection, factoryBSDF and the
//     CudaBSDF Eval/Pdf/Sample_f, the light manager, the sky dome and its
//     CudaDistribution2D, accumulate/scatter/correct_sidedness/rr_terminate,
//     the framebuffer's running mean -- and every manager constructor is the
//     reference's source, included from the reference tree;
//   * prelude.h restates the non-GL part of path_tracer.cuh, shim/ supplies
//     helper_math.h; path_tracer.cuh, path_tracer_data.cuh, render.cuh and
//     path_tracer.cu are not compiled (they open GL, GLEW and CUDA-Samples
//     headers);
//   * k_render restates path_tracer_kernel and pathtracer()
//     (noor/cuda/path_tracer.cu:26-100) statement for statement, minus the
//     look-at write; harness_load restates CudaRenderDevice's constructor
//     (noor/cuda/render.cuh:62-110) without GL;
//   * prescan (noor/cuda/distribution2d.cuh:86-135) is restated: its bank
//     offset macro CONFLICT_FREE_OFFSET(n) expands to n >> (32 + n) >> 10, a
//     shift by 32 or more, undefined in C++; on the hardware a 32-bit shift
//     by 32 or more gives 0 for the non-negative indices it sees, so the
//     restatement is the same Blelloch scan with the offset 0.  The header's
//     own definition is renamed (never launched) by the macro below.
//
// Compiled with -fmad=false: each multiply and add rounds on its own, the
// arithmetic a host build of these routines gives (the reference's own build
// lets nvcc contract them into FMAs, which no host build reproduces).
//
// Hazards kept off the GPU (the reference's own code paths that read out of
// bounds or use an unset value): directMIS (noor/cuda/direct.cuh:119-127)
// reads an uninitialised light index when the light sample fails, so renders
// here run with MIS off (the reference default); the traversal stack
// (noor/cuda/bvh.cuh:147) is a bvh_height slice per thread with no bound
// check, so the harness sizes the slice by the deepest stack the tree can
// need (computed on the host from the node words) instead of bvh_height;
// the reference launches only whole 16x16 tiles, the harness checks x < w,
// y < h.
#include "prelude.h"
#include "onb.cuh"
#include "rng.cuh"
#include "transformimp.cuh"
#include "ray.cuh"
#include "mesh.cuh"
#include "intersection.cuh"
#include "texture.cuh"
#include "distribution1d.cuh"
__global__ void prescan(float* func, float* cdf, int n);
#define prescan(...) prescan_reference_definition_not_launched(__VA_ARGS__)
#include "distribution2d.cuh"
#undef prescan
#include "skydome.cuh"
#include "materialimp.cuh"
#include "stack.cuh"
#include "bbox.cuh"
#include "shapeimp.cuh"
#include "lightimp.cuh"
#include "bvh.cuh"
#include "framebuffer.cuh"
#include "cameraimp.cuh"
#include "bsdf.cuh"
#include "direct.cuh"
#include "scatter.cuh"
#include "accumulate.cuh"

#include <algorithm>
#include <cstdint>

namespace abi {
#include "../../include/noor_b200.h"
}

#define REFDEV_API extern "C" __attribute__((visibility("default")))

// prescan of noor/cuda/distribution2d.cuh:86-135 with the bank offset as the
// hardware evaluates it (0): exclusive Blelloch scan of func[row]/n into
// cdf[row], then cdf[n] = func[n] = the row integral.
__global__ void prescan(float* func, float* cdf, int n) {
    extern __shared__ float temp[];
    const int tid = threadIdx.x;
    const int bid = blockIdx.y;
    int offset = 1;
    const int ai = tid;
    const int bi = tid + (n / 2);
    temp[ai] = func[bid * (n + 1) + ai] / n;
    temp[bi] = func[bid * (n + 1) + bi] / n;
    for (int d = n >> 1; d > 0; d >>= 1) {
        __syncthreads();
        if (tid < d) {
            const int a = offset * (2 * tid + 1) - 1;
            const int b = offset * (2 * tid + 2) - 1;
            temp[b] += temp[a];
        }
        offset *= 2;
    }
    if (tid == 0) temp[n - 1] = 0;
    for (int d = 1; d < n; d *= 2) {
        offset >>= 1;
        __syncthreads();
        if (tid < d) {
            const int a = offset * (2 * tid + 1) - 1;
            const int b = offset * (2 * tid + 2) - 1;
            const float t = temp[a];
            temp[a] = temp[b];
            temp[b] += t;
        }
    }
    __syncthreads();
    cdf[bid * (n + 1) + ai] = temp[ai];
    cdf[bid * (n + 1) + bi] = temp[bi];
    __syncthreads();
    if (tid == 0) {
        const float funcInt = cdf[bid * (n + 1) + n - 1] + func[bid * (n + 1) + n - 1] / n;
        cdf[bid * (n + 1) + n] = funcInt;
        func[bid * (n + 1) + n] = funcInt;
    }
    __syncthreads();
}

// ------------------------------------------------------------------ state
namespace {

std::string g_err;

int fail(const char* what) {
    g_err = what;
    return 1;
}
int fail_cuda(const RefdevError& e) {
    g_err = std::string(e.what) + ": " + cudaGetErrorString(e.code);
    cudaGetLastError();
    return 2;
}

template <class T>
struct Owned {
    T* p = nullptr;
    ~Owned() { reset(); }
    void reset() {
        if (p) {
            try {
                p->free();
            } catch (const RefdevError&) {
            }
            delete p;
            p = nullptr;
        }
    }
};

struct Harness {
    std::unique_ptr<CudaPayload> payload;
    CudaHosekSky hosek;
    CudaCamera camera;
    CudaSpec spec;
    Owned<CudaTextureManager> tex;
    Owned<CudaMeshManager> mesh;
    Owned<CudaMaterialManager> mat;
    Owned<CudaSkyDomeManager> sky;
    Owned<CudaLightManager> light;
    Owned<CudaTransformManager> xf;
    Owned<CudaBxDFManager> bxdf;
    Owned<CudaFrameBufferManager> fb;
    uint32_t slice = 0;      // traversal stack entries per thread
    uint32_t w = 0, h = 0;
};
std::unique_ptr<Harness> g;

__host__ __device__ inline float3 f3p(const float* p) { return make_float3(p[0], p[1], p[2]); }

// Upper bound of the stack the reference's DFS (bvh.cuh:142-191) reaches
// below `node`, popped with `d` entries under it: an inner node pushes two
// (d + 2) and each child is popped with at most d + 1 under it; a mesh leaf
// pushes its count children (child i is popped with d + i - 1 under it); an
// instance pushes its bottom-level root (popped with d under it); light and
// triangle leaves push nothing.  Branches are tested in the traversal's order.
uint32_t max_stack(const CudaPayload& P, uint32_t node, uint32_t d, int level) {
    if (level > 512 || node >= P._bvh_min_right_start_nodes.size()) return d + 1;
    const uint32_t lo_w = P._bvh_min_right_start_nodes[node].w;
    const uint32_t w = P._bvh_max_axis_count_nodes[node].w;
    if (w & LIGHT_NODE_MASK) return d;
    if (w & MESH_INSTANCE_MASK) return std::max(d + 1, max_stack(P, lo_w, d, level + 1));
    if (w & MESH_LEAF_MASK) {
        const uint32_t count = w & COUNT_MASK;
        uint32_t best = d + count;
        for (uint32_t i = 1; i <= count; ++i) best = std::max(best, max_stack(P, node + i, d + i - 1, level + 1));
        return best;
    }
    if (w & TRI_LEAF_MASK) return d;
    return std::max({d + 2, max_stack(P, node + 1, d + 1, level + 1), max_stack(P, lo_w, d + 1, level + 1)});
}

CudaTransform xform_of(const float m[3][4]) {
    return CudaTransform(make_float4(m[0][0], m[0][1], m[0][2], m[0][3]),
                         make_float4(m[1][0], m[1][1], m[1][2], m[1][3]),
                         make_float4(m[2][0], m[2][1], m[2][2], m[2][3]));
}

}  // namespace

// Layout views of the sky dome manager, whose distribution member is private
// (noor/cuda/skydome.cuh:41-44; noor/cuda/distribution2d.cuh:166-173): the
// same member types in the same order, checked by size.  SkyView reaches the
// public sampling routine; DistArrays reads the device array pointers.
struct SkyView {
    CudaMipMap tex;
    CudaDistribution2DManager<CudaMipMap> dist;
    SkydomeType type;
};
struct DistArrays {
    float* func;
    float* cdf;
    int width, height;
    cudaTextureObject_t func_tex, cdf_tex;
    size_t size_bytes;
};
struct SkyArrays {
    CudaMipMap tex;
    DistArrays dist;
    SkydomeType type;
};
static_assert(sizeof(SkyView) == sizeof(CudaSkyDomeManager), "sky dome layout");
static_assert(sizeof(SkyArrays) == sizeof(CudaSkyDomeManager), "sky dome layout");
static_assert(sizeof(DistArrays) == sizeof(CudaDistribution2D<CudaMipMap>), "distribution layout");

// --------------------------------------------------------------- kernels

// path_tracer_kernel + pathtracer (noor/cuda/path_tracer.cu:26-100)
__global__ void k_render(uint frame_number) {
    const uint x = blockIdx.x * blockDim.x + threadIdx.x;
    const uint y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= _constant_camera._w || y >= _constant_camera._h) return;
    const uint gid = y * _constant_camera._w + x;
    const uint tid = threadIdx.y * blockDim.x + threadIdx.x;
    const CudaRNG rng(gid, frame_number);
    CudaRay ray = generateRay(x, y, rng);

    float3 L = _constant_spec._black;
    float3 beta = _constant_spec._white;
    bool specular_bounce = false;
    for (uchar bounce = 0; bounce < _constant_spec._bounces; ++bounce) {
        CudaIntersectionRecord rec(tid);
        if (intersect(ray, rec)) {
            CudaIntersection I(ray, rng, rec);
            if (I.isEmitter() && (bounce == 0 || specular_bounce)) {
                L += beta * (I.isMeshLight() ? _light_manager.Le(ray.getDir(), I.getInsIdx())
                                             : _material_manager.getEmmitance(I));
                break;
            }
            accumulate(I, ray, beta, L);
            if (!correct_sidedness(I)) break;
            if (rr_terminate(I, bounce, beta)) break;
            specular_bounce = I.isSpecular();
            I.spawnRay(ray);
        } else {
            if (_constant_spec.is_sky_light_enabled() && (bounce == 0 || specular_bounce)) {
                L += beta * _skydome_manager.evaluate(normalize(ray.getDir()), false);
            }
            break;
        }
    }
    L = clamp(L, 0, 100.f);
    _framebuffer_manager.set(make_float4(L, 1.f), gid, frame_number);
}

__global__ void k_trace(const abi::noor_ray* rays, abi::noor_hit* hits, uint32_t* occ, size_t n, int any) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint tid = threadIdx.x;
    const abi::noor_ray r = rays[i];
    const CudaRay ray(f3p(r.org), f3p(r.dir), r.tmax);
    if (any) {
        occ[i] = intersectP(ray, tid) ? 1u : 0u;
        return;
    }
    CudaIntersectionRecord rec(tid);
    abi::noor_hit o{};
    if (intersect(ray, rec)) {
        o.t = ray.getTmax();
        o.tri_idx = rec._tri_idx;
        o.ins_idx = rec._ins_idx;
        o.material_type = (uint32_t)rec._material_type;
        o.u = rec._uv.x;
        o.v = rec._uv.y;
        o.hit = 1;
    }
    hits[i] = o;
}

__global__ void k_camera_rays(uint frame, abi::noor_ray* out) {
    const uint x = blockIdx.x * blockDim.x + threadIdx.x;
    const uint y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= _constant_camera._w || y >= _constant_camera._h) return;
    const uint gid = y * _constant_camera._w + x;
    const CudaRNG rng(gid, frame);
    const CudaRay ray = generateRay(x, y, rng);
    abi::noor_ray& o = out[gid];
    o.org[0] = ray.getOrigin().x;
    o.org[1] = ray.getOrigin().y;
    o.org[2] = ray.getOrigin().z;
    o.tmax = ray.getTmax();
    o.dir[0] = ray.getDir().x;
    o.dir[1] = ray.getDir().y;
    o.dir[2] = ray.getDir().z;
    o.pad = 0.0f;
}

// BSDF probe.  The reference's texture reads (evaluateGrad, materialimp.cuh)
// returned wrong channels on this GPU and compiler when the lanes of one warp
// read different texture objects in divergent code; callers group records
// so that every warp probes one material.
// in (16 floats): wo_local[3], wi_local[3], probe ray origin[3],
// probe ray dir[3], seed gid, seed frame, -, -.  The probe ray hits the
// material's triangle; the intersection's own shading frame maps the local
// directions to world.  out (12 floats): f[3], pdf, wi_local[3], sampled
// type, the two uniforms Sample_f drew (in draw order), hit flag, material.
__global__ void k_bsdf(int kind, const float* in, float* out, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* p = in + 16 * i;
    float* q = out + 12 * i;
    for (int k = 0; k < 12; ++k) q[k] = 0.0f;
    const CudaRNG rng((uint)p[12], (uint)p[13]);
    CudaRay ray(f3p(p + 6), f3p(p + 9));
    CudaIntersectionRecord rec(threadIdx.x);
    if (!intersect(ray, rec)) return;
    CudaIntersection I(ray, rng, rec);
    const CudaONB onb(I.getSn(), I.getSdpdu(), I.getSdpdv());
    const float3 wo = onb.toWorld(f3p(p));
    const float3 wi = onb.toWorld(f3p(p + 3));
    CudaBSDF bsdf;
    factoryBSDF(I, bsdf);
    float3 f = make_float3(0.0f);
    float pdf = 0.0f;
    float3 wl = make_float3(0.0f);
    BxDFType st = BxDFType(0);
    if (kind == 0) {
        f = bsdf.Eval(I, wo, wi, BSDF_ALL);
    } else if (kind == 1) {
        pdf = bsdf.Pdf(I, wo, wi, BSDF_ALL);
    } else {
        CudaRNG peek = rng;
        q[8] = peek();
        q[9] = peek();
        float3 wiw = make_float3(0.0f);
        f = bsdf.Sample_f(I, wo, wiw, pdf, BSDF_ALL, st);
        if (pdf != 0.0f) wl = onb.toLocal(wiw);
    }
    q[0] = f.x;
    q[1] = f.y;
    q[2] = f.z;
    q[3] = pdf;
    q[4] = wl.x;
    q[5] = wl.y;
    q[6] = wl.z;
    q[7] = (float)st;
    q[10] = 1.0f;
    q[11] = (float)I.getMatIdx();
}

// Microfacet distributions (noor/cuda/distribution.cuh:58-342) with
// alpha = max(r^2, 1e-3) per axis (the Trowbridge-Reitz constructor's
// mapping; the Beckmann constructor takes alpha as given).
// in (12 floats): roughness[2], wo[3], wh[3], u[2], -, -.
// out (12 floats): D(wh), G(wo, wh), Pdf(wo, wh), Sample_wh(wo, u)[3], 0,
// alpha_x, 0, 0, 0, 0.
__global__ void k_microfacet(int beckmann, const float* in, float* out, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* p = in + 12 * i;
    float* q = out + 12 * i;
    const float3 wo = f3p(p + 2), wh = f3p(p + 5);
    const float2 u = make_float2(p[8], p[9]);
    for (int k = 0; k < 12; ++k) q[k] = 0.0f;
    CudaTrowbridgeReitz alpha_of(make_float2(1.0f));
    const float ax = alpha_of.RoughnessToAlpha(p[0]), ay = alpha_of.RoughnessToAlpha(p[1]);
    float3 s;
    if (beckmann) {
        const CudaBeckmannDistribution d(ax, ay);
        q[0] = d.D(wh);
        q[1] = d.G(wo, wh);
        q[2] = d.Pdf(wo, wh);
        s = d.Sample_wh(wo, u);
    } else {
        const CudaTrowbridgeReitz d(make_float2(p[0], p[1]));
        q[0] = d.D(wh);
        q[1] = d.G(wo, wh);
        q[2] = d.Pdf(wo, wh);
        s = d.Sample_wh(wo, u);
    }
    q[3] = s.x;
    q[4] = s.y;
    q[5] = s.z;
    q[7] = ax;
}

// Fresnel (noor/cuda/fresnel.cuh:58-107).  in (8 floats): cos, etaI, etaT
// (dielectric), eta[3], k[3] (conductor, etaI = 1).  out (4 floats):
// dielectric F, conductor F[3].
__global__ void k_fresnel(const float* in, float* out, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* p = in + 9 * i;
    out[4 * i] = fresnelDielectric(p[0], p[1], p[2]);
    const float3 c = fresnelConductor(p[0], make_float3(1.0f), f3p(p + 3), f3p(p + 6));
    out[4 * i + 1] = c.x;
    out[4 * i + 2] = c.y;
    out[4 * i + 3] = c.z;
}

// Sampling warps and helpers (noor/cuda/utils.cuh:340-550), with the
// handedness the BxDFs call them with (local z up).  in: u[2], x; out (16
// floats): concentricSampleDisk[2], cosineSampleHemisphere[3],
// uniformSampleHemisphere (left handed)[3], sphericalDirection(u)[3] + its
// sinTheta, powerHeuristic(1, u.x, 1, u.y), Erf(x), ErfInv(x), -.
__global__ void k_warps(const float* in, float* out, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* p = in + 3 * i;
    float* q = out + 16 * i;
    const float2 u = make_float2(p[0], p[1]);
    const float2 d = NOOR::concentricSampleDisk(u);
    const float3 c = NOOR::cosineSampleHemisphere(u);
    const float3 h = NOOR::uniformSampleHemisphere(u, LEFT_HANDED);
    float st = 0.0f;
    const float3 s = NOOR::sphericalDirection(u, st);
    q[0] = d.x;
    q[1] = d.y;
    q[2] = c.x;
    q[3] = c.y;
    q[4] = c.z;
    q[5] = h.x;
    q[6] = h.y;
    q[7] = h.z;
    q[8] = s.x;
    q[9] = s.y;
    q[10] = s.z;
    q[11] = st;
    q[12] = NOOR::powerHeuristic(1, u.x, 1, u.y);
    q[13] = NOOR::Erf(p[2]);
    q[14] = NOOR::ErfInv(p[2]);
    q[15] = 0.0f;
}

// Sky: querySkyModel (noor/cuda/hosek.cuh:86-101) on _constant_hosek_sky,
// or the sky dome's evaluate (noor/cuda/skydome.cuh:93-101) of a loaded scene.
__global__ void k_sky(int dome, const float* dirs, float* rgb, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float3 v = f3p(dirs + 3 * i);
    const float3 c = dome ? _skydome_manager.evaluate(v, false) : _constant_hosek_sky.querySkyModel(v);
    rgb[3 * i] = c.x;
    rgb[3 * i + 1] = c.y;
    rgb[3 * i + 2] = c.z;
}

// Sky dome importance sampling (skydome.cuh:78-81,103-107):
// u -> {x, y, pdf of the sample, Pdf(x, y)}
__global__ void k_env_sample(const float* u, float* out, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float pdf = 0.0f;
    const SkyView& sky = reinterpret_cast<const SkyView&>(_skydome_manager);
    const float2 xy = sky.dist._distribution2d.sampleContinuous2D(make_float2(u[2 * i], u[2 * i + 1]), pdf);
    out[4 * i] = xy.x;
    out[4 * i + 1] = xy.y;
    out[4 * i + 2] = pdf;
    out[4 * i + 3] = _skydome_manager.Pdf(xy);
}

// CudaRNG (noor/cuda/rng.cuh:37-76): seed of (id, frame) and `draws` floats
__global__ void k_rng(const uint32_t* seeds, size_t n, int draws, uint32_t* seed_out, float* out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const CudaRNG rng(seeds[2 * i], seeds[2 * i + 1]);
    uint32_t s;
    memcpy(&s, &rng, sizeof(s));
    seed_out[i] = s;
    for (int k = 0; k < draws; ++k) out[i * draws + k] = rng();
}

// ------------------------------------------------------------- host API
namespace {

template <class V, class S>
std::vector<V> vec4s(const S* p, size_t n) {
    std::vector<V> v(n);
    if (p) std::memcpy(v.data(), p, n * sizeof(V));
    return v;
}

ImageTexture& add_texture(CudaPayload& P, int w, int h, cudaTextureFilterMode f, const float* rgba,
                          cudaTextureAddressMode a = cudaAddressModeClamp) {
    P._textures.emplace_back(w, h, 4, f, a);
    ImageTexture& t = P._textures.back();
    if (rgba) std::memcpy(const_cast<float*>(t.getData()), rgba, sizeof(float) * 4 * (size_t)w * h);
    return t;
}

// CudaPayload from the C-ABI mirror (noor/header/payload.h:27-127); the
// environment texture is made as Model::loadMaterials makes it
// (noor/source/model.cpp:313-321): the HDR map linear/clamp, a 2048^2
// linear/clamp surface for the physical sky, a 1x1 constant otherwise.
std::unique_ptr<CudaPayload> make_payload(const abi::noor_payload* A, int sky_type) {
    auto P = std::make_unique<CudaPayload>();
    const size_t nt = A->num_triangles, nv = A->num_vertices, ni = A->num_instances, nn = A->num_bvh_nodes;
    P->_num_triangles = (glm::uint32)nt;
    P->_attribute_indices = vec4s<glm::uvec4>(A->attribute_indices, nt);
    P->_vertices = vec4s<glm::vec4>(A->vertices, nv);
    P->_normals = vec4s<glm::vec4>(A->normals, nv);
    P->_uvs = vec4s<glm::vec2>(A->uvs, nv);
    P->_ai_size_bytes = nt * 16;
    P->_n_size_bytes = nv * 16;
    P->_uv_size_bytes = nv * 8;
    std::vector<glm::vec4>* rows[9] = {&P->_normal_row0,          &P->_normal_row1,          &P->_normal_row2,
                                       &P->_world_to_object_row0, &P->_world_to_object_row1, &P->_world_to_object_row2,
                                       &P->_object_to_world_row0, &P->_object_to_world_row1, &P->_object_to_world_row2};
    for (int r = 0; r < 3; ++r) {
        *rows[r] = vec4s<glm::vec4>(A->normal_row[r], ni);
        *rows[3 + r] = vec4s<glm::vec4>(A->world_to_object_row[r], ni);
        *rows[6 + r] = vec4s<glm::vec4>(A->object_to_world_row[r], ni);
    }
    P->_transforms_size_bytes = ni * 16;
    P->_wald_ax_nu_nv_nd = vec4s<glm::uvec4>(A->wald_ax_nu_nv_nd, nt);
    P->_wald_bnu_bnv_au_av = vec4s<glm::uvec4>(A->wald_bnu_bnv_au_av, nt);
    P->_wald_cnu_cnv_deg_mat = vec4s<glm::uvec4>(A->wald_cnu_cnv_deg_mat, nt);
    P->_wald_size_bytes = nt * 16;
    P->_bvh_root_node = A->bvh_root_node;
    P->_bvh_min_right_start_nodes = vec4s<glm::uvec4>(A->bvh_min_right_start, nn);
    P->_bvh_max_axis_count_nodes = vec4s<glm::uvec4>(A->bvh_max_axis_count, nn);
    P->_bvh_size_bytes = nn * 16;
    // material textures with their own filter and addressing, then the env
    P->_textures.reserve(A->num_textures + 1);
    for (uint32_t i = 0; i + 1 < A->num_textures; ++i) {
        const abi::noor_texture& t = A->textures[i];
        add_texture(*P, t.width, t.height, (cudaTextureFilterMode)t.filter, t.rgba, (cudaTextureAddressMode)t.address);
    }
    const abi::noor_texture* env = A->num_textures ? &A->textures[A->num_textures - 1] : nullptr;
    if (sky_type == HDR && env)
        add_texture(*P, env->width, env->height, cudaFilterModeLinear, env->rgba);
    else if (sky_type == PHYSICAL)
        add_texture(*P, skydome_res.x, skydome_res.y, cudaFilterModeLinear, nullptr);
    else {
        const float c[4] = {SKYDOME_COLOR.x, SKYDOME_COLOR.y, SKYDOME_COLOR.z, 1.0f};
        add_texture(*P, 1, 1, cudaFilterModePoint, c);
    }
    for (int32_t i = 0; i < A->num_area_lights; ++i) {
        const abi::noor_area_light& a = A->area_lights[i];
        CudaShape s;
        s._center = f3p(a.shape.center);
        s._u = f3p(a.shape.u);
        s._v = f3p(a.shape.v);
        s._n = f3p(a.shape.n);
        s._area = a.shape.area;
        s._radius = a.shape.radius;
        s._radius2 = a.shape.radius2;
        s._light_idx = a.shape.light_idx;
        s._type = (AreaMeshLightType)a.shape.type;
        P->_area_light_data.emplace_back(s, f3p(a.ke), a.two_sided != 0);
        P->_shapes.push_back(s);
    }
    P->_num_area_lights = A->num_area_lights;
    for (int32_t i = 0; i < A->num_point_lights; ++i)
        P->_point_light_data.emplace_back(f3p(A->point_lights[i].position), f3p(A->point_lights[i].ke));
    P->_num_point_lights = A->num_point_lights;
    for (int32_t i = 0; i < A->num_spot_lights; ++i) {
        const abi::noor_spot_light& s = A->spot_lights[i];
        P->_spot_light_data.emplace_back(f3p(s.position), f3p(s.direction), f3p(s.ke), s.cos_inner, s.cos_outer);
    }
    P->_num_spot_lights = A->num_spot_lights;
    for (int32_t i = 0; i < A->num_distant_lights; ++i)
        P->_distant_light_data.emplace_back(f3p(A->distant_lights[i].direction), f3p(A->distant_lights[i].ke));
    P->_num_distant_lights = A->num_distant_lights;
    for (int32_t i = 0; i < A->num_infinite_lights; ++i) P->_infinite_light_data.emplace_back(0.0f);
    P->_num_infinite_lights = A->num_infinite_lights;
    P->_num_lights = A->num_area_lights + A->num_point_lights + A->num_spot_lights + A->num_distant_lights +
                     A->num_infinite_lights;
    for (uint32_t i = 0; i < A->num_materials; ++i) {
        const abi::noor_material& m = A->materials[i];
        CudaMaterial c;
        c._diffuse_uvscale = make_float2(m.diffuse_uvscale[0], m.diffuse_uvscale[1]);
        c._specular_uvscale = make_float2(m.specular_uvscale[0], m.specular_uvscale[1]);
        c._transparency_uvscale = make_float2(m.transparency_uvscale[0], m.transparency_uvscale[1]);
        c._emittance_uvscale = make_float2(m.emittance_uvscale[0], m.emittance_uvscale[1]);
        c._bump_uvscale = make_float2(m.bump_uvscale[0], m.bump_uvscale[1]);
        c._roughness_uvscale = make_float2(m.roughness_uvscale[0], m.roughness_uvscale[1]);
        c._metalness_uvscale = make_float2(m.metalness_uvscale[0], m.metalness_uvscale[1]);
        c._diffuse_tex_idx = m.diffuse_tex_idx;
        c._specular_tex_idx = m.specular_tex_idx;
        c._transmission_tex_idx = m.transmission_tex_idx;
        c._emittance_tex_idx = m.emittance_tex_idx;
        c._bump_tex_idx = m.bump_tex_idx;
        c._transparency_tex_idx = m.transparency_tex_idx;
        c._ior_tex_idx = m.ior_tex_idx;
        c._k_tex_idx = m.k_tex_idx;
        c._roughness_tex_idx = m.roughness_tex_idx;
        c._metalness_tex_idx = m.metalness_tex_idx;
        c._bumpfactor = m.bumpfactor;
        c._emitter_scale = m.emitter_scale;
        c._coat_weight = m.coat_weight;
        c._coat_roughness = m.coat_roughness;
        c._coat_thickness = m.coat_thickness;
        c._coat_sigma = m.coat_sigma;
        c._coat_ior = m.coat_ior;
        c._type = m.type;
        P->_materials.push_back(c);
    }
    P->_mat_size_bytes = P->_materials.size() * sizeof(CudaMaterial);
    return P;
}

void set_hosek(CudaHosekSky& H, const abi::noor_hosek_sky* A) {
    CudaArHosekSkyModelState* st[3] = {&H._state_r, &H._state_g, &H._state_b};
    for (int c = 0; c < 3; ++c) {
        const abi::noor_hosek_state& a = A->state[c];
        CudaArHosekSkyModelState& s = *st[c];
        std::memcpy(s._configs, a.configs, sizeof(a.configs));
        s._radiances.x = a.radiances[0];
        s._radiances.y = a.radiances[1];
        s._radiances.z = a.radiances[2];
        s._turbidity = a.turbidity;
        s._solar_radius = a.solar_radius;
        s._emission_correction_factor_sky.x = a.emission_correction_factor_sky[0];
        s._emission_correction_factor_sky.y = a.emission_correction_factor_sky[1];
        s._emission_correction_factor_sky.z = a.emission_correction_factor_sky[2];
        s._emission_correction_factor_sun.x = a.emission_correction_factor_sun[0];
        s._emission_correction_factor_sun.y = a.emission_correction_factor_sun[1];
        s._emission_correction_factor_sun.z = a.emission_correction_factor_sun[2];
        s._albedo = a.albedo;
        s._elevation = a.elevation;
    }
    H._solar_dir = f3p(A->solar_dir);
    H._ground_albedo = f3p(A->ground_albedo);
    H._solar_scale = A->solar_scale;
    H._solar_radius = A->solar_radius;
}

void set_camera(CudaCamera& C, const abi::noor_camera* A) {
    C._cameraToWorld = xform_of(A->camera_to_world);
    C._rasterToCamera = xform_of(A->raster_to_camera);
    C._worldToRaster = xform_of(A->world_to_raster);
    C._dxCamera = f3p(A->dx_camera);
    C._dyCamera = f3p(A->dy_camera);
    C._lens_radius = A->lens_radius;
    C._focal_length = A->focal_length;
    C._image_area = A->image_area;
    C._w = A->w;
    C._h = A->h;
    C._center = A->center;
    C._type = (CameraType)A->type;
}

void set_spec(CudaSpec& S, const abi::noor_spec* A, uint32_t slice) {
    std::memset(&S, 0, sizeof(S));
    S._white = make_float3(1.0f, 1.0f, 1.0f);
    S._black = make_float3(0.0f, 0.0f, 0.0f);
    S._reflection_bias = A->reflection_bias;
    S._shadow_bias = A->shadow_bias;
    S._world_radius = A->world_radius;
    S._wr2 = A->wr2;
    S._bvh_root_node = A->bvh_root_node;
    S._lighting_type = (unsigned short)A->lighting_type;
    S._bounces = (unsigned short)A->bounces;
    S._rr = (unsigned short)A->rr;
    S._bvh_height = (unsigned short)slice;
    S._num_gpus = 1;
    S._skydome_type = (SkydomeType)A->skydome_type;
    S._debug_sky = A->debug_sky != 0;
    S._mis = false;
    S._outofsync = false;
}

int need_scene() { return g ? 0 : fail("refdev: no scene loaded"); }

template <class K>
cudaError_t allow_smem(K kernel, size_t smem) {
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

}  // namespace

REFDEV_API const char* refdev_last_error() { return g_err.c_str(); }

REFDEV_API void refdev_free() {
    if (!g) return;
    cudaDeviceSynchronize();
    g.reset();
}

// CudaRenderDevice's constructor (noor/cuda/render.cuh:62-110) without GL.
// mis must be 0: the reference's MIS path reads an unset light index.
REFDEV_API int refdev_load(const abi::noor_payload* payload, const abi::noor_hosek_sky* hosek,
                           const abi::noor_camera* camera, const abi::noor_spec* spec, uint32_t* stack_slice) {
    if (!payload || !hosek || !camera || !spec) return fail("refdev_load: null argument");
    if (spec->mis) return fail("refdev_load: MIS is not run (the reference's directMIS reads an unset light index)");
    if (payload->num_bvh_nodes == 0 || payload->num_textures == 0) return fail("refdev_load: empty payload");
    refdev_free();
    try {
        auto H = std::make_unique<Harness>();
        H->payload = make_payload(payload, spec->skydome_type);
        H->slice = std::max<uint32_t>(max_stack(*H->payload, payload->bvh_root_node, 0, 0), 1) + 1;
        if (H->slice > 200) return fail("refdev_load: traversal stack bound above 200 entries");
        set_hosek(H->hosek, hosek);
        set_camera(H->camera, camera);
        set_spec(H->spec, spec, H->slice);
        H->w = camera->w;
        H->h = camera->h;
        const CudaPayload* P = H->payload.get();
        H->tex.p = new CudaTextureManager(P);
        H->mesh.p = new CudaMeshManager(P);
        H->mat.p = new CudaMaterialManager(P);
        H->sky.p = new CudaSkyDomeManager(H->tex.p->getEnvTexture(), H->spec._skydome_type);
        H->light.p = new CudaLightManager(P);
        H->xf.p = new CudaTransformManager(P);
        H->bxdf.p = new CudaBxDFManager(1);
        H->fb.p = new CudaFrameBufferManager(CudaRenderTask(camera->w, camera->h, 0));
        checkNoorErrors(NOOR::memcopy_symbol(&_constant_spec, &H->spec));
        checkNoorErrors(NOOR::memcopy_symbol(&_constant_camera, &H->camera));
        checkNoorErrors(NOOR::memcopy_symbol(&_constant_hosek_sky, &H->hosek));
        if (H->spec._skydome_type == PHYSICAL) H->sky.p->update();
        checkNoorErrors(NOOR::memcopy_symbol(&_mesh_manager, H->mesh.p));
        checkNoorErrors(NOOR::memcopy_symbol(&_material_manager, H->mat.p));
        checkNoorErrors(NOOR::memcopy_symbol(&_texture_manager, H->tex.p));
        checkNoorErrors(NOOR::memcopy_symbol(&_light_manager, H->light.p));
        checkNoorErrors(NOOR::memcopy_symbol(&_transform_manager, H->xf.p));
        checkNoorErrors(NOOR::memcopy_symbol(&_skydome_manager, H->sky.p));
        checkNoorErrors(NOOR::memcopy_symbol(&_bxdf_manager, H->bxdf.p));
        checkNoorErrors(NOOR::memcopy_symbol(&_framebuffer_manager, H->fb.p));
        checkNoorErrors(cudaDeviceSynchronize());
        if (stack_slice) *stack_slice = H->slice;
        g = std::move(H);
    } catch (const RefdevError& e) {
        return fail_cuda(e);
    }
    return 0;
}

// frames first..first+n-1, one launch each, folded by the framebuffer's
// running mean (noor/cuda/framebuffer.cuh:62-76); film: host rgba floats
REFDEV_API int refdev_render(uint32_t first_frame, uint32_t n_frames, float* film) {
    if (int rc = need_scene()) return rc;
    if (first_frame == 0) return fail("refdev_render: frames start at 1");
    try {
        const dim3 block(THREAD_W, THREAD_H);
        const dim3 grid((g->w + THREAD_W - 1) / THREAD_W, (g->h + THREAD_H - 1) / THREAD_H);
        const size_t smem = (size_t)THREAD_N * g->slice * sizeof(uint);
        checkNoorErrors(allow_smem(k_render, smem));
        for (uint32_t f = 0; f < n_frames; ++f) {
            k_render<<<grid, block, smem>>>(first_frame + f);
            checkNoorErrors(cudaGetLastError());
        }
        checkNoorErrors(cudaDeviceSynchronize());
        if (film)
            checkNoorErrors(cudaMemcpy(film, g->fb.p->_buffer, (size_t)g->w * g->h * sizeof(float4),
                                       cudaMemcpyDeviceToHost));
    } catch (const RefdevError& e) {
        return fail_cuda(e);
    }
    return 0;
}

// closest hit (any = 0, out = noor_hit per ray) or any hit (any = 1, out =
// uint32 per ray) of host rays
REFDEV_API int refdev_trace(int any, const abi::noor_ray* rays, void* out, size_t n) {
    if (int rc = need_scene()) return rc;
    if (n == 0) return 0;
    abi::noor_ray* d_rays = nullptr;
    void* d_out = nullptr;
    const size_t osz = any ? sizeof(uint32_t) : sizeof(abi::noor_hit);
    int rc = 0;
    try {
        checkNoorErrors(cudaMalloc(&d_rays, n * sizeof(abi::noor_ray)));
        checkNoorErrors(cudaMalloc(&d_out, n * osz));
        checkNoorErrors(cudaMemcpy(d_rays, rays, n * sizeof(abi::noor_ray), cudaMemcpyHostToDevice));
        const int block = 128;
        const size_t smem = (size_t)block * g->slice * sizeof(uint);
        checkNoorErrors(allow_smem(k_trace, smem));
        k_trace<<<(unsigned)((n + block - 1) / block), block, smem>>>(d_rays, (abi::noor_hit*)d_out, (uint32_t*)d_out,
                                                                      n, any);
        checkNoorErrors(cudaGetLastError());
        checkNoorErrors(cudaMemcpy(out, d_out, n * osz, cudaMemcpyDeviceToHost));
    } catch (const RefdevError& e) {
        rc = fail_cuda(e);
    }
    cudaFree(d_rays);
    cudaFree(d_out);
    return rc;
}

// camera rays of every pixel of frame `frame` (noor/cuda/cameraimp.cuh:182-228)
REFDEV_API int refdev_camera_rays(uint32_t frame, abi::noor_ray* out) {
    if (int rc = need_scene()) return rc;
    abi::noor_ray* d = nullptr;
    int rc = 0;
    const size_t n = (size_t)g->w * g->h;
    try {
        checkNoorErrors(cudaMalloc(&d, n * sizeof(abi::noor_ray)));
        const dim3 block(16, 16), grid((g->w + 15) / 16, (g->h + 15) / 16);
        k_camera_rays<<<grid, block>>>(frame, d);
        checkNoorErrors(cudaGetLastError());
        checkNoorErrors(cudaMemcpy(out, d, n * sizeof(abi::noor_ray), cudaMemcpyDeviceToHost));
    } catch (const RefdevError& e) {
        rc = fail_cuda(e);
    }
    cudaFree(d);
    return rc;
}

namespace {
// one batch kernel over host arrays: copy in, launch, copy out
template <class Launch>
int run_batch(const void* in, size_t in_bytes, void* out, size_t out_bytes, Launch launch) {
    void *d_in = nullptr, *d_out = nullptr;
    int rc = 0;
    try {
        checkNoorErrors(cudaMalloc(&d_in, in_bytes ? in_bytes : 4));
        checkNoorErrors(cudaMalloc(&d_out, out_bytes ? out_bytes : 4));
        if (in_bytes) checkNoorErrors(cudaMemcpy(d_in, in, in_bytes, cudaMemcpyHostToDevice));
        launch(d_in, d_out);
        checkNoorErrors(cudaGetLastError());
        if (out_bytes) checkNoorErrors(cudaMemcpy(out, d_out, out_bytes, cudaMemcpyDeviceToHost));
    } catch (const RefdevError& e) {
        rc = fail_cuda(e);
    }
    cudaFree(d_in);
    cudaFree(d_out);
    return rc;
}
unsigned blocks(size_t n, int b) { return (unsigned)((n + b - 1) / b); }
}  // namespace

// BSDF probes of the loaded scene (see k_bsdf); kind 0 Eval, 1 Pdf, 2 Sample_f
REFDEV_API int refdev_bsdf(int kind, const float* in, float* out, size_t n) {
    if (int rc = need_scene()) return rc;
    if (n == 0) return 0;
    const int b = 128;
    const size_t smem = (size_t)b * g->slice * sizeof(uint);
    try {
        checkNoorErrors(allow_smem(k_bsdf, smem));
    } catch (const RefdevError& e) {
        return fail_cuda(e);
    }
    return run_batch(in, n * 16 * 4, out, n * 12 * 4, [&](void* i, void* o) {
        k_bsdf<<<blocks(n, b), b, smem>>>(kind, (const float*)i, (float*)o, n);
    });
}

REFDEV_API int refdev_microfacet(int beckmann, const float* in, float* out, size_t n) {
    return run_batch(in, n * 12 * 4, out, n * 12 * 4, [&](void* i, void* o) {
        k_microfacet<<<blocks(n, 128), 128>>>(beckmann, (const float*)i, (float*)o, n);
    });
}

REFDEV_API int refdev_fresnel(const float* in, float* out, size_t n) {
    return run_batch(in, n * 9 * 4, out, n * 4 * 4, [&](void* i, void* o) {
        k_fresnel<<<blocks(n, 128), 128>>>((const float*)i, (float*)o, n);
    });
}

REFDEV_API int refdev_warps(const float* in, float* out, size_t n) {
    return run_batch(in, n * 3 * 4, out, n * 16 * 4, [&](void* i, void* o) {
        k_warps<<<blocks(n, 128), 128>>>((const float*)i, (float*)o, n);
    });
}

// querySkyModel with the given sky (dome = 0, no scene needed) or the loaded
// scene's sky dome evaluate (dome = 1, hosek ignored)
REFDEV_API int refdev_sky(int dome, const abi::noor_hosek_sky* hosek, const float* dirs, float* rgb, size_t n) {
    if (dome) {
        if (int rc = need_scene()) return rc;
    } else {
        if (!hosek) return fail("refdev_sky: no sky");
        CudaHosekSky H;
        set_hosek(H, hosek);
        try {
            checkNoorErrors(NOOR::memcopy_symbol(&_constant_hosek_sky, &H));
        } catch (const RefdevError& e) {
            return fail_cuda(e);
        }
    }
    const int rc = run_batch(dirs, n * 12, rgb, n * 12, [&](void* i, void* o) {
        k_sky<<<blocks(n, 128), 128>>>(dome, (const float*)i, (float*)o, n);
    });
    if (!dome && g) {  // put the loaded scene's sky back
        try {
            checkNoorErrors(NOOR::memcopy_symbol(&_constant_hosek_sky, &g->hosek));
        } catch (const RefdevError& e) {
            return fail_cuda(e);
        }
    }
    return rc;
}

REFDEV_API int refdev_env_sample(const float* u, float* out, size_t n) {
    if (int rc = need_scene()) return rc;
    return run_batch(u, n * 8, out, n * 16, [&](void* i, void* o) {
        k_env_sample<<<blocks(n, 128), 128>>>((const float*)i, (float*)o, n);
    });
}

// the sky dome's distribution arrays (noor/cuda/distribution2d.cuh:166-220):
// width w, height h; func and cdf hold h*(w+2)+1 floats each: row r at
// r*(w+1) (w values + the row integral), the marginal at h*(w+1) (h values
// + its integral).  Pass null arrays to query w, h.
REFDEV_API int refdev_env_distribution(int* w, int* h, float* func, float* cdf) {
    if (int rc = need_scene()) return rc;
    SkyArrays view;
    std::memcpy(static_cast<void*>(&view), static_cast<const void*>(g->sky.p), sizeof(view));
    if (w) *w = view.dist.width;
    if (h) *h = view.dist.height;
    try {
        if (func) checkNoorErrors(cudaMemcpy(func, view.dist.func, view.dist.size_bytes, cudaMemcpyDeviceToHost));
        if (cdf) checkNoorErrors(cudaMemcpy(cdf, view.dist.cdf, view.dist.size_bytes, cudaMemcpyDeviceToHost));
    } catch (const RefdevError& e) {
        return fail_cuda(e);
    }
    return 0;
}

// seeds: (id, frame) pairs; seed_out: TEA<16> seed; out: `draws` floats each
REFDEV_API int refdev_rng(const uint32_t* seeds, size_t n, int draws, uint32_t* seed_out, float* out) {
    if (n == 0) return 0;
    std::vector<uint8_t> res(n * 4 + n * draws * 4);
    const int rc = run_batch(seeds, n * 8, res.data(), res.size(), [&](void* i, void* o) {
        k_rng<<<blocks(n, 128), 128>>>((const uint32_t*)i, n, draws, (uint32_t*)o, (float*)((uint8_t*)o + n * 4));
    });
    if (rc) return rc;
    std::memcpy(seed_out, res.data(), n * 4);
    std::memcpy(out, res.data() + n * 4, n * draws * 4);
    return 0;
}
