// Device-resident scene: every array the render path reads, in the layouts
// chosen for B200 (one 32-byte sector per BVH node, 64-byte triangle records
// whose first sector holds everything the t-range test needs).
#pragma once
#include "dmath.cuh"
#include "../../include/noor_b200.h"

namespace nb {

// One BVH node = 32 B: [0] = min.xyz | right/start/child-root,
// [1] = max.xyz | flags+count/axis/instance/light.  Same words as the
// reference's two uint4 arrays (noor/cuda/mesh.cuh:43-45), interleaved so one
// node is one aligned sector.
struct __align__(32) DevNode {
    uint4 lo;
    uint4 hi;
};

// Four-wide any-hit node = 128 B (one line): the four entry boxes as
// structure of arrays, the entry words and meta (wide_bvh.h)
struct __align__(128) DevNode4 {
    float4 lox, loy, loz;
    float4 hix, hiy, hiz;
    uint4 child;
    uint4 meta;
};

// Reference-Wald triangle = 64 B: the two records the t-range test reads
// (ax,nu,nv,nd | cnu,cnv,deg,mat) share the first sector, the barycentric
// record and the attribute indices (v0,v1,v2,material) the second.
struct __align__(64) DevWaldTri {
    uint4 ax_nu_nv_nd;
    uint4 cnu_cnv_deg_mat;
    uint4 bnu_bnv_au_av;
    uint4 attr;
};

// Watertight triangle = 64 B: object-space vertices (v0.w = material type
// bits) and the attribute indices.
struct __align__(64) DevWtTri {
    float4 v0;
    float4 v1;
    float4 v2;
    uint4 attr;
};

// Per instance: world->object, object->world and normal rows (9 x float4).
struct DevXform {
    float4 w2o[3];
    float4 o2w[3];
    float4 nrm[3];
};

// Constant material parameters resolved from the 1x1 textures at load.
struct __align__(16) DevMaterial {
    float3 diffuse;
    uint32_t type;
    float3 specular;
    uint32_t distribution;
    float3 transmission;
    float coat_ior;
    float3 emittance;
    float emitter_scale;
    float3 ior;
    float rough_x;
    float3 k;
    float rough_y;
    float coat_weight;      // clear coat
    float coat_sigma;
    float coat_thickness;
    uint32_t tex_mask;      // kTex* slots read through the texture unit (DevMatTex)
};

// Material slots whose texture is an image map (or, for the alpha and bump
// slots of ALPHA / BUMP materials, any texture): fetched per hit by the
// texture unit with the texture's own filter and addressing, at the hit's
// uv times the slot's scale (noor/cuda/materialimp.cuh:121-183).
enum : uint32_t {
    kTexDiffuse = 0,
    kTexSpecular = 1,
    kTexEmittance = 2,
    kTexRoughness = 3,
    kTexTransmission = 4,
    kTexIor = 5,
    kTexK = 6,
    kTexAlpha = 7,
    kTexBump = 8,
    kTexSlots = 9
};
struct DevMatTex {
    cudaTextureObject_t tex[kTexSlots];
    float2 uvscale[kTexSlots];
    float bumpfactor;
    float pad[3];
};

struct DevAreaLight {
    float3 center;
    float area;
    float3 u;
    int two_sided;
    float3 v;
    int type;               // NOOR_SHAPE_*
    float3 n;
    float radius;           // sphere / disk
    float3 ke;
    float radius2;
};

// point, spot and distant lights (noor/cuda/light.cuh:158-238), stored in
// one array in light-index order
enum : int { kDeltaPoint = 0, kDeltaSpot = 1, kDeltaDistant = 2 };
struct DevDeltaLight {
    float3 pos;
    int kind;
    float3 dir;             // spot axis / direction towards a distant light
    float cos_inner;
    float3 ke;
    float cos_outer;
};

struct DevHosek {
    float configs[3][9];  // channel c uses state c's configs[c]
    float radiance[3];
    float3 solar_dir;
    float solar_scale;
    float solar_radius;
};

struct DevCamera {
    float4 c2w[3];
    float4 r2c[3];
    uint32_t w, h, center, type;  // type: NOOR_CAMERA_*
    float lens_radius, focal_length, pad0, pad1;
};
// the raster-to-world transforms and image of a noor_camera, with the
// image size given (a batch frame's own)
inline DevCamera dev_camera(const noor_camera& c, uint32_t w, uint32_t h) {
    DevCamera d{};
    for (int r = 0; r < 3; ++r) {
        d.c2w[r] = make_float4(c.camera_to_world[r][0], c.camera_to_world[r][1], c.camera_to_world[r][2],
                               c.camera_to_world[r][3]);
        d.r2c[r] = make_float4(c.raster_to_camera[r][0], c.raster_to_camera[r][1], c.raster_to_camera[r][2],
                               c.raster_to_camera[r][3]);
    }
    d.w = w;
    d.h = h;
    d.center = c.center;
    d.type = (uint32_t)c.type;
    d.lens_radius = c.lens_radius;
    d.focal_length = c.focal_length;
    return d;
}

// Piecewise-constant 2D distribution over the environment (row = theta).
// Guide tables of a piecewise-constant distribution's CDFs: entry k of a
// row is the largest index i with cdf[i] <= k / kDistGuide, so the inverse
// CDF search for u only has to look between the entries around u *
// kDistGuide (the same index a search over the whole row finds).
constexpr int kDistGuide = 64;
struct DevDist2D {
    const float* func;      // h * w
    const float* cdf;       // h * (w + 1)
    const float* row_int;   // h   (integral of each row's func)
    const float* marg_cdf;  // h + 1
    const int* guide;       // h * (kDistGuide + 1), null: no guides
    const int* mguide;      // kDistGuide + 1 over marg_cdf
    float marg_int;         // integral of row_int
    int w, h;
};

struct DevScene {
    const DevNode* nodes;
    const DevWaldTri* wald;
    const DevWtTri* wtri;
    const float4* vertices;
    const float4* normals;
    const float2* uvs;
    const DevXform* xforms;
    const uint32_t* xf_ident;   // bit i: instance i's world-to-object rows are the identity
    const DevMaterial* materials;
    const DevMatTex* mat_tex;   // per material; read only where tex_mask is set
    const DevAreaLight* area_lights;
    const DevDeltaLight* delta_lights;
    const float4* env;      // env texels (HDR / baked sky / constant), w*h
    uint32_t num_nodes;
    uint32_t num_tris;
    uint32_t num_instances;
    uint32_t num_materials;
    int num_area_lights;
    int num_delta_lights;   // lights num_area_lights .. + num_delta_lights - 1
    int num_lights;         // area lights + infinite light
    int env_w, env_h;
    DevDist2D dist;
    DevHosek hosek;
    // spec
    float bias;
    float world_radius;
    uint32_t root;
    uint32_t bounces;
    uint32_t rr;
    uint32_t mis;
    uint32_t sky_on;
    int sky_type;
    uint32_t isect;
    uint32_t film_mode;
    int stack_cap;
    uint32_t ext_lobes;     // some material uses a lobe beyond Lambert, conductor, Fresnel specular
    uint32_t ext_lights;    // sphere or disk area lights, point, spot or distant lights
    uint32_t has_tex;       // some material reads a texture per hit (image maps, alpha, bump)
    uint32_t has_alpha;     // some material is ALPHA: triangle tests fetch its alpha map
    uint32_t has_bump;      // some material is BUMP: rays carry differentials
    uint32_t shade_kinds;   // bit k: some surface triangle shades in the wavefront's queue k
    // the four-wide tree of the spec's root (null: traversal walks the
    // binary tree), its map from binary inner nodes, and the stack words its
    // traversals can need; stack_words = the largest of the stacks
    const DevNode4* nodes4;
    const uint32_t* map4;
    int stack_cap4;
    uint32_t closest4;      // closest hit may use the four-wide tree
    int stack_words;
    // NOOR_ENV_REFERENCE: the reference's distribution tables (row r at
    // r * (rw + 1), the marginal at rh * (rw + 1)) and the environment as a
    // texture object (linear filter, clamp, normalised coordinates)
    uint32_t env_ref;
    cudaTextureObject_t env_tex;
    const float* rfunc;
    const float* rcdf;
    int rw, rh;
};

#ifdef __CUDACC__
// a texture slot at uv, scaled per component (uvscale * uv), fetched by the
// texture unit (CudaTexture::evaluate, noor/cuda/texture.cuh:113-126)
// (coordinates rounded per operation: the fetch sees the coordinate the
// reference's arithmetic gives, and its 8-bit filter weights amplify any
// last-bit difference)
__device__ __forceinline__ float4 slot_tex(const DevMatTex& T, uint32_t k, float2 uv) {
    const float2 s = T.uvscale[k];
    return tex2D<float4>(T.tex[k], __fmul_rn(s.x, uv.x), __fmul_rn(s.y, uv.y));
}
// texture coordinates of a triangle's vertex as the mesh manager returns
// them, v flipped (noor/cuda/mesh.cuh:145-148)
__device__ __forceinline__ float2 vertex_uv(const DevScene& S, uint32_t i) {
    const float2 t = __ldg(&S.uvs[i]);
    return make_float2(t.x, 1.0f - t.y);
}
// the barycentric interpolation (1 - u - v) uv0 + u uv1 + v uv2
__device__ __forceinline__ float2 lerp_uv(float2 a, float2 b, float2 c, float bu, float bv) {
    const float w = __fsub_rn(__fsub_rn(1.0f, bu), bv);
    return make_float2(__fadd_rn(__fadd_rn(__fmul_rn(w, a.x), __fmul_rn(bu, b.x)), __fmul_rn(bv, c.x)),
                       __fadd_rn(__fadd_rn(__fmul_rn(w, a.y), __fmul_rn(bu, b.y)), __fmul_rn(bv, c.y)));
}
#endif

}  // namespace nb
