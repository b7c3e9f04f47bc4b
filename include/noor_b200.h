/*
 * noor_b200.h -- C-ABI of the B200 path-tracing hot path.
 *
 * This header is the drop-in boundary for Noor's render-frame path.  It has
 * three layers:
 *
 *   1. POD mirrors of the host objects Noor hands to its device side
 *      (noor_payload  <- CudaPayload  noor/header/payload.h:27-127,
 *       noor_camera   <- CudaCamera   noor/cuda/camera.cuh:63-103,
 *       noor_hosek_sky<- CudaHosekSky noor/cuda/hosek.cuh:32-52,
 *       noor_spec     <- CudaSpec     noor/cuda/spec.cuh:41-58).
 *      Arrays are plain pointers + counts; the library deep-copies them
 *      (the caller keeps ownership), as the reference managers do
 *      (noor/cuda/mesh.cuh:64-103).
 *
 *   2. The eight entry points of noor/cuda/path_tracer.cuh:136-151 with the
 *      same names and meaning.  Differences: every call returns an int status
 *      (NOOR_OK or an error code, message via noor_last_error()) instead of
 *      exit()ing (path_tracer.cuh:154-171); `uint&` becomes `unsigned*`; the
 *      GL texture id becomes an opaque handle that may be NULL (there is no
 *      graphics interop, the film stays a device buffer).  These names act on
 *      the calling thread's current context (one context per thread, no other
 *      hidden global state).
 *
 *   3. Additions: film readback, batched multi-frame rendering, ray-batch
 *      traversal for parity tests, device-routine batch evaluators, the host
 *      scene builder (BVH + payload assembly, mirroring Model/BVH in
 *      noor/source/model.cpp and noor/source/bvh.cpp), the persistent
 *      wavefront integrator and the path-replay adjoint.
 *
 * All functions are thread-compatible: distinct contexts may be used from
 * distinct threads concurrently; one context must not be used concurrently.
 */
#ifndef NOOR_B200_H
#define NOOR_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif
#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
enum {
    NOOR_OK = 0,
    NOOR_ERR_INVALID = 1,      /* bad argument or malformed payload          */
    NOOR_ERR_CUDA = 2,         /* a CUDA runtime call failed                  */
    NOOR_ERR_NO_CONTEXT = 3,   /* no current context on this thread           */
    NOOR_ERR_UNSUPPORTED = 4,  /* feature outside the implemented path        */
    NOOR_ERR_OOM = 5,          /* device allocation failed                    */
    NOOR_ERR_DEVICE = 6,       /* a kernel reported a status word (overflow)  */
    NOOR_ERR_CAPACITY = 7      /* a request exceeds a fixed capacity          */
};

/* device status word bits (returned by noor_device_status) */
enum {
    NOOR_DEV_STACK_OVERFLOW = 1u << 0,   /* traversal stack exceeded its depth */
    NOOR_DEV_QUEUE_OVERFLOW = 1u << 1,   /* wavefront queue capacity exceeded  */
    NOOR_DEV_WAIT_TIMEOUT = 1u << 2,     /* a bounded device wait gave up      */
    NOOR_DEV_BAD_INDEX = 1u << 3         /* node/triangle index out of range   */
};

/* BVH node word masks: same bit layout as noor/cuda/path_tracer.cuh:52-64 */
#define NOOR_TRI_LEAF_MASK      0x80000000u
#define NOOR_MESH_LEAF_MASK     0x40000000u
#define NOOR_MESH_INSTANCE_MASK 0x20000000u
#define NOOR_MESH_INNER_MASK    0x10000000u
#define NOOR_MESH_NODE_MASK     0x70000000u
#define NOOR_COUNT_MASK         0x0FFFFFFFu
#define NOOR_TRI_COUNT_MASK     0x7FFFFFFFu
#define NOOR_AXIS_MASK          0x0FFFFFFFu
#define NOOR_TRANS_MASK         0x0FFFFFFFu
#define NOOR_LIGHT_NODE_MASK    0x08000000u
#define NOOR_LIGHT_MASK         0x07FFFFFFu

/* material type bits: noor/cuda/path_tracer.cuh:88-104 */
enum {
    NOOR_DIFFUSE = 1 << 0,
    NOOR_ORENNAYAR = 1 << 1,
    NOOR_TRANSLUCENT = 1 << 2,
    NOOR_GLOSSY = 1 << 3,
    NOOR_MIRROR = 1 << 4,
    NOOR_GLASS = 1 << 5,
    NOOR_ROUGHGLASS = 1 << 6,
    NOOR_METAL = 1 << 7,
    NOOR_SUBSTRATE = 1 << 8,
    NOOR_EMITTER = 1 << 9,
    NOOR_CLEARCOAT = 1 << 10,
    NOOR_SHADOWCATCHER = 1 << 11,
    NOOR_ALPHA = 1 << 12,
    NOOR_BUMP = 1 << 13,
    NOOR_MESHLIGHT = 1 << 14
};

/* skydome types: noor/cuda/path_tracer.cuh:128 */
enum { NOOR_SKY_HDR = 0, NOOR_SKY_PHYSICAL = 1, NOOR_SKY_CONSTANT = 2 };
/* lighting mask bits: noor/cuda/spec.cuh:27-32 */
#define NOOR_LIGHT_AREA_MASK 0x0001u
#define NOOR_LIGHT_SKY_MASK  0x0020u
/* area light shape types: noor/cuda/path_tracer.cuh:127 */
enum { NOOR_SHAPE_QUAD = 0, NOOR_SHAPE_SPHERE = 1, NOOR_SHAPE_DISK = 2 };
/* camera types: noor/cuda/path_tracer.cuh:130 */
enum { NOOR_CAMERA_PERSP = 0, NOOR_CAMERA_ORTHO = 1, NOOR_CAMERA_ENV = 2 };
/* ray-triangle test selector (build addition) */
enum { NOOR_ISECT_WATERTIGHT = 0, NOOR_ISECT_REF_WALD = 1 };
/* film accumulation selector (build addition) */
enum { NOOR_FILM_KAHAN = 0, NOOR_FILM_REF_LERP = 1 };
/* microfacet distribution selector for METAL materials (build addition) */
enum { NOOR_DIST_TROWBRIDGE_REITZ = 0, NOOR_DIST_BECKMANN = 1 };
/* environment sampling selector (build addition).
 * NOOR_ENV_FP64: the build's distribution, one cell per map texel (2048 x
 *   1024 cells of 4x4-supersampled luminance x sin(theta) for the physical
 *   sky) with FP64 prefix sums; map lookups by an FP32 bilinear filter.
 * NOOR_ENV_REFERENCE: the reference's own CudaDistribution2D
 *   (noor/cuda/distribution2d.cuh:63-337): a grid of
 *   clamp(nearestPow2(texture size), 32, 1024) cells per axis, each the 3x3
 *   mean of the texture's luminance read through the texture unit's bilinear
 *   filter, FP32 Blelloch prefix sums, and its sampling routine; the physical
 *   sky is first baked as sin(theta) x radiance into a 2048 x 2048 texture
 *   (update_skydome, noor/cuda/skydome.cuh:27-37), and HDR / constant map
 *   lookups go through the texture unit (tex2D, linear, clamp).  Maps must be
 *   power-of-two sized.  Not available to the adjoint. */
enum { NOOR_ENV_FP64 = 0, NOOR_ENV_REFERENCE = 1 };

/* ---------------------------------------------------------- payload mirror */

/* CudaShape, noor/cuda/shape.cuh:30-69 */
typedef struct noor_shape {
    float center[3];
    float u[3];
    float v[3];
    float n[3];
    float area;
    float radius;
    float radius2;
    int32_t light_idx;
    int32_t type;               /* NOOR_SHAPE_*: QUAD, SPHERE or DISK      */
} noor_shape;
/* The fields hold what the CudaShape constructor (shape.cuh:44-69) leaves:
 * radius = min(|u|, |v|) / 2; for SPHERE and DISK the center is moved to
 * center + (u + v) / 2 and area = 4 pi r^2 (sphere) or pi r^2 (disk); for
 * QUAD area = |u x v|.  n is the quad / disk normal. */

/* CudaAreaLight, noor/cuda/light.cuh:76-121 */
typedef struct noor_area_light {
    noor_shape shape;
    float ke[3];
    int32_t two_sided;
} noor_area_light;

/* CudaPointLight, noor/cuda/light.cuh:158-178 (CudaLight::_ke first) */
typedef struct noor_point_light {
    float ke[3];
    float position[3];
} noor_point_light;

/* CudaSpotLight, noor/cuda/light.cuh:180-214.  falloff() compares
 * `direction` with the direction from the shaded point TO the light:
 * cos >= cos_inner gives 1, cos < cos_outer 0, between ((cos - cos_outer) /
 * (cos_inner - cos_outer))^4. */
typedef struct noor_spot_light {
    float ke[3];
    float position[3];
    float direction[3];
    float cos_inner;
    float cos_outer;
} noor_spot_light;

/* CudaDistantLight, noor/cuda/light.cuh:216-238: `direction` points from
 * the scene towards the light and is a unit vector (the constructor
 * normalises it; noor_build_payload does the same for its input). */
typedef struct noor_distant_light {
    float ke[3];
    float direction[3];
} noor_distant_light;

/* ImageTexture entry of CudaPayload::_textures: constant material
 * parameters are 1x1 textures; the environment texture is the LAST entry
 * (noor/source/model.cpp:313-321).  rgba: width*height*4 floats, row-major,
 * row 0 = v of 0.  filter and address are the ImageTexture's modes
 * (noor/header/texture.h:133-185), with CUDA's values: a material texture
 * larger than 1x1 is fetched by the texture unit with them (normalised
 * coordinates), as the reference's Cuda2DTexture is
 * (noor/cuda/texture.cuh:375-400); 1x1 constants read their one texel. */
enum { NOOR_FILTER_POINT = 0, NOOR_FILTER_LINEAR = 1 };
enum { NOOR_ADDRESS_WRAP = 0, NOOR_ADDRESS_CLAMP = 1 };
typedef struct noor_texture {
    int32_t width;
    int32_t height;
    const float* rgba;
    int32_t filter;             /* NOOR_FILTER_*                             */
    int32_t address;            /* NOOR_ADDRESS_*                            */
} noor_texture;

/* CudaMaterial, noor/cuda/material.cuh:26-58 (+ one build field) */
typedef struct noor_material {
    float diffuse_uvscale[2];
    float specular_uvscale[2];
    float transparency_uvscale[2];
    float emittance_uvscale[2];
    float bump_uvscale[2];
    float roughness_uvscale[2];
    float metalness_uvscale[2];
    uint32_t diffuse_tex_idx;
    uint32_t specular_tex_idx;
    uint32_t transmission_tex_idx;
    uint32_t emittance_tex_idx;
    uint32_t bump_tex_idx;
    uint32_t transparency_tex_idx;
    uint32_t ior_tex_idx;
    uint32_t k_tex_idx;
    uint32_t roughness_tex_idx;
    uint32_t metalness_tex_idx;
    float bumpfactor;
    float emitter_scale;
    float coat_weight;
    float coat_roughness;
    float coat_thickness;
    float coat_sigma;
    float coat_ior;
    uint32_t type;              /* NOOR_* material bits                      */
    uint32_t distribution;      /* NOOR_DIST_*; the reference always uses 0  */
} noor_material;

/* CudaPayload, noor/header/payload.h:27-127.  All arrays are host memory. */
typedef struct noor_payload {
    uint32_t num_triangles;
    const uint32_t* attribute_indices;   /* uint4 per triangle: v0,v1,v2,mat  */
    const float* vertices;               /* float4 per (deduplicated) vertex  */
    const float* normals;                /* float4 per vertex                 */
    const float* uvs;                    /* float2 per vertex                 */
    uint32_t num_vertices;
    /* per mesh/instance 3-row transforms (float4 per row per instance) */
    const float* normal_row[3];
    const float* world_to_object_row[3];
    const float* object_to_world_row[3];
    uint32_t num_instances;
    /* Wald records, uint4 per triangle (noor/header/triangle.h:56-120) */
    const uint32_t* wald_ax_nu_nv_nd;
    const uint32_t* wald_bnu_bnv_au_av;
    const uint32_t* wald_cnu_cnv_deg_mat;
    /* BVH: two uint4 per node (noor/source/bvh.cpp:88-178) */
    uint32_t bvh_root_node;
    const uint32_t* bvh_min_right_start;
    const uint32_t* bvh_max_axis_count;
    uint32_t num_bvh_nodes;
    const noor_texture* textures;
    uint32_t num_textures;
    /* lights, indexed in this order: area, point, spot, distant, infinite
     * (setup_lights, noor/cuda/lightimp.cuh:244-281) */
    const noor_area_light* area_lights;
    int32_t num_area_lights;
    const noor_point_light* point_lights;
    int32_t num_point_lights;
    const noor_spot_light* spot_lights;
    int32_t num_spot_lights;
    const noor_distant_light* distant_lights;
    int32_t num_distant_lights;
    int32_t num_infinite_lights;         /* 0 or 1                            */
    const noor_material* materials;
    uint32_t num_materials;
} noor_payload;

/* CudaCamera, noor/cuda/camera.cuh:63-103.  Transforms are 3 rows of
 * (3x3 | translation), as CudaTransform(row0,row1,row2). */
typedef struct noor_camera {
    float camera_to_world[3][4];
    float raster_to_camera[3][4];
    float world_to_raster[3][4];
    float dx_camera[3];
    float dy_camera[3];
    float lens_radius;
    float focal_length;
    float image_area;
    uint32_t w;
    uint32_t h;
    uint32_t center;
    int32_t type;               /* only NOOR_CAMERA_PERSP, lens_radius 0    */
} noor_camera;

/* ArHosekSkyModelState (noor/external/ArHosekSkyModel.h:346-357) */
typedef struct noor_hosek_state {
    float configs[3][9];
    float radiances[3];
    float turbidity;
    float solar_radius;
    float emission_correction_factor_sky[3];
    float emission_correction_factor_sun[3];
    float albedo;
    float elevation;
} noor_hosek_state;

/* CudaHosekSky, noor/cuda/hosek.cuh:43-52 */
typedef struct noor_hosek_sky {
    noor_hosek_state state[3];  /* r, g, b */
    float solar_dir[3];
    float ground_albedo[3];
    float solar_scale;
    float solar_radius;
} noor_hosek_sky;

/* CudaSpec, noor/cuda/spec.cuh:41-58 (+ build selectors) */
typedef struct noor_spec {
    float reflection_bias;
    float shadow_bias;
    float world_radius;
    float wr2;
    uint32_t bvh_root_node;
    uint32_t lighting_type;     /* NOOR_LIGHT_*_MASK bits                   */
    uint32_t bounces;
    uint32_t rr;
    uint32_t bvh_height;
    uint32_t num_gpus;
    int32_t skydome_type;       /* NOOR_SKY_*                                */
    uint32_t debug_sky;
    uint32_t mis;
    uint32_t intersector;       /* NOOR_ISECT_*                              */
    uint32_t film_mode;         /* NOOR_FILM_*                               */
    uint32_t env_sampling;      /* NOOR_ENV_*                                */
} noor_spec;

/* ------------------------------------------------- reference entry points */
/* These eight carry the reference's names with C-ABI arguments.  A
 * translation unit that also sees the reference's own declarations of them
 * (path_tracer.cuh:136-151, C++ arguments, the same C names) -- the bridge
 * that replaces path_tracer.cu in the reference's host -- defines
 * NOOR_B200_NO_REFERENCE_PROTOTYPES before including this header and
 * resolves the library's versions with dlsym. */
#ifndef NOOR_B200_NO_REFERENCE_PROTOTYPES
/* noor/cuda/path_tracer.cuh:137-142: upload payload, sky, camera and spec
 * into a new context that becomes current on this thread.  hosek, camera and
 * spec are remembered (not copied for later): update_cuda_* re-read them, as
 * the reference device struct keeps references (noor/cuda/render.cuh:38-40).
 * The env/sky importance-sampling distribution is built here.  texture_handle
 * is unused (no graphics interop) and may be NULL.  The payload, spec and
 * camera are checked on the host first; a call they fail leaves the thread's
 * current context as it was. */
int load_cuda_data(const noor_payload* payload, const noor_hosek_sky* hosek,
                   const noor_camera* camera, const noor_spec* spec,
                   void* texture_handle);
/* path_tracer.cuh:144-146; re-upload from the structs given at load time.
 * Each resets the progressive film (noor/source/scene.cpp:124-144). */
int update_cuda_camera(void);
int update_cuda_hosek(void);
int update_cuda_spec(void);
/* path_tracer.cuh:147 / path_tracer.cu:132-155: render one sample per pixel
 * with frame number *frame_count, fold it into the film, then ++*frame_count.
 * A frame number of 1 restarts the film. */
int cuda_path_tracer(unsigned int* frame_count);
/* path_tracer.cuh:148 / path_tracer.cu:102-130: write the sky texture (and,
 * with MIS on, red importance samples) into the film, then ++*frame_count. */
int debug_skydome(unsigned int* frame_count, int width, int height);
/* path_tracer.cuh:149: free the current context and all device memory. */
int device_free_memory(void);
/* path_tracer.cuh:150: hit point of the centre pixel's primary ray from the
 * last frame (w = 1 if it hit, 0 otherwise). */
int get_lookAt(float look_at[4]);
#endif /* NOOR_B200_NO_REFERENCE_PROTOTYPES */

/* ------------------------------------------------------------- additions */
const char* noor_last_error(void);
int noor_device_count(int* count);
/* sizeof of the ABI structs, in declaration order: shape, area_light,
 * texture, material, payload, camera, hosek_state, hosek_sky, spec, ray,
 * hit, bvh_spec, mesh, material_desc, scene_desc, build_stat, wf_frame,
 * wf_params, adjoint_desc, wf_profile, point_light, spot_light,
 * distant_light.  Returns how many were written (<= n). */
int noor_abi_sizes(uint32_t* out, int n);

/* Render frames *frame_count .. *frame_count+n_frames-1 in one launch of the
 * plain megakernel (one path per (pixel, frame)) and fold them into the film
 * in frame order; *frame_count += n_frames. */
int noor_render_frames(unsigned int* frame_count, unsigned int n_frames);
/* Film readback: rgba = mean of the folded samples (w = 1). */
int noor_get_framebuffer(float* host_rgba, size_t n_pixels);
int noor_get_framebuffer_device(float* device_rgba, size_t n_pixels);
int noor_reset_film(void);
/* Headless display (noor/shader/cuda.fs:36-78, which the reference runs as
 * a GL fragment shader over the film texture): the transforms of its
 * `tonemap` subroutine, applied to exposure * rgb, then stored as 8-bit
 * unorm (clamp to [0, 1], round to nearest) with alpha 255. */
enum { NOOR_TONEMAP_NONE = -1, NOOR_TONEMAP_GAMMA = 0, NOOR_TONEMAP_REINHARD = 1, NOOR_TONEMAP_FILMIC = 2,
       NOOR_TONEMAP_UNCHARTED2 = 3 };
/* d_film_rgba: float4 per pixel (16-byte aligned device memory, e.g. from
 * noor_get_framebuffer_device or a wavefront film); d_rgba8: 4 bytes per
 * pixel, device memory, same pixel order. */
int noor_tonemap_device(const float* d_film_rgba, size_t n_pixels, int op, float exposure, uint8_t* d_rgba8);
/* The context's film as an image file: op NOOR_TONEMAP_NONE writes the
 * linear film as PFM (bottom row first, as film row 0 is the bottom of the
 * reference's GL window), any other op writes a binary PPM of the tonemapped
 * film, top row first. */
int noor_save_image(const char* path, int op, float exposure);
/* Rays traced by the megakernel since the last reset (device counters):
 * [0] extension (closest-hit) rays, [1] shadow (any-hit) rays, [2] paths. */
int noor_ray_counters(uint64_t counters[3], int reset);
/* Device status word (NOOR_DEV_* bits) accumulated since the last reset. */
int noor_device_status(uint32_t* status, int reset);
/* CUDA stream the current context launches on (cudaStream_t). */
void* noor_stream(void);
/* The calling thread's render context (NULL if none), and binding a context
 * to the calling thread (NULL unbinds).  A context stays owned by the thread
 * that created it (load_cuda_data) and is freed by device_free_memory on
 * that thread; another thread may borrow it, never concurrently with its
 * owner (e.g. a framework that runs a backward pass on a worker thread while
 * the owner waits). */
void* noor_context_current(void);
int noor_context_bind(void* context);
/* CUDA events on that stream (8 slots) for device-side timing. */
int noor_event_record(int slot);
int noor_event_elapsed(int slot_begin, int slot_end, float* ms);
/* kernels this context has launched so far */
int noor_launch_count(uint64_t* n);

/* Ray batches for parity tests.  Device pointers, launched on noor_stream(). */
typedef struct noor_ray {
    float org[3];
    float tmax;
    float dir[3];
    float pad;
} noor_ray;
typedef struct noor_hit {
    float t;
    uint32_t tri_idx;           /* index into the BVH-ordered triangle arrays */
    uint32_t ins_idx;
    uint32_t material_type;
    float u;
    float v;
    uint32_t hit;
    uint32_t pad;
} noor_hit;
/* closest hit (noor/cuda/bvh.cuh:142-191) with the intersector in the spec */
int noor_trace_closest(const noor_ray* d_rays, noor_hit* d_hits, size_t n);
/* any hit (noor/cuda/bvh.cuh:193-234); d_occluded: one uint32 per ray */
int noor_trace_any(const noor_ray* d_rays, uint32_t* d_occluded, size_t n);
/* camera rays of noor/cuda/cameraimp.cuh:182-228 for every pixel of frame
 * `frame` (RNG seeded as path_tracer.cu:90), device output */
int noor_camera_rays(unsigned int frame, noor_ray* d_rays);

/* Device-routine batch evaluators (parity tests of the shading routines).
 * kind: 0 = BSDF Eval, 1 = BSDF Pdf, 2 = BSDF Sample_f.
 * in: per sample 16 floats {wo_local[3], wi_local[3], u[2], mat_idx, ...}
 * out: per sample 8 floats {f[3], pdf, wi_local[3], sampled_type}.        */
int noor_eval_bsdf(int kind, const float* d_in, float* d_out, size_t n);
/* Stand-alone shading routines (parity tests), device arrays; needs no
 * context (launched on the current context's stream if there is one).
 * kind 0 / 1: Trowbridge-Reitz / Beckmann microfacet distribution
 *   (noor/cuda/distribution.cuh:58-342) with alpha = max(r^2, 1e-3) per
 *   axis; in 12 floats {r_x, r_y, wo[3], wh[3], u[2], -, -}, out 12 floats
 *   {D(wh), G(wo, wh), Pdf(wo, wh), Sample_wh(wo, u)[3], 0, alpha_x, 0...}
 * kind 2: Fresnel (noor/cuda/fresnel.cuh:58-107); in 9 floats {cos, etaI,
 *   etaT, eta[3], k[3]}, out 4 floats {dielectric F, conductor F[3] with
 *   etaI = 1}
 * kind 3: warps (noor/cuda/utils.cuh:364-404,470-486,487-539); in 3 floats
 *   {u[2], x}, out 16 floats {concentricSampleDisk[2],
 *   cosineSampleHemisphere[3], uniformSampleHemisphere[3] (both z up),
 *   sphericalDirection(u)[3], its sinTheta, powerHeuristic(1, u.x, 1, u.y),
 *   Erf(x), ErfInv(x), 0} */
int noor_eval_routines(int kind, const float* d_in, float* d_out, size_t n);
/* Hosek radiance of directions (3 floats each) -> rgb (3 floats each) */
int noor_eval_sky(const float* d_dirs, float* d_rgb, size_t n);
/* environment distribution: u (2 floats) -> {x, y, pdf} and pdf at (x,y) */
int noor_eval_env_sample(const float* d_u, float* d_out, size_t n);
/* copy of the FP64-built env distribution to the host: func (H*W floats),
 * conditional CDFs (H*(W+1)), marginal func (H), marginal CDF (H+1),
 * integrals {marginal integral}.  Pass NULL to query sizes via w,h. */
int noor_get_env_distribution(int* w, int* h, float* func, float* cdf,
                              float* marginal_func, float* marginal_cdf,
                              double* marginal_integral);
/* the NOOR_ENV_REFERENCE tables (built on first use of that mode) as the
 * reference lays them out (noor/cuda/distribution2d.cuh:166-220): func and
 * cdf hold h*(w+2)+1 floats each, row r at r*(w+1) (w values, then the
 * row's integral), the marginal at h*(w+1) (h values, then its integral).
 * Pass NULL arrays to query w, h. */
int noor_get_reference_distribution(int* w, int* h, float* func, float* cdf);

/* -------------------------------------------------- host scene builder */
/* BVHSpec, noor/header/spec.h:27-51 */
typedef struct noor_bvh_spec {
    uint32_t num_bins;
    uint32_t max_height;
    float Ci;
    float Ct;
    uint32_t min_leaf_tris;
    uint32_t max_leaf_tris;
} noor_bvh_spec;

/* Mesh, noor/header/assetLoader.h:45-101.  to_global is column-major
 * (glm::mat4 layout).  instance >= 0 makes this an instance of that source
 * mesh; light_idx >= 0 makes it a light node over area light light_idx
 * (tri_count 0; its bounds are the light shape's, and it gets an empty
 * bottom-level leaf starting at tri_start, as in the reference). */
typedef struct noor_mesh {
    uint32_t tri_start;
    uint32_t tri_count;
    float to_global[16];
    int32_t instance;
    int32_t light_idx;
} noor_mesh;

/* an image map as a texture file decodes (noor/header/texture.h:146-152):
 * width x height RGBA floats, row 0 = v of 0 */
typedef struct noor_image {
    int32_t width;
    int32_t height;
    const float* rgba;
} noor_image;

/* the map slots of a material, in the order of noor_material_desc.map and
 * .map_uvscale (the reference's getMaterial_map_* getters,
 * noor/source/model.cpp:220-300) */
enum {
    NOOR_MAP_DIFFUSE = 0,       /* map_Kd                                    */
    NOOR_MAP_ROUGHNESS = 1,
    NOOR_MAP_METALNESS = 2,
    NOOR_MAP_SPECULAR = 3,      /* map_Ks                                    */
    NOOR_MAP_EMITTANCE = 4,     /* map_Ke                                    */
    NOOR_MAP_ALPHA = 5,         /* map_d: point filtered, sets NOOR_ALPHA    */
    NOOR_MAP_BUMP = 6,          /* map_bump: sets NOOR_BUMP                  */
    NOOR_NUM_MAPS = 7
};

/* material parameters as an AssetLoader reports them
 * (noor/header/assetLoader.h:134-150): the constants, and per map slot an
 * index into noor_scene_desc.images (-1: the constant is used) with its uv
 * scale; bumpfactor scales the bump map's displacement. */
typedef struct noor_material_desc {
    float diffuse[3];
    float specular[3];
    float transmission[3];
    float emittance[3];
    float transparency[3];
    float ior[3];
    float k[3];
    float roughness[2];
    float coat_weight;
    float coat_roughness;
    float coat_thickness;
    float coat_sigma;
    float coat_ior;
    float emitter_scale;
    uint32_t type;
    uint32_t distribution;
    int32_t map[NOOR_NUM_MAPS];
    float map_uvscale[NOOR_NUM_MAPS][2];
    float bumpfactor;
} noor_material_desc;

/* loader output consumed by Model::load (noor/source/model.cpp:132-182) */
typedef struct noor_scene_desc {
    const float* vertices;          /* float4 */
    uint32_t num_vertices;
    const float* normals;           /* float4 */
    uint32_t num_normals;
    const float* uvs;               /* float2 */
    uint32_t num_uvs;
    const uint32_t* vindices;       /* 3 per triangle */
    const uint32_t* nindices;
    const uint32_t* uvindices;
    const uint32_t* material_indices; /* 1 per triangle */
    uint32_t num_triangles;
    const noor_mesh* meshes;
    uint32_t num_meshes;
    const noor_material_desc* materials;
    uint32_t num_materials;
    const noor_area_light* area_lights;
    uint32_t num_area_lights;
    const noor_point_light* point_lights;
    uint32_t num_point_lights;
    const noor_spot_light* spot_lights;
    uint32_t num_spot_lights;
    const noor_distant_light* distant_lights;
    uint32_t num_distant_lights;
    int32_t skydome_type;           /* NOOR_SKY_*                            */
    int32_t env_width;              /* HDR environment map (skydome_type 0)  */
    int32_t env_height;
    const float* env_rgba;
    noor_bvh_spec bvh;
    /* image maps the materials' map_* fields index (decoded texture files,
     * shared by every material that names the same file) */
    const noor_image* images;
    uint32_t num_images;
} noor_scene_desc;

/* Stat, noor/header/stat.h:26-49 (BVH part) + derived scene quantities */
typedef struct noor_build_stat {
    uint32_t height;
    uint32_t num_inner_nodes;
    uint32_t num_leaf_nodes;
    uint32_t max_leaf_tris;
    float scene_min[3];
    float scene_max[3];
    float scene_radius;
    double build_seconds;        /* the whole call                           */
    double box_seconds;          /* triangle and mesh boxes (host)           */
    double tree_seconds;         /* the trees: host, or GPU with transfers   */
    double tree_device_ms;       /* GPU build: device time of the trees      */
    double tail_seconds;         /* vertex de-duplication, Wald records      */
    double tail_device_ms;       /* GPU build: device time of those          */
} noor_build_stat;

typedef struct noor_payload_handle noor_payload_handle;
/* Model::load + BVH build + Model::loadCudaPayload on the host. */
int noor_build_payload(const noor_scene_desc* desc, noor_payload_handle** out,
                       noor_build_stat* stat);
/* The same payload, bit for bit, built on the current CUDA device: the
 * per-mesh bottom-level trees level by level (binning, split search and
 * partition in kernels; the top level over the meshes stays on the host),
 * then the vertex de-duplication in BVH order, the Wald records and the
 * attribute words.  Needs a GPU; errors as noor_build_payload, plus
 * NOOR_ERR_CUDA. */
int noor_build_payload_gpu(const noor_scene_desc* desc, noor_payload_handle** out,
                           noor_build_stat* stat);
/* View of the owned arrays (valid until noor_free_payload). */
int noor_payload_view(const noor_payload_handle* h, noor_payload* out);
/* source triangle index of each BVH-ordered triangle */
int noor_payload_triangle_order(const noor_payload_handle* h, uint32_t* out,
                                size_t n);
/* CudaSpec fields Scene::load derives (noor/source/scene.cpp:51-91):
 * biases, world radius, BVH root and height, sky bit from the light count. */
int noor_payload_default_spec(const noor_payload_handle* h, uint32_t bounces,
                              uint32_t rr, noor_spec* out);
void noor_free_payload(noor_payload_handle* h);
/* The four-wide tree that scene upload builds over the payload's BVH from
 * `root` (host only, no device needed): the number of wide nodes, of binary
 * inner nodes whose children a wide node holds in its own slots, the stack
 * words its traversals can need, and whether closest hit uses it
 * (*closest = 1).  NOOR_ERR_UNSUPPORTED (with the reason) for a tree upload
 * leaves to the binary traversal: a cycle, a NaN bound, or a stack deeper
 * than 96 words. */
int noor_wide_tree_info(const noor_payload* payload, uint32_t root, uint32_t* num_wide,
                        uint32_t* num_expanded, uint32_t* stack_need, uint32_t* closest);

/* Camera::reset + CudaCamera::update for a pinhole perspective camera
 * (noor/header/camera.h:99-153,255-300; noor/cuda/camera.cuh:66-94).
 * fov in radians. */
int noor_camera_lookat(const float eye[3], const float look_at[3],
                       const float up[3], float fov, uint32_t w, uint32_t h,
                       noor_camera* out);

/* Hosek-Wilkie RGB state fit (ArHosekSkyModel.cpp:147-289,667-695) run in
 * FP64 on the GPU.  dataset: the 3 RGB coefficient tables (3 x 1080 floats)
 * followed by the 3 radiance tables (3 x 120 floats).  Fills the three
 * per-channel states and the sun fields as HosekSky::update does
 * (noor/header/hosek.h:61-83); sun_lat is the polar angle of the sun. */
int noor_hosek_fit(const float* dataset, float turbidity,
                   const float ground_albedo[3], float sun_lat, float sun_lon,
                   float solar_scale, float solar_radius_scale,
                   noor_hosek_sky* out);

/* ------------------------------------------------ wavefront integrator */
/* One frame of a batched wavefront render.  Each frame names a loaded
 * context-independent scene (noor_scene_upload) by id. */
typedef struct noor_wf_frame {
    uint32_t scene_id;
    uint32_t width;
    uint32_t height;
    uint32_t spp;
    uint32_t first_frame;       /* RNG frame number of the first sample     */
    uint32_t bounces;
    noor_camera camera;
    float* d_film;              /* device float4 per pixel (mean), or NULL  */
} noor_wf_frame;

typedef struct noor_wf_params {
    uint32_t block_size;        /* threads per block of the stage kernels   */
    uint32_t queue_capacity;    /* path slots in flight                     */
    uint32_t sort_granularity;  /* how finely rays are ordered for SIMT
                                 * coherence: 0 one shading queue; 1 one per
                                 * material kind; 2 also extension rays
                                 * (camera rays compacted in slot order,
                                 * secondary rays by a counting sort on
                                 * (direction octant, origin cell of a 16^3
                                 * grid)); 3 also shadow rays, by the same
                                 * sort; larger values act as 3             */
    uint32_t use_graph;         /* capture one bounce as a CUDA graph       */
    uint32_t max_iterations;    /* bound of the bounce loop; 0: enough for
                                 * every path (slots x bounces); a loop that
                                 * reaches it stops and sets
                                 * NOOR_DEV_WAIT_TIMEOUT                    */
    uint32_t traversal;         /* the trees the extension and shadow
                                 * stages walk (the same hits either way):
                                 * NOOR_TRAVERSAL_*                          */
    uint32_t shade_regs;        /* registers per thread of the shading
                                 * stage: 0 or 80 (24 warps per SM), 128
                                 * (16 warps, no spills); the same results */
} noor_wf_params;
/* BINARY: both stages on the binary tree; WIDE: both on the four-wide tree
 * where every scene of the launch has one (noor_wide_tree_info);
 * WIDE_SHADOW: extension rays on the binary tree, shadow rays on the
 * four-wide one; AUTO: WIDE_SHADOW when every scene of the launch has a
 * four-wide tree and at least 16384 triangles, else BINARY */
enum {
    NOOR_TRAVERSAL_AUTO = 0,
    NOOR_TRAVERSAL_BINARY = 1,
    NOOR_TRAVERSAL_WIDE = 2,
    NOOR_TRAVERSAL_WIDE_SHADOW = 3
};

/* Scenes for the wavefront live in the current context; scene 0 is the one
 * load_cuda_data uploaded.  Adds another payload/sky/spec, returns its id. */
int noor_scene_upload(const noor_payload* payload, const noor_hosek_sky* hosek,
                      const noor_spec* spec, uint32_t* scene_id);
int noor_wavefront_render(const noor_wf_frame* frames, uint32_t n_frames,
                          const noor_wf_params* params);
/* as noor_wavefront_render, also returning the device time of the batch */
int noor_wavefront_render_timed(const noor_wf_frame* frames, uint32_t n_frames,
                                const noor_wf_params* params, float* ms);
/* rays and paths the wavefront traced: [0] extension, [1] shadow, [2] paths */
int noor_wavefront_counters(uint64_t counters[3], int reset);
/* Device time per stage of one wavefront render, for measurement: the batch
 * is rendered in the host-loop form (use_graph ignored) with CUDA events
 * around every stage.  Stages: 0 regen, 1 extension-ray ordering (sort
 * granularity 2 and up), 2 extend, 3 shade (queue binning and all material
 * kinds), 4 shadow-ray ordering (sort granularity 3), 5 shadow, 6 stop
 * test. */
typedef struct noor_wf_profile {
    float ms[7];                /* summed over iterations                   */
    uint32_t launches[7];
    uint32_t iterations;
} noor_wf_profile;
int noor_wavefront_profile(const noor_wf_frame* frames, uint32_t n_frames,
                           const noor_wf_params* params, noor_wf_profile* out);
/* The same frames rendered one after another by the plain megakernel
 * (one launch per frame, film folded with Kahan summation); device time of
 * the whole sequence in *ms. */
int noor_megakernel_batch(const noor_wf_frame* frames, uint32_t n_frames,
                          float* ms);
/* No counterpart in the reference.  One frame with the plain megakernel into
 * the caller's film (frame->d_film, required: float4 per pixel, the mean over
 * frame->spp samples), allocating no device memory: for callers that cannot
 * call cudaMalloc while they render (memory they do not own, hosts that forbid
 * device allocation after start-up).  Scratch comes from one fixed device
 * array of NOOR_NOALLOC_SCRATCH_BYTES, which bounds a frame to
 * NOOR_NOALLOC_SCRATCH_BYTES / 16 pixels (larger frames return
 * NOOR_ERR_CAPACITY).  The first call on a device looks up the array's
 * address (cudaGetSymbolAddress); make it before any stream capture.
 * device_free_memory forgets the address, so the first call after it (and
 * after any reset of the device) looks it up again.  A call waits for its
 * work to finish before it returns.  All calls on a device share the array,
 * so calls that overlap on the GPU race; nothing in it needs clearing
 * between calls. */
#define NOOR_NOALLOC_SCRATCH_BYTES (32u << 20)
int noor_megakernel_frame_noalloc(const noor_wf_frame* frame);
/* Project-written autotuner: coordinate descent on the launch parameters,
 * each candidate timed by one device-timed render of the given batch: slot
 * count (2^18 .. 2^23, at most twice the batch's paths), block size (32, 64,
 * 128), sort granularity (0 .. 3), then the slot count once more around the
 * sort level chosen.  *best = the fastest seen (use_graph as given). */
int noor_wavefront_autotune(const noor_wf_frame* frames, uint32_t n_frames,
                            noor_wf_params* best, float* best_ms);

/* ----------------------------------------------- path-replay adjoint */
/* Differentiable parameters: per material albedo (3) and roughness (1), and
 * the environment texels (3 per texel).  Rendering uses scene 0. */
typedef struct noor_adjoint_desc {
    uint32_t width;
    uint32_t height;
    uint32_t spp;
    uint32_t first_frame;
    uint32_t bounces;
    float* d_albedo;            /* num_materials x 3, device               */
    float* d_roughness;         /* num_materials, device                   */
    float* d_env;               /* env_h x env_w x 3, device               */
} noor_adjoint_desc;
/* forward: render into d_image (float3 per pixel, mean over spp) */
int noor_adjoint_forward(const noor_adjoint_desc* desc, float* d_image);
/* backward: accumulate dLoss/dparams given dLoss/dimage (float3/pixel) */
int noor_adjoint_backward(const noor_adjoint_desc* desc,
                          const float* d_grad_image, float* d_grad_albedo,
                          float* d_grad_roughness, float* d_grad_env);

#ifdef __cplusplus
}
#endif
#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#endif /* NOOR_B200_H */
