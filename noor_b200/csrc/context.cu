// Runtime of the C-ABI: per-thread render context, device residency of the
// payload (the work of CudaRenderDevice / the Cuda*Manager constructors,
// noor/cuda/render.cuh:67-149, mesh.cuh:64-103, lightimp.cuh:299-371), the
// reference entry points of noor/cuda/path_tracer.cuh:136-151 and the
// additions declared in include/noor_b200.h.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "host_common.h"
#include "kernels.h"
#include "runtime.h"
#include "shading.cuh"
#include "wide_bvh.h"

// 1: traversal walks the four-wide tree built at upload; 0: the binary tree
#ifndef NB_WIDE_TREE
#define NB_WIDE_TREE 1
#endif

// ------------------------------------------------------------------ errors
static thread_local std::string tl_err;
int set_error(int code, const std::string& msg) {
    tl_err = msg;
    return code;
}
void clear_error() { tl_err.clear(); }
extern "C" const char* noor_last_error(void) { return tl_err.c_str(); }

namespace nb {

thread_local Context* tl_ctx = nullptr;

int cuda_fail(cudaError_t e, const char* what) {
    return set_error(e == cudaErrorMemoryAllocation ? NOOR_ERR_OOM : NOOR_ERR_CUDA,
                     std::string(what) + ": " + cudaGetErrorString(e));
}

SceneState::~SceneState() {
    if (env_tex) cudaDestroyTextureObject(env_tex);
    if (env_array) cudaFreeArray(env_array);
    for (auto& t : textures) {
        if (t.second.obj) cudaDestroyTextureObject(t.second.obj);
        if (t.second.array) cudaFreeArray(t.second.array);
    }
    for (void* p : allocs) cudaFree(p);
}

// The texture object of payload texture `idx` (made once): an RGBA float
// array with the texture's filter and addressing over normalised
// coordinates, as Cuda2DTexture makes it (noor/cuda/texture.cuh:375-400,
// NOOR::create_2d_texobj).
int SceneState::texture_object(const noor_texture& t, uint32_t idx, cudaTextureObject_t* out) {
    auto it = textures.find(idx);
    if (it != textures.end()) {
        *out = it->second.obj;
        return NOOR_OK;
    }
    TexObj o{};
    const cudaChannelFormatDesc cd = cudaCreateChannelDesc<float4>();
    cudaError_t e = cudaMallocArray(&o.array, &cd, (size_t)t.width, (size_t)t.height);
    if (e != cudaSuccess) return cuda_fail(e, "texture array");
    textures[idx] = o;
    e = cudaMemcpy2DToArray(o.array, 0, 0, t.rgba, (size_t)t.width * 16, (size_t)t.width * 16, (size_t)t.height,
                            cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "texture upload");
    cudaResourceDesc rd;
    std::memset(&rd, 0, sizeof(rd));
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = o.array;
    cudaTextureDesc td;
    std::memset(&td, 0, sizeof(td));
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = (cudaTextureAddressMode)t.address;
    td.filterMode = t.filter == NOOR_FILTER_LINEAR ? cudaFilterModeLinear : cudaFilterModePoint;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 1;
    e = cudaCreateTextureObject(&o.obj, &rd, &td, nullptr);
    if (e != cudaSuccess) return cuda_fail(e, "texture object");
    textures[idx] = o;
    *out = o.obj;
    return NOOR_OK;
}

int SceneState::alloc(void** p, size_t bytes, const char* what) {
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) return cuda_fail(e, what);
    allocs.push_back(*p);
    return NOOR_OK;
}

int SceneState::upload(void** p, const void* host, size_t bytes, const char* what) {
    int rc = alloc(p, bytes, what);
    if (rc) return rc;
    if (host && bytes) {
        cudaError_t e = cudaMemcpy(*p, host, bytes, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return cuda_fail(e, what);
    }
    return NOOR_OK;
}

Context::~Context() {
    if (stream) cudaStreamSynchronize(stream);
    scenes.clear();
    for (void* p : {(void*)film_sum, (void*)film_comp, (void*)film_out, (void*)part_sum, (void*)part_comp,
                    (void*)lookat, (void*)status, (void*)counters, (void*)scratch, adj_buf})
        if (p) cudaFree(p);
    for (auto& e : events)
        if (e) cudaEventDestroy(e);
    wavefront_release(*this);
    if (stream) cudaStreamDestroy(stream);
}

// The constant parameters (the first texel of each texture: a 1x1
// texture's value) and, per slot read through the texture unit, the texture
// object and uv scale.  `object(i)` makes (once) the texture object of
// texture i.
template <class Obj>
static void resolve_textures(const noor_payload* P, const noor_material& m, DevMaterial& d, DevMatTex& t,
                             Obj object) {
    std::memset(&t, 0, sizeof(t));
    auto image = [&](uint32_t idx) { return P->textures[idx].width != 1 || P->textures[idx].height != 1; };
    auto slot = [&](uint32_t k, uint32_t idx, const float* uvscale) {
        t.tex[k] = object(idx);
        t.uvscale[k] = make_float2(uvscale ? uvscale[0] : 1.0f, uvscale ? uvscale[1] : 1.0f);
        d.tex_mask |= 1u << k;
    };
    if (image(m.diffuse_tex_idx)) slot(kTexDiffuse, m.diffuse_tex_idx, m.diffuse_uvscale);
    if (image(m.specular_tex_idx)) slot(kTexSpecular, m.specular_tex_idx, m.specular_uvscale);
    if (image(m.emittance_tex_idx)) slot(kTexEmittance, m.emittance_tex_idx, m.emittance_uvscale);
    if (image(m.roughness_tex_idx)) slot(kTexRoughness, m.roughness_tex_idx, m.roughness_uvscale);
    // transmission, ior and k are read at uv scale 1 (materialimp.cuh:155-182)
    if (image(m.transmission_tex_idx)) slot(kTexTransmission, m.transmission_tex_idx, nullptr);
    if (image(m.ior_tex_idx)) slot(kTexIor, m.ior_tex_idx, nullptr);
    if (image(m.k_tex_idx)) slot(kTexK, m.k_tex_idx, nullptr);
    if (m.type & NOOR_ALPHA) slot(kTexAlpha, m.transparency_tex_idx, m.transparency_uvscale);
    if (m.type & NOOR_BUMP) slot(kTexBump, m.bump_tex_idx, m.bump_uvscale);
    t.bumpfactor = m.bumpfactor;
}

static void resolve_material(const noor_payload* P, const noor_material& m, DevMaterial& d) {
    auto tex = [&](uint32_t idx) -> float3 {
        const float* t = P->textures[idx].rgba;
        return make_float3(t[0], t[1], t[2]);
    };
    d.diffuse = tex(m.diffuse_tex_idx);
    d.specular = tex(m.specular_tex_idx);
    d.transmission = tex(m.transmission_tex_idx);
    d.emittance = tex(m.emittance_tex_idx);
    d.ior = tex(m.ior_tex_idx);
    d.k = tex(m.k_tex_idx);
    const float3 r = tex(m.roughness_tex_idx);
    d.rough_x = r.x;
    d.rough_y = r.y;
    d.coat_ior = m.coat_ior;
    d.coat_weight = m.coat_weight;
    d.coat_sigma = m.coat_sigma;
    d.coat_thickness = m.coat_thickness;
    d.emitter_scale = m.emitter_scale;
    d.type = m.type;
    d.distribution = m.distribution;
}

static int validate_payload(const noor_payload* P) {
    if (!P) return set_error(NOOR_ERR_INVALID, "payload is null");
    if (P->num_triangles == 0 || !P->attribute_indices || !P->wald_ax_nu_nv_nd || !P->wald_bnu_bnv_au_av ||
        !P->wald_cnu_cnv_deg_mat || !P->bvh_min_right_start || !P->bvh_max_axis_count || P->num_bvh_nodes == 0 ||
        !P->vertices || !P->normals || !P->uvs || P->num_vertices == 0)
        return set_error(NOOR_ERR_INVALID, "payload: missing geometry or BVH arrays");
    if (P->bvh_root_node >= P->num_bvh_nodes) return set_error(NOOR_ERR_INVALID, "payload: BVH root out of range");
    if (P->num_area_lights < 0 || (P->num_area_lights > 0 && !P->area_lights))
        return set_error(NOOR_ERR_INVALID, "payload: bad area light array");
    if (P->num_point_lights < 0 || (P->num_point_lights > 0 && !P->point_lights) || P->num_spot_lights < 0 ||
        (P->num_spot_lights > 0 && !P->spot_lights) || P->num_distant_lights < 0 ||
        (P->num_distant_lights > 0 && !P->distant_lights))
        return set_error(NOOR_ERR_INVALID, "payload: bad point, spot or distant light array");
    if (P->num_infinite_lights < 0 || P->num_infinite_lights > 1)
        return set_error(NOOR_ERR_INVALID, "payload: at most one infinite light");
    if (P->num_materials == 0 || !P->materials) return set_error(NOOR_ERR_INVALID, "payload: no materials");
    if (P->num_textures == 0 || !P->textures) return set_error(NOOR_ERR_INVALID, "payload: no textures");
    if (P->num_instances == 0) return set_error(NOOR_ERR_INVALID, "payload: no instance transforms");
    for (int r = 0; r < 3; ++r)
        if (!P->normal_row[r] || !P->world_to_object_row[r] || !P->object_to_world_row[r])
            return set_error(NOOR_ERR_INVALID, "payload: missing transform rows");
    const noor_texture& env = P->textures[P->num_textures - 1];
    if (env.width <= 0 || env.height <= 0 || !env.rgba) return set_error(NOOR_ERR_INVALID, "payload: bad environment texture");
    for (uint32_t i = 0; i + 1 < P->num_textures; ++i) {
        const noor_texture& t = P->textures[i];
        if (t.width <= 0 || t.height <= 0 || !t.rgba) return set_error(NOOR_ERR_INVALID, "payload: empty texture");
        if (t.filter < NOOR_FILTER_POINT || t.filter > NOOR_FILTER_LINEAR || t.address < 0 || t.address > 3)
            return set_error(NOOR_ERR_INVALID, "payload: texture filter or address mode out of range");
    }
    for (uint32_t i = 0; i < P->num_materials; ++i) {
        const noor_material& m = P->materials[i];
        const uint32_t idx[] = {m.diffuse_tex_idx,  m.specular_tex_idx, m.transmission_tex_idx, m.emittance_tex_idx,
                                m.ior_tex_idx,      m.k_tex_idx,        m.roughness_tex_idx,    m.transparency_tex_idx,
                                m.bump_tex_idx,     m.metalness_tex_idx};
        for (uint32_t t : idx)
            if (t + 1 >= P->num_textures)
                return set_error(NOOR_ERR_INVALID, "payload: material texture index out of range");
        // every other type is accepted: the ones factoryBSDF builds no lobe
        // for (Oren-Nayar, mixes of type bits) absorb, as in the reference
        // (bsdf.cuh:425-461)
        if (m.distribution > 1u) return set_error(NOOR_ERR_INVALID, "payload: unknown microfacet distribution");
    }
    for (int i = 0; i < P->num_area_lights; ++i) {
        const noor_shape& sh = P->area_lights[i].shape;
        if (sh.type != NOOR_SHAPE_QUAD && sh.type != NOOR_SHAPE_SPHERE && sh.type != NOOR_SHAPE_DISK)
            return set_error(NOOR_ERR_INVALID, "payload: unknown area light shape type");
        if (sh.type != NOOR_SHAPE_QUAD && !(sh.radius > 0.0f))
            return set_error(NOOR_ERR_INVALID, "payload: sphere or disk light without a radius");
    }
    // attribute and node indices
    for (size_t i = 0; i < (size_t)P->num_triangles; ++i) {
        const uint32_t* a = P->attribute_indices + 4 * i;
        if (a[0] >= P->num_vertices || a[1] >= P->num_vertices || a[2] >= P->num_vertices || a[3] >= P->num_materials)
            return set_error(NOOR_ERR_INVALID, "payload: attribute index out of range");
    }
    for (size_t i = 0; i < (size_t)P->num_bvh_nodes; ++i) {
        const uint32_t w0 = P->bvh_min_right_start[4 * i + 3];
        const uint32_t w1 = P->bvh_max_axis_count[4 * i + 3];
        if (w1 & NOOR_LIGHT_NODE_MASK) {
            if ((int)(w1 & NOOR_LIGHT_MASK) >= P->num_area_lights)
                return set_error(NOOR_ERR_INVALID, "payload: light node names a missing light");
        } else if (w1 & NOOR_MESH_INSTANCE_MASK) {
            if ((w1 & NOOR_TRANS_MASK) >= P->num_instances || w0 >= P->num_bvh_nodes)
                return set_error(NOOR_ERR_INVALID, "payload: instance node out of range");
        } else if (w1 & NOOR_MESH_LEAF_MASK) {
            if (i + (w1 & NOOR_COUNT_MASK) >= P->num_bvh_nodes)
                return set_error(NOOR_ERR_INVALID, "payload: mesh leaf children out of range");
        } else if (w1 & NOOR_TRI_LEAF_MASK) {
            if ((uint64_t)w0 + (w1 & NOOR_TRI_COUNT_MASK) > P->num_triangles)
                return set_error(NOOR_ERR_INVALID, "payload: leaf triangle range out of range");
        } else {
            if (w0 >= P->num_bvh_nodes || i + 1 >= P->num_bvh_nodes || (w1 & NOOR_AXIS_MASK) > 2u)
                return set_error(NOOR_ERR_INVALID, "payload: inner node child out of range");
        }
    }
    return NOOR_OK;
}

void apply_spec(SceneState& st, const noor_spec& s) {
    DevScene& D = st.dev;
    D.bias = s.reflection_bias;
    D.world_radius = s.world_radius;
    D.root = s.bvh_root_node;
    D.bounces = s.bounces;
    D.rr = s.rr;
    D.mis = s.mis;
    D.sky_on = (s.lighting_type & NOOR_LIGHT_SKY_MASK) ? 1u : 0u;
    D.sky_type = st.sky_type;
    D.isect = s.intersector;
    D.film_mode = s.film_mode;
    int cap = (int)s.bvh_height + (int)st.max_mesh_leaf + 4;
    D.stack_cap = cap < 16 ? 16 : (cap > 96 ? 96 : cap);
    // the four-wide tree serves the root it was built from
    const bool wide = st.wide_nodes && s.bvh_root_node == st.wide_root;
    D.nodes4 = wide ? st.wide_nodes : nullptr;
    D.map4 = wide ? st.wide_map : nullptr;
    D.stack_cap4 = wide ? st.wide_cap : 0;
    D.closest4 = wide && st.wide_closest ? 1u : 0u;
    D.stack_words = std::max(D.stack_cap, D.stack_cap4);
}

void apply_hosek(SceneState& st, const noor_hosek_sky& h) {
    DevHosek& H = st.dev.hosek;
    for (int c = 0; c < 3; ++c) {
        for (int i = 0; i < 9; ++i) H.configs[c][i] = h.state[c].configs[c][i];
        H.radiance[c] = h.state[c].radiances[c];
    }
    H.solar_dir = make_float3(h.solar_dir[0], h.solar_dir[1], h.solar_dir[2]);
    H.solar_scale = h.solar_scale;
    H.solar_radius = h.solar_radius;
}

int build_distribution(Context& C, SceneState& st) {
    EnvBuild& b = st.env;
    cudaError_t e;
    if (st.sky_type == NOOR_SKY_PHYSICAL)
        e = launch_env_func_from_sky(st.dev.hosek, b.w, b.h, b.func, C.stream);
    else
        e = launch_env_func_from_texture(st.dev.env, b.w, b.h, b.func, C.stream);
    if (e != cudaSuccess) return cuda_fail(e, "env func");
    e = launch_env_cdf(b, C.stream);
    if (e != cudaSuccess) return cuda_fail(e, "env cdf");
    float mi = 0.0f;
    e = cudaMemcpyAsync(&mi, b.marg_int_out, sizeof(float), cudaMemcpyDeviceToHost, C.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(C.stream);
    if (e != cudaSuccess) return cuda_fail(e, "env integral");
    C.launches += 3;
    st.dev.dist.marg_int = mi;
    return NOOR_OK;
}

// nearestPow2 (noor/cuda/utils.cuh:106-135): the nearer of the powers of two
// around n, the lower one on a tie
static int nearest_pow2(int n) {
    int next = n - 1;
    next |= next >> 1;
    next |= next >> 2;
    next |= next >> 4;
    next |= next >> 8;
    next |= next >> 16;
    next++;
    const int prev = (int)powf(2.0f, (float)(int)log2f((float)n));
    return fabsf((float)(n - next)) < fabsf((float)(n - prev)) ? next : prev;
}

// NOOR_ENV_REFERENCE tables (distribution2d.cuh:166-228), from the map or,
// for the physical sky, from a 2048 x 2048 bake of sin(theta) x radiance
// (skydome.cuh:27-37, the texture model.cpp:318 makes for it); rebuilt when
// the sky changes.
int build_reference_distribution(Context& C, SceneState& st) {
    DevScene& D = st.dev;
    const bool sky = st.sky_type == NOOR_SKY_PHYSICAL;
    const int tw = sky ? 2048 : D.env_w, th = sky ? 2048 : D.env_h;
    if ((tw & (tw - 1)) || (th & (th - 1)))
        return set_error(NOOR_ERR_UNSUPPORTED, "reference env sampling: the map must be power-of-two sized");
    const int w = std::min(std::max(nearest_pow2(tw), 32), 1024), h = std::min(std::max(nearest_pow2(th), 32), 1024);
    const size_t n = (size_t)h * (w + 2) + 1;
    cudaError_t e = cudaSuccess;
    int rc;
    if (!st.ref_built) {
        // two floats of padding past the reference's table size: its
        // searches never select them for u < 1, and they read as zero
        if ((rc = st.alloc((void**)&st.ref_func, (n + 2) * 4, "reference env func"))) return rc;
        if ((rc = st.alloc((void**)&st.ref_cdf, (n + 2) * 4, "reference env cdf"))) return rc;
        if (sky && (rc = st.alloc((void**)&st.ref_bake, (size_t)tw * th * 16, "sky bake"))) return rc;
        const cudaChannelFormatDesc fd = cudaCreateChannelDesc<float4>();
        e = cudaMallocArray(&st.env_array, &fd, tw, th);
        if (e != cudaSuccess) return cuda_fail(e, "environment array");
        cudaResourceDesc rd{};
        rd.resType = cudaResourceTypeArray;
        rd.res.array.array = st.env_array;
        cudaTextureDesc td{};
        td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeClamp;
        // the constant sky is a point-filtered 1x1 texture (texture.h:148-158)
        td.filterMode = st.sky_type == NOOR_SKY_CONSTANT ? cudaFilterModePoint : cudaFilterModeLinear;
        td.readMode = cudaReadModeElementType;
        td.normalizedCoords = 1;
        e = cudaCreateTextureObject(&st.env_tex, &rd, &td, nullptr);
        if (e != cudaSuccess) return cuda_fail(e, "environment texture");
    }
    const float4* src = D.env;
    if (sky) {
        if ((e = launch_ref_sky_bake(D.hosek, tw, th, st.ref_bake, C.stream)) != cudaSuccess) return cuda_fail(e, "sky bake");
        src = st.ref_bake;
        C.launches++;
    }
    e = cudaMemcpy2DToArrayAsync(st.env_array, 0, 0, src, (size_t)tw * 16, (size_t)tw * 16, th, cudaMemcpyDeviceToDevice,
                                 C.stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(st.ref_func, 0, (n + 2) * 4, C.stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(st.ref_cdf, 0, (n + 2) * 4, C.stream);
    if (e == cudaSuccess) e = launch_ref_distribution(st.env_tex, w, h, st.ref_func, st.ref_cdf, C.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(C.stream);
    if (e != cudaSuccess) return cuda_fail(e, "reference env distribution");
    C.launches += 5;
    st.ref_built = true;
    D.env_tex = st.env_tex;
    D.rfunc = st.ref_func;
    D.rcdf = st.ref_cdf;
    D.rw = w;
    D.rh = h;
    return NOOR_OK;
}

// the spec's environment sampling mode, building the reference tables on
// first use
static int apply_env_mode(Context& C, SceneState& st, const noor_spec& s) {
    st.dev.env_ref = s.env_sampling == NOOR_ENV_REFERENCE ? 1u : 0u;
    if (st.dev.env_ref && !st.ref_built) return build_reference_distribution(C, st);
    return NOOR_OK;
}

// every host-side check of a scene, made before any device work
static int check_scene_inputs(const noor_payload* P, const noor_hosek_sky* H, const noor_spec* S) {
    int rc = validate_payload(P);
    if (rc) return rc;
    if (!S) return set_error(NOOR_ERR_INVALID, "spec is null");
    if (S->skydome_type < 0 || S->skydome_type > 2) return set_error(NOOR_ERR_INVALID, "spec: bad skydome type");
    if (S->skydome_type == NOOR_SKY_PHYSICAL && !H) return set_error(NOOR_ERR_INVALID, "physical sky without Hosek state");
    if (S->intersector > 1u || S->film_mode > 1u || S->env_sampling > 1u)
        return set_error(NOOR_ERR_INVALID, "spec: bad selector");
    if (S->bvh_root_node >= P->num_bvh_nodes) return set_error(NOOR_ERR_INVALID, "spec: BVH root out of range");
    return NOOR_OK;
}

int upload_scene(Context& C, const noor_payload* P, const noor_hosek_sky* H, const noor_spec* S, SceneState& st,
                 bool checked = false) {
    int rc = checked ? NOOR_OK : check_scene_inputs(P, H, S);
    if (rc) return rc;
    DevScene& D = st.dev;
    std::memset(&D, 0, sizeof(D));
    const size_t nt = P->num_triangles, nn = P->num_bvh_nodes, nv = P->num_vertices, ni = P->num_instances;
    // nodes: interleave the two uint4 arrays
    {
        std::vector<DevNode> h(nn);
        uint32_t mml = 0;
        for (size_t i = 0; i < nn; ++i) {
            std::memcpy(&h[i].lo, P->bvh_min_right_start + 4 * i, 16);
            std::memcpy(&h[i].hi, P->bvh_max_axis_count + 4 * i, 16);
            if ((h[i].hi.w & NOOR_MESH_LEAF_MASK) && !(h[i].hi.w & NOOR_TRI_LEAF_MASK))
                mml = std::max(mml, h[i].hi.w & NOOR_COUNT_MASK);
        }
        st.max_mesh_leaf = mml;
        if ((rc = st.upload((void**)&D.nodes, h.data(), nn * sizeof(DevNode), "nodes"))) return rc;
#if NB_WIDE_TREE
        // the four-wide tree of the spec's root (shadow rays, and closest hit
        // where it qualifies); a tree it does not suit keeps the binary
        // traversal
        WideTree wt;
        if (build_wide_tree(reinterpret_cast<const uint32_t*>(h.data()), nn, S->bvh_root_node, kWideMaxStack, wt,
                            nullptr)) {
            if ((rc = st.upload((void**)&st.wide_nodes, wt.nodes.data(), wt.nodes.size() * sizeof(DevNode4),
                                "wide nodes")) ||
                (rc = st.upload((void**)&st.wide_map, wt.map.data(), nn * sizeof(uint32_t), "wide map")))
                return rc;
            st.wide_root = wt.root;
            st.wide_cap = wt.stack_need;
            st.wide_closest = wt.closest;
        }
#endif
    }
    {
        std::vector<DevWaldTri> w(nt);
        std::vector<DevWtTri> t(nt);
        uint32_t kinds = 0;
        for (size_t i = 0; i < nt; ++i) {
            std::memcpy(&w[i].ax_nu_nv_nd, P->wald_ax_nu_nv_nd + 4 * i, 16);
            std::memcpy(&w[i].cnu_cnv_deg_mat, P->wald_cnu_cnv_deg_mat + 4 * i, 16);
            std::memcpy(&w[i].bnu_bnv_au_av, P->wald_bnu_bnv_au_av + 4 * i, 16);
            std::memcpy(&w[i].attr, P->attribute_indices + 4 * i, 16);
            const uint32_t* a = P->attribute_indices + 4 * i;
            float4* vv[3] = {&t[i].v0, &t[i].v1, &t[i].v2};
            for (int k = 0; k < 3; ++k) {
                const float* p = P->vertices + 4 * (size_t)a[k];
                *vv[k] = make_float4(p[0], p[1], p[2], 0.0f);
            }
            uint32_t mt = P->wald_cnu_cnv_deg_mat[4 * i + 3];
            std::memcpy(&t[i].v0.w, &mt, 4);
            std::memcpy(&t[i].attr, a, 16);
            if (!(mt & kEmitterMat)) kinds |= 1u << shade_kind(lobe_of(mt));
        }
        D.shade_kinds = kinds;
        if ((rc = st.upload((void**)&D.wald, w.data(), nt * sizeof(DevWaldTri), "wald triangles"))) return rc;
        if ((rc = st.upload((void**)&D.wtri, t.data(), nt * sizeof(DevWtTri), "watertight triangles"))) return rc;
    }
    if ((rc = st.upload((void**)&D.vertices, P->vertices, nv * 16, "vertices"))) return rc;
    if ((rc = st.upload((void**)&D.normals, P->normals, nv * 16, "normals"))) return rc;
    if ((rc = st.upload((void**)&D.uvs, P->uvs, nv * 8, "uvs"))) return rc;
    {
        std::vector<DevXform> x(ni);
        for (size_t i = 0; i < ni; ++i)
            for (int r = 0; r < 3; ++r) {
                std::memcpy(&x[i].w2o[r], P->world_to_object_row[r] + 4 * i, 16);
                std::memcpy(&x[i].o2w[r], P->object_to_world_row[r] + 4 * i, 16);
                std::memcpy(&x[i].nrm[r], P->normal_row[r] + 4 * i, 16);
            }
        if ((rc = st.upload((void**)&D.xforms, x.data(), ni * sizeof(DevXform), "transforms"))) return rc;
        // instances whose world-to-object rows are exactly the identity
        std::vector<uint32_t> ident(ni / 32 + 1, 0u);
        for (size_t i = 0; i < ni; ++i) {
            const float4* r = x[i].w2o;
            const bool id = r[0].x == 1.0f && r[0].y == 0.0f && r[0].z == 0.0f && r[0].w == 0.0f &&
                            r[1].x == 0.0f && r[1].y == 1.0f && r[1].z == 0.0f && r[1].w == 0.0f &&
                            r[2].x == 0.0f && r[2].y == 0.0f && r[2].z == 1.0f && r[2].w == 0.0f;
            if (id) ident[i / 32] |= 1u << (i % 32);
        }
        if ((rc = st.upload((void**)&D.xf_ident, ident.data(), ident.size() * 4, "identity instances"))) return rc;
    }
    {
        std::vector<DevMaterial> m(P->num_materials);
        std::vector<DevMatTex> mt(P->num_materials);
        int terr = NOOR_OK;
        auto object = [&](uint32_t idx) -> cudaTextureObject_t {
            cudaTextureObject_t o = 0;
            if (terr == NOOR_OK) terr = st.texture_object(P->textures[idx], idx, &o);
            return o;
        };
        for (uint32_t i = 0; i < P->num_materials; ++i) {
            std::memset(&m[i], 0, sizeof(DevMaterial));
            resolve_material(P, P->materials[i], m[i]);
            resolve_textures(P, P->materials[i], m[i], mt[i], object);
            if (terr) return terr;
            const uint32_t l = lobe_of(m[i].type);
            if (l > 0xFFFFu || !lobe_common(l)) D.ext_lobes = 1u;
            if (m[i].tex_mask) D.has_tex = 1u;
            if (m[i].type & NOOR_ALPHA) D.has_alpha = 1u;
            if (m[i].type & NOOR_BUMP) D.has_bump = 1u;
        }
        st.materials_host = m;
        if ((rc = st.upload((void**)&D.materials, m.data(), m.size() * sizeof(DevMaterial), "materials"))) return rc;
        if ((rc = st.upload((void**)&D.mat_tex, mt.data(), mt.size() * sizeof(DevMatTex), "material textures")))
            return rc;
    }
    {
        std::vector<DevAreaLight> l(P->num_area_lights);
        st.quad_lights_only = true;
        for (int i = 0; i < P->num_area_lights; ++i) {
            const noor_area_light& a = P->area_lights[i];
            std::memset(&l[i], 0, sizeof(DevAreaLight));
            l[i].center = make_float3(a.shape.center[0], a.shape.center[1], a.shape.center[2]);
            l[i].u = make_float3(a.shape.u[0], a.shape.u[1], a.shape.u[2]);
            l[i].v = make_float3(a.shape.v[0], a.shape.v[1], a.shape.v[2]);
            l[i].n = make_float3(a.shape.n[0], a.shape.n[1], a.shape.n[2]);
            l[i].area = a.shape.area;
            l[i].ke = make_float3(a.ke[0], a.ke[1], a.ke[2]);
            l[i].two_sided = a.two_sided;
            l[i].type = a.shape.type;
            l[i].radius = a.shape.radius;
            l[i].radius2 = a.shape.radius2;
            if (a.shape.type != NOOR_SHAPE_QUAD) {
                st.quad_lights_only = false;
                D.ext_lights = 1u;
            }
        }
        if ((rc = st.upload((void**)&D.area_lights, l.data(), l.size() * sizeof(DevAreaLight), "area lights"))) return rc;
    }
    {
        // point, spot and distant lights in one array, in light-index order
        std::vector<DevDeltaLight> l;
        auto v = [](const float* x) { return make_float3(x[0], x[1], x[2]); };
        for (int i = 0; i < P->num_point_lights; ++i) {
            DevDeltaLight d{};
            d.kind = kDeltaPoint;
            d.pos = v(P->point_lights[i].position);
            d.ke = v(P->point_lights[i].ke);
            l.push_back(d);
        }
        for (int i = 0; i < P->num_spot_lights; ++i) {
            const noor_spot_light& sl = P->spot_lights[i];
            DevDeltaLight d{};
            d.kind = kDeltaSpot;
            d.pos = v(sl.position);
            d.dir = v(sl.direction);
            d.ke = v(sl.ke);
            d.cos_inner = sl.cos_inner;
            d.cos_outer = sl.cos_outer;
            l.push_back(d);
        }
        for (int i = 0; i < P->num_distant_lights; ++i) {
            DevDeltaLight d{};
            d.kind = kDeltaDistant;
            d.dir = v(P->distant_lights[i].direction);
            d.ke = v(P->distant_lights[i].ke);
            l.push_back(d);
        }
        if (!l.empty() &&
            (rc = st.upload((void**)&D.delta_lights, l.data(), l.size() * sizeof(DevDeltaLight), "delta lights")))
            return rc;
        D.num_delta_lights = (int)l.size();
        if (!l.empty()) D.ext_lights = 1u;
    }
    D.num_nodes = (uint32_t)nn;
    D.num_tris = (uint32_t)nt;
    D.num_instances = (uint32_t)ni;
    D.num_materials = P->num_materials;
    D.num_area_lights = P->num_area_lights;
    D.num_lights = P->num_area_lights + D.num_delta_lights + P->num_infinite_lights;
    // environment texture (last texture)
    const noor_texture& env = P->textures[P->num_textures - 1];
    D.env_w = env.width;
    D.env_h = env.height;
    if ((rc = st.upload((void**)&D.env, env.rgba, (size_t)env.width * env.height * 16, "environment"))) return rc;
    st.sky_type = S->skydome_type;
    if (H) apply_hosek(st, *H);
    apply_spec(st, *S);
    // distribution: physical sky at 2048 x 1024, maps at their resolution
    EnvBuild& b = st.env;
    b.w = st.sky_type == NOOR_SKY_PHYSICAL ? 2048 : env.width;
    b.h = st.sky_type == NOOR_SKY_PHYSICAL ? 1024 : env.height;
    const size_t cw = (size_t)b.w, chh = (size_t)b.h;
    if ((rc = st.alloc((void**)&b.func, cw * chh * 4, "env func"))) return rc;
    if ((rc = st.alloc((void**)&b.cdf, chh * (cw + 1) * 4, "env cdf"))) return rc;
    if ((rc = st.alloc((void**)&b.row_int, chh * 4, "env rows"))) return rc;
    if ((rc = st.alloc((void**)&b.marg_cdf, (chh + 1) * 4, "env marginal"))) return rc;
    if ((rc = st.alloc((void**)&b.guide, chh * (kDistGuide + 1) * 4, "env guides"))) return rc;
    if ((rc = st.alloc((void**)&b.mguide, (kDistGuide + 1) * 4, "env marginal guide"))) return rc;
    if ((rc = st.alloc((void**)&b.scratch, (chh * (cw + 1) + 2 * chh + 2) * 8, "env scratch"))) return rc;
    if ((rc = st.alloc((void**)&b.marg_int_out, 16, "env integral"))) return rc;
    D.dist.func = b.func;
    D.dist.cdf = b.cdf;
    D.dist.row_int = b.row_int;
    D.dist.marg_cdf = b.marg_cdf;
    D.dist.guide = b.guide;
    D.dist.mguide = b.mguide;
    D.dist.w = b.w;
    D.dist.h = b.h;
    if ((rc = build_distribution(C, st))) return rc;
    return apply_env_mode(C, st, *S);
}

static void load_camera(Context& C, const noor_camera& cam) { C.cam = dev_camera(cam, cam.w, cam.h); }

static int check_camera(const noor_camera* cam) {
    if (!cam) return set_error(NOOR_ERR_INVALID, "camera is null");
    if (cam->w == 0 || cam->h == 0 || (uint64_t)cam->w * cam->h > (1ull << 28))
        return set_error(NOOR_ERR_INVALID, "camera: bad image size");
    if ((uint32_t)cam->type > NOOR_CAMERA_ENV) return set_error(NOOR_ERR_INVALID, "camera: unknown camera type");
    if (cam->center >= cam->w * cam->h) return set_error(NOOR_ERR_INVALID, "camera: centre pixel out of range");
    return NOOR_OK;
}

int ensure_film(Context& C, uint32_t w, uint32_t h) {
    if (C.film_w == w && C.film_h == h && C.film_sum) return NOOR_OK;
    for (float4** p : {&C.film_sum, &C.film_comp, &C.film_out})
        if (*p) {
            cudaFree(*p);
            *p = nullptr;
        }
    const size_t n = (size_t)w * h * sizeof(float4);
    for (float4** p : {&C.film_sum, &C.film_comp, &C.film_out}) {
        cudaError_t e = cudaMalloc((void**)p, n);
        if (e != cudaSuccess) return cuda_fail(e, "film");
        e = cudaMemsetAsync(*p, 0, n, C.stream);
        if (e != cudaSuccess) return cuda_fail(e, "film");
    }
    C.film_w = w;
    C.film_h = h;
    C.film_count = 0;
    return NOOR_OK;
}

int ensure_parts(Context& C, size_t n) {
    if (C.part_cap >= n) return NOOR_OK;
    if (C.part_sum) cudaFree(C.part_sum);
    if (C.part_comp) cudaFree(C.part_comp);
    C.part_sum = C.part_comp = nullptr;
    C.part_cap = 0;
    cudaError_t e = cudaMalloc((void**)&C.part_sum, n * sizeof(float4));
    if (e == cudaSuccess) e = cudaMalloc((void**)&C.part_comp, n * sizeof(float4));
    if (e != cudaSuccess) return cuda_fail(e, "partial film");
    C.part_cap = n;
    return NOOR_OK;
}

Context* current() { return tl_ctx; }

int need_ctx(Context*& C) {
    C = tl_ctx;
    if (!C) return set_error(NOOR_ERR_NO_CONTEXT, "no render context on this thread (call load_cuda_data first)");
    cudaError_t e = cudaSetDevice(C->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    return NOOR_OK;
}

// render frames [frame0, frame0 + n) with the megakernel
int render_frames(Context& C, uint32_t frame0, uint32_t n) {
    if (n == 0) return NOOR_OK;
    if (frame0 == 0) return set_error(NOOR_ERR_INVALID, "frame numbers start at 1");
    SceneState& st = *C.scenes[0];
    const uint32_t npix = C.cam.w * C.cam.h;
    int rc = ensure_film(C, C.cam.w, C.cam.h);
    if (rc) return rc;
    MegaArgs a{};
    a.frame0 = frame0;
    a.nframes = n;
    a.fresh = frame0 == 1 ? 1u : 0u;
    uint32_t chunks = 1;
    if (st.dev.film_mode == NOOR_FILM_KAHAN) {
        const uint64_t target = (uint64_t)C.sm_count * 1024u;
        chunks = (uint32_t)std::min<uint64_t>(n, std::max<uint64_t>(1, (target + npix - 1) / npix));
    }
    a.chunks = chunks;
    a.film_sum = C.film_sum;
    a.film_comp = C.film_comp;
    if (chunks > 1) {
        if ((rc = ensure_parts(C, (size_t)chunks * npix))) return rc;
        a.part_sum = C.part_sum;
        a.part_comp = C.part_comp;
    }
    a.lookat = C.lookat;
    a.status = C.status;
    a.counters = C.counters;
    cudaError_t e = launch_megakernel(st.dev, C.cam, a, C.stream);
    if (e != cudaSuccess) return cuda_fail(e, "megakernel");
    C.launches += chunks > 1 ? 2 : 1;
    C.film_count = (frame0 == 1) ? n : C.film_count + n;
    C.last_frame = frame0 + n - 1;
    return NOOR_OK;
}

// One frame of a batch with the plain megakernel: film of its own (scratch),
// mean written into d_film (float4 per pixel) when given.
int megakernel_frame(Context& C, const noor_wf_frame& f, float4* sum, float4* comp) {
    if (f.scene_id >= C.scenes.size()) return set_error(NOOR_ERR_INVALID, "megakernel batch: unknown scene id");
    if (f.width == 0 || f.height == 0 || f.spp == 0 || f.first_frame == 0 || f.width != f.camera.w ||
        f.height != f.camera.h)
        return set_error(NOOR_ERR_INVALID, "megakernel batch: bad frame description");
    DevScene S = C.scenes[f.scene_id]->dev;
    if (f.bounces) S.bounces = f.bounces;
    S.film_mode = NOOR_FILM_KAHAN;
    if ((uint32_t)f.camera.type > NOOR_CAMERA_ENV) return set_error(NOOR_ERR_INVALID, "megakernel batch: bad camera type");
    const DevCamera cam = dev_camera(f.camera, f.width, f.height);
    const uint32_t npix = f.width * f.height;
    MegaArgs a{};
    a.frame0 = f.first_frame;
    a.nframes = f.spp;
    a.fresh = 1u;
    const uint64_t target = (uint64_t)C.sm_count * 1024u;
    a.chunks = (uint32_t)std::min<uint64_t>(f.spp, std::max<uint64_t>(1, (target + npix - 1) / npix));
    a.film_sum = sum;
    a.film_comp = comp;
    int rc;
    if (a.chunks > 1) {
        if ((rc = ensure_parts(C, (size_t)a.chunks * npix))) return rc;
        a.part_sum = C.part_sum;
        a.part_comp = C.part_comp;
    }
    a.lookat = C.lookat;
    a.status = C.status;
    a.counters = C.counters;
    cudaError_t e = launch_megakernel(S, cam, a, C.stream);
    if (e == cudaSuccess && f.d_film)
        e = launch_resolve(npix, NOOR_FILM_KAHAN, 1.0f / (float)f.spp, sum, (float4*)f.d_film, C.stream);
    if (e != cudaSuccess) return cuda_fail(e, "megakernel batch");
    C.launches += (a.chunks > 1 ? 2 : 1) + (f.d_film ? 1 : 0);
    return NOOR_OK;
}

int sync_and_check(Context& C, const char* what) {
    cudaError_t e = cudaStreamSynchronize(C.stream);
    if (e != cudaSuccess) return cuda_fail(e, what);
    return NOOR_OK;
}

}  // namespace nb

using namespace nb;

// ================================================== reference entry points
extern "C" int load_cuda_data(const noor_payload* payload, const noor_hosek_sky* hosek, const noor_camera* camera,
                              const noor_spec* spec, void* texture_handle) {
    (void)texture_handle;
    clear_error();
    int rc = check_camera(camera);
    if (rc) return rc;
    if ((rc = check_scene_inputs(payload, hosek, spec))) return rc;
    if (tl_ctx) {
        delete tl_ctx;
        tl_ctx = nullptr;
    }
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return set_error(NOOR_ERR_CUDA, "no CUDA device available");
    std::unique_ptr<Context> C(new Context());
    e = cudaGetDevice(&C->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    cudaDeviceGetAttribute(&C->sm_count, cudaDevAttrMultiProcessorCount, C->device);
    e = cudaStreamCreateWithFlags(&C->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "stream");
    for (auto& ev : C->events)
        if ((e = cudaEventCreate(&ev)) != cudaSuccess) return cuda_fail(e, "event");
    if ((e = cudaMalloc((void**)&C->lookat, 16)) != cudaSuccess) return cuda_fail(e, "lookat");
    if ((e = cudaMalloc((void**)&C->status, 16)) != cudaSuccess) return cuda_fail(e, "status");
    if ((e = cudaMalloc((void**)&C->counters, 64)) != cudaSuccess) return cuda_fail(e, "counters");
    cudaMemsetAsync(C->lookat, 0, 16, C->stream);
    cudaMemsetAsync(C->status, 0, 16, C->stream);
    cudaMemsetAsync(C->counters, 0, 64, C->stream);
    C->hosek_src = hosek;
    C->camera_src = camera;
    C->spec_src = spec;
    C->scenes.emplace_back(new SceneState());
    if ((rc = upload_scene(*C, payload, hosek, spec, *C->scenes[0], true))) return rc;
    load_camera(*C, *camera);
    if ((rc = ensure_film(*C, camera->w, camera->h))) return rc;
    if ((rc = sync_and_check(*C, "load_cuda_data"))) return rc;
    tl_ctx = C.release();
    return NOOR_OK;
}

extern "C" int update_cuda_camera(void) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    if ((rc = check_camera(C->camera_src))) return rc;
    load_camera(*C, *C->camera_src);
    if ((rc = ensure_film(*C, C->cam.w, C->cam.h))) return rc;
    C->film_count = 0;
    return NOOR_OK;
}

extern "C" int update_cuda_hosek(void) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    if (!C->hosek_src) return set_error(NOOR_ERR_INVALID, "no Hosek state was given at load time");
    SceneState& st = *C->scenes[0];
    apply_hosek(st, *C->hosek_src);
    if (st.sky_type == NOOR_SKY_PHYSICAL && (rc = build_distribution(*C, st))) return rc;
    if (st.sky_type == NOOR_SKY_PHYSICAL && st.ref_built && (rc = build_reference_distribution(*C, st))) return rc;
    C->film_count = 0;
    return NOOR_OK;
}

extern "C" int update_cuda_spec(void) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    const noor_spec* s = C->spec_src;
    SceneState& st = *C->scenes[0];
    if (s->intersector > 1u || s->film_mode > 1u || s->env_sampling > 1u)
        return set_error(NOOR_ERR_INVALID, "spec: bad selector");
    if (s->bvh_root_node >= st.dev.num_nodes) return set_error(NOOR_ERR_INVALID, "spec: BVH root out of range");
    if (s->skydome_type != st.sky_type)
        return set_error(NOOR_ERR_UNSUPPORTED, "spec: the skydome type is fixed at load time");
    apply_spec(st, *s);
    if ((rc = apply_env_mode(*C, st, *s))) return rc;
    C->film_count = 0;
    return NOOR_OK;
}

extern "C" int cuda_path_tracer(unsigned int* frame_count) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    if (!frame_count) return set_error(NOOR_ERR_INVALID, "frame_count is null");
    if ((rc = render_frames(*C, *frame_count, 1))) return rc;
    if ((rc = sync_and_check(*C, "cuda_path_tracer"))) return rc;
    ++*frame_count;
    return NOOR_OK;
}

extern "C" int noor_render_frames(unsigned int* frame_count, unsigned int n_frames) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    if (!frame_count) return set_error(NOOR_ERR_INVALID, "frame_count is null");
    if ((rc = render_frames(*C, *frame_count, n_frames))) return rc;
    if ((rc = sync_and_check(*C, "noor_render_frames"))) return rc;
    *frame_count += n_frames;
    return NOOR_OK;
}

extern "C" int debug_skydome(unsigned int* frame_count, int width, int height) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    if (!frame_count || width <= 0 || height <= 0) return set_error(NOOR_ERR_INVALID, "debug_skydome: bad argument");
    DevCamera cam = C->cam;
    if ((uint32_t)width != cam.w || (uint32_t)height != cam.h)
        return set_error(NOOR_ERR_INVALID, "debug_skydome: size differs from the camera's");
    SceneState& st = *C->scenes[0];
    cudaError_t e = launch_debug_skydome(st.dev, cam, *frame_count, C->film_sum, st.dev.mis, C->stream);
    if (e != cudaSuccess) return cuda_fail(e, "debug_skydome");
    C->launches++;
    // the debug image is stored as a mean: read back with count 1
    if ((rc = sync_and_check(*C, "debug_skydome"))) return rc;
    C->film_count = 1;
    C->film_is_mean = true;
    ++*frame_count;
    return NOOR_OK;
}

extern "C" int device_free_memory(void) {
    if (!tl_ctx) return NOOR_OK;
    cudaSetDevice(tl_ctx->device);
    noalloc_forget(tl_ctx->device);
    delete tl_ctx;
    tl_ctx = nullptr;
    return NOOR_OK;
}

extern "C" int get_lookAt(float look_at[4]) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    if (!look_at) return set_error(NOOR_ERR_INVALID, "look_at is null");
    cudaError_t e = cudaMemcpyAsync(look_at, C->lookat, 16, cudaMemcpyDeviceToHost, C->stream);
    if (e != cudaSuccess) return cuda_fail(e, "get_lookAt");
    return sync_and_check(*C, "get_lookAt");
}

// ============================================================== additions
extern "C" int noor_device_count(int* count) {
    if (!count) return set_error(NOOR_ERR_INVALID, "count is null");
    *count = 0;
    cudaError_t e = cudaGetDeviceCount(count);
    if (e != cudaSuccess) {
        *count = 0;
        cudaGetLastError();
    }
    return NOOR_OK;
}

extern "C" int noor_abi_sizes(uint32_t* out, int n) {
    const uint32_t s[] = {sizeof(noor_shape), sizeof(noor_area_light), sizeof(noor_texture), sizeof(noor_material),
                          sizeof(noor_payload), sizeof(noor_camera), sizeof(noor_hosek_state), sizeof(noor_hosek_sky),
                          sizeof(noor_spec), sizeof(noor_ray), sizeof(noor_hit), sizeof(noor_bvh_spec),
                          sizeof(noor_mesh), sizeof(noor_material_desc), sizeof(noor_scene_desc),
                          sizeof(noor_build_stat), sizeof(noor_wf_frame), sizeof(noor_wf_params),
                          sizeof(noor_adjoint_desc), sizeof(noor_wf_profile), sizeof(noor_point_light),
                          sizeof(noor_spot_light), sizeof(noor_distant_light)};
    const int k = (int)(sizeof(s) / sizeof(s[0]));
    int w = 0;
    for (; out && w < n && w < k; ++w) out[w] = s[w];
    return w;
}

extern "C" int noor_get_framebuffer_device(float* device_rgba, size_t n_pixels) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    const size_t npix = (size_t)C->film_w * C->film_h;
    if (!device_rgba || n_pixels < npix) return set_error(NOOR_ERR_INVALID, "framebuffer: buffer too small");
    if (C->film_is_mean || C->scenes[0]->dev.film_mode == NOOR_FILM_REF_LERP) {
        cudaError_t e = cudaMemcpyAsync(device_rgba, C->film_sum, npix * 16, cudaMemcpyDeviceToDevice, C->stream);
        if (e != cudaSuccess) return cuda_fail(e, "framebuffer");
    } else {
        const float inv = C->film_count ? 1.0f / (float)C->film_count : 0.0f;
        cudaError_t e = launch_resolve((uint32_t)npix, NOOR_FILM_KAHAN, inv, C->film_sum, (float4*)device_rgba, C->stream);
        if (e != cudaSuccess) return cuda_fail(e, "framebuffer");
        C->launches++;
    }
    return sync_and_check(*C, "framebuffer");
}

extern "C" int noor_get_framebuffer(float* host_rgba, size_t n_pixels) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    const size_t npix = (size_t)C->film_w * C->film_h;
    if (!host_rgba || n_pixels < npix) return set_error(NOOR_ERR_INVALID, "framebuffer: buffer too small");
    if ((rc = noor_get_framebuffer_device((float*)C->film_out, npix))) return rc;
    cudaError_t e = cudaMemcpyAsync(host_rgba, C->film_out, npix * 16, cudaMemcpyDeviceToHost, C->stream);
    if (e != cudaSuccess) return cuda_fail(e, "framebuffer");
    return sync_and_check(*C, "framebuffer");
}

extern "C" int noor_reset_film(void) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    C->film_count = 0;
    C->film_is_mean = false;
    return NOOR_OK;
}

extern "C" int noor_ray_counters(uint64_t counters[3], int reset) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    unsigned long long h[3] = {0, 0, 0};
    cudaError_t e = cudaMemcpyAsync(h, C->counters, sizeof(h), cudaMemcpyDeviceToHost, C->stream);
    if (e == cudaSuccess && reset) e = cudaMemsetAsync(C->counters, 0, 64, C->stream);
    if (e != cudaSuccess) return cuda_fail(e, "counters");
    if ((rc = sync_and_check(*C, "counters"))) return rc;
    if (counters)
        for (int i = 0; i < 3; ++i) counters[i] = h[i];
    return NOOR_OK;
}

extern "C" int noor_device_status(uint32_t* status, int reset) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    uint32_t h = 0;
    cudaError_t e = cudaMemcpyAsync(&h, C->status, 4, cudaMemcpyDeviceToHost, C->stream);
    if (e == cudaSuccess && reset) e = cudaMemsetAsync(C->status, 0, 4, C->stream);
    if (e != cudaSuccess) return cuda_fail(e, "status");
    if ((rc = sync_and_check(*C, "status"))) return rc;
    if (status) *status = h;
    return NOOR_OK;
}

extern "C" void* noor_stream(void) { return tl_ctx ? (void*)tl_ctx->stream : nullptr; }

extern "C" void* noor_context_current(void) { return tl_ctx; }

extern "C" int noor_context_bind(void* context) {
    clear_error();
    tl_ctx = static_cast<Context*>(context);
    if (tl_ctx) {
        cudaError_t e = cudaSetDevice(tl_ctx->device);
        if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    }
    return NOOR_OK;
}

extern "C" int noor_event_record(int slot) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    if (slot < 0 || slot >= (int)(sizeof(C->events) / sizeof(C->events[0])))
        return set_error(NOOR_ERR_INVALID, "event slot out of range");
    cudaError_t e = cudaEventRecord(C->events[slot], C->stream);
    if (e != cudaSuccess) return cuda_fail(e, "event record");
    return NOOR_OK;
}

extern "C" int noor_event_elapsed(int a, int b, float* ms) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    const int n = (int)(sizeof(C->events) / sizeof(C->events[0]));
    if (a < 0 || b < 0 || a >= n || b >= n || !ms) return set_error(NOOR_ERR_INVALID, "event: bad argument");
    cudaError_t e = cudaEventSynchronize(C->events[b]);
    if (e == cudaSuccess) e = cudaEventElapsedTime(ms, C->events[a], C->events[b]);
    if (e != cudaSuccess) return cuda_fail(e, "event elapsed");
    return NOOR_OK;
}

extern "C" int noor_launch_count(uint64_t* n) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    if (!n) return set_error(NOOR_ERR_INVALID, "n is null");
    *n = C->launches;
    return NOOR_OK;
}

extern "C" int noor_trace_closest(const noor_ray* d_rays, noor_hit* d_hits, size_t n) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    if (n && (!d_rays || !d_hits)) return set_error(NOOR_ERR_INVALID, "trace: null buffer");
    cudaError_t e = launch_trace_closest(C->scenes[0]->dev, d_rays, d_hits, n, C->status, C->stream);
    if (e != cudaSuccess) return cuda_fail(e, "trace_closest");
    C->launches++;
    return sync_and_check(*C, "trace_closest");
}

extern "C" int noor_trace_any(const noor_ray* d_rays, uint32_t* d_occluded, size_t n) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    if (n && (!d_rays || !d_occluded)) return set_error(NOOR_ERR_INVALID, "trace: null buffer");
    cudaError_t e = launch_trace_any(C->scenes[0]->dev, d_rays, d_occluded, n, C->status, C->stream);
    if (e != cudaSuccess) return cuda_fail(e, "trace_any");
    C->launches++;
    return sync_and_check(*C, "trace_any");
}

extern "C" int noor_camera_rays(unsigned int frame, noor_ray* d_rays) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    if (!d_rays) return set_error(NOOR_ERR_INVALID, "camera rays: null buffer");
    cudaError_t e = launch_camera_rays(C->cam, frame, d_rays, C->stream);
    if (e != cudaSuccess) return cuda_fail(e, "camera rays");
    C->launches++;
    return sync_and_check(*C, "camera rays");
}

extern "C" int noor_eval_bsdf(int kind, const float* d_in, float* d_out, size_t n) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    if (kind < 0 || kind > 2 || (n && (!d_in || !d_out))) return set_error(NOOR_ERR_INVALID, "eval_bsdf: bad argument");
    cudaError_t e = launch_eval_bsdf(C->scenes[0]->dev, kind, d_in, d_out, n, C->stream);
    if (e != cudaSuccess) return cuda_fail(e, "eval_bsdf");
    C->launches++;
    return sync_and_check(*C, "eval_bsdf");
}

extern "C" int noor_eval_routines(int kind, const float* d_in, float* d_out, size_t n) {
    if (kind < 0 || kind > 3 || (n && (!d_in || !d_out))) return set_error(NOOR_ERR_INVALID, "eval_routines: bad argument");
    cudaStream_t st = tl_ctx ? tl_ctx->stream : 0;
    cudaError_t e = launch_eval_routines(kind, d_in, d_out, n, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "eval_routines");
    if (tl_ctx) tl_ctx->launches++;
    return NOOR_OK;
}

extern "C" int noor_eval_sky(const float* d_dirs, float* d_rgb, size_t n) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    if (n && (!d_dirs || !d_rgb)) return set_error(NOOR_ERR_INVALID, "eval_sky: bad argument");
    cudaError_t e = launch_eval_sky(C->scenes[0]->dev, d_dirs, d_rgb, n, C->stream);
    if (e != cudaSuccess) return cuda_fail(e, "eval_sky");
    C->launches++;
    return sync_and_check(*C, "eval_sky");
}

extern "C" int noor_eval_env_sample(const float* d_u, float* d_out, size_t n) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    if (n && (!d_u || !d_out)) return set_error(NOOR_ERR_INVALID, "env_sample: bad argument");
    cudaError_t e = launch_env_sample(C->scenes[0]->dev, d_u, d_out, n, C->stream);
    if (e != cudaSuccess) return cuda_fail(e, "env_sample");
    C->launches++;
    return sync_and_check(*C, "env_sample");
}

extern "C" int noor_get_env_distribution(int* w, int* h, float* func, float* cdf, float* marginal_func,
                                         float* marginal_cdf, double* marginal_integral) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    const EnvBuild& b = C->scenes[0]->env;
    if (w) *w = b.w;
    if (h) *h = b.h;
    const size_t W = b.w, H = b.h;
    cudaError_t e = cudaSuccess;
    if (func && e == cudaSuccess) e = cudaMemcpy(func, b.func, W * H * 4, cudaMemcpyDeviceToHost);
    if (cdf && e == cudaSuccess) e = cudaMemcpy(cdf, b.cdf, H * (W + 1) * 4, cudaMemcpyDeviceToHost);
    if (marginal_func && e == cudaSuccess) e = cudaMemcpy(marginal_func, b.row_int, H * 4, cudaMemcpyDeviceToHost);
    if (marginal_cdf && e == cudaSuccess) e = cudaMemcpy(marginal_cdf, b.marg_cdf, (H + 1) * 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "env distribution");
    if (marginal_integral) *marginal_integral = C->scenes[0]->dev.dist.marg_int;
    return NOOR_OK;
}

extern "C" int noor_get_reference_distribution(int* w, int* h, float* func, float* cdf) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    SceneState& st = *C->scenes[0];
    if (!st.ref_built && (rc = build_reference_distribution(*C, st))) return rc;
    if (w) *w = st.dev.rw;
    if (h) *h = st.dev.rh;
    const size_t n = (size_t)st.dev.rh * (st.dev.rw + 2) + 1;
    cudaError_t e = cudaSuccess;
    if (func) e = cudaMemcpy(func, st.ref_func, n * 4, cudaMemcpyDeviceToHost);
    if (cdf && e == cudaSuccess) e = cudaMemcpy(cdf, st.ref_cdf, n * 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "reference distribution");
    return NOOR_OK;
}

extern "C" int noor_megakernel_batch(const noor_wf_frame* frames, uint32_t n_frames, float* ms) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    if (!frames || n_frames == 0) return set_error(NOOR_ERR_INVALID, "megakernel batch: no frames");
    size_t maxpix = 0;
    for (uint32_t i = 0; i < n_frames; ++i) maxpix = std::max<size_t>(maxpix, (size_t)frames[i].width * frames[i].height);
    float4 *sum = nullptr, *comp = nullptr;
    cudaError_t e = cudaMalloc((void**)&sum, maxpix * 16);
    if (e == cudaSuccess) e = cudaMalloc((void**)&comp, maxpix * 16);
    if (e != cudaSuccess) {
        cudaFree(sum);
        return cuda_fail(e, "megakernel batch film");
    }
    cudaEventRecord(C->events[4], C->stream);
    for (uint32_t i = 0; i < n_frames && !rc; ++i) rc = megakernel_frame(*C, frames[i], sum, comp);
    cudaEventRecord(C->events[5], C->stream);
    if (!rc) rc = sync_and_check(*C, "megakernel batch");
    if (!rc && ms) cudaEventElapsedTime(ms, C->events[4], C->events[5]);
    cudaFree(sum);
    cudaFree(comp);
    return rc;
}

extern "C" int noor_scene_upload(const noor_payload* payload, const noor_hosek_sky* hosek, const noor_spec* spec,
                                 uint32_t* scene_id) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    std::unique_ptr<SceneState> st(new SceneState());
    if ((rc = upload_scene(*C, payload, hosek, spec, *st))) return rc;
    if ((rc = sync_and_check(*C, "scene upload"))) return rc;
    C->scenes.emplace_back(std::move(st));
    if (scene_id) *scene_id = (uint32_t)C->scenes.size() - 1;
    return NOOR_OK;
}

// Hosek-Wilkie fit in FP64 on the GPU, then the sun fields of HosekSky::update
// (noor/header/hosek.h:61-83).
extern "C" int noor_hosek_fit(const float* dataset, float turbidity, const float ground_albedo[3], float sun_lat,
                              float sun_lon, float solar_scale, float solar_radius_scale, noor_hosek_sky* out) {
    clear_error();
    if (!dataset || !ground_albedo || !out) return set_error(NOOR_ERR_INVALID, "hosek_fit: null argument");
    if (!(turbidity >= 1.0f && turbidity <= 10.0f)) return set_error(NOOR_ERR_INVALID, "hosek_fit: turbidity outside [1,10]");
    if (!(sun_lat >= 0.0f && sun_lat <= 1.5707964f)) return set_error(NOOR_ERR_INVALID, "hosek_fit: sun below the horizon");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return set_error(NOOR_ERR_CUDA, "no CUDA device available");
    }
    if (tl_ctx) cudaSetDevice(tl_ctx->device);
    const float elevation = 1.5707963267948966f - sun_lat;
    float* d_ds = nullptr;
    float* d_out = nullptr;
    cudaError_t e = cudaMalloc((void**)&d_ds, (3 * 1080 + 3 * 120) * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void**)&d_out, 96 * sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpy(d_ds, dataset, (3 * 1080 + 3 * 120) * sizeof(float), cudaMemcpyHostToDevice);
    const double alb[3] = {ground_albedo[0], ground_albedo[1], ground_albedo[2]};
    if (e == cudaSuccess) e = launch_hosek_fit(d_ds, (double)turbidity, alb, (double)elevation, d_out, 0);
    float h[96];
    if (e == cudaSuccess) e = cudaMemcpy(h, d_out, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d_ds);
    cudaFree(d_out);
    if (e != cudaSuccess) return cuda_fail(e, "hosek_fit");
    std::memset(out, 0, sizeof(*out));
    const float terrestrial_solar_radius = (float)((0.51 * 3.141592653589793 / 180.0) / 2.0);
    for (int s = 0; s < 3; ++s) {
        noor_hosek_state& S = out->state[s];
        for (int c = 0; c < 3; ++c) {
            for (int i = 0; i < 9; ++i) S.configs[c][i] = h[s * 30 + c * 9 + i];
            S.radiances[c] = h[s * 30 + 27 + c];
        }
        S.turbidity = turbidity;
        S.solar_radius = terrestrial_solar_radius;
        S.albedo = ground_albedo[s];
        S.elevation = elevation;
    }
    // NOOR::sphericalDirection(theta=sun_lat, phi=sun_lon), y up, normalised
    const float st = std::sin(sun_lat), ct = std::cos(sun_lat);
    float d[3] = {st * std::cos(sun_lon), ct, st * std::sin(sun_lon)};
    const float inv = 1.0f / std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    for (int k = 0; k < 3; ++k) {
        out->solar_dir[k] = d[k] * inv;
        out->ground_albedo[k] = ground_albedo[k];
    }
    out->solar_scale = solar_scale;
    out->solar_radius = solar_radius_scale * terrestrial_solar_radius;
    return NOOR_OK;
}
