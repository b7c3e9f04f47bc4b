// ORACLE -- test infrastructure.
// C entry points over the reference's own host sources, compiled unmodified
// from the reference tree into oracle/_ref/libnoor_ref.so (see the Makefile):
//   * ref_build_bvh: Model + BVH (noor/source/bvh.cpp, splitter.cpp) on a
//     scene description, returning the node words, root, triangle order and
//     height the reference would hand to the device;
//   * ref_build_payload / ref_payload_view / ref_payload_spec: a whole
//     payload (tree, transforms, de-duplicated vertices, Wald records,
//     materials, lights) and the spec Scene::load derives, for the oracle;
//   * ref_wald: WaldTriangle (noor/header/triangle.h:56-120);
//   * ref_hosek_state / ref_hosek_dataset: the vendored Hosek-Wilkie fit
//     (noor/external/ArHosekSkyModel.cpp:667-695) and its RGB tables.
// Model::computeBBoxes (noor/source/model.cpp:73-108) is restated below with
// the reference's BBox class because model.cpp cannot be compiled without
// its file loaders.
#include "pch.h"
#include "model.h"
#include "bvh.h"
#include "triangle.h"
#include "ArHosekSkyModel.h"
#include "../include/noor_b200.h"

#include <array>
#include <unordered_map>

extern float* datasetsRGB[];
extern float* datasetsRGBRad[];

#define REF_API extern "C" __attribute__((visibility("default")))

static glm::mat4 to_mat4(const float* m) {
    glm::mat4 r(1.0f);
    for (int c = 0; c < 4; ++c)
        for (int k = 0; k < 4; ++k) r[c][k] = m[4 * c + k];
    return r;
}

// Model::load's mesh list and Model::computeBBoxes for a scene description
static void load_model(const noor_scene_desc* d, Model& model) {
    model._num_triangles = d->num_triangles;
    model._meshes.resize(d->num_meshes);
    for (uint32_t i = 0; i < d->num_meshes; ++i) {
        const noor_mesh& m = d->meshes[i];
        Mesh& M = model._meshes[i];
        M._start_count = std::make_pair(m.tri_start, m.tri_count);
        M._to_global = to_mat4(m.to_global);
        M._to_local = glm::inverse(M._to_global);
        M._normal_transform = glm::transpose(glm::inverse(glm::mat3(M._to_global)));
        M._instance = m.instance;
        if (m.light_idx >= 0) {
            M._light_idx = m.light_idx;
            M._is_light = true;
        }
    }
    // Model::computeBBoxes
    model._tri_bboxes.reserve(d->num_triangles);
    auto vtx = [&](uint32_t t, int k) {
        const float* p = d->vertices + 4 * (size_t)d->vindices[3 * (size_t)t + k];
        return glm::vec4(p[0], p[1], p[2], p[3]);
    };
    for (auto& mesh : model._meshes) {
        if (!mesh.isInstance() && !mesh.isLight()) {
            const glm::uint32 start = mesh._start_count.first;
            const glm::uint32 count = start + mesh._start_count.second;
            BBox mesh_bbox, mesh_centbox;
            for (glm::uint32 t = start; t < count; ++t) {
                BBox tri_bbox = BBox(vtx(t, 0), vtx(t, 1), vtx(t, 2));
                model._tri_bboxes.emplace_back(tri_bbox);
                mesh_bbox.merge(tri_bbox);
                mesh_centbox.include(tri_bbox.centroid());
            }
            mesh._bbox = mesh_bbox;
            mesh._centbox = mesh_centbox;
        }
    }
    for (uint32_t i = 0; i < d->num_meshes; ++i) {
        Mesh& mesh = model._meshes[i];
        if (mesh.isLight()) {
            const noor_shape& s = d->area_lights[mesh._light_idx].shape;
            const glm::vec3 c(s.center[0], s.center[1], s.center[2]), u(s.u[0], s.u[1], s.u[2]),
                v(s.v[0], s.v[1], s.v[2]);
            BBox b;
            // CudaShape::getBounds (noor/cuda/shape.cuh:71-90)
            if (s.type == NOOR_SHAPE_SPHERE) {
                const glm::vec3 r(s.radius);
                b.setMin(c - r);
                b.setMax(c + r);
            } else if (s.type == NOOR_SHAPE_DISK) {
                const glm::vec3 un = glm::normalize(u), vn = glm::normalize(v);
                const glm::vec3 pr = c + s.radius * un, pt = c + s.radius * vn;
                const glm::vec3 pl = c - s.radius * un, pb = c - s.radius * vn;
                b.setMin(glm::min(glm::min(glm::min(pl, pr), pt), pb));
                b.setMax(glm::max(glm::max(glm::max(pl, pr), pt), pb));
            } else {
                b.setMin(glm::min(glm::min(glm::min(c, c + u), c + v), c + u + v));
                b.setMax(glm::max(glm::max(glm::max(c, c + u), c + v), c + u + v));
            }
            mesh._instance_bbox = b;
            mesh._bbox = b;
            mesh._instance_centbox.setMin(b.centroid());
            mesh._instance_centbox.setMax(b.centroid());
            mesh._centbox = mesh._instance_centbox;
        } else {
            if (mesh.isInstance()) {
                mesh._bbox = model._meshes[mesh._instance]._bbox;
                mesh._centbox = model._meshes[mesh._instance]._centbox;
            }
            mesh._instance_bbox = mesh._to_global * mesh._bbox;
            mesh._instance_centbox = mesh._to_global * mesh._centbox;
        }
        model._scene_bbox.merge(mesh._instance_bbox);
        model._scene_centbox.include(mesh._instance_bbox.centroid());
    }
}

REF_API int ref_build_bvh(const noor_scene_desc* d, uint32_t* nodes, size_t node_cap, uint32_t* num_nodes,
                          uint32_t* root, uint32_t* tri_order, uint32_t* height) {
    Model model;
    load_model(d, model);
    BVHSpec spec(d->bvh.num_bins, d->bvh.max_height, d->bvh.Ci, d->bvh.Ct, d->bvh.min_leaf_tris,
                 d->bvh.max_leaf_tris);
    Stat stat;
    BVH bvh(model, spec, stat);
    std::unique_ptr<CudaPayload> p(new CudaPayload());
    bvh.loadCudaPayload(p);
    const size_t n = p->_bvh_min_right_start_nodes.size();
    *num_nodes = (uint32_t)n;
    *root = p->_bvh_root_node;
    *height = stat._height;
    if (nodes) {
        if (n > node_cap) return 1;
        for (size_t i = 0; i < n; ++i) {
            const glm::uvec4& a = p->_bvh_min_right_start_nodes[i];
            const glm::uvec4& b = p->_bvh_max_axis_count_nodes[i];
            const uint32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
            std::memcpy(nodes + 8 * i, w, sizeof(w));
        }
    }
    if (tri_order) std::memcpy(tri_order, model._triangle_indices.data(), d->num_triangles * sizeof(uint32_t));
    return 0;
}

// ------------------------------------------------------------------------
// A whole payload on the host from the reference's own builder: the tree and
// the instance transforms come from BVH::loadCudaPayload (bvh.cpp:53-86)
// and the Wald records from WaldTriangle (triangle.h:56-120), both compiled
// unmodified; the steps of Model::loadCudaPayload and Model::loadMaterial
// that need the loaders (model.cpp:184-330,333-458) are restated here.  The
// bench's reference arm renders from this payload with the oracle, so it
// never loads the product library.
struct RefPayload {
    std::vector<uint32_t> attr, wald[3], lo, hi, order;
    std::vector<float> vtx, nrm, uv, xf[9];
    std::vector<std::vector<float>> tex_data;
    std::vector<noor_texture> tex;
    std::vector<noor_material> mats;
    std::vector<noor_area_light> area;
    std::vector<noor_point_light> point;
    std::vector<noor_spot_light> spot;
    std::vector<noor_distant_light> distant;
    uint32_t num_tris = 0, root = 0, height = 0;
    float radius = 0.0f;
    int32_t sky = 0;
};

// ImageTexture(float3): 1 x 1, point filtered, clamped
static uint32_t constant_texture(RefPayload& P, float r, float g, float b) {
    P.tex_data.push_back({r, g, b, 1.0f});
    P.tex.push_back(noor_texture{1, 1, nullptr, NOOR_FILTER_POINT, NOOR_ADDRESS_CLAMP});
    return (uint32_t)P.tex_data.size() - 1;
}

REF_API void* ref_build_payload(const noor_scene_desc* d) {
    std::unique_ptr<RefPayload> P(new RefPayload());
    Model model;
    load_model(d, model);
    BVHSpec spec(d->bvh.num_bins, d->bvh.max_height, d->bvh.Ci, d->bvh.Ct, d->bvh.min_leaf_tris,
                 d->bvh.max_leaf_tris);
    Stat stat;
    BVH bvh(model, spec, stat);
    std::unique_ptr<CudaPayload> cp(new CudaPayload());
    bvh.loadCudaPayload(cp);
    RefPayload& R = *P;
    R.num_tris = d->num_triangles;
    R.root = cp->_bvh_root_node;
    R.height = stat._height;
    R.radius = model.getSceneBBox().radius();
    R.sky = d->skydome_type;
    R.order = model._triangle_indices;
    for (size_t i = 0; i < cp->_bvh_min_right_start_nodes.size(); ++i) {
        const glm::uvec4& a = cp->_bvh_min_right_start_nodes[i];
        const glm::uvec4& b = cp->_bvh_max_axis_count_nodes[i];
        R.lo.insert(R.lo.end(), {a.x, a.y, a.z, a.w});
        R.hi.insert(R.hi.end(), {b.x, b.y, b.z, b.w});
    }
    const std::vector<glm::vec4>* rows[9] = {&cp->_normal_row0,          &cp->_normal_row1,
                                             &cp->_normal_row2,          &cp->_world_to_object_row0,
                                             &cp->_world_to_object_row1, &cp->_world_to_object_row2,
                                             &cp->_object_to_world_row0, &cp->_object_to_world_row1,
                                             &cp->_object_to_world_row2};
    for (int k = 0; k < 9; ++k)
        for (const glm::vec4& v : *rows[k]) R.xf[k].insert(R.xf[k].end(), {v.x, v.y, v.z, v.w});

    // Model::loadMaterial: a texture of 0.5 first, then per material its
    // constants (1 x 1) in the loader's order, an image map instead where the
    // material names one -- one texture per image (the reference's
    // name2index), linear filtered and wrapped, map_d point filtered, which
    // add the ALPHA / BUMP bits.  The CudaMaterial `mt` is one object
    // reused for every material, so fields a material leaves alone keep
    // the previous material's values.
    constant_texture(R, 0.5f, 0.5f, 0.5f);
    std::vector<int64_t> name2index(d->num_images, -1);
    auto image = [&](int32_t img, int32_t filter) -> uint32_t {
        if (name2index[img] < 0) {
            const noor_image& im = d->images[img];
            R.tex_data.emplace_back(im.rgba, im.rgba + 4 * (size_t)im.width * im.height);
            R.tex.push_back(noor_texture{im.width, im.height, nullptr, filter, NOOR_ADDRESS_WRAP});
            name2index[img] = (int64_t)R.tex_data.size() - 1;
        }
        return (uint32_t)name2index[img];
    };
    noor_material mt;
    std::memset(&mt, 0, sizeof(mt));
    for (float* s : {mt.diffuse_uvscale, mt.specular_uvscale, mt.transparency_uvscale, mt.emittance_uvscale,
                     mt.bump_uvscale, mt.roughness_uvscale, mt.metalness_uvscale})
        s[0] = s[1] = 1.0f;
    mt.bumpfactor = 1.0f;
    for (uint32_t i = 0; i < d->num_materials; ++i) {
        const noor_material_desc& m = d->materials[i];
        auto has_map = [&](int slot, float* uvscale) {
            if (m.map[slot] < 0) return false;
            uvscale[0] = m.map_uvscale[slot][0];
            uvscale[1] = m.map_uvscale[slot][1];
            return true;
        };
        mt.coat_weight = m.coat_weight;
        mt.coat_roughness = m.coat_roughness;
        mt.coat_thickness = m.coat_thickness;
        mt.coat_sigma = m.coat_sigma;
        mt.coat_ior = m.coat_ior;
        mt.emitter_scale = m.emitter_scale;
        mt.type = m.type;
        mt.distribution = m.distribution;
        mt.transmission_tex_idx = constant_texture(R, m.transmission[0], m.transmission[1], m.transmission[2]);
        mt.ior_tex_idx = constant_texture(R, m.ior[0], m.ior[1], m.ior[2]);
        mt.k_tex_idx = constant_texture(R, m.k[0], m.k[1], m.k[2]);
        if (has_map(NOOR_MAP_DIFFUSE, mt.diffuse_uvscale))
            mt.diffuse_tex_idx = image(m.map[NOOR_MAP_DIFFUSE], NOOR_FILTER_LINEAR);
        else
            mt.diffuse_tex_idx = constant_texture(R, m.diffuse[0], m.diffuse[1], m.diffuse[2]);
        if (has_map(NOOR_MAP_ROUGHNESS, mt.roughness_uvscale))
            mt.roughness_tex_idx = image(m.map[NOOR_MAP_ROUGHNESS], NOOR_FILTER_LINEAR);
        else
            mt.roughness_tex_idx = constant_texture(R, m.roughness[0], m.roughness[1], 1.0f);
        if (has_map(NOOR_MAP_METALNESS, mt.metalness_uvscale))
            mt.metalness_tex_idx = image(m.map[NOOR_MAP_METALNESS], NOOR_FILTER_LINEAR);
        else
            mt.metalness_tex_idx = constant_texture(R, 1.0f, 1.0f, 1.0f);
        if (has_map(NOOR_MAP_SPECULAR, mt.specular_uvscale))
            mt.specular_tex_idx = image(m.map[NOOR_MAP_SPECULAR], NOOR_FILTER_LINEAR);
        else
            mt.specular_tex_idx = constant_texture(R, m.specular[0], m.specular[1], m.specular[2]);
        if (has_map(NOOR_MAP_EMITTANCE, mt.emittance_uvscale))
            mt.emittance_tex_idx = image(m.map[NOOR_MAP_EMITTANCE], NOOR_FILTER_LINEAR);
        else
            mt.emittance_tex_idx = constant_texture(R, m.emittance[0], m.emittance[1], m.emittance[2]);
        if (has_map(NOOR_MAP_ALPHA, mt.transparency_uvscale)) {
            mt.transparency_tex_idx = image(m.map[NOOR_MAP_ALPHA], NOOR_FILTER_POINT);
            mt.type |= NOOR_ALPHA;
        } else {
            mt.transparency_tex_idx = constant_texture(R, m.transparency[0], m.transparency[1], m.transparency[2]);
        }
        if (has_map(NOOR_MAP_BUMP, mt.bump_uvscale)) {
            mt.bump_tex_idx = image(m.map[NOOR_MAP_BUMP], NOOR_FILTER_LINEAR);
            mt.bumpfactor = m.bumpfactor;
            mt.type |= NOOR_BUMP;
        }
        R.mats.push_back(mt);
    }
    // the sky dome texture last: the HDR map (linear, clamped), else SKYDOME_COLOR
    if (d->skydome_type == NOOR_SKY_HDR) {
        R.tex_data.emplace_back(d->env_rgba, d->env_rgba + 4 * (size_t)d->env_width * d->env_height);
        R.tex.push_back(noor_texture{d->env_width, d->env_height, nullptr, NOOR_FILTER_LINEAR, NOOR_ADDRESS_CLAMP});
    } else {
        constant_texture(R, 0.25f, 0.25f, 0.25f);
    }
    for (size_t i = 0; i < R.tex_data.size(); ++i) R.tex[i].rgba = R.tex_data[i].data();
    R.area.assign(d->area_lights, d->area_lights + d->num_area_lights);
    R.point.assign(d->point_lights, d->point_lights + d->num_point_lights);
    R.spot.assign(d->spot_lights, d->spot_lights + d->num_spot_lights);
    R.distant.assign(d->distant_lights, d->distant_lights + d->num_distant_lights);
    for (noor_distant_light& l : R.distant) {   // CudaDistantLight normalises its direction
        const glm::vec3 w = glm::normalize(glm::vec3(l.direction[0], l.direction[1], l.direction[2]));
        l.direction[0] = w.x;
        l.direction[1] = w.y;
        l.direction[2] = w.z;
    }

    // vertex de-duplication in BVH order: the first (vertex, normal, uv)
    // index triple of a corner appends a vertex, later ones reuse its index
    struct KeyHash {
        size_t operator()(const std::array<uint32_t, 3>& k) const {
            return ((size_t)k[0] * 0x9E3779B97F4A7C15ull) ^ ((size_t)k[1] * 0xC2B2AE3D27D4EB4Full) ^ k[2];
        }
    };
    std::unordered_map<std::array<uint32_t, 3>, uint32_t, KeyHash> seen;
    seen.reserve(3 * (size_t)d->num_triangles);
    std::vector<uint32_t> element;
    element.reserve(3 * (size_t)d->num_triangles);
    for (uint32_t i = 0; i < d->num_triangles; ++i) {
        const size_t t = R.order[i];
        for (int j = 0; j < 3; ++j) {
            const uint32_t vi = d->vindices[3 * t + j], ni = d->nindices[3 * t + j], ui = d->uvindices[3 * t + j];
            auto ins = seen.emplace(std::array<uint32_t, 3>{vi, ni, ui}, (uint32_t)seen.size());
            if (ins.second) {
                R.vtx.insert(R.vtx.end(), d->vertices + 4 * (size_t)vi, d->vertices + 4 * (size_t)vi + 4);
                R.nrm.insert(R.nrm.end(), d->normals + 4 * (size_t)ni, d->normals + 4 * (size_t)ni + 4);
                R.uv.insert(R.uv.end(), d->uvs + 2 * (size_t)ui, d->uvs + 2 * (size_t)ui + 2);
            }
            element.push_back(ins.first->second);
        }
    }
    // Model::buildWaldTriangles: Wald records of the de-duplicated corners,
    // the material type in the last word, attribute words v0, v1, v2, mat
    for (uint32_t i = 0; i < d->num_triangles; ++i) {
        glm::vec3 p[3];
        for (int j = 0; j < 3; ++j) {
            const float* q = R.vtx.data() + 4 * (size_t)element[3 * (size_t)i + j];
            p[j] = glm::vec3(q[0], q[1], q[2]);
        }
        WaldTriangle wt(p[0], p[1], p[2]);
        const uint32_t mi = d->material_indices[R.order[i]];
        const glm::uvec4 r0 = wt.get_ax_nu_nv_nd(), r1 = wt.get_bnu_bnv_au_av(), r2 = wt.get_cnu_cnv_deg_mat();
        R.wald[0].insert(R.wald[0].end(), {r0.x, r0.y, r0.z, r0.w});
        R.wald[1].insert(R.wald[1].end(), {r1.x, r1.y, r1.z, r1.w});
        R.wald[2].insert(R.wald[2].end(), {r2.x, r2.y, r2.z, R.mats[mi].type});
        R.attr.insert(R.attr.end(), {element[3 * (size_t)i], element[3 * (size_t)i + 1], element[3 * (size_t)i + 2], mi});
    }
    return P.release();
}

REF_API void ref_payload_view(const void* h, noor_payload* p) {
    const RefPayload& R = *(const RefPayload*)h;
    std::memset(p, 0, sizeof(*p));
    p->num_triangles = R.num_tris;
    p->attribute_indices = R.attr.data();
    p->vertices = R.vtx.data();
    p->normals = R.nrm.data();
    p->uvs = R.uv.data();
    p->num_vertices = (uint32_t)(R.vtx.size() / 4);
    for (int r = 0; r < 3; ++r) {
        p->normal_row[r] = R.xf[r].data();
        p->world_to_object_row[r] = R.xf[3 + r].data();
        p->object_to_world_row[r] = R.xf[6 + r].data();
    }
    p->num_instances = (uint32_t)(R.xf[0].size() / 4);
    p->wald_ax_nu_nv_nd = R.wald[0].data();
    p->wald_bnu_bnv_au_av = R.wald[1].data();
    p->wald_cnu_cnv_deg_mat = R.wald[2].data();
    p->bvh_root_node = R.root;
    p->bvh_min_right_start = R.lo.data();
    p->bvh_max_axis_count = R.hi.data();
    p->num_bvh_nodes = (uint32_t)(R.lo.size() / 4);
    p->textures = R.tex.data();
    p->num_textures = (uint32_t)R.tex.size();
    p->area_lights = R.area.empty() ? nullptr : R.area.data();
    p->num_area_lights = (int32_t)R.area.size();
    p->point_lights = R.point.empty() ? nullptr : R.point.data();
    p->num_point_lights = (int32_t)R.point.size();
    p->spot_lights = R.spot.empty() ? nullptr : R.spot.data();
    p->num_spot_lights = (int32_t)R.spot.size();
    p->distant_lights = R.distant.empty() ? nullptr : R.distant.data();
    p->num_distant_lights = (int32_t)R.distant.size();
    p->num_infinite_lights = 1;
    p->materials = R.mats.data();
    p->num_materials = (uint32_t)R.mats.size();
}

// the CudaSpec fields Scene::load sets (noor/source/scene.cpp:51-91)
REF_API void ref_payload_spec(const void* h, uint32_t bounces, uint32_t rr, noor_spec* s) {
    const RefPayload& R = *(const RefPayload*)h;
    std::memset(s, 0, sizeof(*s));
    s->reflection_bias = 0.0001f * R.radius;
    s->shadow_bias = 0.0001f * R.radius;
    s->world_radius = R.radius;
    s->wr2 = R.radius * R.radius;
    s->bvh_root_node = R.root;
    s->bvh_height = R.height;
    s->bounces = bounces;
    s->rr = rr;
    s->num_gpus = 1;
    s->skydome_type = R.sky;
    const size_t lights = R.area.size() + R.point.size() + R.spot.size() + R.distant.size() + 1;
    s->lighting_type = lights < 2 ? NOOR_LIGHT_SKY_MASK : 0u;
}

REF_API void ref_free_payload(void* h) { delete (RefPayload*)h; }

// out: ax_nu_nv_nd, bnu_bnv_au_av, cnu_cnv_deg_mat (12 words)
REF_API void ref_wald(const float* v9, uint32_t* out) {
    const glm::vec3 A(v9[0], v9[1], v9[2]), B(v9[3], v9[4], v9[5]), C(v9[6], v9[7], v9[8]);
    WaldTriangle wt(A, B, C);
    const glm::uvec4 r0 = wt.get_ax_nu_nv_nd(), r1 = wt.get_bnu_bnv_au_av(), r2 = wt.get_cnu_cnv_deg_mat();
    const uint32_t w[12] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w, r2.x, r2.y, r2.z, r2.w};
    std::memcpy(out, w, sizeof(w));
}

// configs[3][9] then radiances[3] of one state (HosekSky::update's call)
REF_API void ref_hosek_state(float turbidity, float albedo, float elevation, float* out30) {
    ArHosekSkyModelState st;
    arhosek_rgb_skymodelstate_alloc_update(&st, turbidity, albedo, elevation);
    for (int c = 0; c < 3; ++c)
        for (int i = 0; i < 9; ++i) out30[9 * c + i] = st.configs[c][i];
    for (int c = 0; c < 3; ++c) out30[27 + c] = st.radiances[c];
}

// the RGB coefficient (3 x 1080) and radiance (3 x 120) tables
REF_API void ref_hosek_dataset(float* out) {
    for (int c = 0; c < 3; ++c) std::memcpy(out + 1080 * c, datasetsRGB[c], 1080 * sizeof(float));
    for (int c = 0; c < 3; ++c) std::memcpy(out + 3240 + 120 * c, datasetsRGBRad[c], 120 * sizeof(float));
}
