// ORACLE -- test infrastructure.
// C entry points over the reference's own host sources, compiled unmodified
// from the reference tree into oracle/_ref/libnoor_ref.so (see the Makefile):
//   * ref_build_bvh: Model + BVH (noor/source/bvh.cpp, splitter.cpp) on a
//     scene description, returning the node words, root, triangle order and
//     height the reference would hand to the device;
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

extern float* datasetsRGB[];
extern float* datasetsRGBRad[];

#define REF_API extern "C" __attribute__((visibility("default")))

static glm::mat4 to_mat4(const float* m) {
    glm::mat4 r(1.0f);
    for (int c = 0; c < 4; ++c)
        for (int k = 0; k < 4; ++k) r[c][k] = m[4 * c + k];
    return r;
}

REF_API int ref_build_bvh(const noor_scene_desc* d, uint32_t* nodes, size_t node_cap, uint32_t* num_nodes,
                          uint32_t* root, uint32_t* tri_order, uint32_t* height) {
    Model model;
    model._num_triangles = d->num_triangles;
    model._meshes.resize(d->num_meshes);
    for (uint32_t i = 0; i < d->num_meshes; ++i) {
        const noor_mesh& m = d->meshes[i];
        Mesh& M = model._meshes[i];
        M._start_count = std::make_pair(m.tri_start, m.tri_count);
        M._to_global = to_mat4(m.to_global);
        M._to_local = glm::inverse(M._to_global);
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
