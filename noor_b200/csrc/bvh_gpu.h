// GPU bottom-level BVH builder: the per-mesh trees of BVH::build
// (noor/source/bvh.cpp:88-258) built level by level on the device, with the
// same bytes as the host builder (scene_build.cpp).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace nbg {

// one source mesh: its slice of the triangle order and the boxes the host
// computed for it (Model::computeBBoxes)
struct GpuMesh {
    uint32_t start, count;
    float box[6];   // lo xyz, hi xyz
    float cbox[6];  // centroid box
};
struct GpuBvhParams {
    uint32_t num_bins, max_height, min_leaf, max_leaf;
    float Ci, Ct;
};
// one mesh's tree: 8 words per node in depth-first order, right-child
// indices relative to the tree's first node
struct GpuTree {
    std::vector<uint32_t> nodes;
    uint32_t height = 0, num_inner = 0, num_leaf = 0, max_leaf_tris = 0;
};

// tri_box: 6 floats per triangle (lo, hi); tri_order: the identity on entry,
// each mesh's slice permuted as the host build leaves it on return
int gpu_build_blas(const float* tri_box, uint32_t n_tris, const std::vector<GpuMesh>& meshes,
                   const GpuBvhParams& p, std::vector<uint32_t>& tri_order, std::vector<GpuTree>& trees,
                   double* device_ms, std::string& err);

// The rest of Model::loadCudaPayload on the device (model.cpp:333-458):
// vertex de-duplication in BVH order (the first occurrence of a (vertex,
// normal, uv) index triple gets the next index) and the Wald records and
// attribute words of each triangle in BVH order.
struct GpuTailIn {
    const uint32_t* tri_order;
    uint32_t n_tris;
    const uint32_t *vindices, *nindices, *uvindices;  // 3 per source triangle
    const float* vertices;                            // float4
    uint32_t n_vertices;
    const float* normals;  // float4
    uint32_t n_normals;
    const float* uvs;  // float2
    uint32_t n_uvs;
    const uint32_t* material_indices;  // per source triangle
    const uint32_t* material_types;    // per material
    uint32_t n_materials;
};
struct GpuTailOut {
    std::vector<float> vertices, normals, uvs;
    std::vector<uint32_t> wald[3], attr;
};
int gpu_payload_tail(const GpuTailIn& in, GpuTailOut& out, double* device_ms, std::string& err);

}  // namespace nbg
