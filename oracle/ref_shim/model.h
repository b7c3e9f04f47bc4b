// ORACLE BUILD SHIM -- test infrastructure.
// Stands in for noor/header/model.h: a Model holding exactly what the
// reference BVH builder reads (bvh.cpp, splitter.cpp).  Its bounding boxes
// are computed by a restatement of Model::computeBBoxes
// (noor/source/model.cpp:73-108) using the reference's own BBox class; light
// meshes take their shape bounds (the Mesh(shape, light_idx) constructor,
// noor/header/assetLoader.h:78-91).
#pragma once
#include "pch.h"
#include "payload.h"

struct Mesh {
    std::pair<glm::uint32, glm::uint32> _start_count{std::make_pair(0, 0)};
    BBox _instance_bbox;
    BBox _instance_centbox;
    BBox _bbox;
    BBox _centbox;
    glm::mat4 _to_global{glm::mat4(1.f)};
    glm::mat4 _to_local{glm::mat4(1.f)};
    glm::mat3 _normal_transform{glm::mat3(1.f)};
    int _instance{-1};
    int _mat_idx{0};
    int _light_idx{-1};
    bool _is_light{false};
    bool isInstance() const { return _instance != -1; }
    bool isLight() const { return _is_light; }
};

class BVH;
class Model {
public:
    friend class BVH;
    glm::uint32 _num_triangles = 0;
    std::vector<glm::uint32> _triangle_indices;
    std::vector<glm::uint32> _mesh_indices;
    std::vector<Mesh> _meshes;
    std::vector<BBox> _tri_bboxes;
    BBox _scene_bbox;
    BBox _scene_centbox;

    const BBox& getSceneBBox() const { return _scene_bbox; }
    const BBox& getSceneCentBox() const { return _scene_centbox; }
    const BBox& getMeshBBox(glm::uint32 i) const { return _meshes[i]._bbox; }
    const BBox& getMeshCentBox(glm::uint32 i) const { return _meshes[i]._centbox; }
    const BBox& getInstanceMeshBBox(glm::uint32 i) const { return _meshes[i]._instance_bbox; }
    const BBox& getInstanceMeshCentBox(glm::uint32 i) const { return _meshes[i]._instance_centbox; }
    const BBox& getTriBBox(glm::uint32 i) const { return _tri_bboxes[i]; }
    bool isMeshLight(glm::uint32 i) const { return _meshes[i].isLight(); }
    glm::uint32 getNumTriangles() const { return _num_triangles; }
    glm::uint32 getNumMeshes() const { return (glm::uint32)_meshes.size(); }
};
