// ORACLE BUILD SHIM -- test infrastructure.
// Stands in for noor/header/payload.h with the fields BVH::loadCudaPayload
// (noor/source/bvh.cpp:53-86) writes.
#pragma once
#include "pch.h"

class CudaPayload {
public:
    std::vector<glm::vec4> _normal_row0, _normal_row1, _normal_row2;
    std::vector<glm::vec4> _world_to_object_row0, _world_to_object_row1, _world_to_object_row2;
    std::vector<glm::vec4> _object_to_world_row0, _object_to_world_row1, _object_to_world_row2;
    size_t _transforms_size_bytes = 0;
    glm::uint32 _bvh_root_node = 0;
    std::vector<glm::uvec4> _bvh_min_right_start_nodes;
    std::vector<glm::uvec4> _bvh_max_axis_count_nodes;
    size_t _bvh_size_bytes = 0;
};
