// ORACLE BUILD SHIM -- test infrastructure.
// Stands in for noor/header/pch.h when the reference's host sources are
// compiled for the oracle: the standard headers, the glm subset, the NOOR
// helpers pch.h defines (noor/header/pch.h:57-102) and the BVH word masks of
// noor/cuda/path_tracer.cuh:52-64, then the reference headers pch.h pulls in
// (spec.h, bbox.h, stat.h) -- without GL, GLFW, Windows or CUDA headers.
#pragma once
#include <algorithm>
#include <cassert>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <limits>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "glm/glm.hpp"

#define __forceinline inline

#define TRI_LEAF_MASK 0x80000000
#define MESH_LEAF_MASK 0x40000000
#define MESH_INSTANCE_MASK 0x20000000
#define MESH_INNER_MASK 0x10000000
#define MESH_NODE_MASK 0x70000000
#define COUNT_MASK 0x0FFFFFFF
#define TRI_COUNT_MASK 0x7FFFFFFF
#define AXIS_MASK 0x0FFFFFFF
#define TRANS_MASK 0x0FFFFFFF
#define LIGHT_NODE_MASK 0x08000000
#define LIGHT_MASK 0x07FFFFFF
enum MaterialType { DIFFUSE = 1 << 0 };

namespace NOOR {
inline bool isInf(const glm::vec3& v) { return glm::isinf(v.x) || glm::isinf(v.y) || glm::isinf(v.z); }
inline bool isNan(const glm::vec3& v) { return glm::isnan(v.x) || glm::isnan(v.y) || glm::isnan(v.z); }
inline glm::uint32 float_as_uint(float f) {
    glm::uint32 u;
    std::memcpy(&u, &f, 4);
    return u;
}
template <typename T>
inline std::string to_string(const T a_value, const int n = 4) {
    std::ostringstream out;
    out << std::setprecision(n) << a_value;
    return out.str();
}
}  // namespace NOOR

#include "spec.h"
#include "bbox.h"
#include "stat.h"
