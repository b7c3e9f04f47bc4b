// ORACLE BUILD SHIM -- test infrastructure, not product code.
// Stands in for noor/cuda/path_tracer.cuh when the reference's device
// headers are compiled for the oracle harness (refdev.cu).  path_tracer.cuh
// opens with GL, GLEW and CUDA-Samples includes that are absent here; this
// prelude keeps only what the device headers need from it -- the kernel
// block size, BVH word masks, NOOR_* constants, the material / BxDF /
// shape / sky / camera enums and checkNoorErrors (path_tracer.cuh:46-171) --
// with the same names and values, then includes the same headers in the
// same order (path_tracer.cuh:174-184).
#pragma once
#include <cassert>
#include <cuda.h>
#include <cuda_runtime.h>
#include <math_constants.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <vector>

#include "helper_math.h"
#include "glm/glm.hpp"

// helper_cuda.h's error-name lookup used by checkNoorErrors, and its
// MIN / MAX macros (texture.cuh sizes its mip chain with MAX)
inline const char* _cudaGetErrorEnum(cudaError_t e) { return cudaGetErrorName(e); }
#ifndef MAX
#define MAX(a, b) ((a) > (b) ? (a) : (b))
#endif
#ifndef MIN
#define MIN(a, b) ((a) < (b) ? (a) : (b))
#endif

#define THREAD_W 16
#define THREAD_H 16
#define THREAD_N THREAD_W * THREAD_H

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

#define F2V4(v) glm::vec4(v.x, v.y, v.z, v.w)
#define F2V3(v) glm::vec3(v.x, v.y, v.z)
#define V2F4(v) make_float4(v.x, v.y, v.z, v.w)
#define V2F3(v) make_float3(v.x, v.y, v.z)
#define V2F2(v) make_float2(v.x, v.y)

constexpr float NOOR_EPSILON = std::numeric_limits<float>::epsilon();
constexpr float NOOR_ONE_MINUS_EPSILON = 1.0f - NOOR_EPSILON;
constexpr float NOOR_INF = std::numeric_limits<float>::infinity();
constexpr float NOOR_FLT_MAX = std::numeric_limits<float>::max();
constexpr float NOOR_PI = CUDART_PI_F;
constexpr float NOOR_2PI = 2.0f * CUDART_PI_F;
constexpr float NOOR_4PI = 4.0f * CUDART_PI_F;
constexpr float NOOR_invPI = 1.0f / NOOR_PI;
constexpr float NOOR_inv2PI = 1.0f / NOOR_2PI;
constexpr float NOOR_inv4PI = 1.0f / NOOR_4PI;
constexpr float NOOR_PI_over_2 = NOOR_PI / 2.0f;
constexpr float NOOR_PI_over_4 = NOOR_PI / 4.0f;
constexpr float NOOR_3PI_over_2 = 3.f * NOOR_PI_over_2;

constexpr int2 skydome_res{2048, 2048};
#define SKYDOME_COLOR make_float3(.25f)

enum MaterialType {
    DIFFUSE = 1 << 0,
    ORENNAYAR = 1 << 1,
    TRANSLUCENT = 1 << 2,
    GLOSSY = 1 << 3,
    MIRROR = 1 << 4,
    GLASS = 1 << 5,
    ROUGHGLASS = 1 << 6,
    METAL = 1 << 7,
    SUBSTRATE = 1 << 8,
    EMITTER = 1 << 9,
    CLEARCOAT = 1 << 10,
    SHADOWCATCHER = 1 << 11,
    ALPHA = 1 << 12,
    BUMP = 1 << 13,
    MESHLIGHT = 1 << 14
};
enum BxDFType {
    BSDF_NONE = 1 << 0,
    BSDF_REFLECTION = 1 << 0,
    BSDF_TRANSMISSION = 1 << 1,
    BSDF_DIFFUSE = 1 << 2,
    BSDF_GLOSSY = 1 << 3,
    BSDF_SPECULAR = 1 << 4,
    BSDF_CONDUCTOR = 1 << 5,
    BSDF_DIELECTRIC = 1 << 6,
    BSDF_NOOP = 1 << 7,
    BSDF_ALL = BSDF_DIFFUSE | BSDF_GLOSSY | BSDF_SPECULAR | BSDF_REFLECTION | BSDF_TRANSMISSION |
               BSDF_CONDUCTOR | BSDF_DIELECTRIC | BSDF_NOOP
};
constexpr uint NOOR_NO_BUMP_ALPHA = ~(BUMP | ALPHA);
constexpr uint NOOR_EMITTER = EMITTER | MESHLIGHT;
constexpr uint NOOR_GLASS = GLASS | ROUGHGLASS;
constexpr uint NOOR_TRANSPARENT = TRANSLUCENT | GLASS | ROUGHGLASS;
constexpr uint NOOR_SPECULAR = MIRROR | GLASS | CLEARCOAT;
constexpr uint NOOR_GLOSSY = NOOR_SPECULAR | ROUGHGLASS | CLEARCOAT | METAL | SUBSTRATE | GLOSSY;
enum AreaMeshLightType { QUAD = 0, SPHERE = 1, DISK = 2 };
enum SkydomeType { HDR = 0, PHYSICAL = 1, CONSTANT = 2 };
enum HandedNess { LEFT_HANDED = 0, RIGHT_HANDED = 1 };
enum CameraType { PERSP = 0, ORTHO = 1, ENV = 2 };

class CudaPayload;
class CudaSpec;
class CudaHosekSky;
class CudaCamera;

// the harness reports a failed CUDA call to its caller instead of exiting
struct RefdevError {
    cudaError_t code;
    const char* what;
};
#define checkNoorErrors(val) refdev_check((val), #val)
template <typename T>
static void refdev_check(T result, const char* what) {
    if (result != cudaSuccess) throw RefdevError{static_cast<cudaError_t>(result), what};
}
using uchar = unsigned char;

#include "math.cuh"
#include "utils.cuh"
#include "spec.cuh"
#include "shape.cuh"
#include "light.cuh"
#include "hosek.cuh"
#include "material.cuh"
#include "transform.cuh"
#include "camera.cuh"
#include "texture.h"
#include "payload.h"
