// Stand-in for the reference's noor/cuda/path_tracer.cuh in the bridge
// check (tests/test_bridge_compile.py): the reference's own device headers
// through the oracle's prelude (which replaces path_tracer.cuh's GL and
// CUDA-Samples includes), GLuint as GL defines it, and the extern "C"
// declarations of path_tracer.cuh:136-151 that the bridge defines.
#pragma once
#include "prelude.h"

typedef unsigned int GLuint;
#define NOOR_B200_HEADLESS

extern "C" {
void load_cuda_data(const std::unique_ptr<CudaPayload>& payload, const CudaHosekSky& hosek, const CudaCamera& camera,
                    const CudaSpec& spec, GLuint* textureID);
void update_cuda_camera();
void update_cuda_hosek();
void update_cuda_spec();
void cuda_path_tracer(uint& frameCount);
void debug_skydome(uint& frameCount, int width, int height);
void device_free_memory();
void get_lookAt(float4& lookAt);
}
