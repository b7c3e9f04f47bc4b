// Host-side state of a render context (one per thread).
#pragma once
#include <cuda_runtime.h>
#include <map>
#include <memory>
#include <vector>

#include "kernels.h"

namespace nb {

// one device-resident scene (payload + sky + spec)
struct SceneState {
    DevScene dev{};
    EnvBuild env{};
    std::vector<void*> allocs;
    std::vector<DevMaterial> materials_host;
    bool quad_lights_only = true;   // every area light a quad
    int sky_type = 0;
    uint32_t max_mesh_leaf = 0;
    // the four-wide any-hit tree (wide_bvh.h) and the root it was built from
    const DevNode4* wide_nodes = nullptr;
    const uint32_t* wide_map = nullptr;
    uint32_t wide_root = 0;
    int wide_cap = 0;
    bool wide_closest = false;
    // NOOR_ENV_REFERENCE, built on first use: the environment (or baked sky)
    // as a CUDA array + texture object, the bake buffer and the tables
    cudaArray_t env_array = nullptr;
    cudaTextureObject_t env_tex = 0;
    float4* ref_bake = nullptr;
    float* ref_func = nullptr;
    float* ref_cdf = nullptr;
    bool ref_built = false;
    // material textures read through the texture unit, by payload index
    struct TexObj {
        cudaArray_t array;
        cudaTextureObject_t obj;
    };
    std::map<uint32_t, TexObj> textures;
    ~SceneState();
    int alloc(void** p, size_t bytes, const char* what);
    int upload(void** p, const void* host, size_t bytes, const char* what);
    int texture_object(const noor_texture& t, uint32_t idx, cudaTextureObject_t* out);
};

struct WavefrontState;  // wavefront.cu

struct Context {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    const noor_hosek_sky* hosek_src = nullptr;
    const noor_camera* camera_src = nullptr;
    const noor_spec* spec_src = nullptr;
    std::vector<std::unique_ptr<SceneState>> scenes;
    DevCamera cam{};
    float4* film_sum = nullptr;
    float4* film_comp = nullptr;
    float4* film_out = nullptr;
    uint32_t film_w = 0, film_h = 0;
    uint64_t film_count = 0;
    bool film_is_mean = false;
    uint32_t last_frame = 0;
    float4* part_sum = nullptr;
    float4* part_comp = nullptr;
    size_t part_cap = 0;
    float4* lookat = nullptr;
    uint32_t* status = nullptr;
    unsigned long long* counters = nullptr;
    void* scratch = nullptr;
    void* adj_buf = nullptr;  // adjoint: per-sample radiance of one chunk + the forward's Kahan state
    size_t adj_bytes = 0;
    cudaEvent_t events[8] = {};
    uint64_t launches = 0;
    WavefrontState* wf = nullptr;
    ~Context();
};

extern thread_local Context* tl_ctx;
int cuda_fail(cudaError_t e, const char* what);
int need_ctx(Context*& C);
int sync_and_check(Context& C, const char* what);
int render_frames(Context& C, uint32_t frame0, uint32_t n);
void wavefront_release(Context& C);
void noalloc_forget(int device);  // noalloc.cu

}  // namespace nb
