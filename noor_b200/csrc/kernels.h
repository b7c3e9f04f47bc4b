// Host-visible launchers of the render and parity kernels.
#pragma once
#include "scene_dev.cuh"

namespace nb {

constexpr int kMegaBlock = 128;
constexpr int kTraceBlock = 128;

struct MegaArgs {
    uint32_t frame0;        // RNG frame number of the first sample
    uint32_t nframes;       // samples per pixel in this launch
    uint32_t chunks;        // frame ranges split across threads (>=1)
    uint32_t fresh;         // 1: start the film from zero, 0: fold into it
    float4* film_sum;       // Kahan sum (or running mean in lerp mode)
    float4* film_comp;      // Kahan compensation
    float4* part_sum;       // chunks * npix partial sums (chunks > 1)
    float4* part_comp;
    float4* lookat;         // first hit of the centre pixel
    uint32_t* status;       // NOOR_DEV_* bits
    unsigned long long* counters;  // [ext rays, shadow rays, paths]
};

cudaError_t launch_megakernel(const DevScene& S, const DevCamera& C, const MegaArgs& a, cudaStream_t s);
cudaError_t launch_resolve(uint32_t npix, int mode, float inv_count, const float4* film_sum, float4* out,
                           cudaStream_t s);
cudaError_t launch_trace_closest(const DevScene& S, const noor_ray* rays, noor_hit* hits, size_t n, uint32_t* status,
                                 cudaStream_t s);
cudaError_t launch_trace_any(const DevScene& S, const noor_ray* rays, uint32_t* occ, size_t n, uint32_t* status,
                             cudaStream_t s);
cudaError_t launch_camera_rays(const DevCamera& C, uint32_t frame, noor_ray* rays, cudaStream_t s);
cudaError_t launch_eval_bsdf(const DevScene& S, int kind, const float* in, float* out, size_t n, cudaStream_t s);
cudaError_t launch_eval_sky(const DevScene& S, const float* dirs, float* rgb, size_t n, cudaStream_t s);
cudaError_t launch_eval_routines(int kind, const float* in, float* out, size_t n, cudaStream_t s);
cudaError_t launch_env_sample(const DevScene& S, const float* u, float* out, size_t n, cudaStream_t s);
cudaError_t launch_debug_skydome(const DevScene& S, const DevCamera& C, uint32_t frame, float4* film, int mis,
                                 cudaStream_t s);

// environment distribution (FP64 prefix sums) and sky; envmap.cu
struct EnvBuild {
    float* func;      // h*w
    float* cdf;       // h*(w+1)
    float* row_int;   // h
    float* marg_cdf;  // h+1
    double* scratch;  // h*(w+1) + h + 1 doubles
    float* marg_int_out;  // one float
    int* guide;       // h*(kDistGuide+1) guide entries of the row CDFs
    int* mguide;      // kDistGuide+1 of the marginal CDF
    int w, h;
};
// func from the env texels (luminance x sin(theta) per texel)
cudaError_t launch_env_func_from_texture(const float4* env, int w, int h, float* func, cudaStream_t s);
// func from the Hosek sky (4x4 supersampled luminance x sin(theta) per cell)
cudaError_t launch_env_func_from_sky(const DevHosek& H, int w, int h, float* func, cudaStream_t s);
// FP64 row/marginal prefix sums -> normalised FP32 CDFs
cudaError_t launch_env_cdf(const EnvBuild& b, cudaStream_t s);
// NOOR_ENV_REFERENCE: the physical sky baked as sin(theta) x radiance into a
// w x h texture, and the reference's distribution tables (h * (w + 2) + 1
// floats each) from a texture read with its bilinear filter; w, h powers of
// two in [32, 1024]
cudaError_t launch_ref_sky_bake(const DevHosek& H, int w, int h, float4* out, cudaStream_t s);
cudaError_t launch_ref_distribution(cudaTextureObject_t tex, int w, int h, float* func, float* cdf, cudaStream_t s);
// Hosek-Wilkie RGB fit in FP64: dataset = 3 x 1080 coefficients then 3 x 120
// radiances; writes 3 states x (27 configs + 3 radiances) into out (90 floats
// per state, state-major, configs first).
cudaError_t launch_hosek_fit(const float* dataset, double turbidity, const double* albedo3, double elevation,
                             float* out, cudaStream_t s);

}  // namespace nb
