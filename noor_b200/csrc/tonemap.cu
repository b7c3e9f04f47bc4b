// Headless display path: the film through the display shader's transforms
// (noor/shader/cuda.fs:36-78) into 8-bit RGBA on the device, and image files
// written from it (PPM) or from the linear film (PFM).  The reference draws
// the film as a GL texture; here no graphics API is involved.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <vector>

#include "dmath.cuh"
#include "host_common.h"
#include "runtime.h"

namespace nb {

// gammaCorrect (cuda.fs:37-40): c^(1/2.2)
NB_D float3 gamma22(const float3& c) {
    const float g = 1.0f / 2.2f;
    return f3(powf(c.x, g), powf(c.y, g), powf(c.z, g));
}
// Uncharted2Tonemap (cuda.fs:56-58), John Hable's filmic curve
NB_D float hable(float x) {
    const float A = 0.15f, B = 0.50f, C = 0.10f, D = 0.20f, E = 0.02f, F = 0.30f;
    return ((x * (A * x + C * B) + D * E) / (x * (A * x + B) + D * F)) - E / F;
}
NB_D float3 tonemap_op(int op, const float3& c) {
    if (op == NOOR_TONEMAP_REINHARD) {
        // tonemapReinhard (cuda.fs:42-45)
        return gamma22(f3(c.x / (c.x + 1.0f), c.y / (c.y + 1.0f), c.z / (c.z + 1.0f)));
    }
    if (op == NOOR_TONEMAP_FILMIC) {
        // tonemapFilmic (cuda.fs:47-51): the Hejl-Burgess-Dawson curve,
        // gamma included
        const float3 x = f3(fmaxf(0.0f, c.x - 0.004f), fmaxf(0.0f, c.y - 0.004f), fmaxf(0.0f, c.z - 0.004f));
        return f3((x.x * (6.2f * x.x + 0.5f)) / (x.x * (6.2f * x.x + 1.7f) + 0.06f),
                  (x.y * (6.2f * x.y + 0.5f)) / (x.y * (6.2f * x.y + 1.7f) + 0.06f),
                  (x.z * (6.2f * x.z + 0.5f)) / (x.z * (6.2f * x.z + 1.7f) + 0.06f));
    }
    if (op == NOOR_TONEMAP_UNCHARTED2) {
        // tonemapUncharted2 (cuda.fs:61-68): exposure bias 4, white 11.2
        const float ws = 1.0f / hable(11.2f);
        return gamma22(f3(hable(4.0f * c.x) * ws, hable(4.0f * c.y) * ws, hable(4.0f * c.z) * ws));
    }
    return gamma22(c);
}
// a normalised 8-bit channel: clamp to [0, 1], round to nearest
NB_D uint32_t unorm8(float v) { return __float2uint_rn(fminf(fmaxf(v, 0.0f), 1.0f) * 255.0f); }

// one pixel per thread, grid-stride: 16 B read, 4 B written per pixel
__global__ void __launch_bounds__(256) k_tonemap(const float4* __restrict__ film, uint32_t n, int op, float exposure,
                                                 uchar4* __restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 v = film[i];
        const float3 c = tonemap_op(op, f3(exposure * v.x, exposure * v.y, exposure * v.z));
        out[i] = make_uchar4((unsigned char)unorm8(c.x), (unsigned char)unorm8(c.y), (unsigned char)unorm8(c.z), 255);
    }
}

static int launch_tonemap(Context& C, const float* d_film, size_t n, int op, float exposure, uint8_t* d_out) {
    if (op < NOOR_TONEMAP_GAMMA || op > NOOR_TONEMAP_UNCHARTED2)
        return set_error(NOOR_ERR_INVALID, "tonemap: unknown operator");
    if (n == 0) return NOOR_OK;
    if (n > 0xFFFFFFFFull) return set_error(NOOR_ERR_INVALID, "tonemap: too many pixels");
    if ((reinterpret_cast<uintptr_t>(d_film) & 15u) || (reinterpret_cast<uintptr_t>(d_out) & 3u))
        return set_error(NOOR_ERR_INVALID, "tonemap: film must be 16-byte and output 4-byte aligned");
    const uint32_t blocks = (uint32_t)std::min<size_t>((n + 255) / 256, (size_t)C.sm_count * 8);
    k_tonemap<<<blocks, 256, 0, C.stream>>>(reinterpret_cast<const float4*>(d_film), (uint32_t)n, op, exposure,
                                           reinterpret_cast<uchar4*>(d_out));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "tonemap");
    C.launches++;
    return NOOR_OK;
}

}  // namespace nb

using namespace nb;

extern "C" int noor_tonemap_device(const float* d_film_rgba, size_t n_pixels, int op, float exposure,
                                   uint8_t* d_rgba8) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    if (!d_film_rgba || !d_rgba8) return set_error(NOOR_ERR_INVALID, "tonemap: null buffer");
    if ((rc = launch_tonemap(*C, d_film_rgba, n_pixels, op, exposure, d_rgba8))) return rc;
    return sync_and_check(*C, "tonemap");
}

extern "C" int noor_save_image(const char* path, int op, float exposure) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    if (!path) return set_error(NOOR_ERR_INVALID, "save_image: null path");
    const size_t w = C->film_w, h = C->film_h, n = w * h;
    if (n == 0) return set_error(NOOR_ERR_INVALID, "save_image: no film");
    std::vector<float> lin;
    std::vector<uint8_t> px;
    if ((rc = noor_get_framebuffer_device((float*)C->film_out, n))) return rc;
    if (op == NOOR_TONEMAP_NONE) {
        lin.resize(4 * n);
        cudaError_t e = cudaMemcpyAsync(lin.data(), C->film_out, n * 16, cudaMemcpyDeviceToHost, C->stream);
        if (e != cudaSuccess) return cuda_fail(e, "save_image");
    } else {
        uint8_t* d8 = nullptr;
        cudaError_t e = cudaMalloc((void**)&d8, n * 4);
        if (e != cudaSuccess) return cuda_fail(e, "save_image");
        px.resize(4 * n);
        rc = launch_tonemap(*C, (const float*)C->film_out, n, op, exposure, d8);
        if (!rc) {
            e = cudaMemcpyAsync(px.data(), d8, n * 4, cudaMemcpyDeviceToHost, C->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(C->stream);
            if (e != cudaSuccess) rc = cuda_fail(e, "save_image");
        }
        cudaFree(d8);
        if (rc) return rc;
    }
    if ((rc = sync_and_check(*C, "save_image"))) return rc;
    FILE* f = std::fopen(path, "wb");
    if (!f) return set_error(NOOR_ERR_INVALID, std::string("save_image: cannot open ") + path);
    bool ok = true;
    if (op == NOOR_TONEMAP_NONE) {
        // PFM: linear RGB floats, bottom row first (film row 0 is the bottom
        // of the GL window), little-endian (scale -1)
        ok = std::fprintf(f, "PF\n%zu %zu\n-1.0\n", w, h) > 0;
        std::vector<float> row(3 * w);
        for (size_t y = 0; ok && y < h; ++y) {
            for (size_t x = 0; x < w; ++x)
                for (int c = 0; c < 3; ++c) row[3 * x + c] = lin[4 * (y * w + x) + c];
            ok = std::fwrite(row.data(), sizeof(float), row.size(), f) == row.size();
        }
    } else {
        // binary PPM: top row first, i.e. film row h - 1 first
        ok = std::fprintf(f, "P6\n%zu %zu\n255\n", w, h) > 0;
        std::vector<uint8_t> row(3 * w);
        for (size_t y = h; ok && y-- > 0;) {
            for (size_t x = 0; x < w; ++x)
                for (int c = 0; c < 3; ++c) row[3 * x + c] = px[4 * (y * w + x) + c];
            ok = std::fwrite(row.data(), 1, row.size(), f) == row.size();
        }
    }
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return set_error(NOOR_ERR_INVALID, std::string("save_image: write failed: ") + path);
    return NOOR_OK;
}
