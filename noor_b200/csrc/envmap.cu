// Environment importance-sampling distribution (FP64 prefix sums on the
// GPU) and the FP64 Hosek-Wilkie coefficient fit.
//
// The distribution is PBRT-v3's piecewise-constant Distribution2D over the
// full environment resolution: func = luminance x sin(theta) per cell, each
// row a conditional CDF, the row integrals a marginal CDF.  The reference
// builds an FP32 Blelloch scan over a grid clamped to 1024 x 1024 whose
// sampling reads one entry past each CDF (noor/cuda/distribution2d.cuh:
// 63-228, 326-336); this build uses the whole map and the standard n-entry
// search.  The pdf conversion to solid angle is the reference's
// (skydome.cuh:138, lightimp.cuh:162-173).
#include "kernels.h"
#include "shading.cuh"

namespace nb {

constexpr int kScanThreads = 256;

__global__ void k_env_func_tex(const float4* env, int w, int h, float* func) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w * h) return;
    const int row = i / w;
    const float st = sinf(((float)row + 0.5f) / (float)h * kPi);
    const float4 t = env[i];
    func[i] = fmaxf(0.0f, rgb2y(f3(t))) * st;
}

// querySkyModel (noor/cuda/hosek.cuh:86-101) in FP64, for the distribution
// below only: a sub-sample within FP32 rounding of the sun disc's edge then
// falls on the same side on every machine (FP32 arithmetic libraries differ
// there, and the sun's radiance is 10^4 times the sky's)
__device__ double hosek_channel_d(const float* c, double theta, double gamma) {
    const double cg = cos(gamma), cg2 = cg * cg, ct = cos(theta);
    const double mie = (1.0 + cg2) / pow(1.0 + (double)c[8] * (double)c[8] - 2.0 * (double)c[8] * cg, 1.5);
    return (1.0 + (double)c[0] * exp((double)c[1] / (ct + (double)0.01f))) *
           ((double)c[2] + (double)c[3] * exp((double)c[4] * gamma) + (double)c[5] * cg2 + (double)c[6] * mie +
            (double)c[7] * sqrt(ct));
}
__device__ double inverse_gamma_d(double v) {
    if (v <= (double)0.04045f) return v / (double)12.92f;
    return pow((v + (double)0.055f) / (double)1.055f, (double)2.4f);
}
__device__ double sky_luminance_d(const DevHosek& H, double x, double y, double z) {
    if (y < 0.0) return 0.0;
    const double theta = fmin(fmax(acos(fmin(fmax(y, -1.0), 1.0)), 0.0), 3.141592653589793 / 2.0);
    const double cs = x * (double)H.solar_dir.x + y * (double)H.solar_dir.y + z * (double)H.solar_dir.z;
    const double gamma = acos(fmin(fmax(cs, -1.0), 1.0));
    double rgb[3];
    for (int k = 0; k < 3; ++k) rgb[k] = hosek_channel_d(H.configs[k], theta, gamma) * (double)H.radiance[k];
    if (gamma < (double)H.solar_radius)
        for (int k = 0; k < 3; ++k) rgb[k] *= (double)H.solar_scale;
    else
        for (int k = 0; k < 3; ++k) rgb[k] = inverse_gamma_d(rgb[k] * (double)0.025f);
    return (double)0.2126f * rgb[0] + (double)0.7152f * rgb[1] + (double)0.0722f * rgb[2];
}

// the sky's cells: luminance x sin(theta) averaged over 4 x 4 sub-samples,
// in FP64, rounded once to FP32
__global__ void k_env_func_sky(DevHosek H, int w, int h, float* func) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w * h) return;
    const int row = i / w, col = i % w;
    constexpr double pi = 3.141592653589793;
    double acc = 0.0;
    for (int b = 0; b < 4; ++b) {
        const double theta = ((double)row + ((double)b + 0.5) * 0.25) / (double)h * pi;
        const double st = sin(theta), ct = cos(theta);
        for (int a = 0; a < 4; ++a) {
            const double phi = ((double)col + ((double)a + 0.5) * 0.25) / (double)w * (2.0 * pi);
            double x = st * cos(phi), y = ct, z = st * sin(phi);
            const double inv = 1.0 / sqrt(x * x + y * y + z * z);
            x *= inv;
            y *= inv;
            z *= inv;
            acc += fmax(0.0, sky_luminance_d(H, x, y, z)) * st;
        }
    }
    func[i] = (float)(acc / 16.0);
}

// Inclusive FP64 block scan of kScanThreads values (Hillis-Steele in smem).
__device__ double block_scan_incl(double v, double* sh) {
    const int t = threadIdx.x;
    sh[t] = v;
    __syncthreads();
    for (int off = 1; off < kScanThreads; off <<= 1) {
        const double add = t >= off ? sh[t - off] : 0.0;
        __syncthreads();
        sh[t] += add;
        __syncthreads();
    }
    const double r = sh[t];
    __syncthreads();
    return r;
}

// Prefix sums of one row of n values (FP32 in, FP64 accumulate):
// out[0] = 0, out[i+1] = out[i] + in[i] / n.  Each thread owns a contiguous
// segment; segment totals are scanned across the block.  Returns the total.
__device__ double row_prefix(const float* in, const double* in_d, int n, double* out, double* sh) {
    const int t = threadIdx.x;
    const int seg = (n + kScanThreads - 1) / kScanThreads;
    const int b = t * seg, e = min(b + seg, n);
    const double inv_n = 1.0 / (double)n;
    double local = 0.0;
    for (int i = b; i < e; ++i) local += (in ? (double)in[i] : in_d[i]) * inv_n;
    const double incl = block_scan_incl(local, sh);
    double run = incl - local;
    for (int i = b; i < e; ++i) {
        out[i] = run;
        run += (in ? (double)in[i] : in_d[i]) * inv_n;
    }
    __shared__ double total;
    if (t == kScanThreads - 1) {
        total = incl;
        out[n] = incl;
    }
    __syncthreads();
    return total;
}

// one block per row: conditional CDF of the row, row integral
__global__ void __launch_bounds__(kScanThreads) k_row_cdf(const float* func, int w, int h, float* cdf,
                                                          float* row_int, double* scratch) {
    __shared__ double sh[kScanThreads];
    const int row = blockIdx.x;
    double* cd = scratch + (size_t)row * (w + 1);
    const double total = row_prefix(func + (size_t)row * w, nullptr, w, cd, sh);
    float* c = cdf + (size_t)row * (w + 1);
    for (int i = threadIdx.x; i <= w; i += kScanThreads)
        c[i] = total > 0.0 ? (float)(cd[i] / total) : (float)((double)i / (double)w);
    if (threadIdx.x == 0) {
        row_int[row] = (float)total;
        scratch[(size_t)h * (w + 1) + row] = total;
    }
}

// single block: marginal CDF over the row integrals
__global__ void __launch_bounds__(kScanThreads) k_marg_cdf(int w, int h, float* marg_cdf, double* scratch,
                                                           float* marg_int_out) {
    __shared__ double sh[kScanThreads];
    const double* rows = scratch + (size_t)h * (w + 1);
    double* cd = scratch + (size_t)h * (w + 1) + h;
    // the row integrals are stored as float in row_int; sample with the
    // float values so pdf(sample) == func / integral exactly in FP32
    const double total = row_prefix(nullptr, rows, h, cd, sh);
    for (int i = threadIdx.x; i <= h; i += kScanThreads)
        marg_cdf[i] = total > 0.0 ? (float)(cd[i] / total) : (float)((double)i / (double)h);
    if (threadIdx.x == 0) *marg_int_out = (float)total;
}

cudaError_t launch_env_func_from_texture(const float4* env, int w, int h, float* func, cudaStream_t s) {
    const int n = w * h;
    k_env_func_tex<<<(n + 255) / 256, 256, 0, s>>>(env, w, h, func);
    return cudaGetLastError();
}

cudaError_t launch_env_func_from_sky(const DevHosek& H, int w, int h, float* func, cudaStream_t s) {
    const int n = w * h;
    k_env_func_sky<<<(n + 255) / 256, 256, 0, s>>>(H, w, h, func);
    return cudaGetLastError();
}

// Guide entries of CDF rows (row r of n + 1 values at cdf + r * (n + 1)):
// entry k = largest i in [0, n] with cdf[i] <= k / kDistGuide (exact in
// FP32: kDistGuide is a power of two), by the same search sample_1d runs
__global__ void k_dist_guide(const float* cdf, int n, int rows, int* guide) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= rows * (kDistGuide + 1)) return;
    const int r = t / (kDistGuide + 1), k = t % (kDistGuide + 1);
    const float* c = cdf + (size_t)r * (n + 1);
    const float u = (float)k / (float)kDistGuide;
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (c[mid] <= u)
            lo = mid;
        else
            hi = mid - 1;
    }
    guide[t] = lo;
}

cudaError_t launch_env_cdf(const EnvBuild& b, cudaStream_t s) {
    k_row_cdf<<<b.h, kScanThreads, 0, s>>>(b.func, b.w, b.h, b.cdf, b.row_int, b.scratch);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_marg_cdf<<<1, kScanThreads, 0, s>>>(b.w, b.h, b.marg_cdf, b.scratch, b.marg_int_out);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (b.guide) {
        const int nr = b.h * (kDistGuide + 1);
        k_dist_guide<<<(nr + 255) / 256, 256, 0, s>>>(b.cdf, b.w, b.h, b.guide);
        k_dist_guide<<<1, kDistGuide + 1, 0, s>>>(b.marg_cdf, b.h, 1, b.mguide);
    }
    return cudaGetLastError();
}

// --------------------------------------------------------------- Hosek fit
// Restatement of the published Hosek-Wilkie fit (ArHosekSkyModel.cpp:
// 147-289): each coefficient is a quintic Bezier in elevation^(1/3), blended
// linearly over ground albedo (2 tables) and turbidity (10 tables).  One
// thread per (state, channel, value); value 9 is the radiance scale.
__device__ double bezier5(const float* m, int stride, double se) {
    const double a = 1.0 - se;
    return a * a * a * a * a * (double)m[0] + 5.0 * a * a * a * a * se * (double)m[stride] +
           10.0 * a * a * a * se * se * (double)m[2 * stride] + 10.0 * a * a * se * se * se * (double)m[3 * stride] +
           5.0 * a * se * se * se * se * (double)m[4 * stride] + se * se * se * se * se * (double)m[5 * stride];
}

__global__ void k_hosek_fit(const float* dataset, double turbidity, double a0, double a1, double a2, double elevation,
                            float* out) {
    const int tid = threadIdx.x;  // 0..89
    if (tid >= 90) return;
    const int state = tid / 30, rem = tid % 30, channel = rem / 10, value = rem % 10;
    const double albedo = state == 0 ? a0 : (state == 1 ? a1 : a2);
    const int it = (int)turbidity;
    const double tr = turbidity - (double)it;
    const double se = pow(elevation / (3.141592653589793 / 2.0), 1.0 / 3.0);
    double r;
    if (value < 9) {
        const float* ds = dataset + channel * 1080;
        const int i = value;
        r = (1.0 - albedo) * (1.0 - tr) * bezier5(ds + 54 * (it - 1) + i, 9, se) +
            albedo * (1.0 - tr) * bezier5(ds + 540 + 54 * (it - 1) + i, 9, se);
        if (it != 10)
            r += (1.0 - albedo) * tr * bezier5(ds + 54 * it + i, 9, se) + albedo * tr * bezier5(ds + 540 + 54 * it + i, 9, se);
        out[state * 30 + channel * 9 + value] = (float)r;
    } else {
        const float* ds = dataset + 3 * 1080 + channel * 120;
        r = (1.0 - albedo) * (1.0 - tr) * bezier5(ds + 6 * (it - 1), 1, se) +
            albedo * (1.0 - tr) * bezier5(ds + 60 + 6 * (it - 1), 1, se);
        if (it != 10)
            r += (1.0 - albedo) * tr * bezier5(ds + 6 * it, 1, se) + albedo * tr * bezier5(ds + 60 + 6 * it, 1, se);
        out[state * 30 + 27 + channel] = (float)r;
    }
}

cudaError_t launch_hosek_fit(const float* dataset, double turbidity, const double* albedo3, double elevation,
                             float* out, cudaStream_t s) {
    k_hosek_fit<<<1, 96, 0, s>>>(dataset, turbidity, albedo3[0], albedo3[1], albedo3[2], elevation, out);
    return cudaGetLastError();
}

// ------------------------------------------------ reference distribution
// NOOR_ENV_REFERENCE: the reference's CudaDistribution2D built as it builds
// it (noor/cuda/distribution2d.cuh:63-228), so that sampling maps the same
// uniforms to the same directions.  Its luminance, sums and divisions round
// each operation on its own (the arithmetic of the reference built for the
// host); the texture reads are the texture unit's bilinear filter, as there.

// update_skydome (noor/cuda/skydome.cuh:27-37): texel (x, y) of a w x h
// texture holds sin(theta) x sky radiance at u = (x / w, y / h)
__global__ void k_ref_sky_bake(DevHosek H, int w, int h, float4* out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    float st;
    const float3 dir = spherical_direction(xdiv((float)x, (float)w), xdiv((float)y, (float)h), st);
    const float3 c = hosek_query(H, dir);
    out[(size_t)y * w + x] = make_float4(xmul(st, c.x), xmul(st, c.y), xmul(st, c.z), st);
}

// update_func (distribution2d.cuh:63-83): cell (row, col) of the w x h grid
// = mean luminance of the 3x3 texture reads at ((col + i) / w, (row + j) / h),
// i, j in {-1, 0, 1}; one block per row, one thread per column
__global__ void k_ref_func(cudaTextureObject_t tex, int w, int h, float* func) {
    const int row = blockIdx.y, col = threadIdx.x;
    float acc = 0.0f;
    for (int j = -1; j <= 1; ++j)
        for (int i = -1; i <= 1; ++i) {
            const float4 t = tex2D<float4>(tex, xdiv((float)(i + col), (float)w), xdiv((float)(j + row), (float)h));
            acc = xadd(acc, xdot3(t.x, t.y, t.z, 0.2126f, 0.7152f, 0.0722f));
        }
    func[(size_t)row * (w + 1) + col] = xdiv(acc, 9.0f);
}

// prescan (distribution2d.cuh:86-135): exclusive work-efficient (up-sweep /
// down-sweep) scan of func[row][0..n) / n into cdf[row][0..n), then
// cdf[row][n] = func[row][n] = the row's integral; rows are n + 1 apart,
// one block of n / 2 threads per row, n a power of two.  The reference's
// bank-conflict offset evaluates to 0 for every index it meets.
__global__ void k_ref_scan(float* func, float* cdf, int n) {
    extern __shared__ float tmp[];
    const int tid = threadIdx.x;
    const size_t base = (size_t)blockIdx.y * (n + 1);
    const int ai = tid, bi = tid + n / 2;
    tmp[ai] = xdiv(func[base + ai], (float)n);
    tmp[bi] = xdiv(func[base + bi], (float)n);
    int offset = 1;
    for (int d = n >> 1; d > 0; d >>= 1) {
        __syncthreads();
        if (tid < d) {
            const int a = offset * (2 * tid + 1) - 1, b = offset * (2 * tid + 2) - 1;
            tmp[b] = xadd(tmp[b], tmp[a]);
        }
        offset *= 2;
    }
    if (tid == 0) tmp[n - 1] = 0.0f;
    for (int d = 1; d < n; d *= 2) {
        offset >>= 1;
        __syncthreads();
        if (tid < d) {
            const int a = offset * (2 * tid + 1) - 1, b = offset * (2 * tid + 2) - 1;
            const float t = tmp[a];
            tmp[a] = tmp[b];
            tmp[b] = xadd(tmp[b], t);
        }
    }
    __syncthreads();
    cdf[base + ai] = tmp[ai];
    cdf[base + bi] = tmp[bi];
    __syncthreads();
    if (tid == 0) {
        const float fi = xadd(cdf[base + n - 1], xdiv(func[base + n - 1], (float)n));
        cdf[base + n] = fi;
        func[base + n] = fi;
    }
}

// process_cdf (distribution2d.cuh:137-160): normalise each row's CDF by its
// integral (a uniform CDF for a zero row); with h > 1 the integrals become
// the marginal's func at h * (w + 1)
__global__ void k_ref_normalize(float* func, float* cdf, int w, int h) {
    __shared__ float fi;
    const int row = blockIdx.y, col = threadIdx.x;
    const size_t base = (size_t)row * (w + 1);
    if (col == 0) fi = cdf[base + w];
    __syncthreads();
    cdf[base + col + 1] = fi == 0.0f ? xdiv((float)(col + 1), (float)w) : xdiv(cdf[base + col + 1], fi);
    if (col == 0 && h > 1) func[(size_t)h * (w + 1) + row] = fi;
}

cudaError_t launch_ref_sky_bake(const DevHosek& H, int w, int h, float4* out, cudaStream_t s) {
    const dim3 block(32, 8), grid((w + 31) / 32, (h + 7) / 8);
    k_ref_sky_bake<<<grid, block, 0, s>>>(H, w, h, out);
    return cudaGetLastError();
}

cudaError_t launch_ref_distribution(cudaTextureObject_t tex, int w, int h, float* func, float* cdf, cudaStream_t s) {
    k_ref_func<<<dim3(1, h), w, 0, s>>>(tex, w, h, func);
    k_ref_scan<<<dim3(1, h), w / 2, (w + 1) * sizeof(float), s>>>(func, cdf, w);
    k_ref_normalize<<<dim3(1, h), w, 0, s>>>(func, cdf, w, h);
    float* mf = func + (size_t)h * (w + 1);
    float* mc = cdf + (size_t)h * (w + 1);
    k_ref_scan<<<dim3(1, 1), h / 2, (h + 1) * sizeof(float), s>>>(mf, mc, h);
    k_ref_normalize<<<dim3(1, 1), h, 0, s>>>(mf, mc, h, 1);
    return cudaGetLastError();
}

}  // namespace nb
