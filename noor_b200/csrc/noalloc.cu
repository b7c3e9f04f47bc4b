// Allocation-free variant of the batch megakernel frame
// (noor_megakernel_batch renders each frame into scratch films it allocates
// with cudaMalloc).  Some callers cannot allocate device memory at the
// moment they render: code running inside a memory pool or arena it does not
// own, hosts that forbid device allocation after start-up, or callers that
// must not add allocations to a stream they are about to capture.  This entry
// point takes its scratch -- the compensation film and the per-chunk partial
// films -- from one fixed device array of NOOR_NOALLOC_SCRATCH_BYTES and
// writes the mean into the caller's film, so a render call allocates nothing.
//
// Set-up: the first call on a device (with that device current) looks up the
// array's device address with cudaGetSymbolAddress; make that first call
// before any stream capture.  Every later call reuses the address, until
// device_free_memory on that device forgets it (a caller that resets the
// device afterwards gets a fresh look-up on its next first call).  A call
// waits for its own work to finish before it returns.
//
// Sharing: all calls on a device use the same array, and it keeps the last
// call's contents.  Nothing in it has to start at zero: every element a call
// reads is written earlier in the same call.  Calls whose work overlaps on
// the GPU (two threads rendering on one device at once) race on the array.
#include <algorithm>
#include <mutex>

#include "host_common.h"
#include "runtime.h"

namespace nb {

constexpr size_t kNoAllocElems = NOOR_NOALLOC_SCRATCH_BYTES / sizeof(float4);
static __device__ __align__(256) float4 g_noalloc_scratch[kNoAllocElems];

constexpr int kNoAllocMaxDevices = 64;
static std::mutex g_noalloc_mutex;
static float4* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// device address of the scratch array on the current device (looked up once)
// the cached scratch address of a device is dropped with a render context
// of that device (device_free_memory)
void noalloc_forget(int device) {
    if (device < 0 || device >= kNoAllocMaxDevices) return;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    g_noalloc_ptr[device] = nullptr;
}

static int noalloc_scratch(int device, float4** out) {
    if (device < 0 || device >= kNoAllocMaxDevices)
        return set_error(NOOR_ERR_UNSUPPORTED, "no-alloc render: device index beyond 63");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[device]) {
        float4* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "no-alloc render: cudaGetSymbolAddress of the scratch array");
        g_noalloc_ptr[device] = p;
    }
    *out = g_noalloc_ptr[device];
    return NOOR_OK;
}

}  // namespace nb

using namespace nb;

extern "C" int noor_megakernel_frame_noalloc(const noor_wf_frame* f) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    if (!f) return set_error(NOOR_ERR_INVALID, "no-alloc render: frame is null");
    if (!f->d_film) return set_error(NOOR_ERR_INVALID, "no-alloc render: d_film (the output film) is required");
    if (f->scene_id >= C->scenes.size()) return set_error(NOOR_ERR_INVALID, "no-alloc render: unknown scene id");
    if (f->width == 0 || f->height == 0 || f->spp == 0 || f->first_frame == 0 || f->width != f->camera.w ||
        f->height != f->camera.h)
        return set_error(NOOR_ERR_INVALID, "no-alloc render: bad frame description");
    if ((uint32_t)f->camera.type > NOOR_CAMERA_ENV) return set_error(NOOR_ERR_INVALID, "no-alloc render: bad camera type");
    const uint64_t npix = (uint64_t)f->width * f->height;
    // one compensation value per pixel is the least a call needs
    if (npix > kNoAllocElems)
        return set_error(NOOR_ERR_CAPACITY, "no-alloc render: " + std::to_string(npix) +
                                                " pixels exceed the scratch array (" +
                                                std::to_string(kNoAllocElems) + " pixels, " +
                                                std::to_string(NOOR_NOALLOC_SCRATCH_BYTES >> 20) + " MiB)");
    float4* scratch = nullptr;
    if ((rc = noalloc_scratch(C->device, &scratch))) return rc;

    DevScene S = C->scenes[f->scene_id]->dev;
    if (f->bounces) S.bounces = f->bounces;
    S.film_mode = NOOR_FILM_KAHAN;
    const DevCamera cam = dev_camera(f->camera, f->width, f->height);
    // same split of the samples as the batch megakernel, reduced until the
    // partial films (2 x chunks x pixels) fit beside the compensation film.
    // With 148 SMs the split asks for more than one chunk only below
    // 151,552 pixels, where 1 + 2 x chunks films stay far inside the array:
    // the loop is a guard for GPUs with many more SMs.
    const uint64_t target = (uint64_t)C->sm_count * 1024u;
    uint64_t chunks = std::min<uint64_t>(f->spp, std::max<uint64_t>(1, (target + npix - 1) / npix));
    while (chunks > 1 && npix * (1 + 2 * chunks) > kNoAllocElems) --chunks;
    MegaArgs a{};
    a.frame0 = f->first_frame;
    a.nframes = f->spp;
    a.chunks = (uint32_t)chunks;
    a.fresh = 1u;
    a.film_sum = reinterpret_cast<float4*>(f->d_film);  // the sum, scaled to the mean in place below
    a.film_comp = scratch;
    if (chunks > 1) {
        a.part_sum = scratch + npix;
        a.part_comp = scratch + npix + chunks * npix;
    }
    a.lookat = C->lookat;
    a.status = C->status;
    a.counters = C->counters;
    cudaError_t e = launch_megakernel(S, cam, a, C->stream);
    if (e == cudaSuccess)
        e = launch_resolve((uint32_t)npix, NOOR_FILM_KAHAN, 1.0f / (float)f->spp, a.film_sum, a.film_sum, C->stream);
    if (e != cudaSuccess) return cuda_fail(e, "no-alloc render");
    C->launches += (chunks > 1 ? 2 : 1) + 1;
    return sync_and_check(*C, "no-alloc render");
}
