// Persistent wavefront integrator: the path loop of the megakernel split
// into short kernels over a pool of path slots, so that traversal runs at
// the occupancy of a small kernel, shading runs over slots sorted by
// material kind, and finished slots are refilled with new paths at every
// bounce.  Many frames (different resolutions, scenes and sample counts)
// share one pool and one launch.
//
// Per bounce (one iteration of a CUDA-graph while loop):
//   regen   fold the last step's unblocked direct lighting into each
//           path's radiance (L += beta * (c0' + c1'), as the megakernel); add
//           finished paths to their frame's film; refill free slots with
//           camera rays of the next (frame, sample, pixel) work items, one
//           8x4 pixel tile per warp
//   extend  closest hit for every active slot; misses (their sky term added
//           by the next regen) and emitters finish the path, surface hits
//           are marked with their material kind
//   bin     shading queues per material kind, in slot order
//   shade   one launch per kind: light sample (+ MIS BSDF sample) with the
//           occlusion test deferred to a shadow-ray queue, then scatter,
//           Russian roulette and the next ray
//   shadow  any hit for the queued shadow rays; blocked ones are cancelled
//           (one ray per thread)
//   check   count rays; stop when no slot is active; bounded by an
//           iteration cap
// Counters that every slot touches (work items taken, active slots, queue
// lengths) are reserved with one atomic per block, not per warp: a single
// address serialises its atomics in L2.
//
// Every path draws the same random numbers in the same order as in the
// megakernel (seed TEA(pixel, frame), LCG state carried in the slot), so
// both integrators produce the same samples up to floating-point rounding.
// Films are accumulated with atomic adds whose rounding error is recovered
// exactly by TwoSum and added to a compensation buffer (compensated FP32
// summation that does not depend on completion order).
#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "host_common.h"
#include "integrator.cuh"
#include "runtime.h"

namespace nb {

constexpr int kKinds = 3;  // Lambert, conductor, dielectric

struct WfFrameDev {
    DevCamera cam;
    unsigned long long base;   // first global work index
    unsigned long long count;  // npix * spp
    uint32_t npix;
    uint32_t scene;
    uint32_t first_frame;
    uint32_t bounces;
    uint32_t spp;
    uint32_t pad;
    float4* sum;   // per pixel compensated sum
    float4* comp;
    float* out;    // caller's film (mean, float4 per pixel) or null
};

// slot state: bits 0-1 kFree / kActive / kFinishing; kPend while the direct
// lighting of the last shade step waits for regen to fold it into L; bits
// 3-4 the shading queue (1 + material kind) extend assigned to a surface hit;
// kSkySeen on a finishing slot whose last ray escaped to a sky it counts
// (regen adds beta * sky radiance, evaluated there with converged lanes)
enum : uint32_t { kFree = 0, kActive = 1, kFinishing = 2, kLifeMask = 3, kPend = 4, kKindShift = 3, kSkySeen = 32 };

// counter words
enum : int {
    kCntShadow = kKinds,       // [0, kKinds) shade queue lengths, then the shadow queue length
    kCntActive = kKinds + 1,   // slots holding a path after regen (= rays extend traces)
    kCntIter = kKinds + 2,     // iterations run
    kCntTake = kKinds + 3,     // shadow queue entries taken by wf_shadow's warps
    kCntTakeExt = kKinds + 4,  // extension order entries taken by wf_extend's warps
    kCntWords = kKinds + 5
};

// Ray ordering (sort levels 2 and 3): a counting sort of rays into buckets
// of (direction octant, cell of the origin in a 16^3 grid over the scene's
// root box), so that the lanes of a warp start near each other and head the
// same way.  The bucket of each ray is computed on the device and the
// counts, offsets and permutation never leave it (the pass runs inside the
// graph's loop).
constexpr int kWfStages = 7;  // noor_wf_profile's stages
constexpr int kCellBits = 4;
constexpr int kBuckets = 8 << (3 * kCellBits);
constexpr int kScanThreads = 1024;

// block sizes of the slot sweeps (one block-wide atomic per counter)
#ifndef NB_REGEN_BLOCK
#define NB_REGEN_BLOCK 512
#endif
constexpr int kRegenBlock = NB_REGEN_BLOCK;
constexpr int kBinBlock = 1024;

struct WfDev {
    // path slots
    float4* o;       // origin, w = frame index bits
    float4* d;       // direction, w = pixel bits
    float4* beta;    // throughput, w = bounce | spec << 16
    float4* L;       // radiance, w = RNG state bits
    float4* pend;    // 2 per slot: direct-light contribution, w = 1 while it counts
    float4* pbeta;   // throughput the contributions are weighted by (before the scatter)
    float4* hit;     // t, u, v, tri bits
    uint2* hit2;     // instance, material type
    uint32_t* state;
    float4* diff;           // 4 per slot where some scene has bump maps (else null): the ray's
                            // differentials odx (w = 1 while it has them), ody, ddx, ddy
    uint32_t* qshade;       // kKinds * cap slot indices
    uint32_t* qshadow;      // 2 * cap entries: slot << 1 | which
    float4* sh_o;           // origin, tmax (by queue entry)
    float4* sh_d;           // direction
    uint32_t* counters;     // kCntWords words
    uint32_t* bkt_cnt;      // kBuckets extension-ray bucket sizes (counted by shade for the next iteration)
    uint32_t* bkt_off;      // kBuckets bucket offsets, advanced by the scatter
    uint32_t* sh_bkt_cnt;   // the same for the shadow queue (sort level 3)
    uint32_t* sh_bkt_off;
    uint32_t* sh_key;       // bucket of each shadow queue entry
    uint32_t* sh_perm;      // shadow queue entries in bucket order
    uint32_t* ext_key;      // bucket of each slot's secondary ray
    uint32_t* ext_perm;     // camera-ray slots in slot order, then (at cap) secondary-ray slots in bucket order
    unsigned long long* work_next;  // [0] next work item, [1] the first one of this iteration
    unsigned long long* rays;  // [ext, shadow, paths], added up by wf_check
    uint32_t* status;
    const WfFrameDev* frames;
    const DevScene* scenes;
    uint32_t nframes;
    uint32_t cap;
    uint32_t sort;          // 0: one shade queue, 1: one per kind
    uint32_t level;         // sort granularity: 1 material queues, 2 + extension rays, 3 + shadow rays
    uint32_t max_iters;
    unsigned long long total;
    int stack_cap;
    cudaGraphConditionalHandle cond;
};

// Launch bounds of the traversal stages (extend, shadow): at most 128
// threads per block and 8 such blocks per SM cap their registers at 64
// (32 warps per SM; on the sky-lit 2.6M-triangle scene 76.9 ms per step
// against 78.0 at 9 blocks and 56 registers, where extend spills; the room
// runs the same at both)
#ifndef NB_TRAV_THREADS
#define NB_TRAV_THREADS 128
#endif
#ifndef NB_TRAV_MIN_BLOCKS
#define NB_TRAV_MIN_BLOCKS 8
#endif
// the same for the kernels on the four-wide tree: 8 blocks, 64 registers
// (their wide visits hold four boxes' slab intervals; on the sky-lit
// 2.6M-triangle scene 82.7 ms per step against 85.3 at 9 blocks and 84.8 at 7)
#ifndef NB_TRAV_MIN_BLOCKS_WIDE
#define NB_TRAV_MIN_BLOCKS_WIDE 8
#endif
// minimum resident 256-thread blocks per SM of the shading stage: 3 caps
// its registers at 85 (24 warps per SM instead of 16 at its natural 128)
#ifndef NB_SHADE_MIN_BLOCKS
#define NB_SHADE_MIN_BLOCKS 3
#endif
// 1: shadow rays taken 32 at a time per warp from a counter; 0: grid-stride
#ifndef NB_SHADOW_FETCH
#define NB_SHADOW_FETCH 1
#endif


NB_D uint32_t fbits(float f) { return __float_as_uint(f); }
NB_D float bitsf(uint32_t u) { return __uint_as_float(u); }

// warp-aggregated push: returns this lane's index into the queue.  Lanes of
// one warp may push onto different queues (one per material kind), so the
// lanes are grouped by counter and each group reserves its own range.
NB_D uint32_t queue_push(uint32_t* counter) {
    const uint32_t active = __activemask();
    const uint32_t peers = __match_any_sync(active, reinterpret_cast<unsigned long long>(counter));
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(peers));
    base = __shfl_sync(active, base, leader);
    return base + __popc(peers & ((1u << lane) - 1u));
}

NB_D float two_sum_err(float old, float v) {
    const float s = old + v;
    const float bp = s - old;
    return (old - (s - bp)) + (v - bp);
}
// compensated atomic add of an rgb value to a float4 pixel: one vector
// atomic returns the old sum, TwoSum of (old, v) recovers each channel's
// rounding error exactly, and the errors go to the compensation pixel
NB_D void film_add3(float4* sum, float4* comp, const float3& v) {
    const float4 old = atomicAdd(sum, make_float4(v.x, v.y, v.z, 0.0f));
    const float4 err = make_float4(two_sum_err(old.x, v.x), two_sum_err(old.y, v.y), two_sum_err(old.z, v.z), 0.0f);
    if (err.x != 0.0f || err.y != 0.0f || err.z != 0.0f) atomicAdd(comp, err);
}

NB_D int frame_of(const WfDev& W, unsigned long long k) {
    int lo = 0, hi = (int)W.nframes - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (W.frames[mid].base <= k)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

NB_D uint32_t lanes_below() { return (1u << (threadIdx.x & 31)) - 1u; }

// pixel of the q-th camera ray of a sample: 8x4 tiles in row-major tile
// order, row-major inside a tile, so that the 32 lanes of a warp trace a
// compact bundle; pixels outside the whole tiles follow row by row (the
// right strip, then the bottom rows)
NB_D uint32_t tile_pixel(uint32_t q, uint32_t w, uint32_t h) {
    const uint32_t w8 = w & ~7u, h4 = h & ~3u;
    const uint32_t full = w8 * h4;
    if (q < full) {
        const uint32_t t = q >> 5, r = q & 31u;
        const uint32_t tx = t % (w8 >> 3), ty = t / (w8 >> 3);
        return (ty * 4u + (r >> 3)) * w + tx * 8u + (r & 7u);
    }
    q -= full;
    const uint32_t rw = w - w8;
    if (q < rw * h4) return (q / rw) * w + w8 + q % rw;
    q -= rw * h4;
    return (h4 + q / w) * w + q % w;
}

NB_D void store_diff(const WfDev& W, uint32_t slot, const RayDiff& r) {
    W.diff[4 * slot] = make_float4(r.odx.x, r.odx.y, r.odx.z, r.on ? 1.0f : 0.0f);
    W.diff[4 * slot + 1] = make_float4(r.ody.x, r.ody.y, r.ody.z, 0.0f);
    W.diff[4 * slot + 2] = make_float4(r.ddx.x, r.ddx.y, r.ddx.z, 0.0f);
    W.diff[4 * slot + 3] = make_float4(r.ddy.x, r.ddy.y, r.ddy.z, 0.0f);
}
NB_D RayDiff load_diff(const WfDev& W, uint32_t slot) {
    const float4 a = W.diff[4 * slot], b = W.diff[4 * slot + 1], c = W.diff[4 * slot + 2], e = W.diff[4 * slot + 3];
    RayDiff r;
    r.on = a.w != 0.0f;
    r.odx = f3(a.x, a.y, a.z);
    r.ody = f3(b.x, b.y, b.z);
    r.ddx = f3(c.x, c.y, c.z);
    r.ddy = f3(e.x, e.y, e.z);
    return r;
}

// Regen (every slot): fold the last shade step's direct lighting into L; add
// the sky term of paths whose last ray escaped, and add finished paths to
// their frame's film (one float4 atomic per path, TwoSum-compensated);
// refill free slots with the camera
// rays of the next work items.  The block takes its work items with one
// atomic, in lane order (consecutive lanes: consecutive pixels of one 8x4
// tile), and adds its active slots to the active count with one atomic.
// DIFF: some scene of the batch has bump maps (camera rays with differentials)
template <bool DIFF>
__global__ void __launch_bounds__(kRegenBlock) wf_regen(WfDev W) {
    __shared__ uint32_t warp_off[kRegenBlock / 32];
    __shared__ unsigned long long block_base;
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = slot < W.cap;
    uint32_t st = kFree;
    bool cont = false;  // a continuing path: shade gave its next ray a bucket
    if (valid) {
        st = W.state[slot];
        cont = (st & kLifeMask) == kActive;
        float4 Lw;
        if (st & kPend) {
            // L += beta * (c0' + c1') with c' = c if its shadow ray was
            // unblocked, as the megakernel adds its direct lighting
            const float4 p0 = W.pend[2 * slot], p1 = W.pend[2 * slot + 1];
            Lw = W.L[slot];
            float3 Ld = f3(0.0f);
            if (p0.w != 0.0f) Ld += f3(p0.x, p0.y, p0.z);
            if (p1.w != 0.0f) Ld += f3(p1.x, p1.y, p1.z);
            const float4 b = W.pbeta[slot];
            const float3 c = f3(b.x, b.y, b.z) * Ld;
            Lw.x += c.x;
            Lw.y += c.y;
            Lw.z += c.z;
            if ((st & kLifeMask) == kActive) W.L[slot] = Lw;
        }
        if ((st & kLifeMask) == kFinishing) {
            if (!(st & kPend)) Lw = W.L[slot];
            const uint32_t fi = fbits(W.o[slot].w);
            const uint32_t pix = fbits(W.d[slot].w);
            const WfFrameDev& F = W.frames[fi];
            if (st & kSkySeen) {
                const float4 bw = W.beta[slot], dw = W.d[slot];
                const float3 c = f3(bw.x, bw.y, bw.z) * env_eval<true>(W.scenes[F.scene], normalize_fast(f3(dw.x, dw.y, dw.z)));
                Lw.x += c.x;
                Lw.y += c.y;
                Lw.z += c.z;
            }
            film_add3(F.sum + pix, F.comp + pix, clamp3(f3(Lw.x, Lw.y, Lw.z), 0.0f, 100.0f));
            st = kFree;
        }
        st &= kLifeMask;
    }
    const bool need = valid && st == kFree;
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint32_t ball = __ballot_sync(0xFFFFFFFFu, need);
    if (lane == 0) warp_off[wid] = __popc(ball);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t tot = 0;
        for (int w = 0; w < kRegenBlock / 32; ++w) {
            const uint32_t c = warp_off[w];
            warp_off[w] = tot;
            tot += c;
        }
        block_base = tot ? atomicAdd(W.work_next, (unsigned long long)tot) : 0ull;
    }
    __syncthreads();
    if (need) {
        const unsigned long long k = block_base + warp_off[wid] + __popc(ball & lanes_below());
        if (k < W.total) {
            const int fi = frame_of(W, k);
            const WfFrameDev& F = W.frames[fi];
            // all samples of a pixel are consecutive work items (pixels in
            // 8x4 tile order): the lanes of a warp trace up to 32 camera rays
            // through one pixel, which differ only by their sub-pixel jitter
            const unsigned long long local = k - F.base;
            const uint32_t sample = (uint32_t)(local % F.spp);
            const uint32_t pix = tile_pixel((uint32_t)(local / F.spp), F.cam.w, F.cam.h);
            Rng rng{tea16(pix, F.first_frame + sample)};
            float3 o, d;
            if (DIFF) {
                // a batch with bump maps: camera rays carry differentials
                // where their scene has bump maps
                RayDiff rd{};
                if (W.scenes[F.scene].has_bump)
                    camera_ray_diff(F.cam, pix % F.cam.w, pix / F.cam.w, rng, o, d, rd);
                else
                    camera_ray(F.cam, pix % F.cam.w, pix / F.cam.w, rng, o, d);
                store_diff(W, slot, rd);
            } else {
                camera_ray(F.cam, pix % F.cam.w, pix / F.cam.w, rng, o, d);
            }
            W.o[slot] = make_float4(o.x, o.y, o.z, bitsf((uint32_t)fi));
            W.d[slot] = make_float4(d.x, d.y, d.z, bitsf(pix));
            W.beta[slot] = make_float4(1.0f, 1.0f, 1.0f, bitsf(0u));
            W.L[slot] = make_float4(0.0f, 0.0f, 0.0f, bitsf(rng.s));
            st = kActive;
            // sort level 2: the camera rays in work-item order
            if (W.level >= 2) W.ext_perm[(uint32_t)(k - W.work_next[1])] = slot;
        }
    }
    if (valid && !cont && W.level >= 2) W.ext_key[slot] = 0xFFFFFFFFu;
    if (valid) W.state[slot] = st;
    const int nact = __syncthreads_count(valid && st == kActive);
    if (threadIdx.x == 0 && nact) atomicAdd(W.counters + kCntActive, (uint32_t)nact);
}

// bucket of a ray: direction octant, then the Morton code of its origin's
// cell in a 16^3 grid over the scene's root box
NB_D uint32_t spread3(uint32_t v) {
    v = (v | (v << 8)) & 0x0F00Fu;
    v = (v | (v << 4)) & 0xC30C3u;
    v = (v | (v << 2)) & 0x49249u;
    return v;
}
NB_D uint32_t ray_bucket(const DevScene& S, const float3& o, const float3& d) {
    const DevNode* r = S.nodes + S.root;
    const uint4 lo = __ldg(&r->lo), hi = __ldg(&r->hi);
    const float n = (float)(1 << kCellBits);
    auto cell = [&](float p, uint32_t a, uint32_t b) {
        const float l = __uint_as_float(a), h = __uint_as_float(b);
        const int c = (int)((p - l) / fmaxf(h - l, 1e-30f) * n);
        return (uint32_t)min(max(c, 0), (1 << kCellBits) - 1);
    };
    const uint32_t m = spread3(cell(o.x, lo.x, hi.x)) | (spread3(cell(o.y, lo.y, hi.y)) << 1) |
                       (spread3(cell(o.z, lo.z, hi.z)) << 2);
    const uint32_t oct = (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
    return (oct << (3 * kCellBits)) | m;
}

// warp-aggregated atomicAdd of 1 on counters[key]: lanes with the same key
// share one atomic; returns this lane's old value + its rank among them
NB_D uint32_t bucket_add(uint32_t* counters, uint32_t key) {
    const uint32_t active = __activemask();
    const uint32_t peers = __match_any_sync(active, key);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counters + key, (uint32_t)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    return base + __popc(peers & ((1u << lane) - 1u));
}

// exclusive scan of the bucket sizes into offsets (one block); the sizes
// are cleared for the next pass
__global__ void __launch_bounds__(kScanThreads) wf_bucket_scan(uint32_t* cnt, uint32_t* off) {
    constexpr int per = kBuckets / kScanThreads;
    __shared__ uint32_t part[kScanThreads];
    const int t = threadIdx.x;
    uint32_t v[per];
    uint32_t sum = 0;
    for (int k = 0; k < per; ++k) {
        v[k] = cnt[t * per + k];
        cnt[t * per + k] = 0u;
        sum += v[k];
    }
    part[t] = sum;
    __syncthreads();
    for (int off = 1; off < kScanThreads; off <<= 1) {
        const uint32_t add = t >= off ? part[t - off] : 0u;
        __syncthreads();
        part[t] += add;
        __syncthreads();
    }
    uint32_t run = part[t] - sum;
    for (int k = 0; k < per; ++k) {
        off[t * per + k] = run;
        run += v[k];
    }
}

template <int ISECT, bool EXT, bool WIDE>
NB_D void extend_one(const WfDev& W, const DevScene& S, uint32_t slot, const float4& ow,
                     const SmemStack& stk) {
    const float4 dw = W.d[slot], bw = W.beta[slot];
    const float3 o = f3(ow.x, ow.y, ow.z), d = f3(dw.x, dw.y, dw.z);
    const uint32_t bb = fbits(bw.w);
    const uint32_t bounce = bb & 0xFFFFu;
    const bool spec = (bb >> 16) & 1u;
    float tmax = kInf;
    HitRec rec{0.0f, 0.0f, 0u, 0u, 0u};
    const bool hit = trace_primary<ISECT, EXT, WIDE>(S, o, d, tmax, rec, stk, W.status);
    const float3 beta = f3(bw.x, bw.y, bw.z);
    if (!hit) {
        // the sky term is added by regen (converged lanes), after the
        // direct light regen folded before this extension, as the megakernel
        W.state[slot] = kFinishing | (S.sky_on && (bounce == 0 || spec) ? kSkySeen : 0u);
        return;
    }
    if (rec.mtype & kEmitterMat) {
        if (bounce == 0 || spec) {
            float3 c;
            if (rec.mtype & NOOR_MESHLIGHT) {
                c = beta * area_le<EXT>(S.area_lights[rec.ins], d);
            } else {
                const uint32_t mi = ISECT == NOOR_ISECT_WATERTIGHT ? __ldg(&S.wtri[rec.tri].attr).w
                                                                   : __ldg(&S.wald[rec.tri].attr).w;
                DevMaterial em = S.materials[mi];
                // an emitter's texture is read at the hit's barycentrics
                if (EXT && S.has_tex && em.tex_mask) apply_textures(S, mi, f2(rec.u, rec.v), em);
                c = beta * (em.emitter_scale * em.emittance);
            }
            float4 Lw = W.L[slot];
            W.L[slot] = make_float4(Lw.x + c.x, Lw.y + c.y, Lw.z + c.z, Lw.w);
        }
        W.state[slot] = kFinishing;
        return;
    }
    W.hit[slot] = make_float4(tmax, rec.u, rec.v, bitsf(rec.tri));
    W.hit2[slot] = make_uint2(rec.ins, rec.mtype);
    const uint32_t lobe = lobe_of(rec.mtype);
    const uint32_t kind = W.sort ? shade_kind(lobe) : 0u;
    W.state[slot] = kActive | ((kind + 1u) << kKindShift);  // wf_bin queues it for shading
}

// Sort level 2: the extension order.  Regen lists the camera rays it makes
// in work-item order (consecutive pixels stay together); shade gives each
// continuing path's next ray its bucket and counts it.  After
// wf_bucket_scan, wf_ext_scatter places the secondary rays at cap + their
// position in bucket order.
__global__ void __launch_bounds__(kBinBlock) wf_ext_scatter(WfDev W) {
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= W.cap) return;
    const uint32_t key = W.ext_key[slot];
    if (key != 0xFFFFFFFFu) W.ext_perm[W.cap + bucket_add(W.bkt_off, key)] = slot;
}

// The traversal kernels are instantiated per intersector and per scene
// source: with MULTI false every frame of the launch uses the scene passed as
// the kernel parameter S1 (read from the constant bank); with MULTI true each
// slot's scene comes from its frame, and ISECT may be kIsectMixed (the
// intersector read from that scene).
constexpr int kIsectMixed = -1;

template <int ISECT, bool MULTI>
NB_D const DevScene& slot_scene(const WfDev& W, const DevScene& S1, uint32_t frame) {
    if (!MULTI) return S1;
    return W.scenes[W.frames[frame].scene];
}

// Extend: closest hit for every active slot (one thread per slot).  EXT
// false: no scene of the launch has sphere or disk lights
template <int ISECT, bool MULTI, bool EXT, bool WIDE>
NB_D void extend_slot(const WfDev& W, const DevScene& S1, uint32_t slot, const SmemStack& stk) {
    const float4 ow = W.o[slot];
    const DevScene& S = slot_scene<ISECT, MULTI>(W, S1, fbits(ow.w));
    if (ISECT == kIsectMixed) {
        if (S.isect == NOOR_ISECT_WATERTIGHT)
            extend_one<NOOR_ISECT_WATERTIGHT, EXT, WIDE>(W, S, slot, ow, stk);
        else
            extend_one<NOOR_ISECT_REF_WALD, EXT, WIDE>(W, S, slot, ow, stk);
    } else {
        extend_one<ISECT == kIsectMixed ? 0 : ISECT, EXT, WIDE>(W, S, slot, ow, stk);
    }
}

// Extend.  Below sort level 2 one thread per slot; from level 2 each warp
// takes the next 32 entries of the extension order (camera rays, then
// secondary rays by bucket) when it is done with its last ones.
template <int ISECT, bool MULTI, bool EXT, bool WIDE>
__global__ void __launch_bounds__(NB_TRAV_THREADS, WIDE ? NB_TRAV_MIN_BLOCKS_WIDE : NB_TRAV_MIN_BLOCKS) wf_extend(WfDev W, DevScene S1) {
    extern __shared__ uint32_t smem[];
    SmemStack stk{smem + threadIdx.x, (int)blockDim.x, W.stack_cap};
    if (W.level >= 2) {
        // camera rays: the work items regen took this iteration
        const unsigned long long wn = W.work_next[0] < W.total ? W.work_next[0] : W.total;
        const uint32_t nc = (uint32_t)(wn - W.work_next[1]), n = W.counters[kCntActive];
        const uint32_t lane = threadIdx.x & 31;
        for (;;) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(W.counters + kCntTakeExt, 32u);
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            if (base >= n) break;
            const uint32_t i = base + lane;
            if (i >= n) continue;
            extend_slot<ISECT, MULTI, EXT, WIDE>(W, S1, i < nc ? W.ext_perm[i] : W.ext_perm[W.cap + (i - nc)], stk);
        }
        return;
    }
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= W.cap || W.state[slot] != kActive) return;
    extend_slot<ISECT, MULTI, EXT, WIDE>(W, S1, slot, stk);
}

// Shading queues in slot order: every slot extend left a surface hit goes to
// the queue of its material kind (one block-wide atomic per kind), so that
// shade reads the slots' state in nearly ascending order.
__global__ void __launch_bounds__(kBinBlock) wf_bin(WfDev W) {
    __shared__ uint32_t cnt[kKinds][kBinBlock / 32];
    __shared__ uint32_t base[kKinds];
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t kq = slot < W.cap ? (W.state[slot] >> kKindShift) & 3u : 0u;  // 1 + kind, 0: none
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t mine = 0;
    for (uint32_t k = 0; k < (uint32_t)kKinds; ++k) {
        const uint32_t b = __ballot_sync(0xFFFFFFFFu, kq == k + 1u);
        if (kq == k + 1u) mine = __popc(b & lanes_below());
        if (lane == 0) cnt[k][wid] = __popc(b);
    }
    __syncthreads();
    if (threadIdx.x < (uint32_t)kKinds) {
        const uint32_t k = threadIdx.x;
        uint32_t tot = 0;
        for (int w = 0; w < kBinBlock / 32; ++w) {
            const uint32_t c = cnt[k][w];
            cnt[k][w] = tot;
            tot += c;
        }
        base[k] = tot ? atomicAdd(W.counters + k, tot) : 0u;
    }
    __syncthreads();
    if (kq) {
        const uint32_t k = kq - 1u;
        W.qshade[k * W.cap + base[k] + cnt[k][wid] + mine] = slot;
    }
}

// queues shadow ray `which` (0: light sample, 1: BSDF sample of MIS) of a slot
NB_D void push_shadow(const WfDev& W, const DevScene& S, uint32_t slot, uint32_t which, const ShadowRay& sr) {
    const uint32_t i = queue_push(W.counters + kCntShadow);
    W.qshadow[i] = (slot << 1) | which;
    W.sh_o[i] = make_float4(sr.o.x, sr.o.y, sr.o.z, sr.tmax);
    W.sh_d[i] = make_float4(sr.d.x, sr.d.y, sr.d.z, 0.0f);
    if (W.level >= 3) {
        // sort level 3: the shadow ray's bucket, counted here
        const uint32_t key = ray_bucket(S, sr.o, sr.d);
        W.sh_key[i] = key;
        bucket_add(W.sh_bkt_cnt, key);
    }
}

// EXT false: the queue holds no material with a lobe beyond Lambert,
// conductor and Fresnel specular (those lobes' code is left out).  DIFF:
// some scene has bump maps; its rays' differentials are read, used and
// passed on as the megakernel's DIFF specialisation does.
// MULTI false: every frame of the launch uses scene S1 (a kernel parameter,
// read through the constant cache instead of the scene table)
// BLOCKS: resident 256-thread blocks per SM the kernel is built for (3: 80
// registers, 2: 128, no spills; the launch parameters choose)
template <bool EXT, bool DIFF = false, bool MULTI = true, int BLOCKS = NB_SHADE_MIN_BLOCKS>
__global__ void __launch_bounds__(256, BLOCKS) wf_shade(WfDev W, DevScene S1, uint32_t kind) {
    const uint32_t n = W.counters[kind];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t slot = W.qshade[kind * W.cap + i];
        const float4 ow = W.o[slot], dw = W.d[slot], bw = W.beta[slot], Lw = W.L[slot];  // Lw.w: RNG state
        const float4 hw = W.hit[slot];
        const uint2 h2 = W.hit2[slot];
        const uint32_t fi = fbits(ow.w);
        const WfFrameDev& F = W.frames[fi];
        const DevScene& S = MULTI ? W.scenes[F.scene] : S1;
        const float3 o = f3(ow.x, ow.y, ow.z), d = f3(dw.x, dw.y, dw.z);
        float3 beta = f3(bw.x, bw.y, bw.z);
        const uint32_t bb = fbits(bw.w);
        const uint32_t bounce = bb & 0xFFFFu;
        HitRec rec;
        rec.u = hw.y;
        rec.v = hw.z;
        rec.tri = fbits(hw.w);
        rec.ins = h2.x;
        rec.mtype = h2.y;
        Isect I;
        TangentOut to;
        const bool tex = EXT && S.has_tex;
        if (S.isect == NOOR_ISECT_WATERTIGHT)
            make_isect<NOOR_ISECT_WATERTIGHT, EXT>(S, o, d, hw.x, rec, I, tex ? &to : nullptr);
        else
            make_isect<NOOR_ISECT_REF_WALD, EXT>(S, o, d, hw.x, rec, I, tex ? &to : nullptr);
        DevMaterial m = S.materials[I.mat];
        RayDiff rd{};
        HitDiff hd;
        if (DIFF && S.has_bump) {
            rd = load_diff(W, slot);
            if (rd.on) {
                hd = hit_differential(I, to, rd);
                if (I.mtype & NOOR_BUMP) bump(S, I.mat, I.uv, hd, I.F);
            }
        }
        if (tex && m.tex_mask) apply_textures(S, I.mat, I.uv, m);
        Rng rng{fbits(Lw.w)};
        int li = 0;
        bool picked;
        ShadowRay sr;
        // direct lighting: up to two contributions, each counted only if its
        // shadow ray comes back unblocked; the next regen adds
        // beta * (c0' + c1') to L as the megakernel does
        const float3 c0 = light_sample_contrib<EXT>(S, m, I, rng, S.mis != 0, li, picked, sr);
        const bool has0 = !is_black(c0);
        if (has0) push_shadow(W, S, slot, 0, sr);
        float3 c1 = f3(0.0f);
        bool has1 = false;
        if (S.mis && picked) {
            c1 = bsdf_mis_contrib<EXT>(S, m, I, rng, li, sr);
            has1 = !is_black(c1);
            if (has1) push_shadow(W, S, slot, 1, sr);
        }
        const bool pend = has0 || has1;
        if (pend) {
            W.pend[2 * slot] = has0 ? make_float4(c0.x, c0.y, c0.z, 1.0f) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            W.pend[2 * slot + 1] = has1 ? make_float4(c1.x, c1.y, c1.z, 1.0f) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            W.pbeta[slot] = make_float4(beta.x, beta.y, beta.z, 0.0f);
        }
        // scatter, sidedness, Russian roulette, next ray
        rng.next();
        rng.next();
        float3 wi;
        float pdf;
        uint32_t stype;
        const float3 f = bsdf_sample<EXT>(I.lobe, m, I.F, I.wo, BSDF_ALL, rng, wi, pdf, stype);
        uint32_t st = kActive;
        if (pdf == 0.0f) {
            st = kFinishing;
        } else {
            beta *= (is_catcher<EXT>(I) ? f * catcher_sky<EXT>(S, I) : f) * absdot(wi, I.F.n) / pdf;
            if (!(I.mtype & kTransparentMat) && dot(wi, I.F.ng) < 0.0f) {
                st = kFinishing;
            } else if (bounce >= S.rr) {
                const float q = fmaxf(0.05f, 1.0f - maxcomp(beta));
                if (rng.next() < q)
                    st = kFinishing;
                else
                    beta /= 1.0f - q;
            }
        }
        if (st == kActive) {
            const bool spec = (I.mtype & kSpecularMat) != 0;
            const uint32_t nb_ = bounce + 1;
            const float3 no = spawn_origin(I, wi, S.bias);
            if (DIFF && S.has_bump) {
                RayDiff nd{};
                if (rd.on && (I.mtype & kGlossyMat))
                    nd = spawn_diff(I, hd, rd, no, wi, (I.mtype & kDielectricMat) ? m.coat_ior : 1.0f);
                store_diff(W, slot, nd);
            }
            W.o[slot] = make_float4(no.x, no.y, no.z, ow.w);
            W.d[slot] = make_float4(wi.x, wi.y, wi.z, dw.w);
            W.beta[slot] = make_float4(beta.x, beta.y, beta.z, bitsf(nb_ | (spec ? 1u << 16 : 0u)));
            if (nb_ >= F.bounces) {
                st = kFinishing;
            } else if (W.level >= 2) {
                // the next extension's order: the ray's bucket, counted here
                const uint32_t key = ray_bucket(S, no, wi);
                W.ext_key[slot] = key;
                bucket_add(W.bkt_cnt, key);
            }
        }
        W.L[slot] = make_float4(Lw.x, Lw.y, Lw.z, bitsf(rng.s));
        W.state[slot] = st | (pend ? kPend : 0u);
    }
}

// Sort level 3: shade gave every shadow queue entry its bucket and counted
// it; after wf_bucket_scan, each entry's place in bucket order (grid-stride
// over the queue length the shade stage left).
__global__ void wf_shadow_scatter(WfDev W) {
    const uint32_t n = W.counters[kCntShadow];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        W.sh_perm[bucket_add(W.sh_bkt_off, W.sh_key[i])] = i;
}

// Any hit for each queued shadow ray; a blocked one cancels its pending
// contribution.  Each warp takes the next 32 queue entries when it is done
// with its last ones, so warps that drew long rays do not hold up the launch
// with a fixed share of the queue.
template <int ISECT, bool MULTI, bool EXT, bool WIDE>
__global__ void __launch_bounds__(NB_TRAV_THREADS, WIDE ? NB_TRAV_MIN_BLOCKS_WIDE : NB_TRAV_MIN_BLOCKS) wf_shadow(WfDev W, DevScene S1) {
    extern __shared__ uint32_t smem[];
    const uint32_t n = W.counters[kCntShadow];
    SmemStack stk{smem + threadIdx.x, (int)blockDim.x, W.stack_cap};

#if NB_SHADOW_FETCH
    const uint32_t lane = threadIdx.x & 31;
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(W.counters + kCntTake, 32u);
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (base >= n) break;
        const uint32_t i = base + lane;
        if (i >= n) continue;
#else
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#endif
        const uint32_t q = W.level >= 3 ? W.sh_perm[i] : i;
        const uint32_t e = W.qshadow[q];
        const uint32_t slot = e >> 1;
        const float4 so = W.sh_o[q], sd = W.sh_d[q];
        const DevScene& S = slot_scene<ISECT, MULTI>(W, S1, MULTI ? fbits(W.o[slot].w) : 0u);
        const float3 o = f3(so.x, so.y, so.z), d = f3(sd.x, sd.y, sd.z);
        bool occ;
        if (ISECT == kIsectMixed) {
            if (S.isect == NOOR_ISECT_WATERTIGHT)
                occ = trace_shadow<NOOR_ISECT_WATERTIGHT, EXT, WIDE>(S, o, d, so.w, stk, W.status);
            else
                occ = trace_shadow<NOOR_ISECT_REF_WALD, EXT, WIDE>(S, o, d, so.w, stk, W.status);
        } else {
            occ = trace_shadow<ISECT == kIsectMixed ? 0 : ISECT, EXT, WIDE>(S, o, d, so.w, stk, W.status);
        }
        if (occ) W.pend[e].w = 0.0f;
    }
}

// End of an iteration: count the rays traced (extend traced every active
// slot), stop when regen found no slot holding a path (bounded by an
// iteration cap), reset the per-iteration counters.
__global__ void wf_check(WfDev W, uint32_t* go_out, uint32_t conditional) {
    uint32_t* c = W.counters;
    const uint32_t active = c[kCntActive];
    W.rays[0] += active;
    W.rays[1] += c[kCntShadow];
    const uint32_t it = ++c[kCntIter];
    bool go = active > 0u;
    if (go && it >= W.max_iters) {
        atomicOr(W.status, NOOR_DEV_WAIT_TIMEOUT);
        go = false;
    }
    if (!go) W.rays[2] += *W.work_next < W.total ? *W.work_next : W.total;
    W.work_next[1] = W.work_next[0] < W.total ? W.work_next[0] : W.total;
    for (int k = 0; k <= kCntActive; ++k) c[k] = 0u;
    c[kCntTake] = 0u;
    c[kCntTakeExt] = 0u;
    if (conditional)
        cudaGraphSetConditional(W.cond, go ? 1u : 0u);
    else
        *go_out = go ? 1u : 0u;
}

// mean = (sum + comp) / spp into the caller's film
__global__ void wf_resolve(const WfFrameDev* frames, uint32_t fi) {
    const WfFrameDev& F = frames[fi];
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= F.npix || !F.out) return;
    const float4 s = F.sum[p], c = F.comp[p];
    const float inv = 1.0f / (float)F.spp;
    reinterpret_cast<float4*>(F.out)[p] = make_float4((s.x + c.x) * inv, (s.y + c.y) * inv, (s.z + c.z) * inv, 1.0f);
}

// ------------------------------------------------------------------ host
struct WavefrontState {
    uint32_t cap = 0;
    std::vector<void*> bufs;
    WfDev dev{};
    float4* diff = nullptr;     // ray differentials, made for the first batch with bump maps
    uint32_t* active_host_dev = nullptr;
    // film scratch per frame batch
    void* films = nullptr;
    size_t films_bytes = 0;
    WfFrameDev* frames_dev = nullptr;
    size_t frames_cap = 0;
    DevScene* scenes_dev = nullptr;
    size_t scenes_cap = 0;
    // the instantiated while-loop graph of the last render, reused while the
    // launch (slot buffers, sizes, parameters) is the same
    cudaGraphExec_t exec = nullptr;
    uint64_t graph_key[10] = {};
    ~WavefrontState() {
        if (exec) cudaGraphExecDestroy(exec);
        for (void* p : bufs) cudaFree(p);
        if (films) cudaFree(films);
        if (frames_dev) cudaFree(frames_dev);
        if (scenes_dev) cudaFree(scenes_dev);
        if (active_host_dev) cudaFree(active_host_dev);
        if (diff) cudaFree(diff);
    }
};

void wavefront_release(Context& C) {
    delete C.wf;
    C.wf = nullptr;
}

static int wf_alloc(WavefrontState& S, void** p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) return cuda_fail(e, "wavefront buffers");
    S.bufs.push_back(*p);
    return NOOR_OK;
}

static int wf_ensure(Context& C, uint32_t cap) {
    if (C.wf && C.wf->cap >= cap) return NOOR_OK;
    delete C.wf;
    C.wf = new WavefrontState();
    WavefrontState& S = *C.wf;
    WfDev& W = S.dev;
    int rc;
    const size_t n = cap;
    if ((rc = wf_alloc(S, (void**)&W.o, n * 16)) || (rc = wf_alloc(S, (void**)&W.d, n * 16)) ||
        (rc = wf_alloc(S, (void**)&W.beta, n * 16)) || (rc = wf_alloc(S, (void**)&W.L, n * 16)) ||
        (rc = wf_alloc(S, (void**)&W.pend, 2 * n * 16)) || (rc = wf_alloc(S, (void**)&W.pbeta, n * 16)) ||
        (rc = wf_alloc(S, (void**)&W.hit, n * 16)) ||
        (rc = wf_alloc(S, (void**)&W.hit2, n * 8)) || (rc = wf_alloc(S, (void**)&W.state, n * 4)) ||
        (rc = wf_alloc(S, (void**)&W.qshade, kKinds * n * 4)) || (rc = wf_alloc(S, (void**)&W.qshadow, 2 * n * 4)) ||
        (rc = wf_alloc(S, (void**)&W.sh_o, 2 * n * 16)) || (rc = wf_alloc(S, (void**)&W.sh_d, 2 * n * 16)) ||
        (rc = wf_alloc(S, (void**)&W.counters, kCntWords * 4)) || (rc = wf_alloc(S, (void**)&W.work_next, 16)) ||
        (rc = wf_alloc(S, (void**)&W.rays, 32)) || (rc = wf_alloc(S, (void**)&W.bkt_cnt, kBuckets * 4)) ||
        (rc = wf_alloc(S, (void**)&W.bkt_off, kBuckets * 4)) || (rc = wf_alloc(S, (void**)&W.sh_key, 2 * n * 4)) ||
        (rc = wf_alloc(S, (void**)&W.sh_bkt_cnt, kBuckets * 4)) || (rc = wf_alloc(S, (void**)&W.sh_bkt_off, kBuckets * 4)) ||
        (rc = wf_alloc(S, (void**)&W.sh_perm, 2 * n * 4)) || (rc = wf_alloc(S, (void**)&W.ext_key, n * 4)) ||
        (rc = wf_alloc(S, (void**)&W.ext_perm, 2 * n * 4)))
        return rc;
    cudaError_t e = cudaMalloc((void**)&S.active_host_dev, 16);
    if (e == cudaSuccess) e = cudaMemset(W.rays, 0, 32);
    if (e == cudaSuccess) e = cudaMemset(W.bkt_cnt, 0, kBuckets * 4);
    if (e == cudaSuccess) e = cudaMemset(W.sh_bkt_cnt, 0, kBuckets * 4);
    if (e != cudaSuccess) return cuda_fail(e, "wavefront buffers");
    S.cap = cap;
    return NOOR_OK;
}

using WfTravKernel = void (*)(WfDev, DevScene);

struct WfLaunch {
    int block;
    uint32_t kinds;      // shading queues some scene of the launch can fill
    size_t smem;
    uint32_t grid_slots;    // one thread per slot / queue entry
    uint32_t grid_queue;    // grid-stride stages
    WfTravKernel extend;
    WfTravKernel shadow;
    DevScene scene;         // the launch's scene when every frame uses the same one
    bool ext;               // some frame's scene has extra lobes or lights
    bool ext_lights;        // ... has sphere, disk, point, spot or distant lights
    bool env_ref;           // ... samples its environment as the reference does
    bool tex;               // ... reads textures per hit (image maps, alpha, bump)
    bool diff;              // ... has bump maps: rays carry differentials
    bool multi;             // the frames use more than one scene
    bool shade_wide_regs;   // single-scene shade built for 128 registers
};

// NOOR_TRAVERSAL_AUTO takes the four-wide tree for the shadow rays of scenes
// of at least this many triangles (on the 36-triangle room the binary tree's
// single-box visits are cheaper; on the 2.6M-triangle sky scene shadow rays
// take 11.3 ms per step on the wide tree against 11.7, extension rays 50.2
// against 48.6, so the extension stage keeps the binary tree)
constexpr uint32_t kWideAutoTris = 16384;

// shading launches per iteration: one per queue some scene can fill
static uint32_t shade_launches(const WfDev& W, const WfLaunch& L) {
    return W.sort ? (uint32_t)__builtin_popcount(L.kinds & ((1u << kKinds) - 1u)) : 1u;
}

// one iteration; with `ev` (kWfStages + 1 events), records ev[0] before the
// first stage and ev[k + 1] after stage k (regen, extension ordering,
// extend, shade with its queue binning, shadow ordering, shadow, stop test)
static cudaError_t wf_iteration(const WfDev& W, const WfLaunch& L, cudaStream_t s, bool conditional,
                                uint32_t* go_out, cudaEvent_t* ev = nullptr) {
    if (ev) cudaEventRecord(ev[0], s);
    if (L.diff)
        wf_regen<true><<<(W.cap + kRegenBlock - 1) / kRegenBlock, kRegenBlock, 0, s>>>(W);
    else
        wf_regen<false><<<(W.cap + kRegenBlock - 1) / kRegenBlock, kRegenBlock, 0, s>>>(W);
    if (ev) cudaEventRecord(ev[1], s);
    if (W.level >= 2) {
        // secondary rays in bucket order (shade counted the buckets); camera
        // rays were listed by regen
        wf_bucket_scan<<<1, kScanThreads, 0, s>>>(W.bkt_cnt, W.bkt_off);
        wf_ext_scatter<<<(W.cap + kBinBlock - 1) / kBinBlock, kBinBlock, 0, s>>>(W);
    }
    if (ev) cudaEventRecord(ev[2], s);
    if (W.level >= 2)
        L.extend<<<L.grid_queue, L.block, L.smem, s>>>(W, L.scene);
    else
        L.extend<<<L.grid_slots, L.block, L.smem, s>>>(W, L.scene);
    if (ev) cudaEventRecord(ev[3], s);
    wf_bin<<<(W.cap + kBinBlock - 1) / kBinBlock, kBinBlock, 0, s>>>(W);
    const int nk = W.sort ? kKinds : 1;
    for (int k = 0; k < nk; ++k) {
        // no launch for a queue no triangle of the launch's scenes can fill
        if (W.sort && !((L.kinds >> k) & 1u)) continue;
        // sorted queues 0 and 1 hold Lambert and conductor hits only
        if (L.diff)
            wf_shade<true, true><<<L.grid_queue, 256, 0, s>>>(W, L.scene, (uint32_t)k);
        else if (L.ext && !(W.sort && k < 2 && !L.ext_lights && !L.env_ref && !L.tex))
            wf_shade<true><<<L.grid_queue, 256, 0, s>>>(W, L.scene, (uint32_t)k);
        else if (L.multi)
            wf_shade<false><<<L.grid_queue, 256, 0, s>>>(W, L.scene, (uint32_t)k);
        else if (L.shade_wide_regs)
            wf_shade<false, false, false, 2><<<L.grid_queue, 256, 0, s>>>(W, L.scene, (uint32_t)k);
        else
            wf_shade<false, false, false><<<L.grid_queue, 256, 0, s>>>(W, L.scene, (uint32_t)k);
    }
    if (ev) cudaEventRecord(ev[4], s);
    if (W.level >= 3) {
        // shadow rays in bucket order (shade counted the buckets)
        wf_bucket_scan<<<1, kScanThreads, 0, s>>>(W.sh_bkt_cnt, W.sh_bkt_off);
        wf_shadow_scatter<<<L.grid_queue, 256, 0, s>>>(W);
    }
    if (ev) cudaEventRecord(ev[5], s);
    L.shadow<<<L.grid_queue, L.block, L.smem, s>>>(W, L.scene);
    if (ev) cudaEventRecord(ev[6], s);
    wf_check<<<1, 1, 0, s>>>(W, go_out, conditional ? 1u : 0u);
    if (ev) cudaEventRecord(ev[7], s);
    return cudaGetLastError();
}

// one batch render; returns device-timed ms through `ms` when non-null
int wavefront_render(Context& C, const noor_wf_frame* frames, uint32_t n_frames, const noor_wf_params& P,
                     float* ms_out, noor_wf_profile* prof = nullptr) {
    if (!frames || n_frames == 0) return set_error(NOOR_ERR_INVALID, "wavefront: no frames");
    const uint32_t block = P.block_size ? P.block_size : 128;
    if (block != 32 && block != 64 && block != 128 && block != 256)
        return set_error(NOOR_ERR_INVALID, "wavefront: block_size must be 32, 64, 128 or 256");
    if ((int)block > NB_TRAV_THREADS)
        return set_error(NOOR_ERR_INVALID, "wavefront: block_size above the traversal kernels' launch bound");
    const uint32_t cap = P.queue_capacity ? P.queue_capacity : (1u << 20);
    if (cap < 1024 || cap > (1u << 26)) return set_error(NOOR_ERR_INVALID, "wavefront: queue capacity out of range");
    int rc = wf_ensure(C, cap);
    if (rc) return rc;
    WavefrontState& WS = *C.wf;
    // frames and films
    std::vector<WfFrameDev> fr(n_frames);
    unsigned long long total = 0;
    size_t film_px = 0;
    int stack_cap = 16, stack_words = 16;
    uint32_t max_bounces = 1;
    for (uint32_t i = 0; i < n_frames; ++i) {
        const noor_wf_frame& f = frames[i];
        if (f.scene_id >= C.scenes.size()) return set_error(NOOR_ERR_INVALID, "wavefront: unknown scene id");
        if (f.width == 0 || f.height == 0 || f.spp == 0 || f.first_frame == 0 ||
            f.width != f.camera.w || f.height != f.camera.h)
            return set_error(NOOR_ERR_INVALID, "wavefront: bad frame description");
        if ((uint32_t)f.camera.type > NOOR_CAMERA_ENV) return set_error(NOOR_ERR_INVALID, "wavefront: bad camera type");
        std::memset(&fr[i], 0, sizeof(WfFrameDev));
        fr[i].cam = dev_camera(f.camera, f.width, f.height);
        fr[i].npix = f.width * f.height;
        fr[i].base = total;
        fr[i].count = (unsigned long long)fr[i].npix * f.spp;
        fr[i].scene = f.scene_id;
        fr[i].first_frame = f.first_frame;
        fr[i].bounces = f.bounces ? f.bounces : C.scenes[f.scene_id]->dev.bounces;
        fr[i].spp = f.spp;
        fr[i].out = f.d_film;
        total += fr[i].count;
        film_px += fr[i].npix;
        stack_cap = std::max(stack_cap, C.scenes[f.scene_id]->dev.stack_cap);
        stack_words = std::max(stack_words, C.scenes[f.scene_id]->dev.stack_words);
        max_bounces = std::max(max_bounces, fr[i].bounces);
    }
    const size_t film_bytes = film_px * 32;
    if (WS.films_bytes < film_bytes) {
        if (WS.films) cudaFree(WS.films);
        WS.films = nullptr;
        cudaError_t e = cudaMalloc(&WS.films, film_bytes);
        if (e != cudaSuccess) return cuda_fail(e, "wavefront films");
        WS.films_bytes = film_bytes;
    }
    {
        size_t off = 0;
        for (uint32_t i = 0; i < n_frames; ++i) {
            fr[i].sum = (float4*)((char*)WS.films + off);
            off += (size_t)fr[i].npix * 16;
            fr[i].comp = (float4*)((char*)WS.films + off);
            off += (size_t)fr[i].npix * 16;
        }
    }
    if (WS.frames_cap < n_frames) {
        if (WS.frames_dev) cudaFree(WS.frames_dev);
        cudaError_t e = cudaMalloc((void**)&WS.frames_dev, n_frames * sizeof(WfFrameDev));
        if (e != cudaSuccess) return cuda_fail(e, "wavefront frames");
        WS.frames_cap = n_frames;
    }
    if (WS.scenes_cap < C.scenes.size()) {
        if (WS.scenes_dev) cudaFree(WS.scenes_dev);
        cudaError_t e = cudaMalloc((void**)&WS.scenes_dev, C.scenes.size() * sizeof(DevScene));
        if (e != cudaSuccess) return cuda_fail(e, "wavefront scenes");
        WS.scenes_cap = C.scenes.size();
    }
    std::vector<DevScene> sc(C.scenes.size());
    for (size_t i = 0; i < sc.size(); ++i) sc[i] = C.scenes[i]->dev;
    cudaStream_t s = C.stream;
    cudaError_t e = cudaMemcpyAsync(WS.frames_dev, fr.data(), n_frames * sizeof(WfFrameDev), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(WS.scenes_dev, sc.data(), sc.size() * sizeof(DevScene), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(WS.films, 0, film_bytes, s);
    WfDev& W = WS.dev;
    if (e == cudaSuccess) e = cudaMemsetAsync(W.state, 0, (size_t)cap * 4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(W.counters, 0, kCntWords * 4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(W.work_next, 0, 16, s);
    // shade counts the next iteration's extension buckets: a render cut short
    // by the iteration cap can leave counts behind
    if (e == cudaSuccess) e = cudaMemsetAsync(W.bkt_cnt, 0, kBuckets * 4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(W.sh_bkt_cnt, 0, kBuckets * 4, s);
    if (e != cudaSuccess) return cuda_fail(e, "wavefront setup");
    W.status = C.status;
    W.frames = WS.frames_dev;
    W.scenes = WS.scenes_dev;
    W.nframes = n_frames;
    W.cap = cap;
    W.level = std::min<uint32_t>(P.sort_granularity, 3u);
    W.sort = W.level ? 1u : 0u;
    W.total = total;
    W.stack_cap = stack_cap;
    // every slot finishes within max_bounces iterations of starting; a slot
    // starts at least every iteration while work remains
    W.max_iters = (uint32_t)std::min<unsigned long long>(
        (total + cap - 1) / cap * (max_bounces + 2) + 4 * (max_bounces + 2) + 64, 1u << 30);
    if (P.max_iterations) W.max_iters = std::min(W.max_iters, P.max_iterations);

    WfLaunch L;
    L.block = (int)block;
    // room for the four-wide trees' stacks as well as the binary one's
    L.smem = (size_t)stack_words * block * 4;
    L.grid_slots = (cap + block - 1) / block;
    L.grid_queue = (uint32_t)std::max(1, C.sm_count) * 16;
    const uint32_t scene0 = frames[0].scene_id;
    bool multi = false, mixed = false;
    // the four-wide trees where every scene of the launch has them (and,
    // for NOOR_TRAVERSAL_AUTO, is large enough for them to pay)
    if (P.traversal > NOOR_TRAVERSAL_WIDE_SHADOW)
        return set_error(NOOR_ERR_INVALID, "wavefront: bad traversal selector");
    bool wide_c = P.traversal == NOOR_TRAVERSAL_WIDE, wide_a = P.traversal != NOOR_TRAVERSAL_BINARY;
    L.ext = L.ext_lights = L.env_ref = L.tex = L.diff = false;
    L.kinds = 0;
    for (uint32_t i = 0; i < n_frames; ++i) {
        const DevScene& fs = C.scenes[frames[i].scene_id]->dev;
        const bool big = P.traversal != NOOR_TRAVERSAL_AUTO || fs.num_tris >= kWideAutoTris;
        wide_c &= fs.closest4 != 0u && big;
        wide_a &= fs.nodes4 != nullptr && big;
        L.kinds |= fs.shade_kinds;
        multi |= frames[i].scene_id != scene0;
        mixed |= fs.isect != C.scenes[scene0]->dev.isect;
        L.ext |= fs.ext_lobes != 0u || fs.ext_lights != 0u || fs.env_ref != 0u || fs.has_tex != 0u;
        L.env_ref |= fs.env_ref != 0u;
        // the traversal kernels' full variant also tests alpha maps and reads
        // emitters' textures
        L.ext_lights |= fs.ext_lights != 0u || fs.has_tex != 0u;
        L.tex |= fs.has_tex != 0u;
        L.diff |= fs.has_bump != 0u;
    }
    if (L.diff && !WS.diff) {
        cudaError_t de = cudaMalloc((void**)&WS.diff, (size_t)WS.cap * 64);
        if (de != cudaSuccess) return cuda_fail(de, "wavefront differentials");
    }
    W.diff = L.diff ? WS.diff : nullptr;
    L.scene = C.scenes[scene0]->dev;
    // traversal kernels: per intersector, scene source and light shapes
#define NB_TRAV(I, M)                                                                                      \
    do {                                                                                                   \
        if (wide_c)                                                                                        \
            L.extend = L.ext_lights ? wf_extend<I, M, true, true> : wf_extend<I, M, false, true>;          \
        else                                                                                               \
            L.extend = L.ext_lights ? wf_extend<I, M, true, false> : wf_extend<I, M, false, false>;        \
        if (wide_a)                                                                                        \
            L.shadow = L.ext_lights ? wf_shadow<I, M, true, true> : wf_shadow<I, M, false, true>;          \
        else                                                                                               \
            L.shadow = L.ext_lights ? wf_shadow<I, M, true, false> : wf_shadow<I, M, false, false>;        \
    } while (0)
    if (mixed) {
        NB_TRAV(kIsectMixed, true);
    } else if (L.scene.isect == NOOR_ISECT_WATERTIGHT) {
        if (multi) NB_TRAV(NOOR_ISECT_WATERTIGHT, true);
        else NB_TRAV(NOOR_ISECT_WATERTIGHT, false);
    } else {
        if (multi) NB_TRAV(NOOR_ISECT_REF_WALD, true);
        else NB_TRAV(NOOR_ISECT_REF_WALD, false);
    }
#undef NB_TRAV
    L.multi = multi;
    if (P.shade_regs != 0 && P.shade_regs != 80 && P.shade_regs != 128)
        return set_error(NOOR_ERR_INVALID, "wavefront: shade_regs must be 0, 80 or 128");
    L.shade_wide_regs = P.shade_regs == 128;
    for (WfTravKernel k : {L.extend, L.shadow}) {
        e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.smem);
        if (e != cudaSuccess) return cuda_fail(e, "wavefront smem");
    }
    if (ms_out) cudaEventRecord(C.events[6], s);
    bool done = false;
    if (P.use_graph && !prof) {
        // everything the captured launches take as arguments, apart from the
        // conditional handle (the frame descriptions and the scene table are
        // read from device memory at run time; the single-scene kernels take
        // the scene by value, hashed here)
        uint64_t scene_hash = 1469598103934665603ull;  // FNV-1a over the scene parameter's bytes
        for (size_t b = 0; b < sizeof(DevScene); ++b)
            scene_hash = (scene_hash ^ reinterpret_cast<const unsigned char*>(&L.scene)[b]) * 1099511628211ull;
        const uint64_t key[10] = {(uint64_t)W.cap | (uint64_t)W.level << 32 | (uint64_t)L.ext << 36 |
                                      (uint64_t)L.tex << 37 | (uint64_t)L.diff << 38 | (uint64_t)L.ext_lights << 39 |
                                      (uint64_t)L.env_ref << 40 | (uint64_t)L.kinds << 41 |
                                      (uint64_t)L.shade_wide_regs << 44,
                                  W.total,
                                  (uint64_t)W.max_iters | (uint64_t)W.nframes << 32,
                                  (uint64_t)(uint32_t)W.stack_cap | (uint64_t)L.block << 32,
                                  (uint64_t)L.smem, (uint64_t)L.grid_slots | (uint64_t)L.grid_queue << 32,
                                  (uint64_t)(uintptr_t)W.frames ^ ((uint64_t)(uintptr_t)W.scenes << 1),
                                  (uint64_t)(uintptr_t)W.status ^ ((uint64_t)(uintptr_t)W.diff << 1),
                                  (uint64_t)(uintptr_t)L.extend ^ (uint64_t)(uintptr_t)L.shadow << 1,
                                  scene_hash};
        if (WS.exec && std::memcmp(key, WS.graph_key, sizeof(key)) != 0) {
            cudaGraphExecDestroy(WS.exec);
            WS.exec = nullptr;
        }
        if (!WS.exec) {
            cudaGraph_t graph = nullptr;
            e = cudaGraphCreate(&graph, 0);
            cudaGraphConditionalHandle h;
            if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault);
            cudaGraphNode_t node;
            cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
            cp.conditional.handle = h;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            if (e == cudaSuccess) e = cudaGraphAddNode(&node, graph, nullptr, 0, &cp);
            if (e == cudaSuccess) {
                W.cond = h;
                cudaGraph_t body = cp.conditional.phGraph_out[0];
                e = cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
                if (e == cudaSuccess) {
                    cudaError_t e2 = wf_iteration(W, L, s, true, nullptr);
                    e = cudaStreamEndCapture(s, &body);
                    if (e == cudaSuccess) e = e2;
                }
            }
            if (e == cudaSuccess) e = cudaGraphInstantiate(&WS.exec, graph, 0);
            if (graph) cudaGraphDestroy(graph);
            if (e != cudaSuccess) {
                if (WS.exec) cudaGraphExecDestroy(WS.exec);
                WS.exec = nullptr;
                return cuda_fail(e, "wavefront graph");
            }
            std::memcpy(WS.graph_key, key, sizeof(key));
        }
        e = cudaGraphLaunch(WS.exec, s);
        if (e != cudaSuccess) return cuda_fail(e, "wavefront graph");
        C.launches += (uint64_t)W.max_iters;  // upper bound; refined below
        done = true;
    }
    if (!done) {
        // host loop: one iteration per launch sequence, reading the active
        // count back every iteration (bounded by the iteration cap)
        uint32_t active = 1;
        cudaEvent_t ev[kWfStages + 1] = {};
        if (prof) {
            std::memset(prof, 0, sizeof(*prof));
            for (auto& x : ev)
                if (e == cudaSuccess) e = cudaEventCreate(&x);
        }
        const uint32_t nk = shade_launches(W, L) + (W.level >= 2 ? 2 : 0) + (W.level >= 3 ? 2 : 0);
        for (uint32_t it = 0; e == cudaSuccess && it < W.max_iters && active; ++it) {
            e = wf_iteration(W, L, s, false, WS.active_host_dev, prof ? ev : nullptr);
            if (e == cudaSuccess) e = cudaMemcpyAsync(&active, WS.active_host_dev, 4, cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            C.launches += 5 + nk;
            if (prof && e == cudaSuccess) {
                const uint32_t launches[kWfStages] = {1u, W.level >= 2 ? 2u : 0u, 1u, shade_launches(W, L) + 1u,
                                                      W.level >= 3 ? 2u : 0u, 1u, 1u};
                for (int k = 0; k < kWfStages; ++k) {
                    float ms = 0.0f;
                    cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
                    prof->ms[k] += ms;
                    prof->launches[k] += launches[k];
                }
                ++prof->iterations;
            }
        }
        if (prof)
            for (auto& x : ev)
                if (x) cudaEventDestroy(x);
        if (e != cudaSuccess) return cuda_fail(e, "wavefront iteration");
    }
    for (uint32_t i = 0; i < n_frames; ++i)
        if (fr[i].out) wf_resolve<<<(fr[i].npix + 255) / 256, 256, 0, s>>>(WS.frames_dev, i);
    if (ms_out) cudaEventRecord(C.events[7], s);
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "wavefront render");
    if (ms_out) cudaEventElapsedTime(ms_out, C.events[6], C.events[7]);
    // iterations actually run (for the launch count)
    uint32_t iters = 0;
    cudaMemcpy(&iters, W.counters + kCntIter, 4, cudaMemcpyDeviceToHost);
    if (P.use_graph)
        C.launches += (uint64_t)iters * (5 + shade_launches(W, L) + (W.level >= 2 ? 2 : 0) + (W.level >= 3 ? 2 : 0)) -
                      (uint64_t)W.max_iters;
    return NOOR_OK;
}

}  // namespace nb

using namespace nb;

extern "C" int noor_wavefront_render(const noor_wf_frame* frames, uint32_t n_frames, const noor_wf_params* params) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    noor_wf_params p{};
    if (params) p = *params;
    return wavefront_render(*C, frames, n_frames, p, nullptr);
}

extern "C" int noor_wavefront_render_timed(const noor_wf_frame* frames, uint32_t n_frames,
                                           const noor_wf_params* params, float* ms) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    noor_wf_params p{};
    if (params) p = *params;
    return wavefront_render(*C, frames, n_frames, p, ms);
}

extern "C" int noor_wavefront_profile(const noor_wf_frame* frames, uint32_t n_frames,
                                      const noor_wf_params* params, noor_wf_profile* out) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    if (!out) return set_error(NOOR_ERR_INVALID, "wavefront profile: out is null");
    noor_wf_params p{};
    if (params) p = *params;
    return wavefront_render(*C, frames, n_frames, p, nullptr, out);
}

extern "C" int noor_wavefront_counters(uint64_t counters[3], int reset) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    if (!C->wf) {
        if (counters) counters[0] = counters[1] = counters[2] = 0;
        return NOOR_OK;
    }
    unsigned long long h[3] = {0, 0, 0};
    cudaError_t e = cudaMemcpy(h, C->wf->dev.rays, sizeof(h), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && reset) e = cudaMemset(C->wf->dev.rays, 0, sizeof(h));
    if (e != cudaSuccess) return cuda_fail(e, "wavefront counters");
    if (counters)
        for (int i = 0; i < 3; ++i) counters[i] = h[i];
    return NOOR_OK;
}

// Autotuner: coordinate descent on the launch parameters, each candidate
// timed by one device-timed render of the batch: the slot count first
// (2^18 .. 2^24, none beyond twice the batch's paths), then the block size
// (32, 64, 128), then the sort granularity (0 .. 3), then the trees (binary,
// four-wide, four-wide for shadow rays only), then the shading stage's
// register budget, then the slot count again around the choices made; the
// fastest seen wins.
extern "C" int noor_wavefront_autotune(const noor_wf_frame* frames, uint32_t n_frames, noor_wf_params* best,
                                       float* best_ms) {
    Context* C;
    int rc = need_ctx(C);
    if (rc) return rc;
    if (!best) return set_error(NOOR_ERR_INVALID, "autotune: best is null");
    unsigned long long paths = 0;
    for (uint32_t i = 0; i < n_frames && frames; ++i)
        paths += (unsigned long long)frames[i].width * frames[i].height * frames[i].spp;
    std::vector<uint32_t> caps;
    for (uint32_t c = 1u << 18; c <= (1u << 24); c <<= 1)
        if (c == (1u << 18) || c <= 2 * paths) caps.push_back(c);
    noor_wf_params bp{128, caps.back() >= (1u << 22) ? (1u << 22) : caps.back(), 1, best->use_graph};
    float bms = 3.4e38f;
    auto trial = [&](const noor_wf_params& p) -> int {
        float ms = 0.0f;
        int r = wavefront_render(*C, frames, n_frames, p, &ms);
        if (r) return r;
        if (ms < bms) {
            bms = ms;
            bp = p;
        }
        return NOOR_OK;
    };
    for (uint32_t c : caps) {
        noor_wf_params p = bp;
        p.queue_capacity = c;
        if ((rc = trial(p))) return rc;
    }
    for (uint32_t b : {32u, 64u, 128u}) {
        noor_wf_params p = bp;
        p.block_size = b;
        if (b != bp.block_size && (rc = trial(p))) return rc;
    }
    for (uint32_t so : {0u, 1u, 2u, 3u}) {
        noor_wf_params p = bp;
        p.sort_granularity = so;
        if (so != bp.sort_granularity && (rc = trial(p))) return rc;
    }
    for (uint32_t tv : {(uint32_t)NOOR_TRAVERSAL_BINARY, (uint32_t)NOOR_TRAVERSAL_WIDE,
                        (uint32_t)NOOR_TRAVERSAL_WIDE_SHADOW}) {
        noor_wf_params p = bp;
        p.traversal = tv;
        if ((rc = trial(p))) return rc;
    }
    {
        noor_wf_params p = bp;
        p.shade_regs = 128;
        if ((rc = trial(p))) return rc;
    }
    const uint32_t c0 = bp.queue_capacity;
    for (uint32_t c : caps) {
        if (c != c0 / 2 && c != c0 * 2) continue;
        noor_wf_params p = bp;
        p.queue_capacity = c;
        if ((rc = trial(p))) return rc;
    }
    *best = bp;
    if (best_ms) *best_ms = bms;
    return NOOR_OK;
}

