// GPU bottom-level BVH builder (bvh_gpu.h).  The host builder
// (scene_build.cpp) restates the reference's recursive binned-SAH build
// (noor/source/bvh.cpp:88-258, splitter.cpp:28-161); this file builds the
// same trees level by level and renumbers them depth-first at the end, so
// the node words are the same bytes.  What that takes:
//   * the split search rounds as the host does: this file is compiled with
//     -fmad=false, and the bin edges are accumulated in the host's order;
//   * boxes merged in the host's order keep the first of equal coordinates
//     (+0 / -0): bin boxes are reduced with 64-bit keys (value rank, then
//     position in the node's slice, then the sign of a zero);
//   * the partition is the one libstdc++'s std::partition produces for
//     bidirectional iterators: the k-th element failing the predicate from
//     the left swaps with the k-th element passing it from the right.
// Tasks (nodes to split) of one level run together: leaf tests in one
// kernel, small tasks one block each (binning, split search and partition in
// shared memory), large tasks in chunks with their bins in global memory.
// The payload's tail (gpu_payload_tail) follows: vertex de-duplication in
// BVH order, numbered as the host's sequential table numbers it, and the
// Wald records of the triangles.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "bvh_gpu.h"
#include "../../include/noor_b200.h"

namespace nbg {
namespace {

constexpr uint32_t kMaxBins = 64;
constexpr uint32_t kTinyCap = 256;    // tasks of up to this many triangles: one warp
constexpr uint32_t kSmallCap = 4096;  // up to this many: one 256-thread block
constexpr uint32_t kChunk = 4096;     // larger tasks: one block per this many
constexpr uint32_t kLeafBit = 0x80000000u;

struct Task {
    uint32_t start, count, rec, level, mesh;
    float box[6], cbox[6];
};
struct Rec {
    float box[6];
    uint32_t kind;  // kLeafBit for a leaf; else the split axis
    uint32_t a, b;  // leaf: start, count; inner: left and right record
    uint32_t level, mesh, size, dfs;
};
struct Split {
    uint32_t axis, index, leaf, pad;
    float plane_hi;
    float lbox[6], lcbox[6], rbox[6], rcbox[6];
};
struct Chunk {
    uint32_t task;  // index into the large list
    uint32_t begin, end;  // positions relative to the task's start
};
struct Ctl {
    uint32_t n_next, n_rec, n_tiny, n_small, n_large, overflow;
};
struct Params {
    uint32_t nb, max_height, min_leaf, max_leaf;
    float Ci, Ct;
    uint32_t cap;       // capacity of the record array
    uint32_t task_cap;  // capacity of one level's task array
};

// ------------------------------------------------------------ box algebra
// the host's mn / mx: the first argument wins ties
__device__ __forceinline__ float mn(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float mx(float a, float b) { return (a < b) ? b : a; }

struct DBox {
    float lo[3], hi[3];
};
__device__ __forceinline__ void box_empty(DBox& b) {
    for (int i = 0; i < 3; ++i) {
        b.lo[i] = __int_as_float(0x7f800000);
        b.hi[i] = __int_as_float(0xff800000);
    }
}
__device__ __forceinline__ void box_merge(DBox& a, const DBox& b) {
    for (int i = 0; i < 3; ++i) {
        a.lo[i] = mn(a.lo[i], b.lo[i]);
        a.hi[i] = mx(a.hi[i], b.hi[i]);
    }
}
__device__ __forceinline__ DBox box_merged(const DBox& a, const DBox& b) {
    DBox r = a;
    box_merge(r, b);
    return r;
}
__device__ __forceinline__ float box_area(const DBox& b) {
    const float c[6] = {b.lo[0], b.lo[1], b.lo[2], b.hi[0], b.hi[1], b.hi[2]};
    for (float v : c)
        if (isinf(v) || isnan(v)) return __int_as_float(0x7f800000);
    const float dx = b.hi[0] - b.lo[0], dy = b.hi[1] - b.lo[1], dz = b.hi[2] - b.lo[2];
    return 2.0f * (dx * dy + dy * dz + dx * dz);
}
__device__ __forceinline__ DBox box_load(const float* f) {
    DBox b;
    for (int i = 0; i < 3; ++i) {
        b.lo[i] = f[i];
        b.hi[i] = f[3 + i];
    }
    return b;
}
__device__ __forceinline__ void box_store(float* f, const DBox& b) {
    for (int i = 0; i < 3; ++i) {
        f[i] = b.lo[i];
        f[3 + i] = b.hi[i];
    }
}

// ------------------------------------------------------------ ordered keys
// rank of a float in a total order where -0 and +0 tie
__device__ __forceinline__ uint32_t frank(float f) {
    uint32_t u = __float_as_uint(f);
    if (u == 0x80000000u) u = 0u;
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float funrank(uint32_t o, uint32_t neg_zero) {
    const uint32_t u = (o & 0x80000000u) ? (o & 0x7fffffffu) : ~o;
    return (u == 0u && neg_zero) ? -0.0f : __uint_as_float(u);
}
// min: smallest value, then the earliest position; max: largest value, then
// the earliest position
__device__ __forceinline__ unsigned long long kmin(float v, uint32_t q) {
    return ((unsigned long long)frank(v) << 32) | ((unsigned long long)(q & 0x7fffffffu) << 1) |
           (__float_as_uint(v) >> 31);
}
__device__ __forceinline__ unsigned long long kmax(float v, uint32_t q) {
    return ((unsigned long long)frank(v) << 32) | ((unsigned long long)(0x7fffffffu - (q & 0x7fffffffu)) << 1) |
           (__float_as_uint(v) >> 31);
}
__device__ __forceinline__ float kval(unsigned long long k) { return funrank((uint32_t)(k >> 32), (uint32_t)k & 1u); }

// 12 keys per bin: box lo (min), box hi (max), centroid lo (min), centroid hi (max)
constexpr int kKeys = 12;
__device__ __forceinline__ void keys_init(unsigned long long* k) {
    for (int i = 0; i < 12; ++i) k[i] = (i < 3 || (i >= 6 && i < 9)) ? ~0ull : 0ull;
}

// ------------------------------------------------------------ split search
// bin edges of one axis: the host's sequential accumulation
__device__ void edges_of(const float* cbox, int a, uint32_t nb, float* elo, float* ehi) {
    const float cl = cbox[a], ch = cbox[3 + a];
    const float inv = 1.0f / (float)nb;
    const float dt = (ch - cl) * inv;
    elo[0] = cl;
    ehi[0] = cl + dt;
    for (uint32_t i = 1; i < nb; ++i) {
        elo[i] = elo[i - 1] + dt;
        ehi[i] = ehi[i - 1] + dt;
    }
    ehi[nb - 1] = ch;
}
// first bin whose upper edge is >= c (the host's lower-bound search)
__device__ __forceinline__ uint32_t bin_of(const float* elo, const float* ehi, uint32_t nb, float c) {
    const uint32_t last = nb - 1;
    if (c <= ehi[0]) return 0;
    if (c > elo[last]) return last;
    uint32_t lo = 1, hi = last - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (c <= ehi[mid])
            hi = mid;
        else
            lo = mid + 1;
    }
    return lo;
}
__device__ __forceinline__ void centroid(const float* tb, float* c) {
    for (int i = 0; i < 3; ++i) c[i] = (tb[i] + tb[3 + i]) * 0.5f;
}

struct AxisBest {
    float cost;
    uint32_t index, nl, nr;
};
// decode one axis's keys into bin boxes and run the host's sweep (L, LC,
// NL prefix-merged in place; R, RC, NR suffixes); returns its best plane
__device__ AxisBest sweep_axis(const unsigned long long* keys, const uint32_t* cnt, uint32_t nb, float parent,
                               const Params& P, DBox* L, DBox* LC, DBox* R, DBox* RC, uint32_t* NL, uint32_t* NR) {
    for (uint32_t k = 0; k < nb; ++k) {
        NL[k] = cnt[k];
        NR[k] = 0;
        box_empty(R[k]);
        box_empty(RC[k]);
        if (cnt[k] == 0) {
            box_empty(L[k]);
            box_empty(LC[k]);
        } else {
            const unsigned long long* kk = keys + (size_t)k * kKeys;
            for (int i = 0; i < 3; ++i) {
                L[k].lo[i] = kval(kk[i]);
                L[k].hi[i] = kval(kk[3 + i]);
                LC[k].lo[i] = kval(kk[6 + i]);
                LC[k].hi[i] = kval(kk[9 + i]);
            }
        }
    }
    const uint32_t n = nb - 1;
    R[n] = L[n];
    RC[n] = LC[n];
    NR[n] = NL[n];
    for (uint32_t i = n - 1; i > 0; --i) {
        R[i] = box_merged(L[i], R[i + 1]);
        RC[i] = box_merged(LC[i], RC[i + 1]);
        NR[i] = NL[i] + NR[i + 1];
    }
    for (uint32_t i = 1; i < n; ++i) {
        box_merge(L[i], L[i - 1]);
        box_merge(LC[i], LC[i - 1]);
        NL[i] += NL[i - 1];
    }
    AxisBest best{__int_as_float(0x7f800000), 0u, 0u, 0u};
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t nl = NL[i], nr = NR[i + 1];
        if (nl == 0 || nr == 0) continue;
        const float lc = (float)nl * box_area(L[i]);
        const float rc = (float)nr * box_area(R[i + 1]);
        const float cost = P.Ct + P.Ci * (lc + rc) / parent;
        if (cost < best.cost) best = AxisBest{cost, i, nl, nr};
    }
    return best;
}
__device__ __forceinline__ bool plane_valid(const AxisBest& b) {
    return b.cost != __int_as_float(0x7f800000) && b.nl != 0 && b.nr != 0;
}

// ------------------------------------------------------------ records
struct Out {
    Rec* recs;
    Task* next;
    Ctl* ctl;
    uint32_t* mesh_stats;  // 4 per mesh: height, inner, leaf, max leaf tris
};
__device__ void write_leaf(const Out& o, const Task& t) {
    Rec& r = o.recs[t.rec];
    for (int i = 0; i < 6; ++i) r.box[i] = t.box[i];
    r.kind = kLeafBit;
    r.a = t.start;
    r.b = t.count;
    r.level = t.level;
    r.mesh = t.mesh;
    r.size = 1;
    uint32_t* st = o.mesh_stats + 4 * t.mesh;
    atomicMax(st + 0, t.level);
    atomicAdd(st + 2, 1u);
    atomicMax(st + 3, t.count);
}
// an inner record and its two child tasks; false when out of capacity
__device__ bool write_inner(const Out& o, const Params& P, const Task& t, uint32_t axis, uint32_t nleft,
                            const float* lbox, const float* lcbox, const float* rbox, const float* rcbox) {
    const uint32_t r0 = atomicAdd(&o.ctl->n_rec, 2u);
    const uint32_t q0 = atomicAdd(&o.ctl->n_next, 2u);
    if (r0 + 2 > P.cap || q0 + 2 > P.task_cap) {
        atomicOr(&o.ctl->overflow, 1u);
        return false;
    }
    Rec& r = o.recs[t.rec];
    for (int i = 0; i < 6; ++i) r.box[i] = t.box[i];
    r.kind = axis;
    r.a = r0;
    r.b = r0 + 1;
    r.level = t.level;
    r.mesh = t.mesh;
    atomicAdd(o.mesh_stats + 4 * t.mesh + 1, 1u);
    Task L, R;
    L.start = t.start;
    L.count = nleft;
    R.start = t.start + nleft;
    R.count = t.count - nleft;
    L.rec = r0;
    R.rec = r0 + 1;
    L.level = R.level = t.level + 1;
    L.mesh = R.mesh = t.mesh;
    for (int i = 0; i < 6; ++i) {
        L.box[i] = lbox[i];
        L.cbox[i] = lcbox[i];
        R.box[i] = rbox[i];
        R.cbox[i] = rcbox[i];
    }
    o.next[q0] = L;
    o.next[q0 + 1] = R;
    return true;
}

// ------------------------------------------------------------ kernels
// leaf tests of BVH::recursiveBuild that need no split search (level, count);
// the rest go to the tiny / small / large lists
__global__ void k_classify(const Task* tasks, uint32_t n, Params P, Out o, uint32_t* tiny, uint32_t* small,
                           uint32_t* large, uint32_t* level_recs) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Task t = tasks[i];
    level_recs[i] = t.rec;
    if (t.level >= P.max_height || t.count <= P.min_leaf) {
        write_leaf(o, t);
        return;
    }
    if (t.count <= kTinyCap)
        tiny[atomicAdd(&o.ctl->n_tiny, 1u)] = i;
    else if (t.count <= kSmallCap)
        small[atomicAdd(&o.ctl->n_small, 1u)] = i;
    else
        large[atomicAdd(&o.ctl->n_large, 1u)] = i;
}

// shared memory of k_split for nb bins and `cap` elements
struct SmallSmem {
    size_t keys, cnt, boxes, nlr, edges, best, ids, rank, sF, sT, flags, tsum, total;
};
__host__ __device__ inline SmallSmem small_layout(uint32_t nb, uint32_t cap, uint32_t nt) {
    SmallSmem s{};
    size_t o = 0;
    s.keys = o;
    o += (size_t)3 * nb * kKeys * 8;
    s.cnt = o;
    o += (size_t)3 * nb * 4;
    o = (o + 15) & ~(size_t)15;
    s.boxes = o;
    o += (size_t)4 * 3 * nb * sizeof(DBox);
    s.nlr = o;
    o += (size_t)2 * 3 * nb * 4;
    s.edges = o;
    o += (size_t)2 * 3 * nb * 4;
    s.best = o;
    o += 3 * sizeof(AxisBest) + 32;
    s.ids = o;
    o += (size_t)cap * 4;
    s.rank = o;
    o += (size_t)cap * 4;
    s.sF = o;
    o += (size_t)cap * 4;
    s.sT = o;
    o += (size_t)cap * 4;
    s.flags = o;
    o += ((size_t)cap + 15) & ~(size_t)15;
    s.tsum = o;
    o += (size_t)(nt + 1) * 4;
    s.total = (o + 15) & ~(size_t)15;
    return s;
}

// one block per task of up to CAP triangles: bins, split search, partition
template <uint32_t NT, uint32_t CAP>
__global__ void __launch_bounds__(NT) k_split(const Task* tasks, const uint32_t* list, const float* tri_box,
                                              uint32_t* tri_order, Params P, Out o) {
    extern __shared__ __align__(16) unsigned char sm[];
    const SmallSmem L = small_layout(P.nb, CAP, NT);
    unsigned long long* keys = reinterpret_cast<unsigned long long*>(sm + L.keys);
    uint32_t* cnt = reinterpret_cast<uint32_t*>(sm + L.cnt);
    DBox* bL = reinterpret_cast<DBox*>(sm + L.boxes);
    DBox* bLC = bL + 3 * P.nb;
    DBox* bR = bLC + 3 * P.nb;
    DBox* bRC = bR + 3 * P.nb;
    uint32_t* NL = reinterpret_cast<uint32_t*>(sm + L.nlr);
    uint32_t* NR = NL + 3 * P.nb;
    float* elo = reinterpret_cast<float*>(sm + L.edges);
    float* ehi = elo + 3 * P.nb;
    AxisBest* best = reinterpret_cast<AxisBest*>(sm + L.best);
    uint32_t* dec = reinterpret_cast<uint32_t*>(best + 3);  // [0] leaf, [1] axis, [2] index, [3] plane bits, [4] m
    uint32_t* ids = reinterpret_cast<uint32_t*>(sm + L.ids);
    uint32_t* rank = reinterpret_cast<uint32_t*>(sm + L.rank);
    uint32_t* sF = reinterpret_cast<uint32_t*>(sm + L.sF);
    uint32_t* sT = reinterpret_cast<uint32_t*>(sm + L.sT);
    unsigned char* pred = sm + L.flags;
    uint32_t* tsum = reinterpret_cast<uint32_t*>(sm + L.tsum);

    const uint32_t nb = P.nb;
    const Task t = tasks[list[blockIdx.x]];
    const uint32_t n = t.count;  // <= CAP (checked by the classifier)
    const uint32_t tid = threadIdx.x;
    if (tid < 3) edges_of(t.cbox, (int)tid, nb, elo + tid * nb, ehi + tid * nb);
    for (uint32_t i = tid; i < 3 * nb; i += NT) {
        cnt[i] = 0;
        keys_init(keys + (size_t)i * kKeys);
    }
    __syncthreads();
    for (uint32_t q = tid; q < n; q += NT) {
        const uint32_t id = tri_order[t.start + q];
        ids[q] = id;
        const float* tb = tri_box + 6 * (size_t)id;
        float c[3];
        centroid(tb, c);
        for (int a = 0; a < 3; ++a) {
            const uint32_t k = bin_of(elo + a * nb, ehi + a * nb, nb, c[a]);
            unsigned long long* kk = keys + ((size_t)a * nb + k) * kKeys;
            atomicAdd(cnt + a * nb + k, 1u);
            for (int i = 0; i < 3; ++i) {
                atomicMin(kk + i, kmin(tb[i], q));
                atomicMax(kk + 3 + i, kmax(tb[3 + i], q));
                atomicMin(kk + 6 + i, kmin(c[i], q));
                atomicMax(kk + 9 + i, kmax(c[i], q));
            }
        }
    }
    __syncthreads();
    if (tid < 3) {
        const uint32_t a = tid;
        best[a] = sweep_axis(keys + (size_t)a * nb * kKeys, cnt + a * nb, nb, box_area(box_load(t.box)), P,
                             bL + a * nb, bLC + a * nb, bR + a * nb, bRC + a * nb, NL + a * nb, NR + a * nb);
    }
    __syncthreads();
    if (tid == 0) {
        int ba = -1;
        float bc = __int_as_float(0x7f800000);
        for (int a = 0; a < 3; ++a)
            if (plane_valid(best[a]) && best[a].cost < bc) {
                bc = best[a].cost;
                ba = a;
            }
        const float leaf_cost = P.Ci * (float)n;
        const bool leaf = ba < 0 || (leaf_cost < bc && n <= P.max_leaf);
        dec[0] = leaf ? 1u : 0u;
        if (!leaf) {
            dec[1] = (uint32_t)ba;
            dec[2] = best[ba].index;
            dec[3] = __float_as_uint(ehi[ba * nb + best[ba].index]);
        }
    }
    __syncthreads();
    if (dec[0]) {
        if (tid == 0) write_leaf(o, t);
        return;
    }
    const uint32_t a = dec[1], index = dec[2];
    const float plane = __uint_as_float(dec[3]);
    // predicate and counts: thread tid takes elements [tid*per, (tid+1)*per)
    const uint32_t per = (n + NT - 1) / NT;
    const uint32_t q0 = min(n, tid * per), q1 = min(n, q0 + per);
    uint32_t trues = 0;
    for (uint32_t q = q0; q < q1; ++q) {
        float c[3];
        centroid(tri_box + 6 * (size_t)ids[q], c);
        const unsigned char p = c[a] <= plane ? 1 : 0;
        pred[q] = p;
        trues += p;
    }
    tsum[tid] = trues;
    __syncthreads();
    if (tid == 0) {
        uint32_t s = 0;
        for (uint32_t i = 0; i < NT; ++i) {
            const uint32_t v = tsum[i];
            tsum[i] = s;
            s += v;
        }
        tsum[NT] = s;
    }
    __syncthreads();
    const uint32_t m = tsum[NT];
    uint32_t tb = tsum[tid];  // trues before q
    for (uint32_t q = q0; q < q1; ++q) {
        const uint32_t fb = q - tb;
        if (q < m && !pred[q]) {
            rank[q] = fb;
            sF[fb] = q;
        } else if (q >= m && pred[q]) {
            const uint32_t k = m - tb - 1;  // trues after q: its rank from the right
            rank[q] = k;
            sT[k] = q;
        }
        tb += pred[q];
    }
    __syncthreads();
    for (uint32_t q = q0; q < q1; ++q) {
        uint32_t dst = q;
        if (q < m && !pred[q])
            dst = sT[rank[q]];
        else if (q >= m && pred[q])
            dst = sF[rank[q]];
        tri_order[t.start + dst] = ids[q];
    }
    if (tid == 0) {
        float lb[6], lcb[6], rb[6], rcb[6];
        box_store(lb, bL[a * nb + index]);
        box_store(lcb, bLC[a * nb + index]);
        box_store(rb, bR[a * nb + index + 1]);
        box_store(rcb, bRC[a * nb + index + 1]);
        write_inner(o, P, t, a, m, lb, lcb, rb, rcb);
    }
}

// ---------------------------------------------------- large tasks, chunked
__global__ void __launch_bounds__(256) k_bin_large(const Task* tasks, const uint32_t* large, const Chunk* chunks,
                                                   const float* tri_box, const uint32_t* tri_order, Params P,
                                                   unsigned long long* gkeys, uint32_t* gcnt) {
    extern __shared__ __align__(16) unsigned char sm[];
    const uint32_t nb = P.nb;
    unsigned long long* keys = reinterpret_cast<unsigned long long*>(sm);
    uint32_t* cnt = reinterpret_cast<uint32_t*>(keys + (size_t)3 * nb * kKeys);
    float* elo = reinterpret_cast<float*>(cnt + 3 * nb);
    float* ehi = elo + 3 * nb;
    const Chunk ch = chunks[blockIdx.x];
    const Task t = tasks[large[ch.task]];
    const uint32_t tid = threadIdx.x;
    if (tid < 3) edges_of(t.cbox, (int)tid, nb, elo + tid * nb, ehi + tid * nb);
    for (uint32_t i = tid; i < 3 * nb; i += blockDim.x) {
        cnt[i] = 0;
        keys_init(keys + (size_t)i * kKeys);
    }
    __syncthreads();
    for (uint32_t q = ch.begin + tid; q < ch.end; q += blockDim.x) {
        const float* tb = tri_box + 6 * (size_t)tri_order[t.start + q];
        float c[3];
        centroid(tb, c);
        for (int a = 0; a < 3; ++a) {
            const uint32_t k = bin_of(elo + a * nb, ehi + a * nb, nb, c[a]);
            unsigned long long* kk = keys + ((size_t)a * nb + k) * kKeys;
            atomicAdd(cnt + a * nb + k, 1u);
            for (int i = 0; i < 3; ++i) {
                atomicMin(kk + i, kmin(tb[i], q));
                atomicMax(kk + 3 + i, kmax(tb[3 + i], q));
                atomicMin(kk + 6 + i, kmin(c[i], q));
                atomicMax(kk + 9 + i, kmax(c[i], q));
            }
        }
    }
    __syncthreads();
    unsigned long long* gk = gkeys + (size_t)ch.task * 3 * nb * kKeys;
    uint32_t* gc = gcnt + (size_t)ch.task * 3 * nb;
    for (uint32_t i = tid; i < 3 * nb; i += blockDim.x) {
        if (!cnt[i]) continue;
        atomicAdd(gc + i, cnt[i]);
        const unsigned long long* kk = keys + (size_t)i * kKeys;
        unsigned long long* g = gk + (size_t)i * kKeys;
        for (int j = 0; j < 12; ++j) {
            if (j < 3 || (j >= 6 && j < 9))
                atomicMin(g + j, kk[j]);
            else
                atomicMax(g + j, kk[j]);
        }
    }
}

__global__ void k_init_large_keys(unsigned long long* gkeys, uint32_t* gcnt, uint32_t n_bins) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_bins; i += gridDim.x * blockDim.x) {
        gcnt[i] = 0;
        keys_init(gkeys + (size_t)i * kKeys);
    }
}

// split search of each large task (one 32-thread block each)
__global__ void k_decide_large(const Task* tasks, const uint32_t* large, Params P, const unsigned long long* gkeys,
                               const uint32_t* gcnt, Split* splits, Out o) {
    extern __shared__ __align__(16) unsigned char sm[];
    const uint32_t nb = P.nb;
    DBox* bL = reinterpret_cast<DBox*>(sm);
    DBox* bLC = bL + 3 * nb;
    DBox* bR = bLC + 3 * nb;
    DBox* bRC = bR + 3 * nb;
    uint32_t* NL = reinterpret_cast<uint32_t*>(bRC + 3 * nb);
    uint32_t* NR = NL + 3 * nb;
    AxisBest* best = reinterpret_cast<AxisBest*>(NR + 3 * nb);
    float* ehi = reinterpret_cast<float*>(best + 3);
    float* elo = ehi + 3 * nb;
    const uint32_t j = blockIdx.x;
    const Task t = tasks[large[j]];
    const uint32_t tid = threadIdx.x;
    if (tid < 3) {
        const uint32_t a = tid;
        edges_of(t.cbox, (int)a, nb, elo + a * nb, ehi + a * nb);
        best[a] = sweep_axis(gkeys + ((size_t)j * 3 + a) * nb * kKeys, gcnt + ((size_t)j * 3 + a) * nb, nb,
                             box_area(box_load(t.box)), P, bL + a * nb, bLC + a * nb, bR + a * nb, bRC + a * nb,
                             NL + a * nb, NR + a * nb);
    }
    __syncthreads();
    if (tid != 0) return;
    int ba = -1;
    float bc = __int_as_float(0x7f800000);
    for (int a = 0; a < 3; ++a)
        if (plane_valid(best[a]) && best[a].cost < bc) {
            bc = best[a].cost;
            ba = a;
        }
    const float leaf_cost = P.Ci * (float)t.count;
    Split& s = splits[j];
    s.leaf = (ba < 0 || (leaf_cost < bc && t.count <= P.max_leaf)) ? 1u : 0u;
    if (s.leaf) {
        write_leaf(o, t);
        return;
    }
    const uint32_t index = best[ba].index;
    s.axis = (uint32_t)ba;
    s.index = index;
    s.plane_hi = ehi[ba * nb + index];
    box_store(s.lbox, bL[ba * nb + index]);
    box_store(s.lcbox, bLC[ba * nb + index]);
    box_store(s.rbox, bR[ba * nb + index + 1]);
    box_store(s.rcbox, bRC[ba * nb + index + 1]);
}

// predicate counts per chunk
__global__ void __launch_bounds__(256) k_count_large(const Task* tasks, const uint32_t* large, const Chunk* chunks,
                                                     const Split* splits, const float* tri_box,
                                                     const uint32_t* tri_order, uint32_t* chunk_true) {
    __shared__ uint32_t acc;
    const Chunk ch = chunks[blockIdx.x];
    const Split& s = splits[ch.task];
    if (threadIdx.x == 0) acc = 0;
    __syncthreads();
    if (s.leaf) {
        if (threadIdx.x == 0) chunk_true[blockIdx.x] = 0;
        return;
    }
    const Task t = tasks[large[ch.task]];
    uint32_t c = 0;
    for (uint32_t q = ch.begin + threadIdx.x; q < ch.end; q += blockDim.x) {
        float cc[3];
        centroid(tri_box + 6 * (size_t)tri_order[t.start + q], cc);
        c += cc[s.axis] <= s.plane_hi ? 1u : 0u;
    }
    atomicAdd(&acc, c);
    __syncthreads();
    if (threadIdx.x == 0) chunk_true[blockIdx.x] = acc;
}

// per large task: exclusive prefix of its chunks' counts, then its inner
// record and children (the left child's size is the predicate count)
__global__ void k_scan_emit_large(const Task* tasks, const uint32_t* large, uint32_t n_large,
                                  const uint32_t* task_chunk0, const uint32_t* chunk_true, uint32_t* chunk_before,
                                  const Split* splits, Params P, Out o) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_large) return;
    const Split& s = splits[j];
    if (s.leaf) return;
    uint32_t acc = 0;
    for (uint32_t c = task_chunk0[j]; c < task_chunk0[j + 1]; ++c) {
        chunk_before[c] = acc;
        acc += chunk_true[c];
    }
    const Task t = tasks[large[j]];
    write_inner(o, P, t, s.axis, acc, s.lbox, s.lcbox, s.rbox, s.rcbox);
}

// the partition's destinations: ranks and the swap tables of each chunk
__global__ void __launch_bounds__(256) k_rank_large(const Task* tasks, const uint32_t* large, const Chunk* chunks,
                                                    const uint32_t* task_chunk0, const uint32_t* chunk_true,
                                                    const uint32_t* chunk_before, const Split* splits,
                                                    const float* tri_box, const uint32_t* tri_order, uint32_t* rank,
                                                    uint32_t* sF, uint32_t* sT, unsigned char* pred_out) {
    __shared__ uint32_t tsum[257];
    const Chunk ch = chunks[blockIdx.x];
    const Split& s = splits[ch.task];
    if (s.leaf) return;
    const Task t = tasks[large[ch.task]];
    // total trues of the task
    uint32_t m = 0;
    for (uint32_t c = task_chunk0[ch.task]; c < task_chunk0[ch.task + 1]; ++c) m += chunk_true[c];
    const uint32_t len = ch.end - ch.begin;
    const uint32_t per = (len + 255) / 256;
    const uint32_t q0 = ch.begin + min(len, threadIdx.x * per), q1 = min(ch.end, q0 + per);
    uint32_t trues = 0;
    for (uint32_t q = q0; q < q1; ++q) {
        float cc[3];
        centroid(tri_box + 6 * (size_t)tri_order[t.start + q], cc);
        const unsigned char p = cc[s.axis] <= s.plane_hi ? 1 : 0;
        pred_out[t.start + q] = p;
        trues += p;
    }
    tsum[threadIdx.x] = trues;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t acc = chunk_before[blockIdx.x];
        for (int i = 0; i < 256; ++i) {
            const uint32_t v = tsum[i];
            tsum[i] = acc;
            acc += v;
        }
    }
    __syncthreads();
    uint32_t tb = tsum[threadIdx.x];
    for (uint32_t q = q0; q < q1; ++q) {
        const unsigned char p = pred_out[t.start + q];
        const uint32_t fb = q - tb;
        if (q < m && !p) {
            rank[t.start + q] = fb;
            sF[t.start + fb] = q;
        } else if (q >= m && p) {
            const uint32_t k = m - tb - 1;
            rank[t.start + q] = k;
            sT[t.start + k] = q;
        }
        tb += p;
    }
}

__global__ void __launch_bounds__(256) k_scatter_large(const Task* tasks, const uint32_t* large, const Chunk* chunks,
                                                       const uint32_t* task_chunk0, const uint32_t* chunk_true,
                                                       const Split* splits, const uint32_t* tri_order,
                                                       const uint32_t* rank, const uint32_t* sF, const uint32_t* sT,
                                                       const unsigned char* pred, uint32_t* tri_tmp) {
    const Chunk ch = chunks[blockIdx.x];
    const Split& s = splits[ch.task];
    if (s.leaf) return;
    const Task t = tasks[large[ch.task]];
    uint32_t m = 0;
    for (uint32_t c = task_chunk0[ch.task]; c < task_chunk0[ch.task + 1]; ++c) m += chunk_true[c];
    for (uint32_t q = ch.begin + threadIdx.x; q < ch.end; q += blockDim.x) {
        const unsigned char p = pred[t.start + q];
        uint32_t dst = q;
        if (q < m && !p)
            dst = sT[t.start + rank[t.start + q]];
        else if (q >= m && p)
            dst = sF[t.start + rank[t.start + q]];
        tri_tmp[t.start + dst] = tri_order[t.start + q];
    }
}

__global__ void __launch_bounds__(256) k_copy_large(const Task* tasks, const uint32_t* large, const Chunk* chunks,
                                                    const Split* splits, const uint32_t* tri_tmp,
                                                    uint32_t* tri_order) {
    const Chunk ch = chunks[blockIdx.x];
    if (splits[ch.task].leaf) return;
    const Task t = tasks[large[ch.task]];
    for (uint32_t q = ch.begin + threadIdx.x; q < ch.end; q += blockDim.x)
        tri_order[t.start + q] = tri_tmp[t.start + q];
}

// ---------------------------------------------------- depth-first numbering
__global__ void k_sizes(Rec* recs, const uint32_t* level_recs, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Rec& r = recs[level_recs[i]];
    if (!(r.kind & kLeafBit)) r.size = 1 + recs[r.a].size + recs[r.b].size;
}
__global__ void k_dfs(Rec* recs, const uint32_t* level_recs, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Rec& r = recs[level_recs[i]];
    if (r.kind & kLeafBit) return;
    recs[r.a].dfs = r.dfs + 1;
    recs[r.b].dfs = r.dfs + 1 + recs[r.a].size;
}
__global__ void k_write(const Rec* recs, uint32_t n_rec, const uint32_t* mesh_off, uint32_t* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_rec) return;
    const Rec& r = recs[i];
    uint32_t* w = out + 8 * ((size_t)mesh_off[r.mesh] + r.dfs);
    for (int k = 0; k < 3; ++k) {
        w[k] = __float_as_uint(r.box[k]);
        w[4 + k] = __float_as_uint(r.box[3 + k]);
    }
    if (r.kind & kLeafBit) {
        w[3] = r.a;
        w[7] = NOOR_TRI_LEAF_MASK | r.b;
    } else {
        w[3] = recs[r.b].dfs;
        w[7] = r.kind;
    }
}


// ---------------------------------------------------- payload tail kernels
constexpr uint32_t kEmptySlot = 0xffffffffu;
struct TailArgs {
    const uint32_t *order, *vi, *ni, *ui;
    uint32_t n_corners;
    uint32_t* slots;       // representative corner of each key
    uint32_t* pmin;        // first corner of each key
    uint32_t* corner_slot;
    uint32_t mask;
    uint32_t* fail;
};
__device__ __forceinline__ void corner_key(const TailArgs& A, uint32_t p, uint32_t& v, uint32_t& n, uint32_t& u) {
    const size_t c = 3 * (size_t)A.order[p / 3] + p % 3;
    v = A.vi[c];
    n = A.ni[c];
    u = A.ui[c];
}
__device__ __forceinline__ uint32_t key_hash(uint32_t v, uint32_t n, uint32_t u) {
    uint32_t h = v * 0x9E3779B1u;
    h ^= (n + 0x7F4A7C15u) * 0x85EBCA77u + (h << 6) + (h >> 2);
    h ^= (u + 0x165667B1u) * 0xC2B2AE3Du + (h << 6) + (h >> 2);
    return h ^ (h >> 16);
}
// each corner finds its key's slot (open addressing; a slot holds any corner
// with that key), and the key's first corner by atomicMin
__global__ void k_dedup_insert(TailArgs A) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= A.n_corners) return;
    uint32_t v, n, u;
    corner_key(A, p, v, n, u);
    uint32_t slot = key_hash(v, n, u) & A.mask;
    for (uint32_t probe = 0; probe <= A.mask; ++probe) {
        uint32_t s = A.slots[slot];
        if (s == kEmptySlot) {
            s = atomicCAS(A.slots + slot, kEmptySlot, p);
            if (s == kEmptySlot) s = p;
        }
        uint32_t sv, sn, su;
        corner_key(A, s, sv, sn, su);
        if (sv == v && sn == n && su == u) {
            A.corner_slot[p] = slot;
            atomicMin(A.pmin + slot, p);
            return;
        }
        slot = (slot + 1) & A.mask;
    }
    atomicOr(A.fail, 1u);  // table full (cannot happen at half load)
}
__global__ void k_dedup_flags(TailArgs A, uint32_t* flag) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= A.n_corners) return;
    flag[p] = A.pmin[A.corner_slot[p]] == p ? 1u : 0u;
}
// exclusive scan of n values in three passes: block sums, their scan (one
// block), then each block's scan plus its offset
constexpr uint32_t kScanBlock = 1024;
__global__ void k_scan_sums(const uint32_t* in, uint32_t n, uint32_t* sums) {
    __shared__ uint32_t acc;
    if (threadIdx.x == 0) acc = 0;
    __syncthreads();
    const uint32_t i = blockIdx.x * kScanBlock + threadIdx.x;
    if (i < n) atomicAdd(&acc, in[i]);
    __syncthreads();
    if (threadIdx.x == 0) sums[blockIdx.x] = acc;
}
__global__ void k_scan_top(uint32_t* sums, uint32_t nb, uint32_t* total) {
    // one block of kScanBlock threads; each takes a contiguous run
    __shared__ uint32_t part[kScanBlock + 1];
    const uint32_t per = (nb + kScanBlock - 1) / kScanBlock;
    const uint32_t b0 = min(nb, threadIdx.x * per), b1 = min(nb, b0 + per);
    uint32_t s = 0;
    for (uint32_t i = b0; i < b1; ++i) s += sums[i];
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t a = 0;
        for (uint32_t i = 0; i < kScanBlock; ++i) {
            const uint32_t v = part[i];
            part[i] = a;
            a += v;
        }
        *total = a;
    }
    __syncthreads();
    uint32_t a = part[threadIdx.x];
    for (uint32_t i = b0; i < b1; ++i) {
        const uint32_t v = sums[i];
        sums[i] = a;
        a += v;
    }
}
__global__ void k_scan_block(const uint32_t* in, uint32_t n, const uint32_t* offs, uint32_t* out) {
    __shared__ uint32_t sh[kScanBlock];
    const uint32_t i = blockIdx.x * kScanBlock + threadIdx.x;
    sh[threadIdx.x] = i < n ? in[i] : 0u;
    __syncthreads();
    // Hillis-Steele inclusive scan in shared memory
    for (uint32_t d = 1; d < kScanBlock; d <<= 1) {
        const uint32_t v = threadIdx.x >= d ? sh[threadIdx.x - d] : 0u;
        __syncthreads();
        sh[threadIdx.x] += v;
        __syncthreads();
    }
    if (i < n) out[i] = offs[blockIdx.x] + sh[threadIdx.x] - (i < n ? in[i] : 0u);
}
// the new vertex arrays (first occurrences, in corner order)
__global__ void k_dedup_vertices(TailArgs A, const uint32_t* flag, const uint32_t* first_id, const float4* vtx,
                                 const float4* nrm, const float2* uv, float4* ovtx, float4* onrm, float2* ouv) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= A.n_corners || !flag[p]) return;
    uint32_t v, n, u;
    corner_key(A, p, v, n, u);
    const uint32_t k = first_id[p];
    ovtx[k] = vtx[v];
    onrm[k] = nrm[n];
    ouv[k] = uv[u];
}
// Wald record (header/triangle.h:73-107) of the triangle's de-duplicated
// vertices, as the host computes it (no contraction in this file)
__global__ void k_wald(TailArgs A, const uint32_t* first_id, uint32_t n_tris, const float4* ovtx,
                       const uint32_t* mat_idx, const uint32_t* mat_type, uint4* w0, uint4* w1, uint4* w2,
                       uint4* attr) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_tris) return;
    uint32_t e[3];
    float3 P[3];
    for (int j = 0; j < 3; ++j) {
        e[j] = first_id[A.pmin[A.corner_slot[3 * i + j]]];
        const float4 q = ovtx[e[j]];
        P[j] = make_float3(q.x, q.y, q.z);
    }
    const float3 A0 = P[0];
    const float b[3] = {P[2].x - A0.x, P[2].y - A0.y, P[2].z - A0.z};
    const float c[3] = {P[1].x - A0.x, P[1].y - A0.y, P[1].z - A0.z};
    float N[3] = {c[1] * b[2] - b[1] * c[2], c[2] * b[0] - b[2] * c[0], c[0] * b[1] - b[0] * c[1]};
    const float inv = 1.0f / sqrtf((N[0] * N[0] + N[1] * N[1]) + N[2] * N[2]);
    for (int k = 0; k < 3; ++k) N[k] = N[k] * inv;
    uint32_t axis = 0;
    for (uint32_t k = 0; k < 3; ++k) axis = fabsf(N[k]) > fabsf(N[axis]) ? k : axis;
    const uint32_t mod[4] = {1u, 2u, 0u, 1u};
    const uint32_t u = mod[axis], v = mod[axis + 1];
    const float denom = b[u] * c[v] - b[v] * c[u];
    const float Nk = N[axis];
    const float Aa[3] = {A0.x, A0.y, A0.z};
    uint4 r0 = make_uint4(axis, 0, 0, 0), r1 = make_uint4(0, 0, 0, 0), r2 = make_uint4(0, 0, 0, 0);
    if (denom == 0.0f) {
        r2.z = 1u;
    } else {
        r0.y = __float_as_uint(N[u] / Nk);
        r0.z = __float_as_uint(N[v] / Nk);
        r0.w = __float_as_uint(((N[0] * Aa[0] + N[1] * Aa[1]) + N[2] * Aa[2]) / Nk);
        r1.x = __float_as_uint(b[u] / denom);
        r1.y = __float_as_uint(-b[v] / denom);
        r1.z = __float_as_uint(Aa[u]);
        r1.w = __float_as_uint(Aa[v]);
        r2.x = __float_as_uint(c[v] / denom);
        r2.y = __float_as_uint(-c[u] / denom);
    }
    const uint32_t mi = mat_idx[A.order[i]];
    r2.w = mat_type[mi];
    w0[i] = r0;
    w1[i] = r1;
    w2[i] = r2;
    attr[i] = make_uint4(e[0], e[1], e[2], mi);
}

// ------------------------------------------------------------ host side
// stream-ordered scratch from the device's default pool, which keeps up to
// 4 GiB between calls, so that repeated builds do not pay for allocation
struct DevBuf {
    void* p = nullptr;
    cudaStream_t s = nullptr;
    ~DevBuf() {
        if (p) cudaFreeAsync(p, s);
    }
};
template <class T>
static cudaError_t dalloc(cudaStream_t s, DevBuf& b, size_t n, T** out) {
    b.s = s;
    cudaError_t e = cudaMallocAsync(&b.p, std::max<size_t>(n, 1) * sizeof(T), s);
    *out = static_cast<T*>(b.p);
    return e;
}
// a pair of timing events, released on every return path
struct TimingEvents {
    cudaEvent_t a = nullptr, b = nullptr;
    cudaError_t create() {
        cudaError_t e = cudaEventCreate(&a);
        return e == cudaSuccess ? cudaEventCreate(&b) : e;
    }
    ~TimingEvents() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
};
static void keep_pool() {
    int dev = 0;
    cudaMemPool_t pool;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess) return;
    uint64_t keep = 0;
    if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) == cudaSuccess && keep < (4ull << 30)) {
        keep = 4ull << 30;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
}

}  // namespace

int gpu_build_blas(const float* tri_box, uint32_t n_tris, const std::vector<GpuMesh>& meshes, const GpuBvhParams& bp,
                   std::vector<uint32_t>& tri_order, std::vector<GpuTree>& trees, double* device_ms,
                   std::string& err) {
    auto fail = [&](const char* what, cudaError_t e) {
        err = std::string("GPU BVH build: ") + what + ": " + cudaGetErrorString(e);
        return NOOR_ERR_CUDA;
    };
    const uint32_t M = (uint32_t)meshes.size();
    trees.assign(M, GpuTree());
    if (M == 0) return NOOR_OK;
    if (bp.num_bins < 2 || bp.num_bins > kMaxBins) {
        err = "GPU BVH build: num_bins must be in [2, 64]";
        return NOOR_ERR_INVALID;
    }
    if (n_tris >= 0x7fffffffu) {
        err = "GPU BVH build: too many triangles";
        return NOOR_ERR_INVALID;
    }
    Params P;
    P.nb = bp.num_bins;
    P.max_height = bp.max_height;
    P.min_leaf = bp.min_leaf;
    P.max_leaf = bp.max_leaf;
    P.Ci = bp.Ci;
    P.Ct = bp.Ct;
    // a binary tree over n items has 2n - 1 nodes, and a level has at most
    // one task per triangle; empty children (a partition the bins did not
    // foresee) are covered by the slack and otherwise reported as an overflow
    P.cap = 2 * (n_tris + M) + 64;
    P.task_cap = n_tris + 2 * M + 64;
    // a large task has more than kChunk triangles, so it spans fewer than
    // 2 * count / kChunk chunks
    const size_t max_chunks = 2 * ((size_t)n_tris / kChunk) + M + 8;
    const size_t max_large = (size_t)n_tris / kSmallCap + M + 8;

    cudaStream_t s;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail("stream", e);
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } sg{s};
    keep_pool();
    TimingEvents te;
    if ((e = te.create())) return fail("events", e);
    cudaEvent_t ev0 = te.a, ev1 = te.b;

    DevBuf b_box, b_order, b_tmp, b_rank, b_sF, b_sT, b_pred, b_tasks0, b_tasks1, b_recs, b_levels, b_tiny, b_small,
        b_large, b_ctl, b_stats, b_splits, b_chunks, b_c0, b_ctrue, b_cbefore, b_gkeys, b_gcnt, b_meshoff, b_out;
    float* d_box;
    uint32_t *d_order, *d_tmp, *d_rank, *d_sF, *d_sT, *d_levels, *d_tiny, *d_small, *d_large, *d_stats, *d_c0,
        *d_ctrue, *d_cbefore, *d_gcnt, *d_meshoff, *d_out;
    unsigned char* d_pred;
    Task *d_tasks[2];
    Rec* d_recs;
    Ctl* d_ctl;
    Split* d_splits;
    Chunk* d_chunks;
    unsigned long long* d_gkeys;
    const size_t N = n_tris;
    if ((e = dalloc(s, b_box, 6 * N, &d_box)) || (e = dalloc(s, b_order, N, &d_order)) || (e = dalloc(s, b_tmp, N, &d_tmp)) ||
        (e = dalloc(s, b_rank, N, &d_rank)) || (e = dalloc(s, b_sF, N, &d_sF)) || (e = dalloc(s, b_sT, N, &d_sT)) ||
        (e = dalloc(s, b_pred, N, &d_pred)) || (e = dalloc(s, b_tasks0, P.task_cap, &d_tasks[0])) ||
        (e = dalloc(s, b_tasks1, P.task_cap, &d_tasks[1])) || (e = dalloc(s, b_recs, P.cap, &d_recs)) ||
        (e = dalloc(s, b_levels, P.cap, &d_levels)) || (e = dalloc(s, b_tiny, P.task_cap, &d_tiny)) ||
        (e = dalloc(s, b_small, P.task_cap, &d_small)) || (e = dalloc(s, b_large, max_large, &d_large)) ||
        (e = dalloc(s, b_ctl, 1, &d_ctl)) || (e = dalloc(s, b_stats, 4 * (size_t)M, &d_stats)) ||
        (e = dalloc(s, b_splits, max_large, &d_splits)) || (e = dalloc(s, b_chunks, max_chunks, &d_chunks)) ||
        (e = dalloc(s, b_c0, max_large + 1, &d_c0)) || (e = dalloc(s, b_ctrue, max_chunks, &d_ctrue)) ||
        (e = dalloc(s, b_cbefore, max_chunks, &d_cbefore)) ||
        (e = dalloc(s, b_gkeys, max_large * 3 * P.nb * kKeys, &d_gkeys)) ||
        (e = dalloc(s, b_gcnt, max_large * 3 * P.nb, &d_gcnt)) || (e = dalloc(s, b_meshoff, M, &d_meshoff)))
        return fail("allocation", e);

    // kernel shared memory
    const SmallSmem tiny_l = small_layout(P.nb, kTinyCap, 32), small_l = small_layout(P.nb, kSmallCap, 256);
    const size_t bin_smem = (size_t)3 * P.nb * kKeys * 8 + (size_t)3 * P.nb * 4 + (size_t)2 * 3 * P.nb * 4;
    const size_t dec_smem = (size_t)4 * 3 * P.nb * sizeof(DBox) + (size_t)2 * 3 * P.nb * 4 + 3 * sizeof(AxisBest) +
                            (size_t)2 * 3 * P.nb * 4;
    if ((e = cudaFuncSetAttribute(k_split<32, kTinyCap>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)tiny_l.total)) ||
        (e = cudaFuncSetAttribute(k_split<256, kSmallCap>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)small_l.total)) ||
        (e = cudaFuncSetAttribute(k_bin_large, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bin_smem)) ||
        (e = cudaFuncSetAttribute(k_decide_large, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dec_smem)))
        return fail("shared memory", e);

    // inputs and the roots (records 0..M-1, one task per mesh)
    std::vector<Task> roots(M);
    for (uint32_t i = 0; i < M; ++i) {
        Task& t = roots[i];
        t.start = meshes[i].start;
        t.count = meshes[i].count;
        t.rec = i;
        t.level = 0;
        t.mesh = i;
        std::memcpy(t.box, meshes[i].box, 24);
        std::memcpy(t.cbox, meshes[i].cbox, 24);
        if ((size_t)t.start + t.count > N) {
            err = "GPU BVH build: mesh range outside the triangles";
            return NOOR_ERR_INVALID;
        }
    }
    cudaEventRecord(ev0, s);
    if ((e = cudaMemcpyAsync(d_box, tri_box, 24 * N, cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(d_order, tri_order.data(), 4 * N, cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(d_tasks[0], roots.data(), sizeof(Task) * M, cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemsetAsync(d_stats, 0, 16 * (size_t)M, s)))
        return fail("upload", e);
    Ctl ctl{};
    ctl.n_rec = M;
    if ((e = cudaMemcpyAsync(d_ctl, &ctl, sizeof(Ctl), cudaMemcpyHostToDevice, s))) return fail("upload", e);

    std::vector<uint32_t> level_off{0};
    uint32_t n_cur = M;
    int cur = 0;
    std::vector<Task> ltasks;
    std::vector<Chunk> chunks;
    std::vector<uint32_t> c0;
    for (uint32_t level = 0; n_cur > 0; ++level) {
        if (level > bp.max_height + 1 || level_off.back() + (size_t)n_cur > P.cap || n_cur > P.task_cap) {
            err = "GPU BVH build: tree deeper or larger than expected";
            return NOOR_ERR_CAPACITY;
        }
        Out o{d_recs, d_tasks[cur ^ 1], d_ctl, d_stats};
        // reset the per-level counters
        Ctl* c = d_ctl;
        if ((e = cudaMemsetAsync(&c->n_next, 0, 4, s)) || (e = cudaMemsetAsync(&c->n_tiny, 0, 12, s)))
            return fail("level reset", e);
        k_classify<<<(n_cur + 255) / 256, 256, 0, s>>>(d_tasks[cur], n_cur, P, o, d_tiny, d_small, d_large,
                                                      d_levels + level_off.back());
        Ctl h{};
        if ((e = cudaMemcpyAsync(&h, d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s)) ||
            (e = cudaStreamSynchronize(s)))
            return fail("classify", e);
        if (h.n_tiny)
            k_split<32, kTinyCap><<<h.n_tiny, 32, tiny_l.total, s>>>(d_tasks[cur], d_tiny, d_box, d_order, P, o);
        if (h.n_small)
            k_split<256, kSmallCap><<<h.n_small, 256, small_l.total, s>>>(d_tasks[cur], d_small, d_box, d_order, P,
                                                                         o);
        if (h.n_large) {
            if (h.n_large > max_large) {
                err = "GPU BVH build: too many large tasks";
                return NOOR_ERR_CAPACITY;
            }
            // chunk table on the host (large tasks are few; a level that has
            // them has few tasks in all)
            std::vector<uint32_t> lidx(h.n_large);
            ltasks.resize(n_cur);
            if ((e = cudaMemcpyAsync(lidx.data(), d_large, 4 * (size_t)h.n_large, cudaMemcpyDeviceToHost, s)) ||
                (e = cudaMemcpyAsync(ltasks.data(), d_tasks[cur], sizeof(Task) * (size_t)n_cur, cudaMemcpyDeviceToHost,
                                     s)) ||
                (e = cudaStreamSynchronize(s)))
                return fail("large list", e);
            chunks.clear();
            c0.assign(h.n_large + 1, 0);
            for (uint32_t j = 0; j < h.n_large; ++j) {
                const Task& t = ltasks[lidx[j]];
                c0[j] = (uint32_t)chunks.size();
                for (uint32_t b = 0; b < t.count; b += kChunk) chunks.push_back(Chunk{j, b, std::min(t.count, b + kChunk)});
            }
            c0[h.n_large] = (uint32_t)chunks.size();
            const uint32_t nc = (uint32_t)chunks.size();
            if (nc > max_chunks) {
                err = "GPU BVH build: too many chunks";
                return NOOR_ERR_CAPACITY;
            }
            const uint32_t nbins = h.n_large * 3 * P.nb;
            if ((e = cudaMemcpyAsync(d_chunks, chunks.data(), sizeof(Chunk) * nc, cudaMemcpyHostToDevice, s)) ||
                (e = cudaMemcpyAsync(d_c0, c0.data(), 4 * c0.size(), cudaMemcpyHostToDevice, s)))
                return fail("chunk table", e);
            k_init_large_keys<<<(nbins + 255) / 256, 256, 0, s>>>(d_gkeys, d_gcnt, nbins);
            k_bin_large<<<nc, 256, bin_smem, s>>>(d_tasks[cur], d_large, d_chunks, d_box, d_order, P, d_gkeys, d_gcnt);
            k_decide_large<<<h.n_large, 32, dec_smem, s>>>(d_tasks[cur], d_large, P, d_gkeys, d_gcnt, d_splits, o);
            k_count_large<<<nc, 256, 0, s>>>(d_tasks[cur], d_large, d_chunks, d_splits, d_box, d_order, d_ctrue);
            k_scan_emit_large<<<(h.n_large + 63) / 64, 64, 0, s>>>(d_tasks[cur], d_large, h.n_large, d_c0, d_ctrue,
                                                                  d_cbefore, d_splits, P, o);
            k_rank_large<<<nc, 256, 0, s>>>(d_tasks[cur], d_large, d_chunks, d_c0, d_ctrue, d_cbefore, d_splits,
                                            d_box, d_order, d_rank, d_sF, d_sT, d_pred);
            k_scatter_large<<<nc, 256, 0, s>>>(d_tasks[cur], d_large, d_chunks, d_c0, d_ctrue, d_splits, d_order,
                                               d_rank, d_sF, d_sT, d_pred, d_tmp);
            k_copy_large<<<nc, 256, 0, s>>>(d_tasks[cur], d_large, d_chunks, d_splits, d_tmp, d_order);
        }
        if ((e = cudaGetLastError())) return fail("level kernels", e);
        if ((e = cudaMemcpyAsync(&h, d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s)) || (e = cudaStreamSynchronize(s)))
            return fail("level", e);
        if (h.overflow) {
            err = "GPU BVH build: node capacity exceeded";
            return NOOR_ERR_CAPACITY;
        }
        level_off.push_back(level_off.back() + n_cur);
        n_cur = h.n_next;
        cur ^= 1;
    }
    Ctl h{};
    if ((e = cudaMemcpyAsync(&h, d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s)) || (e = cudaStreamSynchronize(s)))
        return fail("records", e);
    const uint32_t n_rec = h.n_rec;
    const uint32_t n_levels = (uint32_t)level_off.size() - 1;
    for (uint32_t l = n_levels; l-- > 0;) {
        const uint32_t n = level_off[l + 1] - level_off[l];
        k_sizes<<<(n + 255) / 256, 256, 0, s>>>(d_recs, d_levels + level_off[l], n);
    }
    // roots: depth-first index 0 within their mesh's tree
    for (uint32_t i = 0; i < M; ++i)
        if ((e = cudaMemsetAsync(&d_recs[i].dfs, 0, 4, s))) return fail("roots", e);
    for (uint32_t l = 0; l < n_levels; ++l) {
        const uint32_t n = level_off[l + 1] - level_off[l];
        k_dfs<<<(n + 255) / 256, 256, 0, s>>>(d_recs, d_levels + level_off[l], n);
    }
    std::vector<Rec> root_recs(M);
    if ((e = cudaMemcpyAsync(root_recs.data(), d_recs, sizeof(Rec) * M, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaStreamSynchronize(s)))
        return fail("sizes", e);
    std::vector<uint32_t> mesh_off(M);
    size_t total = 0;
    for (uint32_t i = 0; i < M; ++i) {
        mesh_off[i] = (uint32_t)total;
        total += root_recs[i].size;
    }
    if (total != n_rec) {
        err = "GPU BVH build: record count mismatch";
        return NOOR_ERR_CUDA;
    }
    if ((e = dalloc(s, b_out, 8 * total, &d_out)) ||
        (e = cudaMemcpyAsync(d_meshoff, mesh_off.data(), 4 * (size_t)M, cudaMemcpyHostToDevice, s)))
        return fail("output", e);
    k_write<<<(n_rec + 255) / 256, 256, 0, s>>>(d_recs, n_rec, d_meshoff, d_out);
    std::vector<uint32_t> words(8 * total), stats(4 * (size_t)M);
    cudaEventRecord(ev1, s);
    if ((e = cudaGetLastError()) ||
        (e = cudaMemcpyAsync(words.data(), d_out, 32 * total, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(tri_order.data(), d_order, 4 * N, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(stats.data(), d_stats, 16 * (size_t)M, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaStreamSynchronize(s)))
        return fail("download", e);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    if (device_ms) *device_ms = ms;
    for (uint32_t i = 0; i < M; ++i) {
        GpuTree& t = trees[i];
        t.nodes.assign(words.begin() + 8 * (size_t)mesh_off[i], words.begin() + 8 * ((size_t)mesh_off[i] + root_recs[i].size));
        t.height = stats[4 * i];
        t.num_inner = stats[4 * i + 1];
        t.num_leaf = stats[4 * i + 2];
        t.max_leaf_tris = stats[4 * i + 3];
    }
    return NOOR_OK;
}

int gpu_payload_tail(const GpuTailIn& in, GpuTailOut& out, double* device_ms, std::string& err) {
    auto fail = [&](const char* what, cudaError_t e) {
        err = std::string("GPU payload: ") + what + ": " + cudaGetErrorString(e);
        return NOOR_ERR_CUDA;
    };
    const size_t T = in.n_tris, C = 3 * T;
    if (C >= 0x7fffffffu) {
        err = "GPU payload: too many triangles";
        return NOOR_ERR_INVALID;
    }
    size_t cap = 16;
    while (cap < 2 * C) cap <<= 1;
    const uint32_t nblk = (uint32_t)((C + kScanBlock - 1) / kScanBlock);
    cudaStream_t s;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail("stream", e);
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } sg{s};
    keep_pool();
    TimingEvents te;
    if ((e = te.create())) return fail("events", e);
    cudaEvent_t ev0 = te.a, ev1 = te.b;
    DevBuf b_order, b_vi, b_ni, b_ui, b_vtx, b_nrm, b_uv, b_mi, b_mt, b_slots, b_pmin, b_cs, b_flag, b_first, b_sums,
        b_total, b_fail, b_ovtx, b_onrm, b_ouv, b_w0, b_w1, b_w2, b_attr;
    uint32_t *d_order, *d_vi, *d_ni, *d_ui, *d_mi, *d_mt, *d_slots, *d_pmin, *d_cs, *d_flag, *d_first, *d_sums,
        *d_total, *d_fail;
    float4 *d_vtx, *d_nrm, *d_ovtx, *d_onrm;
    float2 *d_uv, *d_ouv;
    uint4 *d_w0, *d_w1, *d_w2, *d_attr;
    if ((e = dalloc(s, b_order, T, &d_order)) || (e = dalloc(s, b_vi, C, &d_vi)) || (e = dalloc(s, b_ni, C, &d_ni)) ||
        (e = dalloc(s, b_ui, C, &d_ui)) || (e = dalloc(s, b_vtx, in.n_vertices, &d_vtx)) ||
        (e = dalloc(s, b_nrm, in.n_normals, &d_nrm)) || (e = dalloc(s, b_uv, in.n_uvs, &d_uv)) ||
        (e = dalloc(s, b_mi, T, &d_mi)) || (e = dalloc(s, b_mt, in.n_materials, &d_mt)) ||
        (e = dalloc(s, b_slots, cap, &d_slots)) || (e = dalloc(s, b_pmin, cap, &d_pmin)) || (e = dalloc(s, b_cs, C, &d_cs)) ||
        (e = dalloc(s, b_flag, C, &d_flag)) || (e = dalloc(s, b_first, C, &d_first)) ||
        (e = dalloc(s, b_sums, nblk, &d_sums)) || (e = dalloc(s, b_total, 1, &d_total)) ||
        (e = dalloc(s, b_fail, 1, &d_fail)) || (e = dalloc(s, b_w0, T, &d_w0)) || (e = dalloc(s, b_w1, T, &d_w1)) ||
        (e = dalloc(s, b_w2, T, &d_w2)) || (e = dalloc(s, b_attr, T, &d_attr)))
        return fail("allocation", e);
    cudaEventRecord(ev0, s);
    if ((e = cudaMemcpyAsync(d_order, in.tri_order, 4 * T, cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(d_vi, in.vindices, 4 * C, cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(d_ni, in.nindices, 4 * C, cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(d_ui, in.uvindices, 4 * C, cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(d_vtx, in.vertices, 16 * (size_t)in.n_vertices, cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(d_nrm, in.normals, 16 * (size_t)in.n_normals, cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(d_uv, in.uvs, 8 * (size_t)in.n_uvs, cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(d_mi, in.material_indices, 4 * T, cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(d_mt, in.material_types, 4 * (size_t)in.n_materials, cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemsetAsync(d_slots, 0xff, 4 * cap, s)) || (e = cudaMemsetAsync(d_pmin, 0xff, 4 * cap, s)) ||
        (e = cudaMemsetAsync(d_fail, 0, 4, s)))
        return fail("upload", e);
    TailArgs A{d_order, d_vi, d_ni, d_ui, (uint32_t)C, d_slots, d_pmin, d_cs, (uint32_t)(cap - 1), d_fail};
    const uint32_t g = (uint32_t)((C + 255) / 256);
    k_dedup_insert<<<g, 256, 0, s>>>(A);
    k_dedup_flags<<<g, 256, 0, s>>>(A, d_flag);
    k_scan_sums<<<nblk, kScanBlock, 0, s>>>(d_flag, (uint32_t)C, d_sums);
    k_scan_top<<<1, kScanBlock, 0, s>>>(d_sums, nblk, d_total);
    k_scan_block<<<nblk, kScanBlock, 0, s>>>(d_flag, (uint32_t)C, d_sums, d_first);
    uint32_t nv = 0, failed = 0;
    if ((e = cudaGetLastError()) || (e = cudaMemcpyAsync(&nv, d_total, 4, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(&failed, d_fail, 4, cudaMemcpyDeviceToHost, s)) || (e = cudaStreamSynchronize(s)))
        return fail("de-duplication", e);
    if (failed) {
        err = "GPU payload: vertex table full";
        return NOOR_ERR_CAPACITY;
    }
    if ((e = dalloc(s, b_ovtx, nv, &d_ovtx)) || (e = dalloc(s, b_onrm, nv, &d_onrm)) || (e = dalloc(s, b_ouv, nv, &d_ouv)))
        return fail("allocation", e);
    k_dedup_vertices<<<g, 256, 0, s>>>(A, d_flag, d_first, d_vtx, d_nrm, d_uv, d_ovtx, d_onrm, d_ouv);
    k_wald<<<(uint32_t)((T + 255) / 256), 256, 0, s>>>(A, d_first, (uint32_t)T, d_ovtx, d_mi, d_mt, d_w0, d_w1, d_w2,
                                                       d_attr);
    cudaEventRecord(ev1, s);
    out.vertices.resize(4 * (size_t)nv);
    out.normals.resize(4 * (size_t)nv);
    out.uvs.resize(2 * (size_t)nv);
    for (auto* w : {&out.wald[0], &out.wald[1], &out.wald[2], &out.attr}) w->resize(4 * T);
    if ((e = cudaGetLastError()) ||
        (e = cudaMemcpyAsync(out.vertices.data(), d_ovtx, 16 * (size_t)nv, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(out.normals.data(), d_onrm, 16 * (size_t)nv, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(out.uvs.data(), d_ouv, 8 * (size_t)nv, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(out.wald[0].data(), d_w0, 16 * T, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(out.wald[1].data(), d_w1, 16 * T, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(out.wald[2].data(), d_w2, 16 * T, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(out.attr.data(), d_attr, 16 * T, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaStreamSynchronize(s)))
        return fail("download", e);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    if (device_ms) *device_ms = ms;
    return NOOR_OK;
}

}  // namespace nbg
