// Host scene builder: the work Model::load, BVH::build and
// Model::loadCudaPayload do before Noor hands a CudaPayload to the device
// (noor/source/model.cpp:73-458, noor/source/bvh.cpp:29-258,
// noor/source/splitter.cpp:28-161).  The output arrays are byte-identical to
// the reference's for the same input, because every step that fixes a bit of
// the output follows the reference's definition:
//   * boxes: component-wise min/max returning the first operand on ties
//     (glm::min/max), centroid (min+max)*0.5, surface area
//     2*((dx*dy + dy*dz) + dx*dz), infinite for non-finite boxes;
//   * binning: num_bins equal slabs of the centroid box whose edges are
//     accumulated by repeated addition of the slab width, last edge pinned to
//     the box maximum; a centroid goes to the first bin whose upper edge is
//     >= it;
//   * SAH: Ct + Ci*(nL*SA_L + nR*SA_R)/SA_parent over the num_bins-1 planes
//     of each axis, first minimum wins, axes in x,y,z order;
//   * leaf rules, depth-first node order (left child = next node), the
//     partition of triangle indices by std::partition with the same
//     predicate, a two-level build (per-mesh trees, then a top tree over
//     mesh instance boxes);
//   * vertex de-duplication on (vertex, normal, uv) index triples in
//     BVH triangle order, Wald precomputation per triangle.
#include <algorithm>
#include <atomic>
#include <exception>
#include <thread>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/noor_b200.h"
#include "bvh_gpu.h"
#include "host_common.h"

namespace nbh {

// ------------------------------------------------------------------ boxes
static inline float mn(float a, float b) { return (b < a) ? b : a; }
static inline float mx(float a, float b) { return (a < b) ? b : a; }

struct V3 {
    float x, y, z;
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
static inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
static inline V3 vadd(const V3& a, const V3& b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 vsub(const V3& a, const V3& b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 vscale(const V3& a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
static inline V3 vmin(const V3& a, const V3& b) { return v3(mn(a.x, b.x), mn(a.y, b.y), mn(a.z, b.z)); }
static inline V3 vmax(const V3& a, const V3& b) { return v3(mx(a.x, b.x), mx(a.y, b.y), mx(a.z, b.z)); }

struct Box {
    V3 lo{kInfF, kInfF, kInfF};
    V3 hi{-kInfF, -kInfF, -kInfF};
    static constexpr float kInfF = std::numeric_limits<float>::infinity();
    void merge(const Box& b) {
        lo = vmin(lo, b.lo);
        hi = vmax(hi, b.hi);
    }
    void include(const V3& p) {
        lo = vmin(lo, p);
        hi = vmax(hi, p);
    }
    V3 centroid() const { return vscale(vadd(lo, hi), 0.5f); }
    bool valid() const {
        const float c[6] = {lo.x, lo.y, lo.z, hi.x, hi.y, hi.z};
        for (float v : c)
            if (std::isinf(v) || std::isnan(v)) return false;
        return true;
    }
    float area() const {
        const V3 d = vsub(hi, lo);
        if (!valid()) return std::numeric_limits<float>::infinity();
        return 2.0f * (d.x * d.y + d.y * d.z + d.x * d.z);
    }
    float radius() const {
        const V3 d = vsub(hi, lo);
        return 0.5f * std::sqrt(d.x * d.x + d.y * d.y + d.z * d.z);
    }
};
static inline Box merged(const Box& a, const Box& b) {
    Box r = a;
    r.merge(b);
    return r;
}

static inline uint32_t f2u(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

// column-major 4x4 (glm layout) times point (x,y,z,1), summed as
// (c0*x + c1*y) + (c2*z + c3*w) like glm's mat4*vec4
static inline V3 xform_point(const float* m, const V3& p) {
    float r[3];
    for (int i = 0; i < 3; ++i) {
        const float a0 = m[0 + i] * p.x, a1 = m[4 + i] * p.y, a2 = m[8 + i] * p.z, a3 = m[12 + i] * 1.0f;
        r[i] = (a0 + a1) + (a2 + a3);
    }
    return v3(r[0], r[1], r[2]);
}
// BBox operator*(mat4, BBox): box of the 8 transformed corners
static Box xform_box(const float* m, const Box& b) {
    V3 p[8];
    p[0] = xform_point(m, v3(b.lo.x, b.lo.y, b.lo.z));
    p[1] = xform_point(m, v3(b.lo.x, b.lo.y, b.hi.z));
    p[2] = xform_point(m, v3(b.lo.x, b.hi.y, b.lo.z));
    p[3] = xform_point(m, v3(b.lo.x, b.hi.y, b.hi.z));
    p[4] = xform_point(m, v3(b.hi.x, b.lo.y, b.lo.z));
    p[5] = xform_point(m, v3(b.hi.x, b.lo.y, b.hi.z));
    p[6] = xform_point(m, v3(b.hi.x, b.hi.y, b.lo.z));
    p[7] = xform_point(m, v3(b.hi.x, b.hi.y, b.hi.z));
    Box r;
    r.lo = vmin(vmin(vmin(vmin(p[0], p[1]), p[2]), p[3]), p[4]);
    r.lo = vmin(vmin(vmin(r.lo, p[5]), p[6]), p[7]);
    r.hi = vmax(vmax(vmax(vmax(p[0], p[1]), p[2]), p[3]), p[4]);
    r.hi = vmax(vmax(vmax(r.hi, p[5]), p[6]), p[7]);
    return r;
}

// ------------------------------------------------------------ matrices
static void inverse4(const float* m, float* out) {
    double a[16], inv[16];
    for (int i = 0; i < 16; ++i) a[i] = m[i];
    inv[0] = a[5] * a[10] * a[15] - a[5] * a[11] * a[14] - a[9] * a[6] * a[15] + a[9] * a[7] * a[14] +
             a[13] * a[6] * a[11] - a[13] * a[7] * a[10];
    inv[4] = -a[4] * a[10] * a[15] + a[4] * a[11] * a[14] + a[8] * a[6] * a[15] - a[8] * a[7] * a[14] -
             a[12] * a[6] * a[11] + a[12] * a[7] * a[10];
    inv[8] = a[4] * a[9] * a[15] - a[4] * a[11] * a[13] - a[8] * a[5] * a[15] + a[8] * a[7] * a[13] +
             a[12] * a[5] * a[11] - a[12] * a[7] * a[9];
    inv[12] = -a[4] * a[9] * a[14] + a[4] * a[10] * a[13] + a[8] * a[5] * a[14] - a[8] * a[6] * a[13] -
              a[12] * a[5] * a[10] + a[12] * a[6] * a[9];
    inv[1] = -a[1] * a[10] * a[15] + a[1] * a[11] * a[14] + a[9] * a[2] * a[15] - a[9] * a[3] * a[14] -
             a[13] * a[2] * a[11] + a[13] * a[3] * a[10];
    inv[5] = a[0] * a[10] * a[15] - a[0] * a[11] * a[14] - a[8] * a[2] * a[15] + a[8] * a[3] * a[14] +
             a[12] * a[2] * a[11] - a[12] * a[3] * a[10];
    inv[9] = -a[0] * a[9] * a[15] + a[0] * a[11] * a[13] + a[8] * a[1] * a[15] - a[8] * a[3] * a[13] -
             a[12] * a[1] * a[11] + a[12] * a[3] * a[9];
    inv[13] = a[0] * a[9] * a[14] - a[0] * a[10] * a[13] - a[8] * a[1] * a[14] + a[8] * a[2] * a[13] +
              a[12] * a[1] * a[10] - a[12] * a[2] * a[9];
    inv[2] = a[1] * a[6] * a[15] - a[1] * a[7] * a[14] - a[5] * a[2] * a[15] + a[5] * a[3] * a[14] +
             a[13] * a[2] * a[7] - a[13] * a[3] * a[6];
    inv[6] = -a[0] * a[6] * a[15] + a[0] * a[7] * a[14] + a[4] * a[2] * a[15] - a[4] * a[3] * a[14] -
             a[12] * a[2] * a[7] + a[12] * a[3] * a[6];
    inv[10] = a[0] * a[5] * a[15] - a[0] * a[7] * a[13] - a[4] * a[1] * a[15] + a[4] * a[3] * a[13] +
              a[12] * a[1] * a[7] - a[12] * a[3] * a[5];
    inv[14] = -a[0] * a[5] * a[14] + a[0] * a[6] * a[13] + a[4] * a[1] * a[14] - a[4] * a[2] * a[13] -
              a[12] * a[1] * a[6] + a[12] * a[2] * a[5];
    inv[3] = -a[1] * a[6] * a[11] + a[1] * a[7] * a[10] + a[5] * a[2] * a[11] - a[5] * a[3] * a[10] -
             a[9] * a[2] * a[7] + a[9] * a[3] * a[6];
    inv[7] = a[0] * a[6] * a[11] - a[0] * a[7] * a[10] - a[4] * a[2] * a[11] + a[4] * a[3] * a[10] +
             a[8] * a[2] * a[7] - a[8] * a[3] * a[6];
    inv[11] = -a[0] * a[5] * a[11] + a[0] * a[7] * a[9] + a[4] * a[1] * a[11] - a[4] * a[3] * a[9] -
              a[8] * a[1] * a[7] + a[8] * a[3] * a[5];
    inv[15] = a[0] * a[5] * a[10] - a[0] * a[6] * a[9] - a[4] * a[1] * a[10] + a[4] * a[2] * a[9] +
              a[8] * a[1] * a[6] - a[8] * a[2] * a[5];
    double det = a[0] * inv[0] + a[1] * inv[4] + a[2] * inv[8] + a[3] * inv[12];
    det = 1.0 / det;
    for (int i = 0; i < 16; ++i) out[i] = (float)(inv[i] * det);
}

// ------------------------------------------------------------- builder
enum BinKind { kTriBin = 0, kMeshBin = 1 };

struct AttrKey {
    uint32_t v, n, u;
    bool operator==(const AttrKey& o) const { return v == o.v && n == o.n && u == o.u; }
};
struct AttrKeyHash {
    size_t operator()(const AttrKey& k) const {
        uint64_t h = (uint64_t)k.v * 0x9E3779B97F4A7C15ull;
        h ^= (uint64_t)k.n * 0xC2B2AE3D27D4EB4Full + (h << 6) + (h >> 2);
        h ^= (uint64_t)k.u * 0x165667B19E3779F9ull + (h << 6) + (h >> 2);
        return (size_t)h;
    }
};


// Vertex de-duplication of the corners in BVH order on all host threads,
// numbered as a sequential find-or-insert pass numbers them (the first
// occurrence of a (vertex, normal, uv) triple takes the next index): every
// corner finds its key's slot in one open-addressing table (a slot holds any
// corner with that key), the key keeps its first corner by an atomic
// minimum, and a prefix count over the "first corner" flags numbers the new
// vertices.  element[p] = new index of corner p; first[k] = the corner that
// introduced new vertex k.  Returns the number of new vertices.
template <class Key>
static uint32_t dedup_corners(size_t C, const Key& key, std::vector<uint32_t>& element, std::vector<uint32_t>& first) {
    constexpr uint32_t kEmpty = 0xFFFFFFFFu;
    size_t cap = 16;
    while (cap < 2 * C) cap <<= 1;
    const size_t mask = cap - 1;
    std::unique_ptr<std::atomic<uint32_t>[]> slot(new std::atomic<uint32_t>[cap]);
    std::unique_ptr<std::atomic<uint32_t>[]> pmin(new std::atomic<uint32_t>[cap]);
    std::vector<uint32_t> cslot(C), id(C);
    const uint32_t nt = std::max(1u, std::min(std::thread::hardware_concurrency(), (uint32_t)(C / 65536 + 1)));
    auto chunks = [&](size_t n, const auto& f) {  // f(thread, begin, end) on nt contiguous chunks
        std::vector<std::thread> pool;
        const size_t per = (n + nt - 1) / nt;
        for (uint32_t t = 0; t < nt; ++t) {
            const size_t b = t * per, e = std::min(n, b + per);
            if (b >= e) break;
            pool.emplace_back([&f, t, b, e]() { f(t, b, e); });
        }
        for (auto& th : pool) th.join();
    };
    chunks(cap, [&](uint32_t, size_t b, size_t e) {
        for (size_t i = b; i < e; ++i) {
            slot[i].store(kEmpty, std::memory_order_relaxed);
            pmin[i].store(kEmpty, std::memory_order_relaxed);
        }
    });
    chunks(C, [&](uint32_t, size_t b, size_t e) {
        for (size_t p = b; p < e; ++p) {
            const AttrKey k = key(p);
            for (size_t i = AttrKeyHash()(k) & mask;; i = (i + 1) & mask) {
                uint32_t s = slot[i].load(std::memory_order_acquire);
                if (s == kEmpty) {
                    uint32_t expect = kEmpty;
                    if (slot[i].compare_exchange_strong(expect, (uint32_t)p, std::memory_order_acq_rel))
                        s = (uint32_t)p;
                    else
                        s = expect;
                }
                if (key(s) == k) {
                    cslot[p] = (uint32_t)i;
                    uint32_t cur = pmin[i].load(std::memory_order_relaxed);
                    while (p < cur && !pmin[i].compare_exchange_weak(cur, (uint32_t)p, std::memory_order_relaxed)) {
                    }
                    break;
                }
            }
        }
    });
    std::vector<uint32_t> count(nt, 0);
    chunks(C, [&](uint32_t t, size_t b, size_t e) {
        uint32_t c = 0;
        for (size_t p = b; p < e; ++p) c += pmin[cslot[p]].load(std::memory_order_relaxed) == p ? 1u : 0u;
        count[t] = c;
    });
    std::vector<uint32_t> off(nt, 0);
    uint32_t nv = 0;
    for (uint32_t t = 0; t < nt; ++t) {
        off[t] = nv;
        nv += count[t];
    }
    first.resize(nv);
    chunks(C, [&](uint32_t t, size_t b, size_t e) {
        uint32_t k = off[t];
        for (size_t p = b; p < e; ++p)
            if (pmin[cslot[p]].load(std::memory_order_relaxed) == p) {
                id[p] = k;
                first[k] = (uint32_t)p;
                ++k;
            }
    });
    element.resize(C);
    chunks(C, [&](uint32_t, size_t b, size_t e) {
        for (size_t p = b; p < e; ++p) element[p] = id[pmin[cslot[p]].load(std::memory_order_relaxed)];
    });
    return nv;
}

// f(i) for i in [0, n) on all host threads (contiguous chunks)
template <class F>
static void parallel_for(uint32_t n, const F& f) {
    const uint32_t nt = std::max(1u, std::min(std::thread::hardware_concurrency(), (n + 65535u) / 65536u));
    std::vector<std::thread> pool;
    const uint32_t chunk = (n + nt - 1) / nt;
    for (uint32_t t = 0; t < nt; ++t) {
        const uint32_t b = t * chunk, e = std::min(n, b + chunk);
        if (b >= e) break;
        pool.emplace_back([&f, b, e]() {
            for (uint32_t i = b; i < e; ++i) f(i);
        });
    }
    for (auto& th : pool) th.join();
}

struct Range {
    uint32_t* b;
    uint32_t* e;
    Box box;
    Box cbox;
    BinKind kind;
    uint32_t count() const { return (uint32_t)(e - b); }
};

struct Plane {
    float cost = std::numeric_limits<float>::infinity();
    uint32_t axis = 0;
    uint32_t index = 0;
    uint32_t nl = 0, nr = 0;
    bool valid() const { return cost != std::numeric_limits<float>::infinity() && nl != 0 && nr != 0; }
};

struct MeshInfo {
    Box box, cbox, ibox, icbox;
    const noor_mesh* src;
};

// Per-tree state of a build: split scratch, the nodes of the tree, and its
// statistics.  Each mesh's tree is built in its own Work (on its own host
// thread); node indices written into a tree are relative to `base`.
struct Work {
    uint32_t nb = 0;
    std::vector<Box> edge;  // slab edges: edge[i].lo/.hi = lower/upper edge
    std::vector<Box> L[3], R[3], LC[3], RC[3];
    std::vector<uint32_t> NL[3], NR[3];
    std::vector<uint32_t> nodes;  // 8 words per node: min.xyz,w0,max.xyz,w1
    uint32_t base = 0;            // index of nodes[0] in the final node array
    noor_build_stat stat{};
    void init(uint32_t bins) {
        nb = bins;
        edge.assign(nb, Box());
        for (int a = 0; a < 3; ++a) {
            L[a].assign(nb, Box());
            R[a].assign(nb, Box());
            LC[a].assign(nb, Box());
            RC[a].assign(nb, Box());
            NL[a].assign(nb, 0u);
            NR[a].assign(nb, 0u);
        }
    }
};

// a failure of the GPU tree build
struct GpuBuildError {
    int code;
    std::string msg;
};

class Builder {
public:
    Builder(const noor_scene_desc& d, bool gpu) : D(d), use_gpu(gpu) {}

    const noor_scene_desc& D;
    bool use_gpu;  // bottom-level trees built on the current CUDA device
    // host trees: subtrees of large ranges above this level are built on
    // threads of their own (when meshes are fewer than threads)
    uint32_t par_levels = 0;
    static constexpr uint32_t kParMinTris = 32768;
    std::vector<Box> tri_box;
    std::vector<MeshInfo> meshes;
    Box scene_box, scene_cbox;
    std::vector<uint32_t> tri_order, mesh_order, mesh_start;
    std::vector<uint32_t> nodes;  // the final node array: mesh trees in mesh order, then the top tree
    uint32_t root = 0;
    noor_build_stat stat{};
    double gpu_ms = 0.0;

    V3 vtx(uint32_t t, int k) const {
        const float* p = D.vertices + 4 * (size_t)D.vindices[3 * (size_t)t + k];
        return v3(p[0], p[1], p[2]);
    }

    // Model::computeBBoxes (model.cpp:73-108); light meshes take the bounds
    // of their shape (CudaShape::getBounds, shape.cuh:71-90)
    void compute_boxes() {
        tri_box.resize(D.num_triangles);
        meshes.resize(D.num_meshes);
        for (uint32_t i = 0; i < D.num_meshes; ++i) {
            const noor_mesh& m = D.meshes[i];
            meshes[i].src = &m;
            if (m.light_idx >= 0 || m.instance >= 0) continue;
            Box mb, mc;
            for (uint32_t t = m.tri_start; t < m.tri_start + m.tri_count; ++t) {
                Box tb;
                const V3 a = vtx(t, 0), b = vtx(t, 1), c = vtx(t, 2);
                tb.lo = vmin(vmin(a, b), c);
                tb.hi = vmax(vmax(a, b), c);
                tri_box[t] = tb;
                mb.merge(tb);
                mc.include(tb.centroid());
            }
            meshes[i].box = mb;
            meshes[i].cbox = mc;
        }
        for (uint32_t i = 0; i < D.num_meshes; ++i) {
            const noor_mesh& m = D.meshes[i];
            MeshInfo& mi = meshes[i];
            if (m.light_idx >= 0) {
                const noor_shape& s = D.area_lights[m.light_idx].shape;
                V3 c = v3(s.center[0], s.center[1], s.center[2]);
                V3 u = v3(s.u[0], s.u[1], s.u[2]), v = v3(s.v[0], s.v[1], s.v[2]);
                Box b;
                if (s.type == NOOR_SHAPE_SPHERE) {
                    const V3 r = v3(s.radius, s.radius, s.radius);
                    b.lo = vsub(c, r);
                    b.hi = vadd(c, r);
                } else if (s.type == NOOR_SHAPE_DISK) {
                    // the four points at radius along +-u and +-v (unit)
                    auto unit = [](const V3& a) { return vscale(a, 1.0f / std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z)); };
                    const V3 un = unit(u), vn = unit(v);
                    const V3 pr = vadd(c, vscale(un, s.radius)), pt = vadd(c, vscale(vn, s.radius));
                    const V3 pl = vsub(c, vscale(un, s.radius)), pb = vsub(c, vscale(vn, s.radius));
                    b.lo = vmin(vmin(vmin(pl, pr), pt), pb);
                    b.hi = vmax(vmax(vmax(pl, pr), pt), pb);
                } else {
                    const V3 cu = vadd(c, u), cv = vadd(c, v), cuv = vadd(vadd(c, u), v);
                    b.lo = vmin(vmin(vmin(c, cu), cv), cuv);
                    b.hi = vmax(vmax(vmax(c, cu), cv), cuv);
                }
                mi.box = mi.ibox = b;
                mi.cbox.lo = mi.cbox.hi = b.centroid();
                mi.icbox = mi.cbox;
            } else {
                if (m.instance >= 0) {
                    mi.box = meshes[m.instance].box;
                    mi.cbox = meshes[m.instance].cbox;
                }
                mi.ibox = xform_box(m.to_global, mi.box);
                mi.icbox = xform_box(m.to_global, mi.cbox);
            }
            scene_box.merge(mi.ibox);
            scene_cbox.include(mi.ibox.centroid());
        }
    }

    const Box& item_box(BinKind k, uint32_t i) const { return k == kTriBin ? tri_box[i] : meshes[i].ibox; }

    void reset_split(Work& w, const Range& r) const {
        const uint32_t nb = w.nb;
        const V3 cl = r.cbox.lo, ch = r.cbox.hi;
        const float inv = 1.0f / (float)nb;
        const V3 dt = vscale(vsub(ch, cl), inv);
        w.edge[0].lo = cl;
        w.edge[0].hi = vadd(cl, dt);
        for (uint32_t i = 1; i < nb; ++i) {
            w.edge[i].lo = vadd(w.edge[i - 1].lo, dt);
            w.edge[i].hi = vadd(w.edge[i - 1].hi, dt);
        }
        w.edge[nb - 1].hi = ch;
        for (int a = 0; a < 3; ++a) {
            std::fill(w.L[a].begin(), w.L[a].end(), Box());
            std::fill(w.R[a].begin(), w.R[a].end(), Box());
            std::fill(w.LC[a].begin(), w.LC[a].end(), Box());
            std::fill(w.RC[a].begin(), w.RC[a].end(), Box());
            std::fill(w.NL[a].begin(), w.NL[a].end(), 0u);
            std::fill(w.NR[a].begin(), w.NR[a].end(), 0u);
        }
    }

    // first bin whose upper edge is >= c; the last bin for c above the last
    // lower edge.  Edges are non-decreasing, so this is a lower-bound search.
    static uint32_t bin_of(const Work& w, float c, int a) {
        const uint32_t last = w.nb - 1;
        if (c <= w.edge[0].hi[a]) return 0;
        if (c > w.edge[last].lo[a]) return last;
        uint32_t lo = 1, hi = last - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (c <= w.edge[mid].hi[a])
                hi = mid;
            else
                lo = mid + 1;
        }
        return lo;
    }

    Plane best_on_axis(Work& w, const Range& r, int a) const {
        auto& L = w.L[a];
        auto& R = w.R[a];
        auto& LC = w.LC[a];
        auto& RC = w.RC[a];
        auto& NL = w.NL[a];
        auto& NR = w.NR[a];
        for (uint32_t* it = r.b; it != r.e; ++it) {
            const Box& bb = item_box(r.kind, *it);
            const V3 c = bb.centroid();
            const uint32_t k = bin_of(w, c[a], a);
            L[k].merge(bb);
            LC[k].include(c);
            ++NL[k];
        }
        const uint32_t n = w.nb - 1;
        R[n] = L[n];
        RC[n] = LC[n];
        NR[n] = NL[n];
        for (uint32_t i = n - 1; i > 0; --i) {
            R[i] = merged(L[i], R[i + 1]);
            RC[i] = merged(LC[i], RC[i + 1]);
            NR[i] = NL[i] + NR[i + 1];
        }
        for (uint32_t i = 1; i < n; ++i) {
            L[i].merge(L[i - 1]);
            LC[i].merge(LC[i - 1]);
            NL[i] += NL[i - 1];
        }
        Plane best;
        const float parent = r.box.area();
        for (uint32_t i = 0; i < n; ++i) {
            const uint32_t nl = NL[i], nr = NR[i + 1];
            if (nl == 0 || nr == 0) continue;
            const float lc = (float)nl * L[i].area();
            const float rc = (float)nr * R[i + 1].area();
            const float cost = D.bvh.Ct + D.bvh.Ci * (lc + rc) / parent;
            if (cost < best.cost) {
                best.cost = cost;
                best.axis = (uint32_t)a;
                best.index = i;
                best.nl = nl;
                best.nr = nr;
            }
        }
        return best;
    }

    Plane best_split(Work& w, const Range& r) const {
        reset_split(w, r);
        Plane best;
        for (int a = 0; a < 3; ++a) {
            const Plane p = best_on_axis(w, r, a);
            if (p.valid() && p.cost < best.cost) best = p;
        }
        return best;
    }

    static uint32_t push_node(Work& w, const Box& b, uint32_t w0, uint32_t w1) {
        const uint32_t v[8] = {f2u(b.lo.x), f2u(b.lo.y), f2u(b.lo.z), w0, f2u(b.hi.x), f2u(b.hi.y), f2u(b.hi.z), w1};
        w.nodes.insert(w.nodes.end(), v, v + 8);
        return num_nodes(w) - 1;
    }
    static uint32_t num_nodes(const Work& w) { return w.base + (uint32_t)(w.nodes.size() / 8); }
    uint32_t num_nodes() const { return (uint32_t)(nodes.size() / 8); }

    // BVH::makeLeaf (bvh.cpp:88-153)
    uint32_t make_leaf(Work& w, const Range& r, uint32_t level) {
        const uint32_t cnt = r.count();
        const uint32_t start = r.kind == kTriBin ? (uint32_t)(r.b - tri_order.data()) : num_nodes(w) + 1;
        const uint32_t w1 = (r.kind == kTriBin ? NOOR_TRI_LEAF_MASK : NOOR_MESH_LEAF_MASK) | cnt;
        const uint32_t id = push_node(w, r.box, start, w1);
        if (r.kind == kMeshBin) {
            uint32_t pos = (uint32_t)(r.b - mesh_order.data());
            for (uint32_t* it = r.b; it != r.e; ++it, ++pos) {
                const MeshInfo& m = meshes[*it];
                uint32_t ww = NOOR_MESH_INSTANCE_MASK | pos;
                if (m.src->light_idx >= 0) ww = NOOR_LIGHT_NODE_MASK | (uint32_t)m.src->light_idx;
                push_node(w, m.ibox, mesh_start[*it], ww);
            }
        }
        if (w.stat.height < level) w.stat.height = level;
        if (r.kind == kTriBin) {
            ++w.stat.num_leaf_nodes;
            w.stat.max_leaf_tris = std::max(w.stat.max_leaf_tris, cnt);
        }
        return id;
    }

    // BVH::recursiveBuild (bvh.cpp:180-214)
    uint32_t build(Work& w, const Range& r, uint32_t level) {
        const uint32_t cnt = r.count();
        if (r.kind == kTriBin) {
            if (level >= D.bvh.max_height || cnt <= D.bvh.min_leaf_tris) return make_leaf(w, r, level);
        } else if (cnt < 2) {
            return make_leaf(w, r, level);
        }
        const Plane p = best_split(w, r);
        const float leaf_cost = D.bvh.Ci * (float)cnt;
        if (r.kind == kTriBin) {
            if (!p.valid() || (leaf_cost < p.cost && cnt <= D.bvh.max_leaf_tris)) return make_leaf(w, r, level);
        } else if (!p.valid()) {
            return make_leaf(w, r, level);
        }
        const int a = (int)p.axis;
        const float plane_hi = w.edge[p.index].hi[a];
        const BinKind k = r.kind;
        uint32_t* mid = std::partition(r.b, r.e, [&](uint32_t i) { return item_box(k, i).centroid()[a] <= plane_hi; });
        Range left{r.b, mid, w.L[a][p.index], w.LC[a][p.index], k};
        Range right{mid, r.e, w.R[a][p.index + 1], w.RC[a][p.index + 1], k};
        const uint32_t id = push_node(w, r.box, 0u, (k == kTriBin ? 0u : NOOR_MESH_INNER_MASK) | p.axis);
        ++w.stat.num_inner_nodes;
        if (k == kTriBin && level < par_levels && cnt >= kParMinTris) {
            // the two subtrees on two threads, each numbered from 0, then
            // appended in depth-first order (left at id + 1, right after it)
            Work wl, wr;
            wl.init(D.bvh.num_bins);
            wr.init(D.bvh.num_bins);
            std::exception_ptr err;
            std::thread t([&]() {
                try {
                    build(wl, left, level + 1);
                } catch (...) {
                    err = std::current_exception();
                }
            });
            build(wr, right, level + 1);
            t.join();
            if (err) std::rethrow_exception(err);
            append_tree(w, wl, id + 1);
            const uint32_t rid = id + 1 + num_nodes(wl);
            append_tree(w, wr, rid);
            w.nodes[8 * (size_t)(id - w.base) + 3] = rid;
            return id;
        }
        build(w, left, level + 1);
        const uint32_t rid = build(w, right, level + 1);
        w.nodes[8 * (size_t)(id - w.base) + 3] = rid;
        return id;
    }

    // nodes of a tree numbered from 0 appended to w at node index `off`
    // (inner nodes' right-child words moved by off), statistics merged
    static void append_tree(Work& w, Work& sub, uint32_t off) {
        for (size_t n = 0; n < sub.nodes.size(); n += 8)
            if (!(sub.nodes[n + 7] & NOOR_TRI_LEAF_MASK)) sub.nodes[n + 3] += off;
        w.nodes.insert(w.nodes.end(), sub.nodes.begin(), sub.nodes.end());
        w.stat.height = std::max(w.stat.height, sub.stat.height);
        w.stat.num_inner_nodes += sub.stat.num_inner_nodes;
        w.stat.num_leaf_nodes += sub.stat.num_leaf_nodes;
        w.stat.max_leaf_tris = std::max(w.stat.max_leaf_tris, sub.stat.max_leaf_tris);
    }

    // BVH::build (bvh.cpp:216-258).  The mesh trees are independent (each
    // partitions its own slice of the triangle order and numbers its nodes
    // from 0), so they are built on all host threads; appended in mesh order
    // with their inner nodes' right-child indices moved by the tree's offset,
    // they are the same bytes as the reference's one-after-another build.
    void build_all() {
        tri_order.resize(D.num_triangles);
        for (uint32_t i = 0; i < D.num_triangles; ++i) tri_order[i] = i;
        mesh_order.resize(D.num_meshes);
        for (uint32_t i = 0; i < D.num_meshes; ++i) mesh_order[i] = i;
        mesh_start.assign(D.num_meshes, 0u);
        std::vector<uint32_t> src;
        // light meshes too: the reference builds each one a bottom-level
        // tree (one empty leaf with the shape's bounds), which its light
        // node points at
        for (uint32_t i = 0; i < D.num_meshes; ++i)
            if (D.meshes[i].instance < 0) src.push_back(i);
        std::vector<Work> trees(src.size());
        std::vector<char> done(src.size(), 0);
        if (use_gpu) {
            // the triangle meshes on the device (bvh_gpu.cu), the light
            // meshes' one-leaf trees below
            std::vector<nbg::GpuMesh> gm;
            std::vector<size_t> gj;
            for (size_t j = 0; j < src.size(); ++j) {
                const noor_mesh& m = D.meshes[src[j]];
                if (m.light_idx >= 0) continue;
                nbg::GpuMesh g;
                g.start = m.tri_start;
                g.count = m.tri_count;
                const MeshInfo& mi = meshes[src[j]];
                const float b[12] = {mi.box.lo.x,  mi.box.lo.y,  mi.box.lo.z,  mi.box.hi.x,  mi.box.hi.y,  mi.box.hi.z,
                                     mi.cbox.lo.x, mi.cbox.lo.y, mi.cbox.lo.z, mi.cbox.hi.x, mi.cbox.hi.y, mi.cbox.hi.z};
                std::memcpy(g.box, b, 24);
                std::memcpy(g.cbox, b + 6, 24);
                gm.push_back(g);
                gj.push_back(j);
            }
            nbg::GpuBvhParams bp{D.bvh.num_bins, D.bvh.max_height, D.bvh.min_leaf_tris, D.bvh.max_leaf_tris,
                                 D.bvh.Ci, D.bvh.Ct};
            std::vector<nbg::GpuTree> gt;
            std::string err;
            static_assert(sizeof(Box) == 24, "Box is 6 floats");
            const int rc = nbg::gpu_build_blas(reinterpret_cast<const float*>(tri_box.data()), D.num_triangles, gm, bp,
                                               tri_order, gt, &gpu_ms, err);
            if (rc) throw GpuBuildError{rc, err};
            for (size_t k = 0; k < gj.size(); ++k) {
                Work& w = trees[gj[k]];
                w.nodes = std::move(gt[k].nodes);
                w.stat.height = gt[k].height;
                w.stat.num_inner_nodes = gt[k].num_inner;
                w.stat.num_leaf_nodes = gt[k].num_leaf;
                w.stat.max_leaf_tris = gt[k].max_leaf_tris;
                done[gj[k]] = 1;
            }
        }
        {
            size_t todo = 0;
            for (size_t j = 0; j < src.size(); ++j) todo += done[j] ? 0 : 1;
            const uint32_t hw = std::max(1u, std::thread::hardware_concurrency());
            par_levels = 0;
            while (todo && (todo << par_levels) < hw && par_levels < 8) ++par_levels;
        }
        std::atomic<size_t> next{0};
        std::vector<std::exception_ptr> errs(src.size());
        auto worker = [&]() {
            for (size_t j; (j = next.fetch_add(1)) < src.size();) {
                if (done[j]) continue;
                try {
                    const uint32_t i = src[j];
                    const noor_mesh& m = D.meshes[i];
                    Work& w = trees[j];
                    w.init(D.bvh.num_bins);
                    w.nodes.reserve(8 * (size_t)2 * m.tri_count);
                    Range r{tri_order.data() + m.tri_start, tri_order.data() + m.tri_start + m.tri_count,
                            meshes[i].box, meshes[i].cbox, kTriBin};
                    build(w, r, 0);
                } catch (...) {
                    errs[j] = std::current_exception();
                }
            }
        };
        const size_t nthreads = std::min<size_t>(src.size(), std::max(1u, std::thread::hardware_concurrency()));
        std::vector<std::thread> pool;
        for (size_t t = 1; t < nthreads; ++t) pool.emplace_back(worker);
        worker();
        for (auto& t : pool) t.join();
        for (auto& e : errs)
            if (e) std::rethrow_exception(e);
        size_t total = 0;
        for (const Work& w : trees) total += w.nodes.size();
        nodes.reserve(total + 8 * (size_t)2 * (D.num_meshes + 1));
        for (size_t j = 0; j < src.size(); ++j) {
            Work& w = trees[j];
            const uint32_t off = num_nodes();
            mesh_start[src[j]] = off;
            for (size_t n = 0; n < w.nodes.size(); n += 8)
                if (!(w.nodes[n + 7] & NOOR_TRI_LEAF_MASK)) w.nodes[n + 3] += off;  // inner: right child
            nodes.insert(nodes.end(), w.nodes.begin(), w.nodes.end());
            stat.height = std::max(stat.height, w.stat.height);
            stat.num_inner_nodes += w.stat.num_inner_nodes;
            stat.num_leaf_nodes += w.stat.num_leaf_nodes;
            stat.max_leaf_tris = std::max(stat.max_leaf_tris, w.stat.max_leaf_tris);
            std::vector<uint32_t>().swap(w.nodes);
        }
        for (uint32_t i = 0; i < D.num_meshes; ++i)
            if (D.meshes[i].instance >= 0) mesh_start[i] = mesh_start[D.meshes[i].instance];
        root = num_nodes();
        Work top;
        top.init(D.bvh.num_bins);
        top.base = root;
        top.stat = stat;
        Range r{mesh_order.data(), mesh_order.data() + D.num_meshes, scene_box, scene_cbox, kMeshBin};
        build(top, r, stat.height);
        nodes.insert(nodes.end(), top.nodes.begin(), top.nodes.end());
        stat = top.stat;
        stat.height += 1;
    }
};

// WaldTriangle(A,B,C) (noor/header/triangle.h:73-107); degenerate triangles
// keep zero coefficients (the reference leaves them uninitialised; they are
// never read because the deg flag is tested first).
static void wald_record(const V3& A, const V3& B, const V3& C, uint32_t* r0, uint32_t* r1, uint32_t* r2) {
    const V3 b = vsub(C, A);
    const V3 c = vsub(B, A);
    // glm::cross(c, b) then glm::normalize (v * 1/sqrt(dot))
    V3 N = v3(c.y * b.z - b.y * c.z, c.z * b.x - b.z * c.x, c.x * b.y - b.x * c.y);
    const float inv = 1.0f / std::sqrt((N.x * N.x + N.y * N.y) + N.z * N.z);
    N = vscale(N, inv);
    uint32_t axis = 0;
    for (uint32_t i = 0; i < 3; ++i) axis = std::fabs(N[(int)i]) > std::fabs(N[(int)axis]) ? i : axis;
    const uint32_t mod[4] = {1u, 2u, 0u, 1u};
    const int u = (int)mod[axis], v = (int)mod[axis + 1];
    const float denom = b[u] * c[v] - b[v] * c[u];
    const float Nk = N[(int)axis];
    std::memset(r0, 0, 16);
    std::memset(r1, 0, 16);
    std::memset(r2, 0, 16);
    r0[0] = axis;
    if (denom == 0.0f) {
        r2[2] = 1u;
        return;
    }
    const float nu = N[u] / Nk, nv = N[v] / Nk;
    const float nd = ((N.x * A.x + N.y * A.y) + N.z * A.z) / Nk;
    r0[1] = f2u(nu);
    r0[2] = f2u(nv);
    r0[3] = f2u(nd);
    r1[0] = f2u(b[u] / denom);
    r1[1] = f2u(-b[v] / denom);
    r1[2] = f2u(A[u]);
    r1[3] = f2u(A[v]);
    r2[0] = f2u(c[v] / denom);
    r2[1] = f2u(-c[u] / denom);
    r2[2] = 0u;
}

}  // namespace nbh

using namespace nbh;

struct noor_payload_handle {
    std::vector<uint32_t> attr;
    std::vector<float> vertices, normals, uvs;
    std::vector<float> xf[9];
    std::vector<uint32_t> wald[3];
    std::vector<uint32_t> bvh_lo, bvh_hi;
    uint32_t root = 0;
    std::vector<std::vector<float>> tex_data;
    std::vector<noor_texture> tex_meta;       // width, height, filter, address of each texture
    std::vector<noor_texture> textures;
    std::vector<noor_area_light> lights;
    std::vector<noor_point_light> point_lights;
    std::vector<noor_spot_light> spot_lights;
    std::vector<noor_distant_light> distant_lights;
    std::vector<noor_material> materials;
    std::vector<uint32_t> tri_order;
    uint32_t num_tris = 0;
    uint32_t height = 0;
    float scene_radius = 0.0f;
    int32_t skydome_type = 0;
};

// a 1x1 constant (ImageTexture(float3), point filtered, clamped)
static uint32_t add_texture(noor_payload_handle* h, const float* rgb, float a) {
    h->tex_data.push_back({rgb[0], rgb[1], rgb[2], a});
    h->tex_meta.push_back(noor_texture{1, 1, nullptr, NOOR_FILTER_POINT, NOOR_ADDRESS_CLAMP});
    return (uint32_t)h->tex_data.size() - 1;
}
// an image map (ImageTexture(file): wrapped, linear unless given)
static uint32_t add_image(noor_payload_handle* h, const noor_image& im, int32_t filter) {
    h->tex_data.emplace_back(im.rgba, im.rgba + 4 * (size_t)im.width * im.height);
    h->tex_meta.push_back(noor_texture{im.width, im.height, nullptr, filter, NOOR_ADDRESS_WRAP});
    return (uint32_t)h->tex_data.size() - 1;
}

static int build_payload(const noor_scene_desc* d, bool gpu, noor_payload_handle** out, noor_build_stat* stat) {
    using namespace nbh;
    if (!d || !out) return set_error(NOOR_ERR_INVALID, "noor_build_payload: null argument");
    *out = nullptr;
    if (d->num_triangles == 0 || !d->vertices || !d->vindices || !d->nindices || !d->uvindices || !d->normals ||
        !d->uvs || !d->material_indices || !d->meshes || d->num_meshes == 0)
        return set_error(NOOR_ERR_INVALID, "noor_build_payload: empty or incomplete scene");
    if (d->num_materials == 0 || !d->materials) return set_error(NOOR_ERR_INVALID, "noor_build_payload: no materials");
    if (d->bvh.num_bins < 2) return set_error(NOOR_ERR_INVALID, "noor_build_payload: num_bins must be >= 2");
    if ((d->num_area_lights && !d->area_lights) || (d->num_point_lights && !d->point_lights) ||
        (d->num_spot_lights && !d->spot_lights) || (d->num_distant_lights && !d->distant_lights))
        return set_error(NOOR_ERR_INVALID, "noor_build_payload: light count without an array");
    // validate indices and mesh ranges (source meshes cover [0,N) in order)
    uint32_t next = 0;
    for (uint32_t i = 0; i < d->num_meshes; ++i) {
        const noor_mesh& m = d->meshes[i];
        if (m.light_idx >= 0) {
            if ((uint32_t)m.light_idx >= d->num_area_lights)
                return set_error(NOOR_ERR_INVALID, "noor_build_payload: light mesh names a missing light");
            if (m.tri_count != 0 || m.tri_start > d->num_triangles)
                return set_error(NOOR_ERR_INVALID, "noor_build_payload: a light mesh carries no triangles");
            continue;
        }
        if (m.instance >= 0) {
            if ((uint32_t)m.instance >= d->num_meshes || d->meshes[m.instance].instance >= 0 ||
                d->meshes[m.instance].light_idx >= 0)
                return set_error(NOOR_ERR_INVALID, "noor_build_payload: instance of a non-source mesh");
            continue;
        }
        if (m.tri_start != next) return set_error(NOOR_ERR_INVALID, "noor_build_payload: mesh ranges not contiguous");
        next += m.tri_count;
    }
    if (next != d->num_triangles) return set_error(NOOR_ERR_INVALID, "noor_build_payload: meshes do not cover triangles");
    for (size_t i = 0; i < 3 * (size_t)d->num_triangles; ++i) {
        if (d->vindices[i] >= d->num_vertices || d->nindices[i] >= d->num_normals || d->uvindices[i] >= d->num_uvs)
            return set_error(NOOR_ERR_INVALID, "noor_build_payload: vertex attribute index out of range");
    }
    for (size_t i = 0; i < 4 * (size_t)d->num_vertices; ++i)
        if (!std::isfinite(d->vertices[i])) return set_error(NOOR_ERR_INVALID, "noor_build_payload: non-finite vertex");
    for (uint32_t i = 0; i < d->num_triangles; ++i)
        if (d->material_indices[i] >= d->num_materials)
            return set_error(NOOR_ERR_INVALID, "noor_build_payload: material index out of range");
    if (d->num_images && !d->images) return set_error(NOOR_ERR_INVALID, "noor_build_payload: image count without an array");
    for (uint32_t i = 0; i < d->num_images; ++i)
        if (d->images[i].width <= 0 || d->images[i].height <= 0 || !d->images[i].rgba)
            return set_error(NOOR_ERR_INVALID, "noor_build_payload: empty image map");
    for (uint32_t i = 0; i < d->num_materials; ++i)
        for (int k = 0; k < NOOR_NUM_MAPS; ++k)
            if (d->materials[i].map[k] < -1 || d->materials[i].map[k] >= (int32_t)d->num_images)
                return set_error(NOOR_ERR_INVALID, "noor_build_payload: material map names a missing image");

    const auto t0 = std::chrono::steady_clock::now();
    std::unique_ptr<noor_payload_handle> h(new (std::nothrow) noor_payload_handle());
    if (!h) return set_error(NOOR_ERR_OOM, "noor_build_payload: out of host memory");
    try {
        Builder B(*d, gpu);
        B.compute_boxes();
        const auto t1 = std::chrono::steady_clock::now();
        B.build_all();
        const auto t2 = std::chrono::steady_clock::now();

        h->num_tris = d->num_triangles;
        h->root = B.root;
        h->height = B.stat.height;
        h->tri_order = B.tri_order;
        h->scene_radius = B.scene_box.radius();
        h->skydome_type = d->skydome_type;
        const uint32_t nn = B.num_nodes();
        h->bvh_lo.resize(4 * (size_t)nn);
        h->bvh_hi.resize(4 * (size_t)nn);
        for (uint32_t i = 0; i < nn; ++i)
            for (int k = 0; k < 4; ++k) {
                h->bvh_lo[4 * (size_t)i + k] = B.nodes[8 * (size_t)i + k];
                h->bvh_hi[4 * (size_t)i + k] = B.nodes[8 * (size_t)i + 4 + k];
            }
        // transforms in mesh_order (BVH::loadCudaPayload, bvh.cpp:59-85)
        for (int k = 0; k < 9; ++k) h->xf[k].reserve(4 * (size_t)d->num_meshes);
        for (uint32_t i = 0; i < d->num_meshes; ++i) {
            const noor_mesh& m = d->meshes[B.mesh_order[i]];
            float tg[16], tl[16];
            std::memcpy(tg, m.to_global, sizeof(tg));
            inverse4(tg, tl);
            // normal transform = transpose(inverse(mat3(to_global)))
            float m3[16] = {tg[0], tg[1], tg[2], 0, tg[4], tg[5], tg[6], 0, tg[8], tg[9], tg[10], 0, 0, 0, 0, 1};
            float im3[16];
            inverse4(m3, im3);
            for (int r = 0; r < 3; ++r) {
                // row r of a column-major matrix: (m[r], m[4+r], m[8+r], m[12+r])
                const float wl[4] = {tl[r], tl[4 + r], tl[8 + r], tl[12 + r]};
                const float wg[4] = {tg[r], tg[4 + r], tg[8 + r], tg[12 + r]};
                // row r of transpose(im3) = column r of im3
                const float wn[4] = {im3[4 * r + 0], im3[4 * r + 1], im3[4 * r + 2], 0.0f};
                h->xf[0 + r].insert(h->xf[0 + r].end(), wn, wn + 4);
                h->xf[3 + r].insert(h->xf[3 + r].end(), wl, wl + 4);
                h->xf[6 + r].insert(h->xf[6 + r].end(), wg, wg + 4);
            }
        }
        // materials and textures (Model::loadMaterial, model.cpp:184-330): a
        // texture of 0.5 first; per material its constants as 1x1 textures
        // and its image maps, one texture per image, made at the image's
        // first use with that use's filter (map_d point, the others linear).
        // One record is carried from material to material, as the reference
        // reuses one CudaMaterial: the uv scale of a slot without a map, and
        // the bump fields of a material without a bump map, keep the values
        // an earlier material set.
        const float half[3] = {0.5f, 0.5f, 0.5f};
        add_texture(h.get(), half, 1.0f);
        std::vector<int64_t> image_tex(d->num_images, -1);
        auto map_texture = [&](int32_t img, int32_t filter) -> uint32_t {
            if (image_tex[img] < 0) image_tex[img] = add_image(h.get(), d->images[img], filter);
            return (uint32_t)image_tex[img];
        };
        noor_material mt;
        std::memset(&mt, 0, sizeof(mt));
        for (float* s : {mt.diffuse_uvscale, mt.specular_uvscale, mt.transparency_uvscale, mt.emittance_uvscale,
                         mt.bump_uvscale, mt.roughness_uvscale, mt.metalness_uvscale})
            s[0] = s[1] = 1.0f;
        mt.bumpfactor = 1.0f;
        for (uint32_t i = 0; i < d->num_materials; ++i) {
            const noor_material_desc& md = d->materials[i];
            auto mapped = [&](int slot, float* uvscale) {
                if (md.map[slot] < 0) return false;
                uvscale[0] = md.map_uvscale[slot][0];
                uvscale[1] = md.map_uvscale[slot][1];
                return true;
            };
            mt.coat_weight = md.coat_weight;
            mt.coat_roughness = md.coat_roughness;
            mt.coat_thickness = md.coat_thickness;
            mt.coat_sigma = md.coat_sigma;
            mt.coat_ior = md.coat_ior;
            mt.emitter_scale = md.emitter_scale;
            mt.type = md.type;
            mt.distribution = md.distribution;
            mt.transmission_tex_idx = add_texture(h.get(), md.transmission, 1.0f);
            mt.ior_tex_idx = add_texture(h.get(), md.ior, 1.0f);
            mt.k_tex_idx = add_texture(h.get(), md.k, 1.0f);
            mt.diffuse_tex_idx = mapped(NOOR_MAP_DIFFUSE, mt.diffuse_uvscale)
                                     ? map_texture(md.map[NOOR_MAP_DIFFUSE], NOOR_FILTER_LINEAR)
                                     : add_texture(h.get(), md.diffuse, 1.0f);
            const float rough[3] = {md.roughness[0], md.roughness[1], 1.0f};
            mt.roughness_tex_idx = mapped(NOOR_MAP_ROUGHNESS, mt.roughness_uvscale)
                                       ? map_texture(md.map[NOOR_MAP_ROUGHNESS], NOOR_FILTER_LINEAR)
                                       : add_texture(h.get(), rough, 1.0f);
            const float metal[3] = {1.0f, 1.0f, 1.0f};
            mt.metalness_tex_idx = mapped(NOOR_MAP_METALNESS, mt.metalness_uvscale)
                                       ? map_texture(md.map[NOOR_MAP_METALNESS], NOOR_FILTER_LINEAR)
                                       : add_texture(h.get(), metal, 1.0f);
            mt.specular_tex_idx = mapped(NOOR_MAP_SPECULAR, mt.specular_uvscale)
                                      ? map_texture(md.map[NOOR_MAP_SPECULAR], NOOR_FILTER_LINEAR)
                                      : add_texture(h.get(), md.specular, 1.0f);
            mt.emittance_tex_idx = mapped(NOOR_MAP_EMITTANCE, mt.emittance_uvscale)
                                       ? map_texture(md.map[NOOR_MAP_EMITTANCE], NOOR_FILTER_LINEAR)
                                       : add_texture(h.get(), md.emittance, 1.0f);
            if (mapped(NOOR_MAP_ALPHA, mt.transparency_uvscale)) {
                mt.transparency_tex_idx = map_texture(md.map[NOOR_MAP_ALPHA], NOOR_FILTER_POINT);
                mt.type |= NOOR_ALPHA;
            } else {
                mt.transparency_tex_idx = add_texture(h.get(), md.transparency, 1.0f);
            }
            if (mapped(NOOR_MAP_BUMP, mt.bump_uvscale)) {
                mt.bump_tex_idx = map_texture(md.map[NOOR_MAP_BUMP], NOOR_FILTER_LINEAR);
                mt.bumpfactor = md.bumpfactor;
                mt.type |= NOOR_BUMP;
            }
            h->materials.push_back(mt);
        }
        // environment texture last
        if (d->skydome_type == NOOR_SKY_HDR) {
            if (!d->env_rgba || d->env_width <= 0 || d->env_height <= 0)
                return set_error(NOOR_ERR_INVALID, "noor_build_payload: HDR sky without an environment map");
            h->tex_data.emplace_back(d->env_rgba, d->env_rgba + 4 * (size_t)d->env_width * d->env_height);
            h->tex_meta.push_back(noor_texture{d->env_width, d->env_height, nullptr, NOOR_FILTER_LINEAR,
                                               NOOR_ADDRESS_CLAMP});
        } else {
            const float sky[3] = {0.25f, 0.25f, 0.25f};
            add_texture(h.get(), sky, 1.0f);
        }
        for (size_t i = 0; i < h->tex_data.size(); ++i) {
            noor_texture t = h->tex_meta[i];
            t.rgba = h->tex_data[i].data();
            h->textures.push_back(t);
        }
        h->lights.assign(d->area_lights, d->area_lights + d->num_area_lights);
        if (d->num_point_lights) h->point_lights.assign(d->point_lights, d->point_lights + d->num_point_lights);
        if (d->num_spot_lights) h->spot_lights.assign(d->spot_lights, d->spot_lights + d->num_spot_lights);
        if (d->num_distant_lights) {
            // CudaDistantLight's constructor normalises the direction (light.cuh:222)
            h->distant_lights.assign(d->distant_lights, d->distant_lights + d->num_distant_lights);
            for (noor_distant_light& l : h->distant_lights) {
                const float* w = l.direction;
                const float inv = 1.0f / std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
                for (int k = 0; k < 3; ++k) l.direction[k] = w[k] * inv;
            }
        }

        double tail_ms = 0.0;
        const auto t3 = std::chrono::steady_clock::now();
        if (gpu) {
            // the same steps on the device (bvh_gpu.cu)
            std::vector<uint32_t> mtypes(d->num_materials);
            for (uint32_t i = 0; i < d->num_materials; ++i) mtypes[i] = h->materials[i].type;
            nbg::GpuTailIn ti{B.tri_order.data(), d->num_triangles, d->vindices, d->nindices, d->uvindices,
                              d->vertices, d->num_vertices, d->normals, d->num_normals, d->uvs, d->num_uvs,
                              d->material_indices, mtypes.data(), d->num_materials};
            nbg::GpuTailOut to;
            std::string err;
            const int rc = nbg::gpu_payload_tail(ti, to, &tail_ms, err);
            if (rc) return set_error(rc, err);
            h->vertices = std::move(to.vertices);
            h->normals = std::move(to.normals);
            h->uvs = std::move(to.uvs);
            for (int k = 0; k < 3; ++k) h->wald[k] = std::move(to.wald[k]);
            h->attr = std::move(to.attr);
        } else {
            // vertex de-duplication in BVH order (Model::loadCudaPayload, model.cpp:376-401):
            // the first occurrence of a (vertex, normal, uv) index triple appends a
            // vertex; later occurrences reuse its index (dedup_corners: the same
            // numbering as the reference's map, on all host threads)
            const size_t nc = 3 * (size_t)d->num_triangles;
            auto key = [&](size_t p) {
                const size_t c = 3 * (size_t)B.tri_order[p / 3] + p % 3;
                return AttrKey{d->vindices[c], d->nindices[c], d->uvindices[c]};
            };
            std::vector<uint32_t> element, first;
            const uint32_t nv = dedup_corners(nc, key, element, first);
            h->vertices.resize(4 * (size_t)nv);
            h->normals.resize(4 * (size_t)nv);
            h->uvs.resize(2 * (size_t)nv);
            parallel_for(nv, [&](uint32_t k) {
                const AttrKey kk = key(first[k]);
                std::memcpy(h->vertices.data() + 4 * (size_t)k, d->vertices + 4 * (size_t)kk.v, 16);
                std::memcpy(h->normals.data() + 4 * (size_t)k, d->normals + 4 * (size_t)kk.n, 16);
                std::memcpy(h->uvs.data() + 2 * (size_t)k, d->uvs + 2 * (size_t)kk.u, 8);
            });
            // Wald triangles + attribute indices (Model::buildWaldTriangles, model.cpp:333-360)
            for (int k = 0; k < 3; ++k) h->wald[k].resize(4 * (size_t)d->num_triangles);
            h->attr.resize(4 * (size_t)d->num_triangles);
            // independent per triangle: split over the host threads
            parallel_for(d->num_triangles, [&](uint32_t i) {
                V3 p[3];
                for (int j = 0; j < 3; ++j) {
                    const float* q = h->vertices.data() + 4 * (size_t)element[3 * (size_t)i + j];
                    p[j] = v3(q[0], q[1], q[2]);
                }
                uint32_t* r0 = h->wald[0].data() + 4 * (size_t)i;
                uint32_t* r1 = h->wald[1].data() + 4 * (size_t)i;
                uint32_t* r2 = h->wald[2].data() + 4 * (size_t)i;
                wald_record(p[0], p[1], p[2], r0, r1, r2);
                const uint32_t mi = d->material_indices[B.tri_order[i]];
                r2[3] = h->materials[mi].type;
                uint32_t* a = h->attr.data() + 4 * (size_t)i;
                a[0] = element[3 * (size_t)i + 0];
                a[1] = element[3 * (size_t)i + 1];
                a[2] = element[3 * (size_t)i + 2];
                a[3] = mi;
            });
        }
        const auto t4 = std::chrono::steady_clock::now();
        if (stat) {
            *stat = B.stat;
            stat->scene_min[0] = B.scene_box.lo.x;
            stat->scene_min[1] = B.scene_box.lo.y;
            stat->scene_min[2] = B.scene_box.lo.z;
            stat->scene_max[0] = B.scene_box.hi.x;
            stat->scene_max[1] = B.scene_box.hi.y;
            stat->scene_max[2] = B.scene_box.hi.z;
            stat->scene_radius = h->scene_radius;
            stat->build_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            stat->box_seconds = std::chrono::duration<double>(t1 - t0).count();
            stat->tree_seconds = std::chrono::duration<double>(t2 - t1).count();
            stat->tree_device_ms = B.gpu_ms;
            stat->tail_seconds = std::chrono::duration<double>(t4 - t3).count();
            stat->tail_device_ms = tail_ms;
        }
    } catch (const std::bad_alloc&) {
        return set_error(NOOR_ERR_OOM, "noor_build_payload: out of host memory");
    } catch (const GpuBuildError& g) {
        return set_error(g.code, g.msg);
    }
    *out = h.release();
    return NOOR_OK;
}

extern "C" int noor_build_payload(const noor_scene_desc* d, noor_payload_handle** out, noor_build_stat* stat) {
    return build_payload(d, false, out, stat);
}
extern "C" int noor_build_payload_gpu(const noor_scene_desc* d, noor_payload_handle** out, noor_build_stat* stat) {
    return build_payload(d, true, out, stat);
}

extern "C" int noor_payload_view(const noor_payload_handle* h, noor_payload* p) {
    if (!h || !p) return set_error(NOOR_ERR_INVALID, "noor_payload_view: null argument");
    std::memset(p, 0, sizeof(*p));
    p->num_triangles = h->num_tris;
    p->attribute_indices = h->attr.data();
    p->vertices = h->vertices.data();
    p->normals = h->normals.data();
    p->uvs = h->uvs.data();
    p->num_vertices = (uint32_t)(h->vertices.size() / 4);
    for (int r = 0; r < 3; ++r) {
        p->normal_row[r] = h->xf[0 + r].data();
        p->world_to_object_row[r] = h->xf[3 + r].data();
        p->object_to_world_row[r] = h->xf[6 + r].data();
    }
    p->num_instances = (uint32_t)(h->xf[0].size() / 4);
    p->wald_ax_nu_nv_nd = h->wald[0].data();
    p->wald_bnu_bnv_au_av = h->wald[1].data();
    p->wald_cnu_cnv_deg_mat = h->wald[2].data();
    p->bvh_root_node = h->root;
    p->bvh_min_right_start = h->bvh_lo.data();
    p->bvh_max_axis_count = h->bvh_hi.data();
    p->num_bvh_nodes = (uint32_t)(h->bvh_lo.size() / 4);
    p->textures = h->textures.data();
    p->num_textures = (uint32_t)h->textures.size();
    p->area_lights = h->lights.empty() ? nullptr : h->lights.data();
    p->num_area_lights = (int32_t)h->lights.size();
    p->point_lights = h->point_lights.empty() ? nullptr : h->point_lights.data();
    p->num_point_lights = (int32_t)h->point_lights.size();
    p->spot_lights = h->spot_lights.empty() ? nullptr : h->spot_lights.data();
    p->num_spot_lights = (int32_t)h->spot_lights.size();
    p->distant_lights = h->distant_lights.empty() ? nullptr : h->distant_lights.data();
    p->num_distant_lights = (int32_t)h->distant_lights.size();
    p->num_infinite_lights = 1;
    p->materials = h->materials.data();
    p->num_materials = (uint32_t)h->materials.size();
    return NOOR_OK;
}

extern "C" int noor_payload_triangle_order(const noor_payload_handle* h, uint32_t* out, size_t n) {
    if (!h || !out || n < h->tri_order.size()) return set_error(NOOR_ERR_INVALID, "noor_payload_triangle_order: bad argument");
    std::memcpy(out, h->tri_order.data(), h->tri_order.size() * sizeof(uint32_t));
    return NOOR_OK;
}

// Scene::load (noor/source/scene.cpp:51-91)
extern "C" int noor_payload_default_spec(const noor_payload_handle* h, uint32_t bounces, uint32_t rr, noor_spec* s) {
    if (!h || !s) return set_error(NOOR_ERR_INVALID, "noor_payload_default_spec: null argument");
    std::memset(s, 0, sizeof(*s));
    const float r = h->scene_radius;
    s->reflection_bias = 0.0001f * r;
    s->shadow_bias = 0.0001f * r;
    s->world_radius = r;
    s->wr2 = r * r;
    s->bvh_root_node = h->root;
    s->bvh_height = h->height;
    s->bounces = bounces;
    s->rr = rr;
    s->num_gpus = 1;
    s->skydome_type = h->skydome_type;
    const int num_lights = (int)(h->lights.size() + h->point_lights.size() + h->spot_lights.size() +
                                 h->distant_lights.size()) + 1;
    s->lighting_type = num_lights < 2 ? NOOR_LIGHT_SKY_MASK : 0u;
    s->mis = 0;
    s->intersector = NOOR_ISECT_WATERTIGHT;
    s->film_mode = NOOR_FILM_KAHAN;
    return NOOR_OK;
}

extern "C" void noor_free_payload(noor_payload_handle* h) { delete h; }

// Camera(...) + CudaCamera::update for a pinhole perspective camera
// (noor/header/camera.h:99-153,255-300; noor/cuda/camera.cuh:66-94), in FP64.
extern "C" int noor_camera_lookat(const float eye[3], const float look_at[3], const float up[3], float fov,
                                  uint32_t w, uint32_t h, noor_camera* out) {
    if (!eye || !look_at || !up || !out || w == 0 || h == 0 || !(fov > 0.0f))
        return set_error(NOOR_ERR_INVALID, "noor_camera_lookat: bad argument");
    auto norm = [](double* v) {
        const double l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        v[0] /= l;
        v[1] /= l;
        v[2] /= l;
    };
    double fwd[3] = {(double)eye[0] - look_at[0], (double)eye[1] - look_at[1], (double)eye[2] - look_at[2]};
    const double scale = std::sqrt(fwd[0] * fwd[0] + fwd[1] * fwd[1] + fwd[2] * fwd[2]);
    norm(fwd);
    const double u[3] = {up[0], up[1], up[2]};
    double right[3] = {u[1] * fwd[2] - u[2] * fwd[1], u[2] * fwd[0] - u[0] * fwd[2], u[0] * fwd[1] - u[1] * fwd[0]};
    norm(right);
    // cameraToWorld = translate(lookAt) * [right up forward] * translate(0,0,scale)
    std::memset(out, 0, sizeof(*out));
    for (int r = 0; r < 3; ++r) {
        out->camera_to_world[r][0] = (float)right[r];
        out->camera_to_world[r][1] = (float)u[r];
        out->camera_to_world[r][2] = (float)fwd[r];
        out->camera_to_world[r][3] = (float)((double)look_at[r] + fwd[r] * scale);
    }
    // rasterToCamera: raster -> screen window -> camera plane z = -1
    const double aspect = (double)w / (double)h;
    double smin[2], smax[2];
    if (aspect > 1.0) {
        smin[0] = -aspect; smax[0] = aspect; smin[1] = -1.0; smax[1] = 1.0;
    } else {
        smin[0] = -1.0; smax[0] = 1.0; smin[1] = -1.0 / aspect; smax[1] = 1.0 / aspect;
    }
    const double cot = 1.0 / std::tan((double)fov / 2.0);
    const double sx = (smax[0] - smin[0]) / (double)w / cot, sy = (smax[1] - smin[1]) / (double)h / cot;
    out->raster_to_camera[0][0] = (float)sx;
    out->raster_to_camera[0][3] = (float)(smin[0] / cot);
    out->raster_to_camera[1][1] = (float)sy;
    out->raster_to_camera[1][3] = (float)(smin[1] / cot);
    out->raster_to_camera[2][3] = -1.0f;
    out->dx_camera[0] = (float)sx;
    out->dy_camera[1] = (float)sy;
    out->image_area = (float)std::fabs((smax[0] - smin[0]) / cot * (smax[1] - smin[1]) / cot);
    out->lens_radius = 0.0f;
    out->focal_length = (float)scale;
    out->w = w;
    out->h = h;
    out->center = w * (h >> 1) + (w >> 1);
    out->type = NOOR_CAMERA_PERSP;
    return NOOR_OK;
}
