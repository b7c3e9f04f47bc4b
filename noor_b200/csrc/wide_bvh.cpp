// Host collapse of a payload's binary BVH into the four-wide any-hit tree
// (layout and rules in wide_bvh.h).
#include "wide_bvh.h"

#include <algorithm>
#include <cmath>
#include <cstring>

#include "noor_b200.h"

namespace nb {

namespace {

constexpr uint32_t kKindMask =
    NOOR_LIGHT_NODE_MASK | NOOR_MESH_INSTANCE_MASK | NOOR_MESH_LEAF_MASK | NOOR_TRI_LEAF_MASK;

enum Kind : uint8_t { kInner, kLight, kInstance, kMeshLeaf, kTriLeaf };

struct Tree {
    const uint32_t* w;
    size_t nn;
    uint32_t w0(uint32_t n) const { return w[8 * (size_t)n + 3]; }
    uint32_t w1(uint32_t n) const { return w[8 * (size_t)n + 7]; }
    float lo(uint32_t n, int a) const { return bits(w[8 * (size_t)n + a]); }
    float hi(uint32_t n, int a) const { return bits(w[8 * (size_t)n + 4 + a]); }
    static float bits(uint32_t u) {
        float f;
        std::memcpy(&f, &u, 4);
        return f;
    }
    // the node kinds in the order the traversal tells them apart
    Kind kind(uint32_t n) const {
        const uint32_t f = w1(n);
        if (!(f & kKindMask)) return kInner;
        if (f & NOOR_LIGHT_NODE_MASK) return kLight;
        if (f & NOOR_MESH_INSTANCE_MASK) return kInstance;
        if (f & NOOR_MESH_LEAF_MASK) return kMeshLeaf;
        return kTriLeaf;
    }
    // the traversal resets the ray to world space on taking this node
    bool world(uint32_t n) const { return (w1(n) & NOOR_MESH_NODE_MASK) != 0u; }
    uint32_t axis(uint32_t n) const { return w1(n) & NOOR_AXIS_MASK; }
    uint32_t count(uint32_t n) const { return w1(n) & NOOR_COUNT_MASK; }
    bool nan_box(uint32_t n) const {
        for (int a = 0; a < 3; ++a)
            if (std::isnan(lo(n, a)) || std::isnan(hi(n, a))) return true;
        return false;
    }
    bool contains(uint32_t c, uint32_t g) const {
        for (int a = 0; a < 3; ++a)
            if (!(lo(g, a) >= lo(c, a) && hi(g, a) <= hi(c, a))) return false;
        return true;
    }
    // the i-th successor the traversal can take from n (i < num_succ)
    uint32_t num_succ(uint32_t n) const {
        switch (kind(n)) {
            case kInner: return 2;
            case kInstance: return 1;
            case kMeshLeaf: return count(n);
            default: return 0;
        }
    }
    uint32_t succ(uint32_t n, uint32_t i) const {
        switch (kind(n)) {
            case kInner: return i == 0 ? n + 1 : w0(n);
            case kInstance: return w0(n);
            default: return n + 1 + i;
        }
    }
};

}  // namespace

bool build_wide_tree(const uint32_t* nodes8, size_t nn, uint32_t root, int max_stack, WideTree& out,
                     std::string* why) {
    out = WideTree{};
    auto fail = [&](const char* m) {
        if (why) *why = m;
        out = WideTree{};
        return false;
    };
    if (nn == 0 || nn >= (size_t)kWIndex || root >= nn) return fail("node count or root out of range");
    const Tree T{nodes8, nn};

    // every node the traversal can reach, in post order (successors first),
    // with cycles refused; pure = no instance, mesh or light node in the
    // subtree, so the ray cannot change while the subtree is walked
    std::vector<uint8_t> state(nn, 0);  // 0 new, 1 on the path, 2 done
    std::vector<uint8_t> pure(nn, 0);
    std::vector<uint32_t> post;
    {
        std::vector<std::pair<uint32_t, uint32_t>> path;  // node, next successor
        path.emplace_back(root, 0u);
        state[root] = 1;
        while (!path.empty()) {
            auto& top = path.back();
            const uint32_t n = top.first;
            if (top.second < T.num_succ(n)) {
                const uint32_t s = T.succ(n, top.second++);
                if (s >= nn) return fail("successor out of range");
                if (state[s] == 1) return fail("the tree has a cycle");
                if (state[s] == 0) {
                    state[s] = 1;
                    path.emplace_back(s, 0u);
                }
                continue;
            }
            if (T.nan_box(n)) return fail("NaN box bound");
            const Kind k = T.kind(n);
            bool p = !T.world(n) && k != kLight && k != kInstance && k != kMeshLeaf;
            if (p && k == kInner) p = pure[n + 1] && pure[T.w0(n)];
            pure[n] = p ? 1 : 0;
            state[n] = 2;
            post.push_back(n);
            path.pop_back();
        }
    }

    out.map.assign(nn, kWNone);
    std::vector<uint32_t> work;
    bool deferred = false;
    auto get_wide = [&](uint32_t n) -> uint32_t {
        if (out.map[n] == kWNone) {
            out.map[n] = (uint32_t)out.nodes.size();
            out.nodes.emplace_back();
            work.push_back(n);
        }
        return out.map[n];
    };
    // inner nodes taken from refs: the root, mesh-leaf members, instance roots
    if (T.kind(root) == kInner) get_wide(root);
    for (uint32_t n : post) {
        const Kind k = T.kind(n);
        if (k != kMeshLeaf && k != kInstance) continue;
        for (uint32_t i = 0; i < T.num_succ(n); ++i)
            if (T.kind(T.succ(n, i)) == kInner) get_wide(T.succ(n, i));
    }
    while (!work.empty()) {
        const uint32_t P = work.back();
        work.pop_back();
        const bool world = T.world(P);
        // whether the binary traversal tests x against the ray of P's visit
        auto testable = [&](uint32_t x) { return world ? T.world(x) : (bool)pure[P]; };
        auto entry = [&](uint32_t x) -> uint32_t {
            if (!testable(x)) {
                deferred = true;
                if (T.kind(x) == kInner) get_wide(x);
                return kWRef | kWUntested | x;
            }
            if (T.kind(x) == kInner) return get_wide(x);
            return kWRef | x;
        };
        WideNodeHost h;
        std::memset(&h, 0, sizeof(h));
        uint32_t flags = (world ? kW4World : 0u) | (T.axis(P) << 4);
        const uint32_t cs[2] = {P + 1, T.w0(P)};
        for (int c = 0; c < 2; ++c) {
            const uint32_t C = cs[c];
            uint32_t slot_nodes[2] = {C, kWNone};
            bool expand = false;
            if (T.kind(C) == kInner && testable(C)) {
                const uint32_t g0 = C + 1, g1 = T.w0(C);
                expand = testable(g0) && testable(g1) && T.contains(C, g0) && T.contains(C, g1);
                if (expand) {
                    slot_nodes[0] = g0;
                    slot_nodes[1] = g1;
                    flags |= (c == 0 ? kW4ExpandL : kW4ExpandR) | (T.axis(C) << (c == 0 ? 6 : 8));
                }
            }
            for (int j = 0; j < 2; ++j) {
                const int s = 2 * c + j;
                const uint32_t x = slot_nodes[j];
                if (x == kWNone) {
                    h.child[s] = kWNone;
                    continue;
                }
                // entry() may grow out.nodes: write through the index afterwards
                h.child[s] = entry(x);
                for (int a = 0; a < 3; ++a) {
                    h.lo[a][s] = T.lo(x, a);
                    h.hi[a][s] = T.hi(x, a);
                }
            }
        }
        h.meta[0] = flags;
        // the visiting order of the four slots for each ray octant (bit a of
        // the octant: direction component a <= 0): the near side of P's split
        // axis first, within it the near side of an expanded child's; two
        // bits per slot, first visited lowest, one byte per octant
        for (uint32_t o = 0; o < 8; ++o) {
            const bool right_first = (o >> T.axis(P)) & 1u;
            const uint32_t ax_l = (flags >> 6) & 3u, ax_r = (flags >> 8) & 3u;
            const bool swap_l = (flags & kW4ExpandL) && ((o >> ax_l) & 1u);
            const bool swap_r = (flags & kW4ExpandR) && ((o >> ax_r) & 1u);
            const uint32_t l = swap_l ? 0x1u : 0x4u;  // slots (1,0) or (0,1)
            const uint32_t r = swap_r ? 0xBu : 0xEu;  // slots (3,2) or (2,3)
            const uint32_t order = right_first ? (r | l << 4) : (l | r << 4);
            h.meta[1 + o / 4] |= order << (8 * (o % 4));
        }
        out.nodes[out.map[P]] = h;
    }

    // deepest stack: a wide node with k entries pushes k - 1 of them before
    // taking the first, a mesh leaf of n members pushes n - 1, and below a
    // ray that may not skip boxes inner nodes are walked one by one (one push
    // each); the larger of the two counts
    std::vector<int> need(nn, 0);
    for (uint32_t n : post) {
        int v = 0;
        switch (T.kind(n)) {
            case kInner:
                if (out.map[n] != kWNone) {
                    const WideNodeHost& h = out.nodes[out.map[n]];
                    int k = 0, m = 0;
                    for (int s = 0; s < 4; ++s) {
                        if (h.child[s] == kWNone) continue;
                        ++k;
                        // the entry's binary node: the ref's, else slot s's (the
                        // left or right child, or one of their children)
                        uint32_t bx = (h.child[s] & kWRef) ? (h.child[s] & kWIndex) : kWNone;
                        if (bx == kWNone) {
                            const uint32_t C = s < 2 ? n + 1 : T.w0(n);
                            const bool ex = (h.meta[0] & (s < 2 ? kW4ExpandL : kW4ExpandR)) != 0u;
                            bx = !ex ? C : ((s & 1) ? T.w0(C) : C + 1);
                        }
                        m = std::max(m, need[bx]);
                    }
                    v = (k > 0 ? k - 1 : 0) + m;
                }
                v = std::max(v, 1 + std::max(need[n + 1], need[T.w0(n)]));
                break;
            case kMeshLeaf: {
                const uint32_t cnt = T.count(n);
                int m = 0;
                for (uint32_t i = 1; i <= cnt; ++i) m = std::max(m, need[n + i]);
                v = cnt ? (int)cnt - 1 + m : 0;
                break;
            }
            case kInstance: v = need[T.w0(n)]; break;
            default: break;
        }
        need[n] = v;
    }
    out.stack_need = need[root];
    out.root = root;
    if (out.stack_need > max_stack) return fail("the four-wide traversal needs a deeper stack than allowed");
    // closest hit re-tests every binary node when it is taken and relies on
    // each entry box being tested against the ray of its parent's visit: no
    // deferred entries
    out.closest = !deferred;
    return true;
}

}  // namespace nb

#include "host_common.h"

extern "C" int noor_wide_tree_info(const noor_payload* payload, uint32_t root, uint32_t* num_wide,
                                   uint32_t* num_expanded, uint32_t* stack_need, uint32_t* closest) {
    if (!payload || !payload->bvh_min_right_start || !payload->bvh_max_axis_count || !num_wide || !num_expanded ||
        !stack_need || !closest || root >= payload->num_bvh_nodes)
        return set_error(NOOR_ERR_INVALID, "noor_wide_tree_info: bad argument");
    const size_t nn = payload->num_bvh_nodes;
    std::vector<uint32_t> w(8 * nn);
    for (size_t i = 0; i < nn; ++i) {
        std::memcpy(&w[8 * i], payload->bvh_min_right_start + 4 * i, 16);
        std::memcpy(&w[8 * i + 4], payload->bvh_max_axis_count + 4 * i, 16);
    }
    nb::WideTree t;
    std::string why;
    if (!nb::build_wide_tree(w.data(), nn, root, nb::kWideMaxStack, t, &why))
        return set_error(NOOR_ERR_UNSUPPORTED, "four-wide tree: " + why);
    uint32_t ex = 0;
    for (const nb::WideNodeHost& h : t.nodes)
        ex += ((h.meta[0] & nb::kW4ExpandL) ? 1u : 0u) + ((h.meta[0] & nb::kW4ExpandR) ? 1u : 0u);
    *num_wide = (uint32_t)t.nodes.size();
    *num_expanded = ex;
    *stack_need = (uint32_t)t.stack_need;
    *closest = t.closest ? 1u : 0u;
    clear_error();
    return NOOR_OK;
}
