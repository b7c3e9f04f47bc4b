// Four-wide tree over a payload's binary BVH, built on the host at scene
// upload (wide_bvh.cpp) and walked by trace_any4 and trace_closest4
// (traverse.cuh).
//
// A wide node stands for a binary inner node P and holds up to four entries:
// for each child C of P, C's two children when C is an inner node whose box
// contains theirs (C is "expanded"), else C itself.  Entries are kept in
// the binary tree's order (left child's side first), so a traversal that
// orders them by the ray's sign on P's and C's split axes visits leaves in
// exactly the order of the binary traversal (noor/cuda/bvh.cuh:193-234).
// Skipping C's own slab test changes no outcome: for a ray whose direction
// components are all normal floats and whose origin is finite, the slab
// test's per-axis intervals are monotone in the box bounds, so a box inside
// C can only pass where C passes; other rays walk the binary tree below
// that point, node by node.
//
// Entries whose slab test the binary traversal runs against a ray that may
// differ from the one at P's visit (an entry without instance bits under a
// top-level node, where an earlier sibling may have left an object-space
// ray; anything under an inner node whose subtree holds instance or light
// nodes) are deferred: pushed untested, in order, and tested when taken,
// against the ray of that moment, as the binary traversal does.
//
// Closest hit shrinks the hit distance as it goes, so a wide node's tests
// (at its visit) may pass an entry the binary traversal (later, with a
// shorter distance) would miss.  trace_closest4 therefore tests every binary
// node again when it takes it, with the distance of that moment; an inner
// entry passed in this way only leads to boxes inside it, which miss
// whenever it misses.  Trees with deferred entries keep the binary closest
// hit.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace nb {

// stack and child-slot words
constexpr uint32_t kWRef = 0x80000000u;       // a binary node (else the index of a wide node)
constexpr uint32_t kWUntested = 0x40000000u;  // with kWRef: its box is tested when it is taken
constexpr uint32_t kWIndex = 0x3FFFFFFFu;
constexpr uint32_t kWNone = 0xFFFFFFFFu;
// deepest stack a tree may need to be used (words per thread)
constexpr int kWideMaxStack = 96;
// meta[0] bits; the split axes of P, the left and the right child at bits
// 4, 6 and 8
constexpr uint32_t kW4World = 1u;    // P resets the ray to world space (a top-level node)
constexpr uint32_t kW4ExpandL = 2u;  // slots 0, 1 hold the left child's children
constexpr uint32_t kW4ExpandR = 4u;  // slots 2, 3 hold the right child's children

// 128 bytes: the four entry boxes as structure of arrays, the entry words,
// and meta = {flags and axes, slot order for ray octants 0-3, for octants
// 4-7, 0}
struct WideNodeHost {
    float lo[3][4];
    float hi[3][4];
    uint32_t child[4];
    uint32_t meta[4];
};
static_assert(sizeof(WideNodeHost) == 128, "wide node layout");

struct WideTree {
    std::vector<WideNodeHost> nodes;
    std::vector<uint32_t> map;  // binary inner node -> its wide node (kWNone where there is none)
    uint32_t root = 0;          // the binary root the tree was built from
    int stack_need = 0;         // the deepest stack trace_any4 / trace_closest4 can reach
    bool closest = false;       // trace_closest4 may use the tree
};

// Collapse the binary tree (8 words per node: min.xyz, w0, max.xyz, w1, as
// the payload's two uint4 arrays interleaved) reachable from `root`.
// Returns false, with the reason in *why, when the tree has a cycle, a NaN
// box bound, more nodes than the stack words can address or a deeper stack
// than `max_stack`; trace_any4 is then not used for the scene.
bool build_wide_tree(const uint32_t* nodes8, size_t nn, uint32_t root, int max_stack, WideTree& out,
                     std::string* why);

}  // namespace nb
