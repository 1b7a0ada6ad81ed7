// Wide BVH for the GPU traversal, derived from the reference's binary BVH
// (BVHNode, scene/bvh.h:30-52) without changing what a traversal finds.
//
// A wide node stands for one interior binary node N. Its children are the
// "frontier" of N's subtree after collapsing up to width - 2 interior nodes below N
// (the largest surface area first), kept in the reference's visiting order: depth
// first, right child before left (scene.h:114-116). Each child keeps the exact box
// of its binary node. A traversal tests a wide node's children when it expands the
// node, pushes the ones that pass in reverse visiting order together with their
// entry distance, and culls an entry at its pop when that distance exceeds the
// best hit so far, as the reference does for every node it pops.
//
// The collapsed binary nodes are never tested. That changes nothing: a child box
// lies inside its parent's box (the builder takes unions), and the slab test of
// BVHNode::intersect is monotone under containment (per axis, the entry distance of
// an inner box is at least the outer box's and its exit at most; NaN bounds are
// ignored by both), so a child passes only if its parent does, with an entry
// distance at least the parent's. The nodes that pass are therefore visited in the
// reference's order with the reference's culling decisions, and the primitives are
// tested in the same order against the same best distance.
#pragma once

#include <cstdint>
#include <vector>

#include "lambda_gpu.h"

namespace lambda_host {

struct WideBvh {
    int width = 0;
    // width child records per node, each 8 floats: min.xyz, code (int bits), max.xyz, 0.
    // code >= 0: the child's wide node; code < 0: leaf -(code + 1) of `leaves`.
    // Unused slots have an empty box (min +inf, max -inf), which no ray enters.
    std::vector<float> records;
    std::vector<int32_t> leaves;  // pairs (index, count) of the binary leaves
    std::vector<int32_t> code;    // per binary node: its wide node or leaf code (-1 - leaf); INT32_MIN for
                                  // binary nodes collapsed into a wide node (only roots are looked up)
    int stack_tlas = 0;           // entries a TLAS traversal can hold at once (every child passing)
    int stack_blas = 0;           // the same for the deepest BLAS
};

// nodes: the binary BVH (TLAS rooted at node 0, BLAS roots given by the instances).
WideBvh build_wide_bvh(const lambda_bvh_node *nodes, int num_nodes, const lambda_instance *instances,
                       int num_instances, int width);

}  // namespace lambda_host
