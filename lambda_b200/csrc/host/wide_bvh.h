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
//
// The compressed layout (quant below) adds a conservative 8-bit box per child. A
// traversal over it tests those boxes when it expands a node, pushes the children
// that pass with their (lower or equal) entry distances, and at each pop tests the
// child's exact record before it uses it: a child whose quantized test fails would
// fail the exact test too, so the nodes expanded, their order and the culling
// decisions are the exact layout's.
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
    // The compressed layout: per wide node `quant_stride` 16-byte words. Word 0 is
    // the node's origin o (the least child min per axis, 3 floats) and a packed word:
    // the biased float exponents e_x, e_y, e_z of the per-axis scales s = 2^(e - 127)
    // in bits 0-23, the child count in bits 24-27, bit 31 set when the node could not
    // be quantized (its children are then tested on their exact records). Then 6
    // bytes per child: lo x y z, hi x y z. A child's quantized box is
    // [o + lo * s, o + hi * s], computed in FP32 (one multiply, one add, no fused
    // multiply-add) and checked here to contain the child's exact box, so it passes
    // a ray's slab test whenever the exact box does, with an entry distance no larger.
    std::vector<uint32_t> quant;
    int quant_stride = 0;
};

// nodes: the binary BVH (TLAS rooted at node 0, BLAS roots given by the instances).
WideBvh build_wide_bvh(const lambda_bvh_node *nodes, int num_nodes, const lambda_instance *instances,
                       int num_instances, int width);

}  // namespace lambda_host
