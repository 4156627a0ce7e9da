// Compressed 8-wide BVH: the layout the traversal kernels walk.
//
// The binary SAH tree of the compiled geometry (the reference's buildBvh
// tree, src/bvh.ts:16-178, kept as it is so it stays comparable with the
// reference's) is collapsed into nodes of up to eight children, after the
// compressed wide BVH of Ylitie, Karras and Laine ("Efficient Incoherent Ray
// Traversal on GPUs Through Compressed Wide BVHs", HPG 2017):
//
//   * A wide node is 80 bytes: the origin p and power-of-two scales 2^e of a
//     grid over its box, and each child's box as 8-bit grid coordinates,
//     rounded outwards, so the decoded box p + q * 2^e contains the child.
//   * Inner children are stored contiguously from child_base in slot order;
//     `imask` marks which slots are inner, so a child's index is child_base
//     plus the inner slots before it.
//   * Leaf children hold one to three triangles. A node's leaf triangles are
//     stored contiguously from tri_base in a copy of the triangles in wide
//     order (wtris); each child's meta byte holds its offset there and its
//     count in unary, so the children a ray hits become a 24-bit mask of
//     triangles to test.
//   * Children sit in slots by the direction of their centre from the
//     node's, so visiting the hit slots in the order given by the ray's
//     direction octant approximates near to far without a sort.
//
// wtris keeps the watertight test's vertices and, in its third w lane, the
// triangle's index in the compiled geometry, which every hit reports.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "device_scene.cuh"

namespace mcrt {

// Five 16-byte words per node:
//   w0  p.x, p.y, p.z (float bits), e.x | e.y << 8 | e.z << 16 | imask << 24
//       (e: the scale's biased float exponent byte)
//   w1  child_base, tri_base, meta of slots 0-3, meta of slots 4-7
//   w2  qlo.x of slots 0-7 (two words), qlo.y of slots 0-7
//   w3  qlo.z, qhi.x
//   w4  qhi.y, qhi.z
// meta: 0 an empty slot; 0x38 + slot an inner child (bits 5-7 = 001, bits
// 0-4 = 24 + slot, its bit in the traversal's hit mask before the octant
// swizzle); otherwise a leaf, count in unary in bits 5-7 (1, 3 or 7) and the
// offset of its first triangle from tri_base in bits 0-4 (0 to 21).
constexpr int kWideNodeWords = 5;
constexpr int kWideLeafMax = 3;

// Builds the wide tree of a binary tree in the reference's layout (nodes:
// first, count, axis; the children of inner node i at nodes[i].first and
// first + 1; bounds: lo xyz, hi xyz per node) over `tris` (3 float4 per
// triangle in binary order, as the traversal packs them). `root_count` > 0
// when the root itself is a leaf of that many triangles. Outputs: wnodes
// (kWideNodeWords uint4 per node; room for max(n, 1) nodes), wtris (3 float4
// per triangle), `items` scratch for 2 n work items, `counters` 4 device
// unsigned. Writes the node count to *wide_nodes. Synchronises the stream.
// Returns cudaErrorInvalidValue, having written nothing out of bounds, when
// the binary tree reaches a node or a triangle twice (it is not a tree).
cudaError_t build_wide_bvh(const int* nodes, const float* bounds, int root_count, const float4* tris, int n,
                           uint4* wnodes, float4* wtris, void* items, unsigned* counters, int* wide_nodes,
                           cudaStream_t s);

// Bytes of the `items` scratch build_wide_bvh needs for n triangles.
size_t wide_bvh_item_bytes(int n);

}  // namespace mcrt
