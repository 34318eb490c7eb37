// Compressed 8-wide BVH for traversal, converted on the GPU from the binary
// Karras hierarchy of an LBVH build (the same tree whose collapsed form is
// exported in the reference's BvhNode layout).
//
// The format follows the idea of Ylitie, Karras and Laine, "Efficient
// Incoherent Ray Traversal on GPUs Through Compressed Wide BVHs" (HPG 2017):
// child boxes are stored as 8-bit offsets on a per-node power-of-two grid,
// internal children are stored contiguously, leaf primitives of a node are
// stored contiguously, and children are placed in slots by direction octant so
// that a ray visits them roughly near to far without sorting. The layout and
// the conversion below are this project's own:
//
//   * 80-byte node, five 16-byte loads;
//   * every quantised box contains its child's exact box with a margin of one
//     grid step on every side (directed rounding), so that the box test,
//     computed as t = q * (2^e * invDir) + (p - origin) * invDir, never culls a
//     box that contains a hit point (the step is far larger than the rounding
//     error of that expression);
//   * leaves hold at most WIDE_LEAF_MAX primitives of one contiguous range;
//     meta[slot] = (count << 5) | offset, offset relative to the node's
//     primitive base, so a node's hit leaves become one 32-bit primitive mask.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mb {

constexpr int WIDE_LEAF_MAX = 3;       // primitives per leaf in object hierarchies
constexpr int WIDE_TLAS_LEAF_MAX = 1;  // instances per leaf in the instance hierarchy

struct alignas(16) WideNode {
	float p[3];            // grid origin
	uint32_t eimask;       // biased exponents ex | ey << 8 | ez << 16, internal-slot mask << 24
	uint32_t childBase;    // index of the first internal child
	uint32_t primBase;     // first slot of this node's leaf primitives
	uint32_t meta[2];      // per slot (count << 5) | offset, 0 for internal / empty slots
	uint32_t qlo[3][2];    // per axis, 8 slots of 8 bits
	uint32_t qhi[3][2];
};
static_assert(sizeof(WideNode) == 80, "WideNode layout");

// Upper bound on the number of wide nodes for n primitives: every node with
// eight children expands seven binary nodes of its own; the others are
// disjoint subtrees of more than leafMax primitives.
inline size_t wide_node_capacity(size_t n, int leafMax) { return n / 7 + n / size_t(leafMax + 1) + 2; }

struct WideBuildArgs {
	int n;                          // leaves of the binary tree (primitives in use)
	int numInternal;                // n - 1
	int leafMax;
	const int32_t* children;        // 2 per binary internal node
	const int2* ranges;             // first/last sorted leaf per binary internal node
	const float4* nodeData;         // 2 per binary node: min.xyz, max.xyz (exact boxes)
	const int32_t* sortedIds;       // sorted leaf index -> primitive / instance id
	WideNode* nodes;                // capacity wide_node_capacity(n, leafMax)
	int32_t* prims;                 // n: wide leaf slot -> primitive / instance id
	uint32_t nodeCapacity;
	uint32_t* counters;             // device scratch, WIDE_COUNTERS entries
	int2* queueA;                   // device scratch, nodeCapacity entries each
	int2* queueB;
};
constexpr int WIDE_COUNTERS = 8;

// Converts the binary tree into the wide one on `stream`. Reads back the
// node count once (one synchronisation). Returns cudaErrorInvalidValue if
// the capacity was exceeded or the levels did not terminate.
cudaError_t build_wide(const WideBuildArgs& a, int32_t* numNodesOut, cudaStream_t stream);

} // namespace mb
