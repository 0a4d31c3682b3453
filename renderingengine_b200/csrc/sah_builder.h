// Host-side binned-SAH BVH builder and the conversion of its flattened tree
// into the device layout the traversal kernels read.
//
// The build reproduces the deterministic topology of the reference CPU build
// Rt::Cpu::Bvh<float>::Rebuild (include/rt/cpu/Bvh.hpp:82-133, BuildRange
// :562-616, FindSahSplit :434-504, MedianPartition :506-537): the same binning
// arithmetic (promoted to double), the same strict-less tie rule (lowest axis,
// then lowest bin wins), the same stable partition and the same stable
// (centroid, primitive ID, index) median fallback.  Node numbering is the
// reference's pre-order, so the flattened 48-byte records equal the ones
// SoftwareGpu::FlattenCanonicalL3BinnedSah (src/rt/software_gpu/SoftwareGpu.cpp
// :1109-1247) produces.  Sub-trees below the top levels are built on separate
// host threads; each thread writes a contiguous pre-order range, so the
// result does not depend on the thread count.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "re_b200.h"

namespace re {

struct HostTriangle {
    float v[3][3];
    uint32_t primitive_id;  // stable traversal ID
};

struct FlatBvh {
    std::vector<re_software_node> nodes;     // pre-order, reference layout
    std::vector<uint32_t> leaf_order;        // source triangle index per leaf slot
    uint32_t max_depth = 0;
    uint32_t leaf_count = 0;
};

// Builds the binned-SAH tree.  Returns false with `error` set on invalid input
// (non-finite triangle, zero leaf size, depth above 128).
bool build_binned_sah(const std::vector<HostTriangle>& triangles, uint32_t bins,
                      uint32_t max_leaf_size, uint32_t threads, FlatBvh& out,
                      std::string& error);

// Device node: the two children of one interior node side by side, 64 bytes,
// so one node fetch is four aligned 16-byte loads and yields both child boxes.
//   a = (L.min.x, L.max.x, L.min.y, L.max.y)
//   b = (L.min.z, L.max.z, R.min.x, R.max.x)
//   c = (R.min.y, R.max.y, R.min.z, R.max.z)
//   d = (left ref, right ref, left leaf count, right leaf count)
// A child with leaf count 0 is an interior node (ref = device node index);
// otherwise ref is the first leaf-ordered triangle of that leaf.  The original
// binary node index of each child is kept in `orig` for traversal counters and
// tie order (reference near-first rule compares node indices).
struct alignas(16) DeviceNode {
    float a[4];
    float b[4];
    float c[4];
    uint32_t d[4];
};
static_assert(sizeof(DeviceNode) == 64, "device node is 64 bytes");

// Device triangle, 64 bytes, leaf order:
//   p0 = (v0.xyz, flags as bits)   e1 = (v1 - v0, 0)   e2 = (v2 - v0, 0)
//   key = (instance, primitive, traversal ID, canonical source index)
// The edges are the same float subtractions the Moller-Trumbore test in
// software_common.hlsli:125-172 performs, so the test is bit-identical.
// Triangle record of the traversal: p0 and the two edges, the flags in p0[3]
// and the (instance, primitive) key also in e1[3] / e2[3] (as bits), so a
// triangle test reads the first 48 bytes; key[] repeats the key with the
// traversal ID and the original index for the host.
struct alignas(16) DeviceTriangle {
    float p0[4];
    float e1[4];
    float e2[4];
    uint32_t key[4];
};
static_assert(sizeof(DeviceTriangle) == 64, "device triangle is 64 bytes");

// Flag bits packed into DeviceTriangle::p0[3].
enum : uint32_t {
    kTriDoubleSided = 1u << 0,
    kTriCastsShadow = 1u << 1,
    kTriAlphaMask = 1u << 2,    // GeometryFlagAlphaMask or MaterialFlagAlphaMask (SceneAbiV0.hpp:20, 42)
};

struct DeviceLayout {
    std::vector<DeviceNode> nodes;           // interior nodes, pre-order; root = 0
    std::vector<uint32_t> node_original;     // 2 per device node: original child indices
    uint32_t root_is_leaf = 0;
};

// Converts the flattened binary tree into child-pair device nodes.
void build_device_layout(const FlatBvh& flat, DeviceLayout& out);

// Four-wide device node, 128 bytes: the boxes of up to four children stored
// per axis (one 16-byte lane per bound and axis, so a node is eight aligned
// 16-byte loads) and the child references.  count[c] == 0: interior child,
// its reference a wide node index; 1..15: leaf of that many leaf-ordered
// triangles starting at its reference; kWideEmpty: no child (its box is +inf
// on every bound, which no slab test enters).  entry[c] is the child as the
// traversal stacks it, reference | count << kWideLeafShift (kWideEmpty for
// no child), so a traversal step loads the six plane vectors and the entries.
constexpr uint32_t kWideEmpty = 0xffffffffu;
constexpr uint32_t kWideLeafShift = 28u;
struct alignas(16) WideNode {
    float lo_x[4], hi_x[4];
    float lo_y[4], hi_y[4];
    float lo_z[4], hi_z[4];
    uint32_t entry[4];
    uint32_t count[4];
};
static_assert(sizeof(WideNode) == 128, "wide node is 128 bytes");

struct WideLayout {
    std::vector<WideNode> nodes;  // root = 0; a node's interior children are numbered consecutively
    uint32_t max_depth = 0;       // wide levels
    uint32_t stack_bound = 0;     // most stack entries a near-first traversal can hold
};

// Collapses the flattened binary tree into four-wide nodes over the same
// leaf-ordered triangles: a wide node takes its binary node's two children
// and repeatedly opens the interior child with the largest surface area
// until it has four children or only leaves.  Children keep the binary
// tree's left-to-right order.
void build_wide_layout(const FlatBvh& flat, WideLayout& out);

// Eight-wide nodes, collapsed from the same binary tree with the same rule
// (open the largest interior child until eight children or only leaves).
// Plain form: the children's exact boxes, lo / hi per axis as two 16-byte
// lanes each (the entry planes of an axis are one 32-byte pair), then the
// child entries (reference | count << kWideLeafShift, kWideEmpty for none):
// 224 bytes, padded to 256.  An empty slot's box is +inf on every bound.
struct alignas(16) Wide8Node {
    float lo_x[8], hi_x[8];
    float lo_y[8], hi_y[8];
    float lo_z[8], hi_z[8];
    uint32_t entry[8];
    uint32_t pad[8];
};
static_assert(sizeof(Wide8Node) == 256, "eight-wide node is 256 bytes");

// Compressed form (96 bytes, six 16-byte lanes): the node's origin (the
// minimum corner of its children's union) and a power-of-two scale 2^e per
// axis; per child and axis an 8-bit lower and upper bound q such that
// origin + q * 2^e, added with rounding toward -inf (lower) or +inf (upper),
// contains the child's exact box.  Empty slots carry an inverted box
// (lo 255, hi 0), which no slab test enters.
struct alignas(16) Wide8QNode {
    float origin[3];
    uint8_t exponent[3];   // scale = 2^(exponent - 127), as a float's biased exponent
    uint8_t pad0;
    uint8_t lo_x[8], hi_x[8];
    uint8_t lo_y[8], hi_y[8];
    uint8_t lo_z[8], hi_z[8];
    uint32_t entry[8];
};
static_assert(sizeof(Wide8QNode) == 96, "compressed eight-wide node is 96 bytes");

struct Wide8Layout {
    std::vector<Wide8Node> nodes;   // root = 0
    std::vector<Wide8QNode> qnodes;  // the same nodes compressed
    uint32_t max_depth = 0;
    uint32_t stack_bound = 0;
};
void build_wide8_layout(const FlatBvh& flat, Wide8Layout& out);

}  // namespace re
