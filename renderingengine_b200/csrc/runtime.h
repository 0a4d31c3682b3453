// Internal runtime helpers shared by the C-ABI translation units: error
// reporting, CUDA checks and the scene object.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "re_b200.h"
#include "sah_builder.h"

namespace re {

re_status set_error(re_status code, const std::string& message);
re_status clear_error();

#define RE_CUDA_TRY(expr)                                                             \
    do {                                                                              \
        cudaError_t re_err_ = (expr);                                                 \
        if (re_err_ != cudaSuccess) {                                                 \
            return ::re::set_error(re_err_ == cudaErrorMemoryAllocation               \
                                       ? RE_OUT_OF_MEMORY                             \
                                       : RE_CUDA_ERROR,                               \
                                   std::string(#expr) + ": " +                        \
                                       cudaGetErrorString(re_err_));                  \
        }                                                                             \
    } while (0)

// Device attribute record per leaf-ordered triangle (64 B): the data only the
// final hit needs (shading normals and the canonical identity tuple).
struct alignas(16) DeviceAttr {
    float n0[4];   // n0.xyz, w unused
    float n1[4];
    float n2[4];
    uint32_t ids[4];  // instance, primitive, geometry, material
};
static_assert(sizeof(DeviceAttr) == 64, "attribute record is 64 bytes");

// Scratch buffer that grows on demand and is reused between calls.
struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    int device = 0;
    cudaError_t reserve(size_t n);
    void release();
    ~DeviceBuffer() { release(); }
};

}  // namespace re

struct re_scene;

namespace re {
// GPU LBVH build of a scene (Morton codes, radix sort, Karras hierarchy,
// refit); fills sc->flat and uploads the device layout.
re_status build_lbvh_on_device(re_scene* sc, const re_canonical_triangle* tris);
// The same build from CanonicalTraversalTriangle records already in device
// memory (validated on the device; traversal IDs must be a permutation of
// 0 .. triangle_count - 1); the leaf-ordered triangle and attribute records
// are made on the device.
re_status build_lbvh_from_device_records(re_scene* sc, const re_canonical_triangle* d_tris);
// Child-pair device nodes of sc->flat.
re_status upload_scene_nodes(re_scene* sc);
// Leaf-ordered device triangle and attribute records from host records.
re_status upload_scene_triangles(re_scene* sc, const re_canonical_triangle* src_in_leaf_order_or_null,
                                 const re_canonical_triangle* src, const std::vector<uint32_t>& leaf_order);

// Renderer services for the render server (wavefront.cu).
// Film mean of paths [offset, offset + n) into pinned host memory, queued on
// `s` without synchronising.
re_status renderer_copy_mean_async(re_renderer* r, uint32_t offset, uint32_t n, void* host_dst, cudaStream_t s);
// Allocates the ReSTIR state now (so a budget can account for it).
re_status renderer_reserve_restir(re_renderer* r);
// Device bytes held by the renderer (path pool, tables, ReSTIR state).
uint64_t renderer_device_bytes(const re_renderer* r);
// Running totals since creation: launches' path rays and shadow rays.
re_status renderer_ray_totals(re_renderer* r, uint64_t* path_rays, uint64_t* shadow_rays);
}  // namespace re

struct re_scene {
    int device = 0;
    uint64_t fingerprint = 0;
    uint32_t generation = 0;
    uint32_t triangle_count = 0;
    uint32_t build_kind = 0;
    re::FlatBvh flat;               // host copy of the flattened tree
    re::DeviceLayout layout_meta;   // node_original / root flag (nodes freed after upload)
    // Resident device buffers.
    re::DeviceBuffer nodes;         // DeviceNode[]
    re::DeviceBuffer tris;          // DeviceTriangle[]
    re::DeviceBuffer attrs;         // DeviceAttr[]
    uint32_t device_node_count = 0;
    double build_ms = 0.0;
    double lbvh_gpu_ms = 0.0;    // device time of the GPU LBVH passes
    double lbvh_total_ms = 0.0;
    // Per-scene staging for host-memory trace batches and the work counter of
    // the persistent traversal kernels.
    re::DeviceBuffer stage_rays;
    re::DeviceBuffer stage_hits;
    re::DeviceBuffer work_counter;
    re::DeviceBuffer counters;
    // Four-wide nodes over the same triangles (re::WideNode), built on first
    // use by a renderer tuned for them.
    re::DeviceBuffer wide_nodes;
    uint32_t wide_node_count = 0;
    uint32_t wide_stack_bound = 0;
    // Eight-wide nodes, plain (re::Wide8Node) and compressed (re::Wide8QNode),
    // built on first use by a renderer tuned for them.
    re::DeviceBuffer eight_nodes, eight_qnodes;
    uint32_t eight_node_count = 0;
    uint32_t eight_stack_bound = 0;
    // Alpha masks: per leaf-ordered triangle texture coordinates + material
    // (2 x float4, made when any triangle is alpha-masked), and the tables
    // of re_scene_set_alpha_masks with their device AlphaView.
    bool alpha_masked = false;
    re::DeviceBuffer alpha_tc, alpha_materials, alpha_atlas, alpha_view;
    // Copy streams of chunked host-memory trace batches (created on first use).
    cudaStream_t copy_in = nullptr, copy_out = nullptr;
    ~re_scene() {
        if (copy_in) cudaStreamDestroy(copy_in);
        if (copy_out) cudaStreamDestroy(copy_out);
    }
};

namespace re {
// Builds and uploads the scene's four-wide nodes if it has none yet.
re_status ensure_wide_layout(re_scene* sc);
// Builds and uploads the scene's eight-wide nodes (plain and compressed).
re_status ensure_eight_layout(re_scene* sc);
}  // namespace re
