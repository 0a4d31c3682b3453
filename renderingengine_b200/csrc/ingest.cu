// Scene ingestion: instance expansion of object-space SceneAbiV0 records
// into world-space CanonicalTraversalTriangle records on the GPU
// (BuildCanonicalTraversalScene, src/rt/gpu/CanonicalTraversalScene.cpp:69).
//
// The host checks the per-instance / per-geometry ranges (O(instances x
// geometries)) and lays out one segment per visible (instance, geometry)
// pair with its first output index, so the traversal ID of every triangle
// is known up front; one device thread then expands one triangle.  Positions
// are transformed as TransformPosition (:14-25) and normals as
// TransformNormal (:27-47), in the reference's operand order with explicit
// round-to-nearest operations, the normal length in double precision.  A
// triangle that references a vertex out of range or transforms to a
// non-finite value raises a flag that the host turns into the reference's
// error.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "re_b200.h"
#include "runtime.h"

static_assert(sizeof(re_gpu_vertex_v0) == 64, "GpuVertexV0");
static_assert(sizeof(re_gpu_geometry_v0) == 64, "GpuGeometryV0");
static_assert(sizeof(re_gpu_instance_v0) == 224, "GpuInstanceV0");
static_assert(sizeof(re_gpu_material_v0) == 128, "GpuMaterialV0");
static_assert(sizeof(re_canonical_triangle) == 176, "CanonicalTraversalTriangle");

namespace re {
namespace {

// One visible (instance, geometry) pair.
struct Segment {
    uint32_t first_out;    // traversal ID of its first triangle
    uint32_t instance;
    uint32_t geometry;
    uint32_t material;
};

constexpr uint32_t kBadVertex = 1u, kNonFinite = 2u;

struct ExpandArgs {
    const re_gpu_vertex_v0* vertices;
    const uint32_t* indices;
    const re_gpu_geometry_v0* geometries;
    const re_gpu_instance_v0* instances;
    const re_gpu_material_v0* materials;
    const Segment* segments;
    uint32_t segment_count, triangle_count, vertex_count, pad;
    re_canonical_triangle* out;
    uint32_t* flags;
};

__device__ __forceinline__ float dot_row(const re_float4& r, const re_float4& p) {
    return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(r.x, p.x), __fmul_rn(r.y, p.y)), __fmul_rn(r.z, p.z)), r.w);
}

__device__ __forceinline__ bool finite3(float x, float y, float z) { return isfinite(x) && isfinite(y) && isfinite(z); }

__global__ void k_expand(ExpandArgs a) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.triangle_count) return;
    // Segment of triangle t: the last one starting at or before t.
    uint32_t lo = 0, hi = a.segment_count;
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a.segments[mid].first_out <= t) lo = mid;
        else hi = mid;
    }
    const Segment sg = a.segments[lo];
    const re_gpu_instance_v0& inst = a.instances[sg.instance];
    const re_gpu_geometry_v0& geo = a.geometries[sg.geometry];
    const re_gpu_material_v0& mat = a.materials[sg.material];
    const uint32_t local = t - sg.first_out;
    const uint32_t first_index = geo.index_range.x + local * 3u;
    re_canonical_triangle out;
    const re_mat4_rows& o2w = inst.object_to_world;
    const re_mat4_rows& w2o = inst.world_to_object;
    for (int c = 0; c < 3; ++c) {
        const uint32_t vi = a.indices[first_index + c] + geo.index_range.z;
        if (vi >= a.vertex_count) {
            atomicOr(a.flags, kBadVertex);
            return;
        }
        const re_gpu_vertex_v0& v = a.vertices[vi];
        const float px = dot_row(o2w.row0, v.position), py = dot_row(o2w.row1, v.position),
                    pz = dot_row(o2w.row2, v.position);
        // World-to-object transposed, without the translation column.
        float nx = __fadd_rn(__fadd_rn(__fmul_rn(w2o.row0.x, v.normal.x), __fmul_rn(w2o.row1.x, v.normal.y)),
                             __fmul_rn(w2o.row2.x, v.normal.z));
        float ny = __fadd_rn(__fadd_rn(__fmul_rn(w2o.row0.y, v.normal.x), __fmul_rn(w2o.row1.y, v.normal.y)),
                             __fmul_rn(w2o.row2.y, v.normal.z));
        float nz = __fadd_rn(__fadd_rn(__fmul_rn(w2o.row0.z, v.normal.x), __fmul_rn(w2o.row1.z, v.normal.y)),
                             __fmul_rn(w2o.row2.z, v.normal.z));
        const double l2 = __dadd_rn(__dadd_rn(__dmul_rn(double(nx), double(nx)), __dmul_rn(double(ny), double(ny))),
                                    __dmul_rn(double(nz), double(nz)));
        if (!(l2 > 0.0) || !isfinite(l2)) {
            nx = ny = nz = 0.0f;
        } else {
            const float inv = __double2float_rn(__ddiv_rn(1.0, __dsqrt_rn(l2)));
            nx = __fmul_rn(nx, inv);
            ny = __fmul_rn(ny, inv);
            nz = __fmul_rn(nz, inv);
        }
        if (!finite3(px, py, pz) || !finite3(nx, ny, nz)) {
            atomicOr(a.flags, kNonFinite);
            return;
        }
        out.positions[c] = re_float4{px, py, pz, 1.0f};
        out.normals[c] = re_float4{nx, ny, nz, 0.0f};
        out.texcoords[c] = v.texcoord0;
    }
    out.identity = re_uint4{inst.metadata.z, geo.index_range.w + local, geo.identity.x, mat.metadata.z};
    out.metadata = re_uint4{geo.identity.w, mat.metadata.y, t, inst.metadata.w};
    a.out[t] = out;
}

}  // namespace
}  // namespace re

extern "C" RE_API re_status re_scene_expand_canonical(
    const re_gpu_vertex_v0* vertices, uint32_t vertex_count, const uint32_t* indices, uint32_t index_count,
    const re_gpu_geometry_v0* geometries, uint32_t geometry_count, const re_gpu_instance_v0* instances,
    uint32_t instance_count, const re_gpu_material_v0* materials, uint32_t material_count, re_canonical_triangle* out,
    uint32_t out_capacity, uint32_t* out_count, uint32_t memory, uint32_t device, void* stream) {
    using namespace re;
    if (out_count == nullptr) return set_error(RE_INVALID_ARGUMENT, "null count output");
    *out_count = 0u;
    if (vertices == nullptr || vertex_count == 0u || indices == nullptr || index_count == 0u || geometries == nullptr ||
        geometry_count == 0u || instances == nullptr || instance_count == 0u || materials == nullptr ||
        material_count == 0u || out == nullptr)
        return set_error(RE_INVALID_ARGUMENT,
                         "Canonical traversal expansion requires a validated, identified scene view.");
    if (memory != RE_MEMORY_HOST && memory != RE_MEMORY_DEVICE)
        return set_error(RE_INVALID_ARGUMENT, "memory kind is invalid");
    if (uint64_t(index_count / 3u) * instance_count > 0xffffffffull)
        return set_error(RE_INVALID_ARGUMENT, "Canonical traversal expansion exceeds uint32 triangle identity.");
    // Segments in the reference's output order, with its range checks.
    std::vector<Segment> segs;
    uint64_t total = 0;
    for (uint32_t i = 0; i < instance_count; ++i) {
        const re_uint4 m = instances[i].metadata;
        if ((m.w & RE_INSTANCE_FLAG_VISIBLE) == 0u) continue;
        if (m.x >= geometry_count || m.y > geometry_count - m.x)
            return set_error(RE_INVALID_ARGUMENT, "Canonical instance geometry range is invalid during traversal expansion.");
        for (uint32_t g = m.x; g < m.x + m.y; ++g) {
            const re_gpu_geometry_v0& geo = geometries[g];
            if (geo.identity.z >= material_count)
                return set_error(RE_INVALID_ARGUMENT, "Canonical traversal geometry references an invalid material.");
            const uint32_t tris = uint32_t((uint64_t(geo.index_range.y) + 2u) / 3u);  // one per started index triple
            if (tris == 0u) continue;
            const uint64_t last_first = uint64_t(geo.index_range.x) + uint64_t(tris - 1u) * 3u;
            if (last_first > index_count || 3u > index_count - last_first)
                return set_error(RE_INVALID_ARGUMENT, "Canonical traversal triangle index range is invalid.");
            segs.push_back(Segment{uint32_t(total), i, g, geo.identity.z});
            total += tris;
        }
    }
    if (total == 0u) return set_error(RE_INVALID_ARGUMENT, "Canonical traversal expansion produced no visible triangles.");
    if (total > out_capacity) return set_error(RE_INVALID_ARGUMENT, "output holds fewer records than the expansion");
    RE_CUDA_TRY(cudaSetDevice(int(device)));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    DeviceBuffer d_v, d_i, d_g, d_inst, d_m, d_seg, d_out, d_flags;
    RE_CUDA_TRY(d_v.reserve(size_t(vertex_count) * sizeof(re_gpu_vertex_v0)));
    RE_CUDA_TRY(d_i.reserve(size_t(index_count) * 4u));
    RE_CUDA_TRY(d_g.reserve(size_t(geometry_count) * sizeof(re_gpu_geometry_v0)));
    RE_CUDA_TRY(d_inst.reserve(size_t(instance_count) * sizeof(re_gpu_instance_v0)));
    RE_CUDA_TRY(d_m.reserve(size_t(material_count) * sizeof(re_gpu_material_v0)));
    RE_CUDA_TRY(d_seg.reserve(segs.size() * sizeof(Segment)));
    RE_CUDA_TRY(d_flags.reserve(4u));
    re_canonical_triangle* dst = out;
    if (memory == RE_MEMORY_HOST) {
        RE_CUDA_TRY(d_out.reserve(size_t(total) * sizeof(re_canonical_triangle)));
        dst = static_cast<re_canonical_triangle*>(d_out.ptr);
    }
    RE_CUDA_TRY(cudaMemcpyAsync(d_v.ptr, vertices, size_t(vertex_count) * sizeof(re_gpu_vertex_v0),
                                cudaMemcpyHostToDevice, s));
    RE_CUDA_TRY(cudaMemcpyAsync(d_i.ptr, indices, size_t(index_count) * 4u, cudaMemcpyHostToDevice, s));
    RE_CUDA_TRY(cudaMemcpyAsync(d_g.ptr, geometries, size_t(geometry_count) * sizeof(re_gpu_geometry_v0),
                                cudaMemcpyHostToDevice, s));
    RE_CUDA_TRY(cudaMemcpyAsync(d_inst.ptr, instances, size_t(instance_count) * sizeof(re_gpu_instance_v0),
                                cudaMemcpyHostToDevice, s));
    RE_CUDA_TRY(cudaMemcpyAsync(d_m.ptr, materials, size_t(material_count) * sizeof(re_gpu_material_v0),
                                cudaMemcpyHostToDevice, s));
    RE_CUDA_TRY(cudaMemcpyAsync(d_seg.ptr, segs.data(), segs.size() * sizeof(Segment), cudaMemcpyHostToDevice, s));
    RE_CUDA_TRY(cudaMemsetAsync(d_flags.ptr, 0, 4u, s));
    ExpandArgs a{};
    a.vertices = static_cast<const re_gpu_vertex_v0*>(d_v.ptr);
    a.indices = static_cast<const uint32_t*>(d_i.ptr);
    a.geometries = static_cast<const re_gpu_geometry_v0*>(d_g.ptr);
    a.instances = static_cast<const re_gpu_instance_v0*>(d_inst.ptr);
    a.materials = static_cast<const re_gpu_material_v0*>(d_m.ptr);
    a.segments = static_cast<const Segment*>(d_seg.ptr);
    a.segment_count = uint32_t(segs.size());
    a.triangle_count = uint32_t(total);
    a.vertex_count = vertex_count;
    a.out = dst;
    a.flags = static_cast<uint32_t*>(d_flags.ptr);
    k_expand<<<(a.triangle_count + 255u) / 256u, 256, 0, s>>>(a);
    RE_CUDA_TRY(cudaGetLastError());
    uint32_t flags = 0;
    RE_CUDA_TRY(cudaMemcpyAsync(&flags, d_flags.ptr, 4u, cudaMemcpyDeviceToHost, s));
    if (memory == RE_MEMORY_HOST)
        RE_CUDA_TRY(cudaMemcpyAsync(out, dst, size_t(total) * sizeof(re_canonical_triangle), cudaMemcpyDeviceToHost, s));
    RE_CUDA_TRY(cudaStreamSynchronize(s));
    if (flags & kBadVertex)
        return set_error(RE_INVALID_ARGUMENT, "Canonical traversal triangle references an invalid vertex.");
    if (flags & kNonFinite)
        return set_error(RE_INVALID_ARGUMENT, "Canonical traversal transform produced non-finite geometry.");
    *out_count = uint32_t(total);
    return clear_error();
}
