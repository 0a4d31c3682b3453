// Scene residency (IGpuTraversalBackend::BuildOrUpdateScene) and the
// trace-batch entry points (RecordTraceClosestBatch / RecordTraceAnyBatch).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <thread>

#include "runtime.h"
#include "traverse.cuh"

namespace re {

static thread_local std::string g_last_error;

re_status set_error(re_status code, const std::string& message) {
    g_last_error = message;
    return code;
}

re_status clear_error() {
    g_last_error.clear();
    return RE_SUCCESS;
}

cudaError_t DeviceBuffer::reserve(size_t n) {
    if (n <= bytes && ptr != nullptr) return cudaSuccess;
    release();
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    e = cudaMalloc(&ptr, n == 0 ? 16 : n);
    if (e != cudaSuccess) {
        ptr = nullptr;
        bytes = 0;
        return e;
    }
    bytes = n;
    return cudaSuccess;
}

void DeviceBuffer::release() {
    if (ptr != nullptr) {
        int cur = 0;
        cudaGetDevice(&cur);
        if (cur != device) cudaSetDevice(device);
        cudaFree(ptr);
        if (cur != device) cudaSetDevice(cur);
    }
    ptr = nullptr;
    bytes = 0;
}

TraceSceneView scene_view(const re_scene* sc) {
    TraceSceneView v;
    v.nodes = static_cast<const float4*>(sc->nodes.ptr);
    v.tris = static_cast<const float4*>(sc->tris.ptr);
    v.node_count = sc->device_node_count;
    v.tri_count = sc->triangle_count;
    const re_software_node& r = sc->flat.nodes[0];
    v.root_lo[0] = r.bounds_min.x; v.root_lo[1] = r.bounds_min.y; v.root_lo[2] = r.bounds_min.z;
    v.root_hi[0] = r.bounds_max.x; v.root_hi[1] = r.bounds_max.y; v.root_hi[2] = r.bounds_max.z;
    v.wide = static_cast<const float4*>(sc->wide_nodes.ptr);
    v.wide_count = sc->wide_node_count;
    v.wide_stack = sc->wide_stack_bound;
    v.alpha = static_cast<const AlphaView*>(sc->alpha_view.ptr);
    v.eight = static_cast<const float4*>(sc->eight_nodes.ptr);
    v.eightq = static_cast<const float4*>(sc->eight_qnodes.ptr);
    v.eight_count = sc->eight_node_count;
    v.eight_stack = sc->eight_stack_bound;
    return v;
}

re_status ensure_eight_layout(re_scene* sc) {
    if (sc->eight_node_count != 0u) return RE_SUCCESS;
    Wide8Layout w;
    build_wide8_layout(sc->flat, w);
    if (w.nodes.empty()) return set_error(RE_INVALID_ARGUMENT, "scene has no hierarchy");
    RE_CUDA_TRY(cudaSetDevice(sc->device));
    RE_CUDA_TRY(sc->eight_nodes.reserve(w.nodes.size() * sizeof(Wide8Node)));
    RE_CUDA_TRY(cudaMemcpy(sc->eight_nodes.ptr, w.nodes.data(), w.nodes.size() * sizeof(Wide8Node),
                           cudaMemcpyHostToDevice));
    RE_CUDA_TRY(sc->eight_qnodes.reserve(w.qnodes.size() * sizeof(Wide8QNode)));
    RE_CUDA_TRY(cudaMemcpy(sc->eight_qnodes.ptr, w.qnodes.data(), w.qnodes.size() * sizeof(Wide8QNode),
                           cudaMemcpyHostToDevice));
    sc->eight_node_count = uint32_t(w.nodes.size());
    sc->eight_stack_bound = w.stack_bound;
    return RE_SUCCESS;
}

re_status ensure_wide_layout(re_scene* sc) {
    if (sc->wide_node_count != 0u) return RE_SUCCESS;
    WideLayout w;
    build_wide_layout(sc->flat, w);
    if (w.nodes.empty()) return set_error(RE_INVALID_ARGUMENT, "scene has no hierarchy");
    RE_CUDA_TRY(cudaSetDevice(sc->device));
    RE_CUDA_TRY(sc->wide_nodes.reserve(w.nodes.size() * sizeof(WideNode)));
    RE_CUDA_TRY(cudaMemcpy(sc->wide_nodes.ptr, w.nodes.data(), w.nodes.size() * sizeof(WideNode),
                           cudaMemcpyHostToDevice));
    sc->wide_node_count = uint32_t(w.nodes.size());
    sc->wide_stack_bound = w.stack_bound;
    return RE_SUCCESS;
}

namespace {

constexpr uint32_t kInvalid = 0xffffffffu;
constexpr int kWarp = 32;

struct HitWriteView {
    const float4* attrs;  // DeviceAttr as 4 x float4
    const float4* tris;
};

// Builds the abi-v1 hit record the way PbrPopulateSoftwareTraversalHitL6
// (pbr_software_traversal.hlsli:150-186) reconstructs a hit.
__device__ __forceinline__ void write_hit_record(const HitWriteView& v, const TraceRay& ray,
                                                 const TraceHit& h, uint4 ray_identity,
                                                 float4* out) {
    if (h.status != 0u) {
        out[0] = make_float4(0.f, 0.f, 0.f, ray.tmax);
        out[1] = make_float4(0.f, 0.f, 0.f, 0.f);
        out[2] = make_float4(0.f, 0.f, 0.f, 0.f);
        reinterpret_cast<uint4*>(out)[3] = make_uint4(kInvalid, kInvalid, kInvalid, kInvalid);
        reinterpret_cast<uint4*>(out)[4] = make_uint4(ray_identity.x, RE_HIT_KIND_INVALID, h.status, ray_identity.y);
        reinterpret_cast<uint4*>(out)[5] = make_uint4(0, 0, 0, 0);
        return;
    }
    if (h.tri == kInvalid) {
        out[0] = make_float4(0.f, 0.f, 0.f, ray.tmax);
        out[1] = make_float4(0.f, 0.f, 0.f, 0.f);
        out[2] = make_float4(0.f, 0.f, 0.f, 0.f);
        reinterpret_cast<uint4*>(out)[3] = make_uint4(kInvalid, kInvalid, kInvalid, kInvalid);
        reinterpret_cast<uint4*>(out)[4] = make_uint4(ray_identity.x, RE_HIT_KIND_MISS, 0u, ray_identity.y);
        reinterpret_cast<uint4*>(out)[5] = make_uint4(0, 0, 0, 0);
        return;
    }
    const float4* a = v.attrs + size_t(h.tri) * 4u;
    const float4* tp = v.tris + size_t(h.tri) * 4u;
    const f3 e1 = from4(__ldg(tp + 1));
    const f3 e2 = from4(__ldg(tp + 2));
    const float w0 = 1.0f - h.u - h.v;
    f3 gn = normalize3(cross(e1, e2));
    const f3 n0 = from4(__ldg(a + 0)), n1 = from4(__ldg(a + 1)), n2 = from4(__ldg(a + 2));
    f3 sn = normalize3(w0 * n0 + h.u * n1 + h.v * n2);
    if (!h.front) {
        gn = -gn;
        sn = -sn;
    }
    const uint4 ids = __ldg(reinterpret_cast<const uint4*>(a + 3));
    const f3 p = ray.o + ray.d * h.t;
    out[0] = to4(p, h.t);
    out[1] = to4(gn, h.u);
    out[2] = to4(sn, h.v);
    reinterpret_cast<uint4*>(out)[3] = ids;
    reinterpret_cast<uint4*>(out)[4] =
        make_uint4(ray_identity.x, RE_HIT_KIND_TRIANGLE, h.front ? RE_HIT_FLAG_FRONT_FACE : 0u, ray_identity.y);
    reinterpret_cast<uint4*>(out)[5] = make_uint4(0, 0, 0, 0);
}

struct BatchArgs {
    TraceSceneView scene;
    HitWriteView view;
    const float4* rays;   // re_ray_record as 4 x float4
    float4* hits;         // re_hit_record as 6 x float4
    uint32_t count;
    uint32_t* work;       // persistent work counter
    unsigned long long* counters;  // 9 slots (re_traversal_counters order)
};

__device__ __forceinline__ void flush_counters(const TraceCounters& c, unsigned long long* g) {
    // Warp-aggregated accumulation of the per-ray counters.
    uint32_t vals[4] = {c.node_tests, c.tri_tests, c.leaf_visits, c.leaf_prims};
    unsigned long long sum[4];
    for (int k = 0; k < 4; ++k) {
        unsigned long long x = vals[k];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        sum[k] = x;
    }
    uint32_t mx_leaf = c.max_leaf, mx_stack = c.max_stack;
    for (int o = 16; o > 0; o >>= 1) {
        mx_leaf = max(mx_leaf, __shfl_xor_sync(0xffffffffu, mx_leaf, o));
        mx_stack = max(mx_stack, __shfl_xor_sync(0xffffffffu, mx_stack, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(g + 0, sum[0]);
        atomicAdd(g + 1, sum[1]);
        atomicAdd(g + 6, sum[2]);
        atomicAdd(g + 7, sum[3]);
        atomicMax(g + 5, (unsigned long long)mx_stack);
        atomicMax(g + 8, (unsigned long long)mx_leaf);
    }
}

// Persistent traversal: every warp pulls 32 consecutive rays from a global
// work counter until the batch is exhausted.
template <bool ANY, bool COUNT, int STACK>
__global__ void __launch_bounds__(128) trace_batch_kernel(BatchArgs args) {
    const int lane = threadIdx.x & 31;
    TraceOptions opt;
    opt.ignore_instance = kInvalid;
    opt.ignore_primitive = kInvalid;
    opt.shadow = false;
    while (true) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(args.work, uint32_t(kWarp));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= args.count) break;
        const uint32_t i = base + lane;
        TraceCounters c{};
        if (i < args.count) {
            const float4* rp = args.rays + size_t(i) * 4u;
            const float4 ot = __ldg(rp + 0);
            const float4 dt = __ldg(rp + 1);
            const uint4 ident = __ldg(reinterpret_cast<const uint4*>(rp + 2));
            TraceRay ray{mk(ot.x, ot.y, ot.z), mk(dt.x, dt.y, dt.z), ot.w, dt.w};
            const TraceHit h = trace<ANY, COUNT, STACK>(args.scene, ray, opt, &c);
            if (COUNT) {
                if (h.status == 1u) atomicAdd(args.counters + 3, 1ull);
                if (h.status == 2u) atomicAdd(args.counters + 2, 1ull);
                if (h.status == 3u) atomicAdd(args.counters + 4, 1ull);
            }
            write_hit_record(args.view, ray, h, ident, args.hits + size_t(i) * 6u);
        }
        if (COUNT) flush_counters(c, args.counters);
    }
}

struct LaunchShape {
    int grid = 0;
    int block = 128;
};

template <typename K>
LaunchShape persistent_shape(K kernel, int device) {
    static std::mutex mu;
    LaunchShape s;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, s.block, 0);
    if (per_sm <= 0) per_sm = 1;
    s.grid = sms * per_sm;
    return s;
}

template <bool ANY, bool COUNT>
cudaError_t launch_batch(re_scene* sc, BatchArgs args, cudaStream_t stream) {
    const uint32_t depth = sc->flat.max_depth;
    if (depth <= 64) {
        auto k = trace_batch_kernel<ANY, COUNT, 64>;
        const LaunchShape s = persistent_shape(k, sc->device);
        const int need = int((args.count + 127) / 128);
        k<<<need < s.grid ? need : s.grid, s.block, 0, stream>>>(args);
    } else {
        auto k = trace_batch_kernel<ANY, COUNT, 128>;
        const LaunchShape s = persistent_shape(k, sc->device);
        const int need = int((args.count + 127) / 128);
        k<<<need < s.grid ? need : s.grid, s.block, 0, stream>>>(args);
    }
    return cudaGetLastError();
}

re_status validate_batch(const re_scene* sc, const re_trace_batch* b) {
    if (b == nullptr) return set_error(RE_INVALID_ARGUMENT, "trace batch is null");
    if (b->fingerprint != sc->fingerprint || b->generation != sc->generation)
        return set_error(RE_MISSING_SCENE,
                         "trace batch fingerprint/generation does not match the resident scene");
    if (b->ray_count == 0) return RE_SUCCESS;
    if (b->rays == nullptr || b->hits == nullptr)
        return set_error(RE_INVALID_ARGUMENT, "trace batch rays/hits must be non-null");
    if (b->memory != RE_MEMORY_HOST && b->memory != RE_MEMORY_DEVICE)
        return set_error(RE_INVALID_ARGUMENT, "trace batch memory kind is invalid");
    return RE_SUCCESS;
}

// Host-memory batch in chunks: ray uploads on one copy stream, the
// traversal of chunk k on the caller's stream once its rays are in, hit
// downloads on a second copy stream once its traversal is done, so the two
// PCIe directions and the traversal overlap (with pinned host memory).
// Same kernel per chunk, so the same hits as one launch.
constexpr uint32_t kTraceChunk = 1u << 18;

template <bool ANY>
re_status run_trace_chunked(re_scene* sc, const re_trace_batch* b, cudaStream_t stream) {
    const uint32_t n = b->ray_count;
    RE_CUDA_TRY(sc->stage_rays.reserve(size_t(n) * sizeof(re_ray_record)));
    RE_CUDA_TRY(sc->stage_hits.reserve(size_t(n) * sizeof(re_hit_record)));
    RE_CUDA_TRY(sc->work_counter.reserve(sizeof(uint32_t)));
    if (sc->copy_in == nullptr) {
        RE_CUDA_TRY(cudaStreamCreateWithFlags(&sc->copy_in, cudaStreamNonBlocking));
        RE_CUDA_TRY(cudaStreamCreateWithFlags(&sc->copy_out, cudaStreamNonBlocking));
    }
    const uint32_t chunks = (n + kTraceChunk - 1u) / kTraceChunk;
    std::vector<cudaEvent_t> in(chunks, nullptr), run(chunks, nullptr);
    re_status st = RE_SUCCESS;
    auto ok = [&](cudaError_t e) {
        if (e != cudaSuccess && st == RE_SUCCESS)
            st = set_error(RE_RECORDING_FAILED, std::string("CUDA error: ") + cudaGetErrorString(e));
        return st == RE_SUCCESS;
    };
    auto* d_rays = static_cast<re_ray_record*>(sc->stage_rays.ptr);
    auto* d_hits = static_cast<re_hit_record*>(sc->stage_hits.ptr);
    for (uint32_t k = 0; k < chunks && st == RE_SUCCESS; ++k) {
        ok(cudaEventCreateWithFlags(&in[k], cudaEventDisableTiming));
        ok(cudaEventCreateWithFlags(&run[k], cudaEventDisableTiming));
    }
    for (uint32_t k = 0; k < chunks && st == RE_SUCCESS; ++k) {
        const uint32_t off = k * kTraceChunk, cnt = std::min(kTraceChunk, n - off);
        ok(cudaMemcpyAsync(d_rays + off, b->rays + b->ray_offset + off, size_t(cnt) * sizeof(re_ray_record),
                           cudaMemcpyHostToDevice, sc->copy_in)) &&
            ok(cudaEventRecord(in[k], sc->copy_in));
    }
    for (uint32_t k = 0; k < chunks && st == RE_SUCCESS; ++k) {
        const uint32_t off = k * kTraceChunk, cnt = std::min(kTraceChunk, n - off);
        if (!ok(cudaStreamWaitEvent(stream, in[k], 0)) ||
            !ok(cudaMemsetAsync(sc->work_counter.ptr, 0, sizeof(uint32_t), stream)))
            break;
        BatchArgs args;
        args.scene = scene_view(sc);
        args.view.attrs = static_cast<const float4*>(sc->attrs.ptr);
        args.view.tris = args.scene.tris;
        args.rays = reinterpret_cast<const float4*>(d_rays + off);
        args.hits = reinterpret_cast<float4*>(d_hits + off);
        args.count = cnt;
        args.work = static_cast<uint32_t*>(sc->work_counter.ptr);
        args.counters = nullptr;
        if (!ok(launch_batch<ANY, false>(sc, args, stream)) || !ok(cudaEventRecord(run[k], stream)) ||
            !ok(cudaStreamWaitEvent(sc->copy_out, run[k], 0)))
            break;
        ok(cudaMemcpyAsync(b->hits + b->hit_offset + off, d_hits + off, size_t(cnt) * sizeof(re_hit_record),
                           cudaMemcpyDeviceToHost, sc->copy_out));
    }
    ok(cudaStreamSynchronize(sc->copy_out));
    ok(cudaStreamSynchronize(stream));
    for (uint32_t k = 0; k < chunks; ++k) {
        if (in[k]) cudaEventDestroy(in[k]);
        if (run[k]) cudaEventDestroy(run[k]);
    }
    return st == RE_SUCCESS ? clear_error() : st;
}

re_status run_trace(re_scene* sc, const re_trace_batch* b, bool any, re_traversal_counters* out_counters) {
    if (sc == nullptr) return set_error(RE_MISSING_SCENE, "scene is null");
    re_status st = validate_batch(sc, b);
    if (st != RE_SUCCESS || b->ray_count == 0) return st;
    RE_CUDA_TRY(cudaSetDevice(sc->device));
    cudaStream_t stream = static_cast<cudaStream_t>(b->stream);
    if (b->memory == RE_MEMORY_HOST && out_counters == nullptr && b->ray_count > kTraceChunk)
        return any ? run_trace_chunked<true>(sc, b, stream) : run_trace_chunked<false>(sc, b, stream);
    const size_t ray_bytes = size_t(b->ray_count) * sizeof(re_ray_record);
    const size_t hit_bytes = size_t(b->ray_count) * sizeof(re_hit_record);
    const re_ray_record* d_rays = b->rays + b->ray_offset;
    re_hit_record* d_hits = b->hits + b->hit_offset;
    const bool host = b->memory == RE_MEMORY_HOST;
    if (host) {
        RE_CUDA_TRY(sc->stage_rays.reserve(ray_bytes));
        RE_CUDA_TRY(sc->stage_hits.reserve(hit_bytes));
        RE_CUDA_TRY(cudaMemcpyAsync(sc->stage_rays.ptr, b->rays + b->ray_offset, ray_bytes,
                                    cudaMemcpyHostToDevice, stream));
        d_rays = static_cast<const re_ray_record*>(sc->stage_rays.ptr);
        d_hits = static_cast<re_hit_record*>(sc->stage_hits.ptr);
    }
    RE_CUDA_TRY(sc->work_counter.reserve(sizeof(uint32_t)));
    RE_CUDA_TRY(cudaMemsetAsync(sc->work_counter.ptr, 0, sizeof(uint32_t), stream));
    BatchArgs args;
    args.scene = scene_view(sc);
    args.view.attrs = static_cast<const float4*>(sc->attrs.ptr);
    args.view.tris = args.scene.tris;
    args.rays = reinterpret_cast<const float4*>(d_rays);
    args.hits = reinterpret_cast<float4*>(d_hits);
    args.count = b->ray_count;
    args.work = static_cast<uint32_t*>(sc->work_counter.ptr);
    args.counters = nullptr;
    cudaError_t e;
    if (out_counters != nullptr) {
        RE_CUDA_TRY(sc->counters.reserve(9 * sizeof(unsigned long long)));
        RE_CUDA_TRY(cudaMemsetAsync(sc->counters.ptr, 0, 9 * sizeof(unsigned long long), stream));
        args.counters = static_cast<unsigned long long*>(sc->counters.ptr);
        e = any ? launch_batch<true, true>(sc, args, stream) : launch_batch<false, true>(sc, args, stream);
    } else {
        e = any ? launch_batch<true, false>(sc, args, stream) : launch_batch<false, false>(sc, args, stream);
    }
    RE_CUDA_TRY(e);
    if (out_counters != nullptr) {
        unsigned long long c[9];
        RE_CUDA_TRY(cudaMemcpyAsync(c, sc->counters.ptr, sizeof(c), cudaMemcpyDeviceToHost, stream));
        RE_CUDA_TRY(cudaStreamSynchronize(stream));
        out_counters->node_tests += c[0];
        out_counters->triangle_tests += c[1];
        out_counters->stack_overflows += c[2];
        out_counters->invalid_rays += c[3];
        out_counters->invalid_hits += c[4];
        out_counters->max_stack_depth = std::max<uint64_t>(out_counters->max_stack_depth, c[5]);
        out_counters->leaf_visits += c[6];
        out_counters->leaf_primitives += c[7];
        out_counters->max_leaf_occupancy = std::max<uint64_t>(out_counters->max_leaf_occupancy, c[8]);
    }
    if (host) {
        RE_CUDA_TRY(cudaMemcpyAsync(b->hits + b->hit_offset, d_hits, hit_bytes, cudaMemcpyDeviceToHost, stream));
        RE_CUDA_TRY(cudaStreamSynchronize(stream));
    }
    return clear_error();
}

bool finite4(const re_float4& v) {
    return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z);
}

}  // namespace

// Uploads a built tree and its leaf-ordered triangles; shared by the SAH path
// and the GPU LBVH path.
// Child-pair device nodes of the flattened tree.
re_status upload_scene_nodes(re_scene* sc) {
    DeviceLayout layout;
    build_device_layout(sc->flat, layout);
    sc->layout_meta.root_is_leaf = layout.root_is_leaf;
    sc->layout_meta.node_original = layout.node_original;
    RE_CUDA_TRY(cudaSetDevice(sc->device));
    RE_CUDA_TRY(sc->nodes.reserve(layout.nodes.size() * sizeof(DeviceNode)));
    RE_CUDA_TRY(cudaMemcpy(sc->nodes.ptr, layout.nodes.data(), layout.nodes.size() * sizeof(DeviceNode),
                           cudaMemcpyHostToDevice));
    sc->device_node_count = uint32_t(layout.nodes.size());
    return RE_SUCCESS;
}

re_status upload_scene_geometry(re_scene* sc, const re_canonical_triangle* src_in_leaf_order_or_null,
                                const re_canonical_triangle* src, const std::vector<uint32_t>& leaf_order) {
    const re_status nst = upload_scene_nodes(sc);
    if (nst != RE_SUCCESS) return nst;
    return upload_scene_triangles(sc, src_in_leaf_order_or_null, src, leaf_order);
}

re_status upload_scene_triangles(re_scene* sc, const re_canonical_triangle* src_in_leaf_order_or_null,
                                 const re_canonical_triangle* src, const std::vector<uint32_t>& leaf_order) {
    const size_t n = sc->triangle_count;
    std::vector<DeviceTriangle> tris(n);
    std::vector<DeviceAttr> attrs(n);
    bool any_masked = false;
    for (size_t i = 0; i < n; ++i) {
        const re_canonical_triangle& t =
            src_in_leaf_order_or_null != nullptr ? src_in_leaf_order_or_null[i] : src[leaf_order[i]];
        DeviceTriangle& d = tris[i];
        const re_float4* p = t.positions;
        const bool double_sided = (t.metadata.x & RE_GEOMETRY_FLAG_DOUBLE_SIDED) != 0u ||
                                  (t.metadata.y & RE_MATERIAL_FLAG_DOUBLE_SIDED) != 0u;
        const bool casts = (t.metadata.w & RE_INSTANCE_FLAG_CASTS_SHADOW) != 0u;
        const bool masked = (t.metadata.x & RE_GEOMETRY_FLAG_ALPHA_MASK) != 0u ||
                            (t.metadata.y & RE_MATERIAL_FLAG_ALPHA_MASK) != 0u;
        uint32_t flags = (double_sided ? kTriDoubleSided : 0u) | (casts ? kTriCastsShadow : 0u) |
                         (masked ? kTriAlphaMask : 0u);
        any_masked |= masked;
        d.p0[0] = p[0].x; d.p0[1] = p[0].y; d.p0[2] = p[0].z;
        std::memcpy(&d.p0[3], &flags, 4);
        d.e1[0] = p[1].x - p[0].x; d.e1[1] = p[1].y - p[0].y; d.e1[2] = p[1].z - p[0].z;
        d.e2[0] = p[2].x - p[0].x; d.e2[1] = p[2].y - p[0].y; d.e2[2] = p[2].z - p[0].z;
        std::memcpy(&d.e1[3], &t.identity.x, 4);
        std::memcpy(&d.e2[3], &t.identity.y, 4);
        d.key[0] = t.identity.x;
        d.key[1] = t.identity.y;
        d.key[2] = t.metadata.z;
        d.key[3] = src_in_leaf_order_or_null != nullptr ? uint32_t(i) : leaf_order[i];
        DeviceAttr& a = attrs[i];
        a.n0[0] = t.normals[0].x; a.n0[1] = t.normals[0].y; a.n0[2] = t.normals[0].z; a.n0[3] = 0.0f;
        a.n1[0] = t.normals[1].x; a.n1[1] = t.normals[1].y; a.n1[2] = t.normals[1].z; a.n1[3] = 0.0f;
        a.n2[0] = t.normals[2].x; a.n2[1] = t.normals[2].y; a.n2[2] = t.normals[2].z; a.n2[3] = 0.0f;
        a.ids[0] = t.identity.x; a.ids[1] = t.identity.y; a.ids[2] = t.identity.z; a.ids[3] = t.identity.w;
    }
    RE_CUDA_TRY(cudaSetDevice(sc->device));
    if (any_masked) {
        // Texture coordinates and material of every leaf slot, for the alpha test.
        std::vector<float4> alpha_tc(2 * n);
        for (size_t i = 0; i < n; ++i) {
            const re_canonical_triangle& t =
                src_in_leaf_order_or_null != nullptr ? src_in_leaf_order_or_null[i] : src[leaf_order[i]];
            float mat;
            std::memcpy(&mat, &t.identity.w, 4);
            alpha_tc[2 * i] = make_float4(t.texcoords[0].x, t.texcoords[0].y, t.texcoords[1].x, t.texcoords[1].y);
            alpha_tc[2 * i + 1] = make_float4(t.texcoords[2].x, t.texcoords[2].y, mat, 0.f);
        }
        sc->alpha_masked = true;
        RE_CUDA_TRY(sc->alpha_tc.reserve(alpha_tc.size() * sizeof(float4)));
        RE_CUDA_TRY(cudaMemcpy(sc->alpha_tc.ptr, alpha_tc.data(), alpha_tc.size() * sizeof(float4),
                               cudaMemcpyHostToDevice));
    }
    RE_CUDA_TRY(sc->tris.reserve(n * sizeof(DeviceTriangle)));
    RE_CUDA_TRY(sc->attrs.reserve(n * sizeof(DeviceAttr)));
    RE_CUDA_TRY(cudaMemcpy(sc->tris.ptr, tris.data(), n * sizeof(DeviceTriangle), cudaMemcpyHostToDevice));
    RE_CUDA_TRY(cudaMemcpy(sc->attrs.ptr, attrs.data(), n * sizeof(DeviceAttr), cudaMemcpyHostToDevice));
    return RE_SUCCESS;
}

}  // namespace re

using namespace re;

extern "C" {

RE_API const char* re_last_error(void) { return g_last_error.c_str(); }

RE_API uint32_t re_abi_version(void) { return RE_ABI_VERSION; }

RE_API const char* re_execution_architecture_token(void) { return "cuda-wavefront"; }

RE_API int re_capability_is_built(uint32_t transport, uint32_t backend, uint32_t estimator,
                                  const char** reason) {
    const char* why = nullptr;
    if (transport != RE_TRANSPORT_PBR) why = "cuda-wavefront implements the PBR transport only";
    else if (backend != RE_BACKEND_GPU_FLATTENED_SAH && backend != RE_BACKEND_GPU_LBVH)
        why = "cuda-wavefront traverses the flattened SAH or the GPU LBVH only";
    else if (estimator > 3u) why = "unknown direct-light estimator";
    if (reason != nullptr) *reason = why != nullptr ? why : "";
    return why == nullptr ? 1 : 0;
}

RE_API re_status re_scene_create(const re_scene_desc* desc, re_scene** out_scene) {
    if (out_scene == nullptr || desc == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    *out_scene = nullptr;
    if (desc->fingerprint == 0 || desc->generation == 0)
        return set_error(RE_INVALID_ARGUMENT, "scene fingerprint and generation must be non-zero");
    if (desc->triangle_count == 0 || desc->triangles == nullptr)
        return set_error(RE_INVALID_ARGUMENT, "scene needs at least one triangle");
    if (desc->triangle_count >= (1u << kLeafShift))
        return set_error(RE_INVALID_ARGUMENT, "scene exceeds 2^28 triangles");
    if (desc->build_kind != RE_BUILD_FLATTENED_SAH && desc->build_kind != RE_BUILD_LBVH)
        return set_error(RE_INVALID_ARGUMENT, "unknown build kind");
    const uint32_t max_leaf = desc->max_leaf_size == 0 ? 4u : desc->max_leaf_size;
    if (max_leaf > 15u) return set_error(RE_INVALID_ARGUMENT, "leaf size must be <= 15");
    // Fail closed on malformed primitives exactly where the reference's
    // IsPrimitiveValid / HasUniqueIds reject them (SoftwareGpu.cpp:134-170).
    std::vector<uint32_t> ids(desc->triangle_count);
    for (uint32_t i = 0; i < desc->triangle_count; ++i) {
        const re_canonical_triangle& t = desc->triangles[i];
        if (!finite4(t.positions[0]) || !finite4(t.positions[1]) || !finite4(t.positions[2]))
            return set_error(RE_INVALID_ARGUMENT, "A BVH cannot contain a non-finite triangle");
        const float e0[3] = {t.positions[1].x - t.positions[0].x, t.positions[1].y - t.positions[0].y,
                             t.positions[1].z - t.positions[0].z};
        const float e1[3] = {t.positions[2].x - t.positions[0].x, t.positions[2].y - t.positions[0].y,
                             t.positions[2].z - t.positions[0].z};
        const float c[3] = {(e0[1] * e1[2]) - (e0[2] * e1[1]), (e0[2] * e1[0]) - (e0[0] * e1[2]),
                            (e0[0] * e1[1]) - (e0[1] * e1[0])};
        const float area2 = (c[0] * c[0]) + (c[1] * c[1]) + (c[2] * c[2]);
        const float l0 = (e0[0] * e0[0]) + (e0[1] * e0[1]) + (e0[2] * e0[2]);
        const float l1 = (e1[0] * e1[0]) + (e1[1] * e1[1]) + (e1[2] * e1[2]);
        const float scale = l0 > l1 ? l0 : l1;
        if (!std::isfinite(area2) || !(area2 > scale * scale * 1.0e-14f))
            return set_error(RE_INVALID_ARGUMENT, "scene contains a degenerate triangle");
        if (t.metadata.z == 0xffffffffu) return set_error(RE_INVALID_ARGUMENT, "triangle has no traversal ID");
        ids[i] = t.metadata.z;
    }
    std::sort(ids.begin(), ids.end());
    if (std::adjacent_find(ids.begin(), ids.end()) != ids.end())
        return set_error(RE_INVALID_ARGUMENT, "traversal IDs must be unique");
    int ndev = 0;
    RE_CUDA_TRY(cudaGetDeviceCount(&ndev));
    if (int(desc->device) >= ndev) return set_error(RE_INVALID_ARGUMENT, "device ordinal out of range");

    auto sc = new re_scene();
    sc->device = int(desc->device);
    sc->fingerprint = desc->fingerprint;
    sc->generation = desc->generation;
    sc->triangle_count = desc->triangle_count;
    sc->build_kind = desc->build_kind;
    const auto t0 = std::chrono::steady_clock::now();
    re_status st = RE_SUCCESS;
    if (desc->build_kind == RE_BUILD_LBVH) {
        if (cudaSetDevice(sc->device) != cudaSuccess) st = set_error(RE_CUDA_ERROR, "cudaSetDevice failed");
        else st = build_lbvh_on_device(sc, desc->triangles);
    } else if (desc->nodes != nullptr) {
        // Caller-flattened SAH: triangles are already in leaf order.
        sc->flat.nodes.assign(desc->nodes, desc->nodes + desc->node_count);
        sc->flat.leaf_order.resize(desc->triangle_count);
        uint32_t depth = 0, leaves = 0;
        for (uint32_t i = 0; i < desc->triangle_count; ++i) sc->flat.leaf_order[i] = i;
        // Depth and structural sanity: every index in range.
        std::vector<uint32_t> d(desc->node_count, 0);
        if (desc->node_count > 0) d[0] = 1;
        for (uint32_t i = 0; i < desc->node_count && st == RE_SUCCESS; ++i) {
            const re_uint4& l = desc->nodes[i].links;
            if (l.y != 0) {
                ++leaves;
                if (uint64_t(l.x) + l.y > desc->triangle_count || l.y > 15u)
                    st = set_error(RE_INVALID_ARGUMENT, "flattened leaf range is out of bounds");
            } else if (l.x >= desc->node_count || l.z >= desc->node_count || l.x <= i || l.z <= i) {
                st = set_error(RE_INVALID_ARGUMENT, "flattened interior child index is invalid");
            } else {
                d[l.x] = d[l.z] = d[i] + 1;
            }
            depth = std::max(depth, d[i]);
        }
        sc->flat.max_depth = depth;
        sc->flat.leaf_count = leaves;
        if (st == RE_SUCCESS && depth > 128) st = set_error(RE_INVALID_ARGUMENT, "flattened depth exceeds 128");
        if (st == RE_SUCCESS) st = upload_scene_geometry(sc, desc->triangles, nullptr, {});
    } else {
        std::vector<HostTriangle> tris(desc->triangle_count);
        for (uint32_t i = 0; i < desc->triangle_count; ++i) {
            const re_canonical_triangle& t = desc->triangles[i];
            for (int v = 0; v < 3; ++v) {
                tris[i].v[v][0] = t.positions[v].x;
                tris[i].v[v][1] = t.positions[v].y;
                tris[i].v[v][2] = t.positions[v].z;
            }
            tris[i].primitive_id = t.metadata.z;
        }
        std::string err;
        const uint32_t threads = std::max(1u, std::thread::hardware_concurrency());
        if (!build_binned_sah(tris, desc->sah_bins == 0 ? 16u : desc->sah_bins, max_leaf, threads,
                              sc->flat, err)) {
            st = set_error(RE_INVALID_ARGUMENT, err);
        } else {
            st = upload_scene_geometry(sc, nullptr, desc->triangles, sc->flat.leaf_order);
        }
    }
    if (st != RE_SUCCESS) {
        delete sc;
        return st;
    }
    sc->build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    *out_scene = sc;
    return clear_error();
}

RE_API re_status re_scene_create_from_device(const re_scene_desc* desc, re_scene** out_scene) {
    if (out_scene == nullptr || desc == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    *out_scene = nullptr;
    if (desc->fingerprint == 0 || desc->generation == 0)
        return set_error(RE_INVALID_ARGUMENT, "scene fingerprint and generation must be non-zero");
    if (desc->triangle_count == 0 || desc->triangles == nullptr)
        return set_error(RE_INVALID_ARGUMENT, "scene needs at least one triangle");
    if (desc->triangle_count >= (1u << kLeafShift))
        return set_error(RE_INVALID_ARGUMENT, "scene exceeds 2^28 triangles");
    if (desc->build_kind != RE_BUILD_LBVH || desc->nodes != nullptr)
        return set_error(RE_UNSUPPORTED, "a scene from device records is built as a GPU LBVH");
    int ndev = 0;
    RE_CUDA_TRY(cudaGetDeviceCount(&ndev));
    if (int(desc->device) >= ndev) return set_error(RE_INVALID_ARGUMENT, "device ordinal out of range");
    auto sc = new re_scene();
    sc->device = int(desc->device);
    sc->fingerprint = desc->fingerprint;
    sc->generation = desc->generation;
    sc->triangle_count = desc->triangle_count;
    sc->build_kind = desc->build_kind;
    const auto t0 = std::chrono::steady_clock::now();
    re_status st = RE_SUCCESS;
    if (cudaSetDevice(sc->device) != cudaSuccess) st = set_error(RE_CUDA_ERROR, "cudaSetDevice failed");
    else st = build_lbvh_from_device_records(sc, desc->triangles);
    if (st != RE_SUCCESS) {
        delete sc;
        return st;
    }
    sc->build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    *out_scene = sc;
    return clear_error();
}

RE_API re_status re_scene_destroy(re_scene* scene) {
    delete scene;
    return clear_error();
}

RE_API re_status re_scene_info_get(const re_scene* sc, re_scene_info* out) {
    if (sc == nullptr || out == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    out->triangle_count = sc->triangle_count;
    out->node_count = uint32_t(sc->flat.nodes.size());
    out->max_depth = sc->flat.max_depth;
    out->leaf_count = sc->flat.leaf_count;
    out->device_bytes = uint64_t(sc->nodes.bytes) + sc->tris.bytes + sc->attrs.bytes + sc->wide_nodes.bytes;
    out->build_ms = sc->build_ms;
    out->node_bytes = sizeof(DeviceNode);
    out->triangle_bytes = sizeof(DeviceTriangle);
    out->gpu_build_ms = sc->lbvh_gpu_ms;
    return clear_error();
}

RE_API re_status re_scene_export_flat(const re_scene* sc, re_software_node* nodes, uint32_t node_capacity,
                                      uint32_t* leaf_order, uint32_t order_capacity) {
    if (sc == nullptr) return set_error(RE_INVALID_ARGUMENT, "scene is null");
    if (nodes != nullptr) {
        if (node_capacity < sc->flat.nodes.size()) return set_error(RE_INVALID_ARGUMENT, "node capacity too small");
        std::memcpy(nodes, sc->flat.nodes.data(), sc->flat.nodes.size() * sizeof(re_software_node));
    }
    if (leaf_order != nullptr) {
        if (order_capacity < sc->flat.leaf_order.size())
            return set_error(RE_INVALID_ARGUMENT, "order capacity too small");
        std::memcpy(leaf_order, sc->flat.leaf_order.data(), sc->flat.leaf_order.size() * sizeof(uint32_t));
    }
    return clear_error();
}

RE_API re_status re_sah_build_host(const re_canonical_triangle* triangles, uint32_t count, uint32_t sah_bins,
                                   uint32_t max_leaf_size, re_software_node* nodes_out, uint32_t node_capacity,
                                   uint32_t* node_count_out, uint32_t* leaf_order_out, uint32_t* max_depth_out) {
    if (triangles == nullptr || nodes_out == nullptr || node_count_out == nullptr || leaf_order_out == nullptr)
        return set_error(RE_INVALID_ARGUMENT, "null argument");
    std::vector<HostTriangle> tris(count);
    for (uint32_t i = 0; i < count; ++i) {
        for (int v = 0; v < 3; ++v) {
            tris[i].v[v][0] = triangles[i].positions[v].x;
            tris[i].v[v][1] = triangles[i].positions[v].y;
            tris[i].v[v][2] = triangles[i].positions[v].z;
        }
        tris[i].primitive_id = triangles[i].metadata.z;
    }
    FlatBvh flat;
    std::string err;
    const uint32_t threads = std::max(1u, std::thread::hardware_concurrency());
    if (!build_binned_sah(tris, sah_bins == 0 ? 16u : sah_bins, max_leaf_size == 0 ? 4u : max_leaf_size, threads,
                          flat, err))
        return set_error(RE_INVALID_ARGUMENT, err);
    if (flat.nodes.size() > node_capacity) return set_error(RE_INVALID_ARGUMENT, "node capacity too small");
    std::memcpy(nodes_out, flat.nodes.data(), flat.nodes.size() * sizeof(re_software_node));
    std::memcpy(leaf_order_out, flat.leaf_order.data(), flat.leaf_order.size() * sizeof(uint32_t));
    *node_count_out = uint32_t(flat.nodes.size());
    if (max_depth_out != nullptr) *max_depth_out = flat.max_depth;
    return clear_error();
}

RE_API re_status re_trace_closest(re_scene* scene, const re_trace_batch* batch) {
    return run_trace(scene, batch, false, nullptr);
}

RE_API re_status re_trace_any(re_scene* scene, const re_trace_batch* batch) {
    return run_trace(scene, batch, true, nullptr);
}

RE_API re_status re_trace_counted(re_scene* scene, const re_trace_batch* batch, uint32_t any_hit,
                                  re_traversal_counters* counters) {
    if (counters == nullptr) return set_error(RE_INVALID_ARGUMENT, "counters is null");
    return run_trace(scene, batch, any_hit != 0, counters);
}

}  // extern "C"

extern "C" RE_API re_status re_scene_set_alpha_masks(re_scene* sc, const re_gpu_material_v0* materials,
                                                     uint32_t material_count, const float* atlas_alpha,
                                                     uint32_t width, uint32_t height, uint32_t layers,
                                                     uint32_t sampler_id) {
    using namespace re;
    if (sc == nullptr) return set_error(RE_MISSING_SCENE, "scene is null");
    if (material_count != 0u && materials == nullptr) return set_error(RE_INVALID_ARGUMENT, "null materials");
    if (layers != 0u && (atlas_alpha == nullptr || width == 0u || height == 0u))
        return set_error(RE_INVALID_ARGUMENT, "an alpha atlas needs texels and non-zero dimensions");
    if (uint64_t(width) * height * layers > (uint64_t(1) << 31))
        return set_error(RE_INVALID_ARGUMENT, "alpha atlas too large");
    // Per material: alpha factor (baseColorFactor.w), cutoff (surfaceParams.w),
    // alpha layer (textureImageIndices.x) and sampler (textureSamplerIndices.x).
    std::vector<float4> mats(std::max(1u, material_count));
    for (uint32_t i = 0; i < material_count; ++i) {
        const re_gpu_material_v0& m = materials[i];
        float layer, sampler;
        std::memcpy(&layer, &m.texture_image_indices.x, 4);
        std::memcpy(&sampler, &m.texture_sampler_indices.x, 4);
        mats[i] = make_float4(m.base_color_factor.w, m.surface_params.w, layer, sampler);
    }
    RE_CUDA_TRY(cudaSetDevice(sc->device));
    RE_CUDA_TRY(cudaDeviceSynchronize());  // launches in flight may read the old tables
    RE_CUDA_TRY(sc->alpha_materials.reserve(mats.size() * sizeof(float4)));
    RE_CUDA_TRY(cudaMemcpy(sc->alpha_materials.ptr, mats.data(), mats.size() * sizeof(float4), cudaMemcpyHostToDevice));
    const size_t texels = size_t(width) * height * layers;
    RE_CUDA_TRY(sc->alpha_atlas.reserve(std::max<size_t>(1, texels) * sizeof(float)));
    if (texels)
        RE_CUDA_TRY(cudaMemcpy(sc->alpha_atlas.ptr, atlas_alpha, texels * sizeof(float), cudaMemcpyHostToDevice));
    AlphaView v{};
    v.tc = static_cast<const float4*>(sc->alpha_tc.ptr);
    v.materials = static_cast<const float4*>(sc->alpha_materials.ptr);
    v.atlas = static_cast<const float*>(sc->alpha_atlas.ptr);
    v.material_count = material_count;
    v.width = width;
    v.height = height;
    v.layers = layers;
    v.sampler_id = sampler_id;
    if (!sc->alpha_masked) v.material_count = 0u;  // no masked triangle reads it
    RE_CUDA_TRY(sc->alpha_view.reserve(sizeof(AlphaView)));
    RE_CUDA_TRY(cudaMemcpy(sc->alpha_view.ptr, &v, sizeof(AlphaView), cudaMemcpyHostToDevice));
    return clear_error();
}
