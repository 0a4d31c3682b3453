// TEST INFRASTRUCTURE ONLY -- the CPU oracle for the traversal stage.  Only
// tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load it.
//
// A plain scalar restatement of the reference's production flattened-SAH
// traversal over 48-byte SoftwareNodeRecords:
//   - ray validity           resources/shaders/traversal/software_common.hlsli:69-75
//   - reciprocal slab test   software_common.hlsli:77-118
//   - Moller-Trumbore        software_common.hlsli:120-172 (CPU mirror order,
//                            src/rt/software_gpu/SoftwareGpu.cpp:661-703)
//   - cull / casts-shadow / ignored primitive / lower-(instance, primitive)
//     tie rule               resources/shaders/integrators/pbr_software_traversal.hlsli:288-535
//   - stack DFS, near child first, near pruning
//                            src/rt/software_gpu/SoftwareGpu.cpp:1529-1700
// Built with -ffp-contract=off so every float operation rounds once, as on
// the GPU side.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "oracle_common.h"

namespace {

constexpr uint32_t kInvalid = 0xffffffffu;

struct V3 {
    float x, y, z;
};

V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
float dot(V3 a, V3 b) { return (a.x * b.x) + (a.y * b.y) + (a.z * b.z); }
V3 cross(V3 a, V3 b) { return {(a.y * b.z) - (a.z * b.y), (a.z * b.x) - (a.x * b.z), (a.x * b.y) - (a.y * b.x)}; }
float axis(V3 v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }

struct Node {
    float bmin[4];
    float bmax[4];
    uint32_t links[4];
};

struct Ray {
    V3 o, d;
    float tmin, tmax;
};

bool ray_valid(const Ray& r) {
    const float l2 = dot(r.d, r.d);
    return std::isfinite(r.o.x) && std::isfinite(r.o.y) && std::isfinite(r.o.z) && std::isfinite(r.d.x) &&
           std::isfinite(r.d.y) && std::isfinite(r.d.z) && std::isfinite(l2) && std::fabs(l2 - 1.0f) <= 1.0e-4f &&
           !std::isnan(r.tmin) && !std::isnan(r.tmax) && r.tmin < r.tmax;
}

// SoftwareIntersectBounds with the per-axis reciprocal.
bool bounds(const Ray& r, const Node& n, float limit, bool inclusive, float& near_out) {
    float tn = -INFINITY, tf = INFINITY;
    for (int a = 0; a < 3; ++a) {
        const float d = axis(r.d, a), o = axis(r.o, a);
        if (d == 0.0f) {
            if (o < n.bmin[a] || o > n.bmax[a]) return false;
            continue;
        }
        const float inv = 1.0f / d;
        float an = (n.bmin[a] - o) * inv;
        float af = (n.bmax[a] - o) * inv;
        if (an > af) std::swap(an, af);
        tn = std::fmax(tn, an);
        tf = std::fmin(tf, af);
        if (tf < tn) return false;
    }
    const bool within_ray = tn < r.tmax;
    const bool within_limit = inclusive ? tn <= limit : tn < limit;
    if (!(tf > r.tmin && within_ray && within_limit)) return false;
    near_out = std::fmax(tn, r.tmin);
    return true;
}

bool triangle(const Ray& r, const float* v, float limit, bool inclusive, float& t, float& u, float& w, bool& front) {
    const V3 v0{v[0], v[1], v[2]};
    const V3 e1 = sub(V3{v[3], v[4], v[5]}, v0);
    const V3 e2 = sub(V3{v[6], v[7], v[8]}, v0);
    const V3 p = cross(r.d, e2);
    const float det = dot(e1, p);
    if (det == 0.0f || !std::isfinite(det)) return false;
    const float inv = 1.0f / det;
    const V3 tv = sub(r.o, v0);
    const float uu = dot(tv, p) * inv;
    if (!(uu >= 0.0f && uu <= 1.0f)) return false;
    const V3 q = cross(tv, e1);
    const float vv = dot(r.d, q) * inv;
    if (!(vv >= 0.0f && uu + vv <= 1.0f)) return false;
    const float tt = dot(e2, q) * inv;
    const bool within_limit = inclusive ? tt <= limit : tt < limit;
    if (!(std::isfinite(tt) && tt > r.tmin && tt < r.tmax && within_limit)) return false;
    t = tt;
    u = uu;
    w = vv;
    front = det > 0.0f;
    return true;
}

struct Result {
    uint32_t tri = kInvalid;
    float t = 0, u = 0, v = 0;
    uint32_t front = 0, status = 0;
    uint64_t node_tests = 0, tri_tests = 0;
};

// Alpha-masked candidate acceptance (pbr_software_traversal.hlsli:207-240,
// 430-470): 1 keeps, 0 skips (alpha below the cutoff), -1 invalid mapping.
int alpha_accept(const oracle::AlphaData* a, uint32_t ti, float u, float v) {
    if (a == nullptr || a->tc == nullptr) return -1;
    const float* t = a->tc + size_t(ti) * 8u;
    uint32_t mat;
    std::memcpy(&mat, t + 6, 4);
    if (mat >= a->material_count) return -1;
    const float* m = a->materials + size_t(mat) * 4u;
    uint32_t layer, sampler;
    std::memcpy(&layer, m + 2, 4);
    std::memcpy(&sampler, m + 3, 4);
    float alpha = m[0];
    if (layer == kInvalid) {
        if (sampler != kInvalid) return -1;
    } else if (layer >= a->layers || sampler != a->sampler_id) {
        return -1;
    } else {
        const float w0 = (1.0f - u) - v;
        const float su = (w0 * t[0] + u * t[2]) + v * t[4];
        const float sv = (w0 * t[1] + u * t[3]) + v * t[5];
        const int i = std::min(std::max(int(std::floor(su * float(a->width))), 0), int(a->width) - 1);
        const int j = std::min(std::max(int(std::floor(sv * float(a->height))), 0), int(a->height) - 1);
        alpha = alpha * a->atlas[(size_t(layer) * a->height + size_t(j)) * a->width + size_t(i)];
    }
    return alpha < m[1] ? 0 : 1;
}

// flags word: bit0 double-sided, bit1 casts shadow, bit2 alpha-masked.
Result trace_one(const Node* nodes, uint32_t node_count, const float* tv, const uint32_t* key,
                 const Ray& ray, bool any, bool shadow, uint32_t ign_inst, uint32_t ign_prim,
                 const oracle::AlphaData* alpha = nullptr) {
    Result res;
    res.t = ray.tmax;
    if (!ray_valid(ray)) { res.status = 1; return res; }
    if (node_count == 0) return res;
    struct Entry { uint32_t node; float near; };
    Entry stack[128];
    int sp = 0;
    float root_near = 0;
    ++res.node_tests;
    if (!bounds(ray, nodes[0], ray.tmax, false, root_near)) return res;
    stack[sp++] = {0u, root_near};
    bool found = false;
    float limit = ray.tmax;
    uint32_t bi = kInvalid, bp = kInvalid;
    size_t visited = 0;
    while (sp > 0) {
        const Entry e = stack[--sp];
        if (++visited > node_count) { res.status = 3; res.tri = kInvalid; return res; }
        if (found ? e.near > limit : e.near >= limit) continue;
        const Node& n = nodes[e.node];
        if (n.links[1] != 0) {
            for (uint32_t k = 0; k < n.links[1]; ++k) {
                const uint32_t ti = n.links[0] + k;
                const uint32_t* kk = key + size_t(ti) * 4u;
                if (kk[0] == ign_inst && kk[1] == ign_prim) continue;
                if (shadow && (kk[3] & 2u) == 0u) continue;
                ++res.tri_tests;
                float t, u, v;
                bool front;
                if (!triangle(ray, tv + size_t(ti) * 9u, limit, found, t, u, v, front)) continue;
                if (!front && (kk[3] & 1u) == 0u) continue;
                if ((kk[3] & 4u) != 0u) {
                    const int acc = alpha_accept(alpha, ti, u, v);
                    if (acc < 0) { res.status = 3; res.tri = kInvalid; return res; }
                    if (acc == 0) continue;
                }
                if (any) {
                    res.tri = ti; res.t = t; res.u = u; res.v = v; res.front = front;
                    return res;
                }
                const bool lower = t == limit && (kk[0] < bi || (kk[0] == bi && kk[1] < bp));
                if (!found || t < limit || lower) {
                    found = true;
                    limit = t;
                    bi = kk[0];
                    bp = kk[1];
                    res.tri = ti; res.t = t; res.u = u; res.v = v; res.front = front;
                }
            }
            continue;
        }
        const uint32_t l = n.links[0], r = n.links[2];
        if (l >= node_count || r >= node_count) { res.status = 3; res.tri = kInvalid; return res; }
        float nl = 0, nr = 0;
        res.node_tests += 2;
        const bool hl = bounds(ray, nodes[l], limit, found, nl);
        const bool hr = bounds(ray, nodes[r], limit, found, nr);
        if (hl && hr) {
            const bool left_first = nl < nr || (!(nr < nl) && l < r);
            if (sp + 2 > 128) { res.status = 2; res.tri = kInvalid; return res; }
            stack[sp++] = left_first ? Entry{r, nr} : Entry{l, nl};
            stack[sp++] = left_first ? Entry{l, nl} : Entry{r, nr};
        } else if (hl) {
            stack[sp++] = {l, nl};
        } else if (hr) {
            stack[sp++] = {r, nr};
        }
    }
    return res;
}

}  // namespace

namespace oracle {
TraceResult trace_flat(const void* nodes, uint32_t node_count, const float* tri_v, const uint32_t* tri_key,
                       V3 o, float tmin, V3 d, float tmax, bool any, bool shadow, uint32_t ign_inst,
                       uint32_t ign_prim, const AlphaData* alpha) {
    const Ray ray{{o.x, o.y, o.z}, {d.x, d.y, d.z}, tmin, tmax};
    const Result r = trace_one(static_cast<const Node*>(nodes), node_count, tri_v, tri_key, ray, any, shadow,
                               ign_inst, ign_prim, alpha);
    return {r.tri, r.t, r.u, r.v, r.front, r.status, r.node_tests, r.tri_tests};
}
}  // namespace oracle

extern "C" {

// rays: n x 8 floats (origin.xyz, tMin, direction.xyz, tMax).
// tri_v: leaf-ordered 9 floats per triangle.  tri_key: 4 words per triangle
// (instance, primitive, traversal ID, flags).
// out: tri index (leaf order) or 0xffffffff, t/u/v, front, status.
void oracle_trace_alpha(const void* nodes, uint32_t node_count, const float* tri_v, const uint32_t* tri_key,
                        const float* rays, uint32_t n, uint32_t any, uint32_t shadow, uint32_t threads,
                        uint32_t* out_tri, float* out_tuv, uint32_t* out_front, uint32_t* out_status,
                        uint64_t* out_counters, const oracle::AlphaData* alpha);

void oracle_trace(const void* nodes, uint32_t node_count, const float* tri_v, const uint32_t* tri_key,
                  const float* rays, uint32_t n, uint32_t any, uint32_t shadow, uint32_t threads,
                  uint32_t* out_tri, float* out_tuv, uint32_t* out_front, uint32_t* out_status,
                  uint64_t* out_counters) {
    oracle_trace_alpha(nodes, node_count, tri_v, tri_key, rays, n, any, shadow, threads, out_tri, out_tuv, out_front,
                       out_status, out_counters, nullptr);
}

// oracle_trace with alpha-mask data (null: no masked triangle may be met).
void oracle_trace_alpha(const void* nodes, uint32_t node_count, const float* tri_v, const uint32_t* tri_key,
                        const float* rays, uint32_t n, uint32_t any, uint32_t shadow, uint32_t threads,
                        uint32_t* out_tri, float* out_tuv, uint32_t* out_front, uint32_t* out_status,
                        uint64_t* out_counters, const oracle::AlphaData* alpha) {
    const Node* nd = static_cast<const Node*>(nodes);
    const uint32_t nt = std::max(1u, threads);
    std::vector<uint64_t> cn(size_t(nt) * 2, 0);
    auto work = [&](uint32_t tid) {
        for (uint32_t i = tid; i < n; i += nt) {
            const float* rr = rays + size_t(i) * 8u;
            const Ray ray{{rr[0], rr[1], rr[2]}, {rr[4], rr[5], rr[6]}, rr[3], rr[7]};
            const Result r =
                trace_one(nd, node_count, tri_v, tri_key, ray, any != 0, shadow != 0, kInvalid, kInvalid, alpha);
            out_tri[i] = r.tri;
            out_tuv[size_t(i) * 3 + 0] = r.t;
            out_tuv[size_t(i) * 3 + 1] = r.u;
            out_tuv[size_t(i) * 3 + 2] = r.v;
            out_front[i] = r.front;
            out_status[i] = r.status;
            cn[size_t(tid) * 2] += r.node_tests;
            cn[size_t(tid) * 2 + 1] += r.tri_tests;
        }
    };
    std::vector<std::thread> pool;
    for (uint32_t t = 1; t < nt; ++t) pool.emplace_back(work, t);
    work(0);
    for (auto& th : pool) th.join();
    if (out_counters != nullptr) {
        out_counters[0] = out_counters[1] = 0;
        for (uint32_t t = 0; t < nt; ++t) {
            out_counters[0] += cn[size_t(t) * 2];
            out_counters[1] += cn[size_t(t) * 2 + 1];
        }
    }
}

}  // extern "C"
