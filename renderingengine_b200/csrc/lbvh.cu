// GPU LBVH build: scene bounds, 30-bit Morton codes, a stable LSD radix sort
// on (code, stable primitive ID), the Karras hierarchy and a bottom-up refit,
// all on the device.  Semantics follow the reference's CPU mirror
// (src/rt/software_gpu/SoftwareGpu.cpp):
//   - MortonCode / QuantizeMortonAxis / ExpandMortonBits   :184-207, 814-838
//   - centroid = midpoint of the primitive bounds         :92-98
//   - StableRadixSortMorton: lexicographic (code, ID)      :840-884
//   - FindKarrasSplit on the 64-bit key code << 32 | ID    :540-571
//   - one primitive per leaf; RefitBottomUp                 :1265-1527
// and the GPU passes software_lbvh_{morton,radix,hierarchy,bounds}.hlsl.
// The hierarchy is identical to the reference's (the split of a key range is
// the first differing bit of its end keys, a unique position), only the node
// numbering differs: Karras numbering on the device, the reference's pre-order
// in the exported flat records.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "runtime.h"
#include "traverse.cuh"

namespace re {

re_status upload_scene_geometry(re_scene* sc, const re_canonical_triangle* src_in_leaf_order_or_null,
                                const re_canonical_triangle* src, const std::vector<uint32_t>& leaf_order);

namespace {

constexpr uint32_t kRadixThreads = 256;
constexpr uint32_t kRadixItems = 16;
constexpr uint32_t kRadixTile = kRadixThreads * kRadixItems;
constexpr uint32_t kRadixBins = 16;  // 4-bit digits, 16 passes over the 64-bit key

// Order-preserving float <-> uint mapping for atomic min / max.
__device__ __forceinline__ uint32_t f2o(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float o2f(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__global__ void k_bounds(const float4* pos, uint32_t n, uint32_t* out /* 6: minx miny minz maxx maxy maxz */) {
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        for (int v = 0; v < 3; ++v) {
            const float4 p = pos[size_t(i) * 3 + v];
            lo[0] = fminf(lo[0], p.x); lo[1] = fminf(lo[1], p.y); lo[2] = fminf(lo[2], p.z);
            hi[0] = fmaxf(hi[0], p.x); hi[1] = fmaxf(hi[1], p.y); hi[2] = fmaxf(hi[2], p.z);
        }
    }
    for (int a = 0; a < 3; ++a) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[a] = fminf(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
            hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
        }
    }
    if ((threadIdx.x & 31) == 0) {
        for (int a = 0; a < 3; ++a) {
            atomicMin(out + a, f2o(lo[a]));
            atomicMax(out + 3 + a, f2o(hi[a]));
        }
    }
}

__device__ __forceinline__ uint32_t expand_bits(uint32_t v) {
    v &= 0x000003ffu;
    v = (v | (v << 16u)) & 0x030000ffu;
    v = (v | (v << 8u)) & 0x0300f00fu;
    v = (v | (v << 4u)) & 0x030c30c3u;
    v = (v | (v << 2u)) & 0x09249249u;
    return v;
}

// QuantizeMortonAxis in double precision.
__device__ __forceinline__ uint32_t quantize(float v, float lo, float hi) {
    const double extent = double(hi) - double(lo);
    const double nrm = extent > 0.0 ? (double(v) - double(lo)) / extent : 0.5;
    const double c = fmin(fmax(nrm, 0.0), 1.0);
    return min(uint32_t(c * 1024.0), 1023u);
}

__device__ __forceinline__ float midpoint(float a, float b) {
    // std::midpoint for finite floats of normal magnitude: (a + b) / 2.
    return (a + b) / 2.0f;
}

__global__ void k_morton(const float4* pos, const uint32_t* ids, uint32_t n, const uint32_t* bounds,
                         unsigned long long* keys, uint32_t* vals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] = o2f(bounds[a]);
        hi[a] = o2f(bounds[3 + a]);
    }
    const float4 p0 = pos[size_t(i) * 3], p1 = pos[size_t(i) * 3 + 1], p2 = pos[size_t(i) * 3 + 2];
    const float c[3] = {midpoint(fminf(p0.x, fminf(p1.x, p2.x)), fmaxf(p0.x, fmaxf(p1.x, p2.x))),
                        midpoint(fminf(p0.y, fminf(p1.y, p2.y)), fmaxf(p0.y, fmaxf(p1.y, p2.y))),
                        midpoint(fminf(p0.z, fminf(p1.z, p2.z)), fmaxf(p0.z, fmaxf(p1.z, p2.z)))};
    const uint32_t code = (expand_bits(quantize(c[0], lo[0], hi[0])) << 2u) |
                          (expand_bits(quantize(c[1], lo[1], hi[1])) << 1u) | expand_bits(quantize(c[2], lo[2], hi[2]));
    keys[i] = (static_cast<unsigned long long>(code) << 32) | ids[i];
    vals[i] = i;
}

// Radix pass, kernel 1: per-block digit histogram, stored digit-major.
__global__ void __launch_bounds__(kRadixThreads) k_radix_hist(const unsigned long long* keys, uint32_t n,
                                                              uint32_t shift, uint32_t* hist, uint32_t blocks) {
    __shared__ uint32_t h[kRadixBins];
    if (threadIdx.x < kRadixBins) h[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t base = blockIdx.x * kRadixTile + threadIdx.x * kRadixItems;
    uint32_t local[kRadixBins] = {};
    for (uint32_t k = 0; k < kRadixItems; ++k) {
        const uint32_t i = base + k;
        if (i < n) ++local[(keys[i] >> shift) & 0xFu];
    }
    for (uint32_t b = 0; b < kRadixBins; ++b)
        if (local[b]) atomicAdd(&h[b], local[b]);
    __syncthreads();
    if (threadIdx.x < kRadixBins) hist[threadIdx.x * blocks + blockIdx.x] = h[threadIdx.x];
}

// Exclusive scan of the digit-major histogram in one block.
__global__ void __launch_bounds__(1024) k_radix_scan(uint32_t* hist, uint32_t count) {
    __shared__ uint32_t part[1024];
    const uint32_t per = (count + 1023u) / 1024u;
    const uint32_t b = threadIdx.x * per;
    uint32_t sum = 0;
    for (uint32_t k = 0; k < per; ++k)
        if (b + k < count) sum += hist[b + k];
    part[threadIdx.x] = sum;
    __syncthreads();
    for (uint32_t off = 1; off < 1024; off <<= 1) {
        const uint32_t v = threadIdx.x >= off ? part[threadIdx.x - off] : 0u;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t run = part[threadIdx.x] - sum;
    for (uint32_t k = 0; k < per; ++k) {
        if (b + k < count) {
            const uint32_t v = hist[b + k];
            hist[b + k] = run;
            run += v;
        }
    }
}

// Radix pass, kernel 3: stable scatter.  Each thread owns 16 consecutive
// keys; a block-wide exclusive scan over the (digit, thread) counts gives
// every key its rank among equal digits in key order.
__global__ void __launch_bounds__(kRadixThreads) k_radix_scatter(const unsigned long long* keys_in,
                                                                 const uint32_t* vals_in, unsigned long long* keys_out,
                                                                 uint32_t* vals_out, uint32_t n, uint32_t shift,
                                                                 const uint32_t* hist, uint32_t blocks) {
    __shared__ uint32_t scan[kRadixBins * kRadixThreads];
    __shared__ uint32_t warp_tot[kRadixBins * kRadixThreads / 32];
    const uint32_t t = threadIdx.x;
    const uint32_t base = blockIdx.x * kRadixTile + t * kRadixItems;
    uint32_t local[kRadixBins] = {};
    for (uint32_t k = 0; k < kRadixItems; ++k) {
        const uint32_t i = base + k;
        if (i < n) ++local[(keys_in[i] >> shift) & 0xFu];
    }
    for (uint32_t b = 0; b < kRadixBins; ++b) scan[b * kRadixThreads + t] = local[b];
    __syncthreads();
    // Exclusive scan over each digit's row (digit-major rows of 256 entries):
    // each thread scans 16 consecutive entries of the flattened array.
    const uint32_t seg = t * kRadixBins;
    uint32_t s = 0;
    for (uint32_t k = 0; k < kRadixBins; ++k) s += scan[seg + k];
    // Scan the per-thread segment sums (256 of them) with warp shuffles.
    uint32_t incl = s;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if ((t & 31) >= uint32_t(o)) incl += v;
    }
    if ((t & 31) == 31) warp_tot[t >> 5] = incl;
    __syncthreads();
    if (t < 32) {
        uint32_t w = t < kRadixThreads / 32 ? warp_tot[t] : 0u;
        uint32_t wi = w;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, wi, o);
            if (t >= uint32_t(o)) wi += v;
        }
        if (t < kRadixThreads / 32) warp_tot[t] = wi - w;
    }
    __syncthreads();
    uint32_t run = warp_tot[t >> 5] + incl - s;
    for (uint32_t k = 0; k < kRadixBins; ++k) {
        const uint32_t v = scan[seg + k];
        scan[seg + k] = run;
        run += v;
    }
    __syncthreads();
    // scan[b * 256 + t] is now the count of keys with digit < b in the block
    // plus digit b in threads < t; subtract the digit's block start.
    uint32_t pos[kRadixBins];
    for (uint32_t b = 0; b < kRadixBins; ++b)
        pos[b] = hist[b * blocks + blockIdx.x] + (scan[b * kRadixThreads + t] - scan[b * kRadixThreads]);
    for (uint32_t k = 0; k < kRadixItems; ++k) {
        const uint32_t i = base + k;
        if (i < n) {
            const unsigned long long key = keys_in[i];
            const uint32_t dgt = uint32_t((key >> shift) & 0xFu);
            const uint32_t dst = pos[dgt]++;
            keys_out[dst] = key;
            vals_out[dst] = vals_in[i];
        }
    }
}

// Common-prefix length of sorted keys i and j (-1 outside the array).  With
// kIndexTieBreak, equal keys compare by their sorted positions instead
// (64 + the common prefix of i and j, Karras 2012 section 4), so duplicate
// keys still give every node exactly one parent; without it the keys must be
// unique, which the scene builds check before they get here.
template <bool kIndexTieBreak>
__device__ __forceinline__ int delta(const unsigned long long* k, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    const unsigned long long x = k[i] ^ k[j];
    if (kIndexTieBreak && x == 0ull) return 64 + __clz(uint32_t(i) ^ uint32_t(j));
    return __clzll(x);
}

// Karras hierarchy (Karras 2012, "Maximizing parallelism in the construction
// of BVHs, octrees, and k-d trees"): internal node i covers [first, last] and
// splits after gamma.  Child codes: bit 31 set = leaf (primitive index).
template <bool kIndexTieBreak = false>
__global__ void k_karras(const unsigned long long* k, int n, uint32_t* left, uint32_t* right, uint32_t* parent_int,
                         uint32_t* parent_leaf, uint32_t* range_first, uint32_t* range_last) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    auto dl = [&](int j) { return delta<kIndexTieBreak>(k, n, i, j); };
    const int d = (dl(i + 1) - dl(i - 1)) >= 0 ? 1 : -1;
    const int dmin = dl(i - d);
    int lmax = 2;
    while (dl(i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (dl(i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = dl(j);
    int s = 0;
    int t = l;
    do {
        t = (t + 1) >> 1;
        if (dl(i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    const int gamma = i + s * d + min(d, 0);
    const int first = min(i, j), last = max(i, j);
    const uint32_t lc = (first == gamma) ? (0x80000000u | uint32_t(gamma)) : uint32_t(gamma);
    const uint32_t rc = (last == gamma + 1) ? (0x80000000u | uint32_t(gamma + 1)) : uint32_t(gamma + 1);
    left[i] = lc;
    right[i] = rc;
    range_first[i] = uint32_t(first);
    range_last[i] = uint32_t(last);
    if (lc & 0x80000000u) parent_leaf[lc & 0x7fffffffu] = uint32_t(i);
    else parent_int[lc] = uint32_t(i);
    if (rc & 0x80000000u) parent_leaf[rc & 0x7fffffffu] = uint32_t(i);
    else parent_int[rc] = uint32_t(i);
}

// Bottom-up refit with arrival counters; each internal node is finished by
// the second child that reaches it.  Box layout: 6 floats (lo xyz, hi xyz).
__global__ void k_refit(const float4* pos_sorted, uint32_t n, const uint32_t* left, const uint32_t* right,
                        const uint32_t* parent_int, const uint32_t* parent_leaf, uint32_t* arrivals, float* box_int,
                        float* box_leaf) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p0 = pos_sorted[size_t(i) * 3], p1 = pos_sorted[size_t(i) * 3 + 1], p2 = pos_sorted[size_t(i) * 3 + 2];
    float* lb = box_leaf + size_t(i) * 6;
    lb[0] = fminf(p0.x, fminf(p1.x, p2.x)); lb[1] = fminf(p0.y, fminf(p1.y, p2.y)); lb[2] = fminf(p0.z, fminf(p1.z, p2.z));
    lb[3] = fmaxf(p0.x, fmaxf(p1.x, p2.x)); lb[4] = fmaxf(p0.y, fmaxf(p1.y, p2.y)); lb[5] = fmaxf(p0.z, fmaxf(p1.z, p2.z));
    if (n == 1) return;
    uint32_t node = parent_leaf[i];
    for (uint32_t guard = 0; guard < n; ++guard) {
        __threadfence();
        if (atomicAdd(arrivals + node, 1u) == 0u) return;  // first arrival: sibling not done yet
        __threadfence();
        const uint32_t l = left[node], r = right[node];
        const volatile float* bl = (l & 0x80000000u) ? box_leaf + size_t(l & 0x7fffffffu) * 6 : box_int + size_t(l) * 6;
        const volatile float* br = (r & 0x80000000u) ? box_leaf + size_t(r & 0x7fffffffu) * 6 : box_int + size_t(r) * 6;
        float* out = box_int + size_t(node) * 6;
        for (int a = 0; a < 3; ++a) {
            out[a] = fminf(bl[a], br[a]);
            out[3 + a] = fmaxf(bl[3 + a], br[3 + a]);
        }
        if (node == 0u) return;
        node = parent_int[node];
    }
}

__global__ void k_gather_positions(const float4* pos, const uint32_t* order, uint32_t n, float4* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t s = order[i];
    out[size_t(i) * 3] = pos[size_t(s) * 3];
    out[size_t(i) * 3 + 1] = pos[size_t(s) * 3 + 1];
    out[size_t(i) * 3 + 2] = pos[size_t(s) * 3 + 2];
}

}  // namespace

namespace {

constexpr uint32_t kFlatUnrefit = 1u, kFlatTooDeep = 2u;
constexpr uint32_t kMaxLbvhDepth = 128u;

// One thread per node of the Karras hierarchy (internal nodes first, then
// leaves): its pre-order index is 2 x (leaves left of its range) + (its
// depth) - (right turns on its path from the root), since every ancestor
// entered on the left precedes it and every subtree it passes on the right
// holds 2 L - 1 nodes for L leaves.  Writes the SoftwareNodeRecord there:
// bounds, and links (left / first, count, right, parent) as the
// reference's buildRange emits them; state[0] collects errors, state[1]
// the maximum depth (root 1).
__global__ void k_flatten_preorder(uint32_t n, const uint32_t* left, const uint32_t* right, const uint32_t* parent_int,
                                   const uint32_t* parent_leaf, const uint32_t* range_first,
                                   const uint32_t* range_last, const uint32_t* arrivals, const float* box_int,
                                   const float* box_leaf, re_software_node* out, DeviceNode* dev_nodes,
                                   uint32_t* state) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t internal = n - 1u;
    if (t >= internal + n) return;
    const bool leaf = t >= internal;
    const uint32_t idx = leaf ? t - internal : t;
    const uint32_t code = leaf ? (0x80000000u | idx) : idx;
    auto leaves_of = [&](uint32_t c) -> uint32_t {
        return (c & 0x80000000u) ? 1u : range_last[c] - range_first[c] + 1u;
    };
    if (!leaf && arrivals[idx] != 2u) atomicOr(state, kFlatUnrefit);
    // Walk to the root: depth and right turns.
    uint32_t depth = 0u, rights = 0u, cur = code;
    bool is_right = false;  // of this node under its parent
    uint32_t parent = 0xffffffffu;
    while (n > 1u && cur != 0u) {
        const uint32_t p = (cur & 0x80000000u) ? parent_leaf[cur & 0x7fffffffu] : parent_int[cur];
        const bool r = right[p] == cur;
        if (depth == 0u) {
            is_right = r;
            parent = p;
        }
        rights += r ? 1u : 0u;
        cur = p;
        if (++depth > kMaxLbvhDepth) {
            atomicOr(state, kFlatTooDeep);
            return;
        }
    }
    const uint32_t first = leaf ? idx : range_first[idx];
    const uint32_t pre = 2u * first + depth - rights;
    atomicMax(state + 1, depth + 1u);
    if (depth + 1u > kMaxLbvhDepth) atomicOr(state, kFlatTooDeep);
    uint32_t parent_pre = 0xffffffffu;
    if (parent != 0xffffffffu) parent_pre = is_right ? pre - 2u * leaves_of(left[parent]) : pre - 1u;
    const float* b = leaf ? box_leaf + size_t(idx) * 6 : box_int + size_t(idx) * 6;
    re_software_node rec;
    rec.bounds_min = re_float4{b[0], b[1], b[2], 0.f};
    rec.bounds_max = re_float4{b[3], b[4], b[5], 0.f};
    if (leaf) rec.links = re_uint4{idx, 1u, 0xffffffffu, parent_pre};
    else rec.links = re_uint4{pre + 1u, 0u, pre + 2u * leaves_of(left[idx]), parent_pre};
    out[pre] = rec;
    if (leaf || dev_nodes == nullptr) return;
    // Child-pair device node (build_device_layout's record), numbered among
    // the interior nodes in pre-order: pre - first, the leaves before it
    // being exactly the first leaves of the order.
    const uint32_t lc = left[idx], rc = right[idx];
    const uint32_t ll = leaves_of(lc);
    const float* lb = (lc & 0x80000000u) ? box_leaf + size_t(lc & 0x7fffffffu) * 6 : box_int + size_t(lc) * 6;
    const float* rb = (rc & 0x80000000u) ? box_leaf + size_t(rc & 0x7fffffffu) * 6 : box_int + size_t(rc) * 6;
    float4* dn = reinterpret_cast<float4*>(dev_nodes + (pre - first));
    dn[0] = make_float4(lb[0], lb[3], lb[1], lb[4]);
    dn[1] = make_float4(lb[2], lb[5], rb[0], rb[3]);
    dn[2] = make_float4(rb[1], rb[4], rb[2], rb[5]);
    const uint32_t lref = (lc & 0x80000000u) ? (lc & 0x7fffffffu) : (pre + 1u) - first;
    const uint32_t rref = (rc & 0x80000000u) ? (rc & 0x7fffffffu) : (pre + 2u * ll) - (first + ll);
    reinterpret_cast<uint4*>(dn)[3] =
        make_uint4(lref, rref, (lc & 0x80000000u) ? 1u : 0u, (rc & 0x80000000u) ? 1u : 0u);
}

// The GPU LBVH passes over device positions (3 float4 per triangle) and
// stable IDs: Morton codes, the 16-pass radix sort, the Karras hierarchy and
// the refit, then sc->flat in the reference's pre-order (leaf order set).
re_status lbvh_core(re_scene* sc, DeviceBuffer& d_pos, DeviceBuffer& d_ids) {
    const uint32_t n = sc->triangle_count;
    const uint32_t blocks = (n + kRadixTile - 1) / kRadixTile;
    DeviceBuffer d_bounds, keys_a, keys_b, vals_a, vals_b, hist, d_left, d_right, d_pint, d_pleaf, d_first,
        d_last, d_arr, d_boxi, d_boxl, d_pos_sorted;
    const size_t ni = n > 1 ? n - 1 : 1;
    RE_CUDA_TRY(d_bounds.reserve(64));
    RE_CUDA_TRY(keys_a.reserve(size_t(n) * 8));
    RE_CUDA_TRY(keys_b.reserve(size_t(n) * 8));
    RE_CUDA_TRY(vals_a.reserve(size_t(n) * 4));
    RE_CUDA_TRY(vals_b.reserve(size_t(n) * 4));
    RE_CUDA_TRY(hist.reserve(size_t(blocks) * kRadixBins * 4));
    RE_CUDA_TRY(d_left.reserve(ni * 4));
    RE_CUDA_TRY(d_right.reserve(ni * 4));
    RE_CUDA_TRY(d_pint.reserve(ni * 4));
    RE_CUDA_TRY(d_pleaf.reserve(size_t(n) * 4));
    RE_CUDA_TRY(d_first.reserve(ni * 4));
    RE_CUDA_TRY(d_last.reserve(ni * 4));
    RE_CUDA_TRY(d_arr.reserve(ni * 4));
    RE_CUDA_TRY(d_boxi.reserve(ni * 24));
    RE_CUDA_TRY(d_boxl.reserve(size_t(n) * 24));
    RE_CUDA_TRY(d_pos_sorted.reserve(size_t(n) * 3 * sizeof(float4)));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    const uint32_t init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    RE_CUDA_TRY(cudaMemcpy(d_bounds.ptr, init, sizeof(init), cudaMemcpyHostToDevice));
    k_bounds<<<std::min<uint32_t>(1184, (n + 255) / 256), 256>>>(static_cast<const float4*>(d_pos.ptr), n,
                                                                   static_cast<uint32_t*>(d_bounds.ptr));
    k_morton<<<(n + 255) / 256, 256>>>(static_cast<const float4*>(d_pos.ptr), static_cast<const uint32_t*>(d_ids.ptr), n,
                                       static_cast<const uint32_t*>(d_bounds.ptr),
                                       static_cast<unsigned long long*>(keys_a.ptr), static_cast<uint32_t*>(vals_a.ptr));
    // 16 stable 4-bit passes over the 64-bit (code << 32 | ID) key.
    unsigned long long* kin = static_cast<unsigned long long*>(keys_a.ptr);
    unsigned long long* kout = static_cast<unsigned long long*>(keys_b.ptr);
    uint32_t* vin = static_cast<uint32_t*>(vals_a.ptr);
    uint32_t* vout = static_cast<uint32_t*>(vals_b.ptr);
    for (uint32_t shift = 0; shift < 64; shift += 4) {
        k_radix_hist<<<blocks, kRadixThreads>>>(kin, n, shift, static_cast<uint32_t*>(hist.ptr), blocks);
        k_radix_scan<<<1, 1024>>>(static_cast<uint32_t*>(hist.ptr), blocks * kRadixBins);
        k_radix_scatter<<<blocks, kRadixThreads>>>(kin, vin, kout, vout, n, shift, static_cast<uint32_t*>(hist.ptr),
                                                   blocks);
        std::swap(kin, kout);
        std::swap(vin, vout);
    }
    k_gather_positions<<<(n + 255) / 256, 256>>>(static_cast<const float4*>(d_pos.ptr), vin, n,
                                                 static_cast<float4*>(d_pos_sorted.ptr));
    if (n > 1) {
        k_karras<false><<<(n - 1 + 255) / 256, 256>>>(kin, int(n), static_cast<uint32_t*>(d_left.ptr),
                                               static_cast<uint32_t*>(d_right.ptr), static_cast<uint32_t*>(d_pint.ptr),
                                               static_cast<uint32_t*>(d_pleaf.ptr), static_cast<uint32_t*>(d_first.ptr),
                                               static_cast<uint32_t*>(d_last.ptr));
        RE_CUDA_TRY(cudaMemset(d_arr.ptr, 0, ni * 4));
    }
    k_refit<<<(n + 255) / 256, 256>>>(static_cast<const float4*>(d_pos_sorted.ptr), n,
                                      static_cast<const uint32_t*>(d_left.ptr), static_cast<const uint32_t*>(d_right.ptr),
                                      static_cast<const uint32_t*>(d_pint.ptr), static_cast<const uint32_t*>(d_pleaf.ptr),
                                      static_cast<uint32_t*>(d_arr.ptr), static_cast<float*>(d_boxi.ptr),
                                      static_cast<float*>(d_boxl.ptr));
    cudaEventRecord(e1);
    RE_CUDA_TRY(cudaEventSynchronize(e1));
    float gpu_ms = 0.f;
    cudaEventElapsedTime(&gpu_ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    RE_CUDA_TRY(cudaGetLastError());
    sc->lbvh_gpu_ms = gpu_ms;

    // Flattened records in the reference's pre-order numbering
    // (BuildKarrasLbvh's buildRange order), written on the device.
    std::vector<uint32_t> order(n);
    RE_CUDA_TRY(cudaMemcpy(order.data(), vin, size_t(n) * 4, cudaMemcpyDeviceToHost));
    const uint32_t nodes = 2u * n - 1u;
    DeviceBuffer d_flat, d_state;
    RE_CUDA_TRY(d_flat.reserve(size_t(nodes) * sizeof(re_software_node)));
    // The child-pair device nodes straight from the flattening (a single
    // leaf keeps the host layout's synthetic root).
    DeviceNode* dev_nodes = nullptr;
    if (n > 1u) {
        RE_CUDA_TRY(sc->nodes.reserve(size_t(n - 1u) * sizeof(DeviceNode)));
        dev_nodes = static_cast<DeviceNode*>(sc->nodes.ptr);
    }
    RE_CUDA_TRY(d_state.reserve(8));
    RE_CUDA_TRY(cudaMemset(d_state.ptr, 0, 8));
    k_flatten_preorder<<<(nodes + 255) / 256, 256>>>(n, static_cast<const uint32_t*>(d_left.ptr),
                                                     static_cast<const uint32_t*>(d_right.ptr),
                                                     static_cast<const uint32_t*>(d_pint.ptr),
                                                     static_cast<const uint32_t*>(d_pleaf.ptr),
                                                     static_cast<const uint32_t*>(d_first.ptr),
                                                     static_cast<const uint32_t*>(d_last.ptr),
                                                     static_cast<const uint32_t*>(d_arr.ptr),
                                                     static_cast<const float*>(d_boxi.ptr),
                                                     static_cast<const float*>(d_boxl.ptr),
                                                     static_cast<re_software_node*>(d_flat.ptr), dev_nodes,
                                                     static_cast<uint32_t*>(d_state.ptr));
    RE_CUDA_TRY(cudaGetLastError());
    uint32_t state[2] = {0, 0};
    RE_CUDA_TRY(cudaMemcpy(state, d_state.ptr, 8, cudaMemcpyDeviceToHost));
    if (state[0] & kFlatUnrefit)
        return set_error(RE_RECORDING_FAILED, "LBVH bottom-up refit did not reach every node");
    if (state[0] & kFlatTooDeep)
        return set_error(RE_INVALID_ARGUMENT, "LBVH hierarchy exceeds its configured maximum depth");
    FlatBvh& flat = sc->flat;
    flat = FlatBvh{};
    flat.nodes.resize(nodes);
    RE_CUDA_TRY(cudaMemcpy(flat.nodes.data(), d_flat.ptr, size_t(nodes) * sizeof(re_software_node),
                           cudaMemcpyDeviceToHost));
    flat.max_depth = state[1];
    flat.leaf_count = n;
    if (dev_nodes != nullptr) {
        sc->device_node_count = n - 1u;
        sc->layout_meta.root_is_leaf = 0;
        sc->layout_meta.node_original.clear();
    }
    flat.leaf_order = order;
    return RE_SUCCESS;
}

}  // namespace

re_status build_lbvh_on_device(re_scene* sc, const re_canonical_triangle* tris) {
    const uint32_t n = sc->triangle_count;
    const auto t0 = std::chrono::steady_clock::now();
    // Upload positions and stable IDs.
    std::vector<float4> pos(size_t(n) * 3);
    std::vector<uint32_t> ids(n);
    for (uint32_t i = 0; i < n; ++i) {
        for (int v = 0; v < 3; ++v)
            pos[size_t(i) * 3 + v] = make_float4(tris[i].positions[v].x, tris[i].positions[v].y,
                                                 tris[i].positions[v].z, 0.f);
        ids[i] = tris[i].metadata.z;
    }
    DeviceBuffer d_pos, d_ids;
    RE_CUDA_TRY(d_pos.reserve(pos.size() * sizeof(float4)));
    RE_CUDA_TRY(d_ids.reserve(size_t(n) * 4));
    RE_CUDA_TRY(cudaMemcpy(d_pos.ptr, pos.data(), pos.size() * sizeof(float4), cudaMemcpyHostToDevice));
    RE_CUDA_TRY(cudaMemcpy(d_ids.ptr, ids.data(), size_t(n) * 4, cudaMemcpyHostToDevice));
    re_status st = lbvh_core(sc, d_pos, d_ids);
    if (st != RE_SUCCESS) return st;
    st = n > 1u ? upload_scene_triangles(sc, nullptr, tris, sc->flat.leaf_order)
                : upload_scene_geometry(sc, nullptr, tris, sc->flat.leaf_order);
    if (st != RE_SUCCESS) return st;
    sc->lbvh_total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return RE_SUCCESS;
}

// ---------------------------------------------------------------------------
// Scene build from device records (re_scene_create_from_device): the host
// path's primitive checks on the device (re_scene_create: finite vertices,
// the degenerate-area rule, traversal IDs present and unique -- here they
// must also be below the triangle count, so a bitmap checks uniqueness),
// the LBVH passes, then the leaf-ordered triangle and attribute records
// packed on the device exactly as upload_scene_geometry packs them on the
// host.
// ---------------------------------------------------------------------------
namespace {

constexpr uint32_t kBadFinite = 1u, kBadDegenerate = 2u, kBadNoId = 4u, kBadIdRange = 8u, kBadIdDup = 16u;
constexpr uint32_t kHasAlphaMask = 32u;  // not an error: some record is alpha-masked

__global__ void k_check_extract(const re_canonical_triangle* t, uint32_t n, float4* pos, uint32_t* ids,
                                uint32_t* seen, uint32_t* flags) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const re_canonical_triangle& r = t[i];
    const re_float4 p0 = r.positions[0], p1 = r.positions[1], p2 = r.positions[2];
    uint32_t bad = 0u;
    if (!(isfinite(p0.x) && isfinite(p0.y) && isfinite(p0.z) && isfinite(p1.x) && isfinite(p1.y) && isfinite(p1.z) &&
          isfinite(p2.x) && isfinite(p2.y) && isfinite(p2.z))) {
        bad |= kBadFinite;
    } else {
        const float e0x = __fsub_rn(p1.x, p0.x), e0y = __fsub_rn(p1.y, p0.y), e0z = __fsub_rn(p1.z, p0.z);
        const float e1x = __fsub_rn(p2.x, p0.x), e1y = __fsub_rn(p2.y, p0.y), e1z = __fsub_rn(p2.z, p0.z);
        const float cx = __fsub_rn(__fmul_rn(e0y, e1z), __fmul_rn(e0z, e1y));
        const float cy = __fsub_rn(__fmul_rn(e0z, e1x), __fmul_rn(e0x, e1z));
        const float cz = __fsub_rn(__fmul_rn(e0x, e1y), __fmul_rn(e0y, e1x));
        const float area2 = __fadd_rn(__fadd_rn(__fmul_rn(cx, cx), __fmul_rn(cy, cy)), __fmul_rn(cz, cz));
        const float l0 = __fadd_rn(__fadd_rn(__fmul_rn(e0x, e0x), __fmul_rn(e0y, e0y)), __fmul_rn(e0z, e0z));
        const float l1 = __fadd_rn(__fadd_rn(__fmul_rn(e1x, e1x), __fmul_rn(e1y, e1y)), __fmul_rn(e1z, e1z));
        const float scale = l0 > l1 ? l0 : l1;
        if (!isfinite(area2) || !(area2 > __fmul_rn(__fmul_rn(scale, scale), 1.0e-14f))) bad |= kBadDegenerate;
    }
    const uint32_t id = r.metadata.z;
    if (id == 0xffffffffu) bad |= kBadNoId;
    else if (id >= n) bad |= kBadIdRange;
    else if (atomicOr(seen + (id >> 5), 1u << (id & 31u)) & (1u << (id & 31u))) bad |= kBadIdDup;
    if ((r.metadata.x & RE_GEOMETRY_FLAG_ALPHA_MASK) != 0u || (r.metadata.y & RE_MATERIAL_FLAG_ALPHA_MASK) != 0u)
        bad |= kHasAlphaMask;
    if (bad != 0u) atomicOr(flags, bad);
    pos[size_t(i) * 3 + 0] = make_float4(p0.x, p0.y, p0.z, 0.f);
    pos[size_t(i) * 3 + 1] = make_float4(p1.x, p1.y, p1.z, 0.f);
    pos[size_t(i) * 3 + 2] = make_float4(p2.x, p2.y, p2.z, 0.f);
    ids[i] = id;
}

__global__ void k_pack_leaf_order(const re_canonical_triangle* t, const uint32_t* order, uint32_t n,
                                  DeviceTriangle* tris, DeviceAttr* attrs, float4* alpha_tc) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t src = order[i];
    const re_canonical_triangle& r = t[src];
    const re_float4* p = r.positions;
    const bool double_sided = (r.metadata.x & RE_GEOMETRY_FLAG_DOUBLE_SIDED) != 0u ||
                              (r.metadata.y & RE_MATERIAL_FLAG_DOUBLE_SIDED) != 0u;
    const bool casts = (r.metadata.w & RE_INSTANCE_FLAG_CASTS_SHADOW) != 0u;
    const bool masked = (r.metadata.x & RE_GEOMETRY_FLAG_ALPHA_MASK) != 0u ||
                        (r.metadata.y & RE_MATERIAL_FLAG_ALPHA_MASK) != 0u;
    const uint32_t flags = (double_sided ? kTriDoubleSided : 0u) | (casts ? kTriCastsShadow : 0u) |
                           (masked ? kTriAlphaMask : 0u);
    if (alpha_tc != nullptr) {
        alpha_tc[2 * size_t(i)] = make_float4(r.texcoords[0].x, r.texcoords[0].y, r.texcoords[1].x, r.texcoords[1].y);
        alpha_tc[2 * size_t(i) + 1] =
            make_float4(r.texcoords[2].x, r.texcoords[2].y, __uint_as_float(r.identity.w), 0.f);
    }
    float4* d = reinterpret_cast<float4*>(tris + i);
    d[0] = make_float4(p[0].x, p[0].y, p[0].z, __uint_as_float(flags));
    d[1] = make_float4(__fsub_rn(p[1].x, p[0].x), __fsub_rn(p[1].y, p[0].y), __fsub_rn(p[1].z, p[0].z),
                       __uint_as_float(r.identity.x));
    d[2] = make_float4(__fsub_rn(p[2].x, p[0].x), __fsub_rn(p[2].y, p[0].y), __fsub_rn(p[2].z, p[0].z),
                       __uint_as_float(r.identity.y));
    reinterpret_cast<uint4*>(d)[3] = make_uint4(r.identity.x, r.identity.y, r.metadata.z, src);
    float4* a = reinterpret_cast<float4*>(attrs + i);
    a[0] = make_float4(r.normals[0].x, r.normals[0].y, r.normals[0].z, 0.f);
    a[1] = make_float4(r.normals[1].x, r.normals[1].y, r.normals[1].z, 0.f);
    a[2] = make_float4(r.normals[2].x, r.normals[2].y, r.normals[2].z, 0.f);
    reinterpret_cast<uint4*>(a)[3] = make_uint4(r.identity.x, r.identity.y, r.identity.z, r.identity.w);
}

}  // namespace

re_status build_lbvh_from_device_records(re_scene* sc, const re_canonical_triangle* d_tris) {
    const uint32_t n = sc->triangle_count;
    const auto t0 = std::chrono::steady_clock::now();
    DeviceBuffer d_pos, d_ids, d_seen, d_flags;
    RE_CUDA_TRY(d_pos.reserve(size_t(n) * 3 * sizeof(float4)));
    RE_CUDA_TRY(d_ids.reserve(size_t(n) * 4));
    RE_CUDA_TRY(d_seen.reserve((size_t(n) + 31) / 32 * 4));
    RE_CUDA_TRY(d_flags.reserve(4));
    RE_CUDA_TRY(cudaMemset(d_seen.ptr, 0, (size_t(n) + 31) / 32 * 4));
    RE_CUDA_TRY(cudaMemset(d_flags.ptr, 0, 4));
    k_check_extract<<<(n + 255) / 256, 256>>>(d_tris, n, static_cast<float4*>(d_pos.ptr),
                                              static_cast<uint32_t*>(d_ids.ptr), static_cast<uint32_t*>(d_seen.ptr),
                                              static_cast<uint32_t*>(d_flags.ptr));
    RE_CUDA_TRY(cudaGetLastError());
    uint32_t bad = 0;
    RE_CUDA_TRY(cudaMemcpy(&bad, d_flags.ptr, 4, cudaMemcpyDeviceToHost));
    if (bad & kBadFinite) return set_error(RE_INVALID_ARGUMENT, "A BVH cannot contain a non-finite triangle");
    if (bad & kBadDegenerate) return set_error(RE_INVALID_ARGUMENT, "scene contains a degenerate triangle");
    if (bad & kBadNoId) return set_error(RE_INVALID_ARGUMENT, "triangle has no traversal ID");
    if (bad & kBadIdRange)
        return set_error(RE_INVALID_ARGUMENT, "traversal IDs of device records must be below the triangle count");
    if (bad & kBadIdDup) return set_error(RE_INVALID_ARGUMENT, "traversal IDs must be unique");
    re_status st = lbvh_core(sc, d_pos, d_ids);
    if (st != RE_SUCCESS) return st;
    if (n == 1u) {
        st = upload_scene_nodes(sc);
        if (st != RE_SUCCESS) return st;
    }
    DeviceBuffer d_order;
    RE_CUDA_TRY(d_order.reserve(size_t(n) * 4));
    RE_CUDA_TRY(cudaMemcpy(d_order.ptr, sc->flat.leaf_order.data(), size_t(n) * 4, cudaMemcpyHostToDevice));
    RE_CUDA_TRY(sc->tris.reserve(size_t(n) * sizeof(DeviceTriangle)));
    RE_CUDA_TRY(sc->attrs.reserve(size_t(n) * sizeof(DeviceAttr)));
    sc->alpha_masked = (bad & kHasAlphaMask) != 0u;
    if (sc->alpha_masked) RE_CUDA_TRY(sc->alpha_tc.reserve(size_t(n) * 2 * sizeof(float4)));
    k_pack_leaf_order<<<(n + 255) / 256, 256>>>(d_tris, static_cast<const uint32_t*>(d_order.ptr), n,
                                                static_cast<DeviceTriangle*>(sc->tris.ptr),
                                                static_cast<DeviceAttr*>(sc->attrs.ptr),
                                                sc->alpha_masked ? static_cast<float4*>(sc->alpha_tc.ptr) : nullptr);
    RE_CUDA_TRY(cudaGetLastError());
    RE_CUDA_TRY(cudaDeviceSynchronize());
    sc->lbvh_total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return RE_SUCCESS;
}

// ---------------------------------------------------------------------------
// Allocation-free LBVH build (re_lbvh_build_static).  The same passes as
// build_lbvh_on_device, with every intermediate array carved out of one
// file-scope device array instead of cudaMalloc'd buffers, launched on the
// caller's stream, with the Karras hierarchy written to caller buffers.
// ---------------------------------------------------------------------------
namespace {

constexpr uint32_t kStaticMaxTris = RE_LBVH_STATIC_MAX_TRIANGLES;
constexpr size_t kStaticAlign = 256;
constexpr size_t static_slot(size_t bytes) { return (bytes + kStaticAlign - 1) / kStaticAlign * kStaticAlign; }
constexpr size_t kStaticHistBytes = size_t((kStaticMaxTris + kRadixTile - 1) / kRadixTile) * kRadixBins * 4;
constexpr size_t kStaticScratchBytes =
    2 * static_slot(size_t(kStaticMaxTris) * 8) +   // radix keys, ping-pong
    2 * static_slot(size_t(kStaticMaxTris) * 4) +   // radix values, ping-pong
    static_slot(kStaticHistBytes) +                 // digit histograms
    static_slot(6 * 4) +                            // scene bounds
    6 * static_slot(size_t(kStaticMaxTris) * 4) +   // left, right, parent_int, first, last, arrivals
    static_slot(size_t(kStaticMaxTris) * 4) +       // parent_leaf
    2 * static_slot(size_t(kStaticMaxTris) * 24) +  // internal and leaf boxes
    static_slot(size_t(kStaticMaxTris) * 48);       // positions in sorted order

// Scratch of re_lbvh_build_static: about 9.3 MB per device the library is
// loaded on.  Nothing in it needs an initial value: each call re-initialises
// the scene bounds and the refit arrival counters before using them.
static __device__ __align__(256) unsigned char g_lbvh_static_scratch[kStaticScratchBytes];

// Device address of g_lbvh_static_scratch per device, resolved once with that
// device current.
std::mutex g_static_mutex;
void* g_static_addr[64] = {};

__global__ void k_static_init(uint32_t* bounds, uint32_t* arrivals, uint32_t arrival_count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 6) bounds[i] = i < 3 ? 0xffffffffu : 0u;
    for (uint32_t k = i; k < arrival_count; k += gridDim.x * blockDim.x) arrivals[k] = 0u;
}

// Packs the Karras hierarchy into the caller's 32-byte node records.
__global__ void k_static_pack(const uint32_t* left, const uint32_t* right, const float* box_int, uint32_t count,
                              re_lbvh_node* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float* b = box_int + size_t(i) * 6;
    float4* o = reinterpret_cast<float4*>(out + i);
    o[0] = make_float4(b[0], b[1], b[2], __uint_as_float(left[i]));
    o[1] = make_float4(b[3], b[4], b[5], __uint_as_float(right[i]));
}

}  // namespace

}  // namespace re

extern "C" RE_API re_status re_lbvh_build_static(const re_float4* positions, const uint32_t* stable_ids,
                                                 uint32_t count, uint32_t* order_out, re_lbvh_node* nodes_out,
                                                 void* stream) {
    using namespace re;
    if (positions == nullptr || stable_ids == nullptr || order_out == nullptr || (count > 1 && nodes_out == nullptr))
        return set_error(RE_INVALID_ARGUMENT, "null argument");
    if (count == 0) return set_error(RE_INVALID_ARGUMENT, "LBVH build of zero triangles");
    if (count > kStaticMaxTris)
        return set_error(RE_INVALID_ARGUMENT, "re_lbvh_build_static: " + std::to_string(count) +
                                                  " triangles exceed the static scratch capacity of " +
                                                  std::to_string(kStaticMaxTris));
    if ((reinterpret_cast<uintptr_t>(positions) & 15u) != 0 || (reinterpret_cast<uintptr_t>(nodes_out) & 15u) != 0 ||
        (reinterpret_cast<uintptr_t>(stable_ids) & 3u) != 0 || (reinterpret_cast<uintptr_t>(order_out) & 3u) != 0)
        return set_error(RE_INVALID_ARGUMENT, "re_lbvh_build_static: misaligned buffer");
    // A launch error left by the caller's earlier work would otherwise be
    // picked up by the check after this call's launches and reported as this
    // build's failure: report it as what it is, before launching anything.
    const cudaError_t pending = cudaGetLastError();
    if (pending != cudaSuccess)
        return set_error(RE_CUDA_ERROR, std::string("re_lbvh_build_static: CUDA error pending from earlier work: ") +
                                            cudaGetErrorString(pending));
    int device = 0;
    RE_CUDA_TRY(cudaGetDevice(&device));
    if (device < 0 || device >= 64) return set_error(RE_INVALID_ARGUMENT, "device ordinal out of range");
    char* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_static_mutex);
        if (g_static_addr[device] == nullptr) {
            void* addr = nullptr;
            RE_CUDA_TRY(cudaGetSymbolAddress(&addr, g_lbvh_static_scratch));
            g_static_addr[device] = addr;
        }
        base = static_cast<char*>(g_static_addr[device]);
    }
    const uint32_t n = count;
    const size_t N = kStaticMaxTris;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char* p = base + off;
        off += static_slot(bytes);
        return p;
    };
    auto* keys_a = reinterpret_cast<unsigned long long*>(take(N * 8));
    auto* keys_b = reinterpret_cast<unsigned long long*>(take(N * 8));
    auto* vals_a = reinterpret_cast<uint32_t*>(take(N * 4));
    auto* vals_b = reinterpret_cast<uint32_t*>(take(N * 4));
    auto* hist = reinterpret_cast<uint32_t*>(take(kStaticHistBytes));
    auto* bounds = reinterpret_cast<uint32_t*>(take(6 * 4));
    auto* left = reinterpret_cast<uint32_t*>(take(N * 4));
    auto* right = reinterpret_cast<uint32_t*>(take(N * 4));
    auto* pint = reinterpret_cast<uint32_t*>(take(N * 4));
    auto* first = reinterpret_cast<uint32_t*>(take(N * 4));
    auto* last = reinterpret_cast<uint32_t*>(take(N * 4));
    auto* arrivals = reinterpret_cast<uint32_t*>(take(N * 4));
    auto* pleaf = reinterpret_cast<uint32_t*>(take(N * 4));
    auto* box_int = reinterpret_cast<float*>(take(N * 24));
    auto* box_leaf = reinterpret_cast<float*>(take(N * 24));
    auto* pos_sorted = reinterpret_cast<float4*>(take(N * 48));
    if (off > kStaticScratchBytes) return set_error(RE_FATAL_QUEUE, "static LBVH scratch layout overflow");

    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const float4* pos = reinterpret_cast<const float4*>(positions);
    const uint32_t blocks = (n + kRadixTile - 1) / kRadixTile;
    const uint32_t ni = n - 1;
    k_static_init<<<std::max<uint32_t>(1, std::min<uint32_t>(148, (ni + 255) / 256)), 256, 0, st>>>(bounds, arrivals,
                                                                                                      ni);
    k_bounds<<<std::min<uint32_t>(1184, (n + 255) / 256), 256, 0, st>>>(pos, n, bounds);
    k_morton<<<(n + 255) / 256, 256, 0, st>>>(pos, stable_ids, n, bounds, keys_a, vals_a);
    unsigned long long* kin = keys_a;
    unsigned long long* kout = keys_b;
    uint32_t* vin = vals_a;
    uint32_t* vout = vals_b;
    for (uint32_t shift = 0; shift < 64; shift += 4) {
        k_radix_hist<<<blocks, kRadixThreads, 0, st>>>(kin, n, shift, hist, blocks);
        k_radix_scan<<<1, 1024, 0, st>>>(hist, blocks * kRadixBins);
        k_radix_scatter<<<blocks, kRadixThreads, 0, st>>>(kin, vin, kout, vout, n, shift, hist, blocks);
        std::swap(kin, kout);
        std::swap(vin, vout);
    }
    // 16 passes: the sorted keys and order are back in keys_a / vals_a.
    RE_CUDA_TRY(cudaMemcpyAsync(order_out, vin, size_t(n) * 4, cudaMemcpyDeviceToDevice, st));
    if (n > 1) {
        k_gather_positions<<<(n + 255) / 256, 256, 0, st>>>(pos, vin, n, pos_sorted);
        // Stable IDs are not checked for uniqueness here (that would need a
        // read-back): equal (code, ID) keys are split by sorted position.
        k_karras<true><<<(ni + 255) / 256, 256, 0, st>>>(kin, int(n), left, right, pint, pleaf, first, last);
        k_refit<<<(n + 255) / 256, 256, 0, st>>>(pos_sorted, n, left, right, pint, pleaf, arrivals, box_int,
                                                 box_leaf);
        k_static_pack<<<(ni + 255) / 256, 256, 0, st>>>(left, right, box_int, ni, nodes_out);
    }
    RE_CUDA_TRY(cudaGetLastError());
    return clear_error();
}
