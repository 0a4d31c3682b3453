#include "sah_builder.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <future>
#include <limits>
#include <stdexcept>

namespace re {
namespace {

constexpr uint32_t kInvalid = 0xffffffffu;
constexpr uint32_t kMaxDepth = 128u;  // Bvh.hpp:70, SoftwareGpu.hpp:18
constexpr uint32_t kMaxBins = 64u;

struct Box {
    float lo[3] = {INFINITY, INFINITY, INFINITY};
    float hi[3] = {-INFINITY, -INFINITY, -INFINITY};

    bool valid() const {
        for (int a = 0; a < 3; ++a) {
            if (!std::isfinite(lo[a]) || !std::isfinite(hi[a]) || !(lo[a] <= hi[a])) return false;
        }
        return true;
    }
    // Point expansion without a validity test (Aabb::Expand(point), Geometry.hpp:80-84).
    void grow_point(const float p[3]) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = lo[a] < p[a] ? lo[a] : p[a];
            hi[a] = hi[a] > p[a] ? hi[a] : p[a];
        }
    }
    // Box expansion skips invalid boxes (Aabb::Expand(Aabb), Geometry.hpp:86-98).
    void grow_box(const Box& b) {
        if (!b.valid()) return;
        if (!valid()) { *this = b; return; }
        for (int a = 0; a < 3; ++a) {
            lo[a] = lo[a] < b.lo[a] ? lo[a] : b.lo[a];
            hi[a] = hi[a] > b.hi[a] ? hi[a] : b.hi[a];
        }
    }
    double area() const {
        if (!valid()) return 0.0;
        const double ex = double(hi[0]) - double(lo[0]);
        const double ey = double(hi[1]) - double(lo[1]);
        const double ez = double(hi[2]) - double(lo[2]);
        return 2.0 * ((ex * ey) + (ey * ez) + (ez * ex));
    }
};

struct Ref {
    uint32_t index;     // source triangle index
    uint32_t id;        // stable primitive ID
    Box box;
    float c[3];         // centroid
};

struct Node {
    Box box;
    uint32_t left = kInvalid, right = kInvalid;
    uint32_t first = 0, count = 0;
    uint32_t parent = kInvalid;
};

struct Builder {
    std::vector<Ref>& refs;
    uint32_t bins;
    uint32_t max_leaf;
    std::vector<Ref> scratch;  // stable-partition workspace, same size as refs

    uint32_t bin_of(float c, float cmin, float cext) const {
        const double normalized = (double(c) - double(cmin)) / double(cext);
        const double scaled = normalized * double(bins);
        if (!(scaled > 0.0)) return 0u;
        if (scaled >= double(bins)) return bins - 1u;
        return uint32_t(scaled);
    }

    struct Split { bool valid = false; uint32_t axis = 0, last_left = 0; double cost = INFINITY; };

    Split find_split(size_t begin, size_t end, const Box& cb) const {
        Split best;
        float ext[3];
        for (int a = 0; a < 3; ++a) ext[a] = cb.hi[a] - cb.lo[a];
        Box bbox[kMaxBins];
        uint32_t bcount[kMaxBins];
        Box right_box[kMaxBins];
        uint32_t right_count[kMaxBins];
        for (uint32_t axis = 0; axis < 3; ++axis) {
            if (!(ext[axis] > 0.0f)) continue;
            for (uint32_t b = 0; b < bins; ++b) { bbox[b] = Box{}; bcount[b] = 0u; }
            for (size_t i = begin; i < end; ++i) {
                const uint32_t b = bin_of(refs[i].c[axis], cb.lo[axis], ext[axis]);
                ++bcount[b];
                bbox[b].grow_box(refs[i].box);
            }
            // Suffix sweep; min/max unions are exact, so this equals the
            // per-split re-summation of the reference.
            Box acc;
            uint32_t n = 0;
            for (int b = int(bins) - 1; b >= 1; --b) {
                acc.grow_box(bbox[b]);
                n += bcount[b];
                right_box[b] = acc;
                right_count[b] = n;
            }
            Box lacc;
            uint32_t ln = 0;
            for (uint32_t s = 0; s + 1 < bins; ++s) {
                lacc.grow_box(bbox[s]);
                ln += bcount[s];
                const uint32_t rn = right_count[s + 1];
                if (ln == 0 || rn == 0) continue;
                const double cost = lacc.area() * double(ln) + right_box[s + 1].area() * double(rn);
                if (!best.valid || cost < best.cost) {
                    best.valid = true;
                    best.axis = axis;
                    best.last_left = s;
                    best.cost = cost;
                }
            }
        }
        return best;
    }

    size_t sah_partition(size_t begin, size_t end, const Box& cb, const Split& s) {
        const float cmin = cb.lo[s.axis];
        const float cext = cb.hi[s.axis] - cb.lo[s.axis];
        size_t l = begin, r = 0;
        Ref* tmp = scratch.data() + begin;
        for (size_t i = begin; i < end; ++i) {
            if (bin_of(refs[i].c[s.axis], cmin, cext) <= s.last_left) refs[l++] = refs[i];
            else tmp[r++] = refs[i];
        }
        std::copy(tmp, tmp + r, refs.begin() + l);
        return l;
    }

    size_t median_partition(size_t begin, size_t end, const Box& cb) {
        float ext[3];
        for (int a = 0; a < 3; ++a) ext[a] = cb.hi[a] - cb.lo[a];
        uint32_t axis = 0;  // LongestAxis (Math.hpp:197-209)
        if (ext[1] > ext[0]) axis = 1;
        if (ext[2] > ext[axis]) axis = 2;
        std::stable_sort(refs.begin() + begin, refs.begin() + end,
                         [axis](const Ref& l, const Ref& r) {
                             if (l.c[axis] < r.c[axis]) return true;
                             if (l.c[axis] > r.c[axis]) return false;
                             if (l.id < r.id) return true;
                             if (l.id > r.id) return false;
                             return l.index < r.index;
                         });
        return begin + (end - begin) / 2u;
    }

    // Decides the split of [begin, end) and partitions it.  Returns `end`
    // marker semantics: leaf when count <= max_leaf.
    size_t split_range(size_t begin, size_t end, Box& bounds) {
        for (size_t i = begin; i < end; ++i) bounds.grow_box(refs[i].box);
        if (end - begin <= max_leaf) return begin;  // leaf
        Box cb;
        for (size_t i = begin; i < end; ++i) cb.grow_point(refs[i].c);
        size_t middle = begin;
        const Split s = find_split(begin, end, cb);
        if (s.valid) middle = sah_partition(begin, end, cb, s);
        if (middle == begin || middle == end) middle = median_partition(begin, end, cb);
        return middle;
    }

    // Sequential pre-order build appending to `out`; indices are relative to
    // `base` (the final index of out[0]).
    uint32_t build_seq(std::vector<Node>& out, uint32_t base, size_t begin, size_t end,
                       uint32_t depth, uint32_t& max_depth) {
        if (depth > kMaxDepth) throw std::length_error("BVH depth exceeds 128");
        const uint32_t local = uint32_t(out.size());
        out.emplace_back();
        if (depth > max_depth) max_depth = depth;
        Box bounds;
        const size_t middle = split_range(begin, end, bounds);
        if (end - begin <= max_leaf) {
            Node& leaf = out[local];
            leaf.box = bounds;
            leaf.first = uint32_t(begin);
            leaf.count = uint32_t(end - begin);
            return base + local;
        }
        const uint32_t l = build_seq(out, base, begin, middle, depth + 1, max_depth);
        const uint32_t r = build_seq(out, base, middle, end, depth + 1, max_depth);
        Node& in = out[local];
        in.box = bounds;
        in.left = l;
        in.right = r;
        return base + local;
    }

    // Parallel variant for the top levels: returns a self-contained pre-order
    // sub-tree with indices relative to its own root (0).
    std::vector<Node> build_par(size_t begin, size_t end, uint32_t depth, int spawn_levels,
                                uint32_t& max_depth) {
        std::vector<Node> out;
        if (spawn_levels <= 0 || end - begin < 65536) {
            out.reserve((end - begin) * 2);
            build_seq(out, 0, begin, end, depth, max_depth);
            return out;
        }
        if (depth > kMaxDepth) throw std::length_error("BVH depth exceeds 128");
        if (depth > max_depth) max_depth = depth;
        Box bounds;
        const size_t middle = split_range(begin, end, bounds);
        // end - begin >= 65536 > max_leaf, so this is always an interior node.
        uint32_t depth_l = 0, depth_r = 0;
        auto fut = std::async(std::launch::async, [&] {
            return build_par(begin, middle, depth + 1, spawn_levels - 1, depth_l);
        });
        std::vector<Node> right = build_par(middle, end, depth + 1, spawn_levels - 1, depth_r);
        std::vector<Node> left = fut.get();
        max_depth = std::max(max_depth, std::max(depth_l, depth_r));
        out.resize(1 + left.size() + right.size());
        const uint32_t lo = 1, ro = uint32_t(1 + left.size());
        auto shift = [](Node n, uint32_t off) {
            if (n.count == 0) { n.left += off; n.right += off; }
            return n;
        };
        for (size_t i = 0; i < left.size(); ++i) out[lo + i] = shift(left[i], lo);
        for (size_t i = 0; i < right.size(); ++i) out[ro + i] = shift(right[i], ro);
        out[0].box = bounds;
        out[0].left = lo;
        out[0].right = ro;
        return out;
    }
};

}  // namespace

bool build_binned_sah(const std::vector<HostTriangle>& triangles, uint32_t bins,
                      uint32_t max_leaf_size, uint32_t threads, FlatBvh& out,
                      std::string& error) {
    out = FlatBvh{};
    if (bins < 2 || bins > kMaxBins) { error = "SAH bin count must be in [2, 64]"; return false; }
    if (max_leaf_size == 0) { error = "A BVH leaf must allow at least one primitive"; return false; }
    for (const HostTriangle& t : triangles) {
        for (int v = 0; v < 3; ++v)
            for (int a = 0; a < 3; ++a)
                if (!std::isfinite(t.v[v][a])) { error = "A BVH cannot contain a non-finite triangle"; return false; }
    }
    if (triangles.empty()) return true;

    std::vector<Ref> refs(triangles.size());
    for (size_t i = 0; i < triangles.size(); ++i) {
        const HostTriangle& t = triangles[i];
        Ref& r = refs[i];
        r.index = uint32_t(i);
        r.id = t.primitive_id;
        for (int v = 0; v < 3; ++v) r.box.grow_point(t.v[v]);
        // Triangle::Centroid promotes to double (Geometry.hpp:160-176).
        for (int a = 0; a < 3; ++a)
            r.c[a] = float((double(t.v[0][a]) + double(t.v[1][a]) + double(t.v[2][a])) / 3.0);
    }
    Builder b{refs, bins, max_leaf_size, std::vector<Ref>(refs.size())};
    std::vector<Node> nodes;
    uint32_t max_depth = 0;
    try {
        int levels = 0;
        while ((1u << levels) < std::max(1u, threads)) ++levels;
        nodes = b.build_par(0, refs.size(), 1, levels, max_depth);
    } catch (const std::exception& e) {
        error = e.what();
        return false;
    }

    // Parents (SoftwareGpu.cpp:1010-1030 records them while validating).
    std::vector<uint32_t> parent(nodes.size(), kInvalid);
    for (uint32_t i = 0; i < nodes.size(); ++i) {
        if (nodes[i].count == 0) {
            parent[nodes[i].left] = i;
            parent[nodes[i].right] = i;
        }
    }
    out.nodes.resize(nodes.size());
    for (size_t i = 0; i < nodes.size(); ++i) {
        const Node& n = nodes[i];
        re_software_node& r = out.nodes[i];
        r.bounds_min = {n.box.lo[0], n.box.lo[1], n.box.lo[2], 0.0f};
        r.bounds_max = {n.box.hi[0], n.box.hi[1], n.box.hi[2], 0.0f};
        if (n.count != 0) {
            r.links = {n.first, n.count, kInvalid, parent[i]};
            ++out.leaf_count;
        } else {
            r.links = {n.left, 0u, n.right, parent[i]};
        }
    }
    out.leaf_order.resize(refs.size());
    for (size_t i = 0; i < refs.size(); ++i) out.leaf_order[i] = refs[i].index;
    out.max_depth = max_depth;
    return true;
}

void build_device_layout(const FlatBvh& flat, DeviceLayout& out) {
    out = DeviceLayout{};
    const auto& n = flat.nodes;
    if (n.empty()) return;
    // Interior nodes get device indices in pre-order.
    std::vector<uint32_t> dev(n.size(), kInvalid);
    uint32_t count = 0;
    for (size_t i = 0; i < n.size(); ++i)
        if (n[i].links.y == 0) dev[i] = count++;
    auto put_child = [&](DeviceNode& d, int side, uint32_t child) {
        const re_software_node& c = n[child];
        float* bx = side == 0 ? d.a : d.b + 2;
        (void)bx;
        if (side == 0) {
            d.a[0] = c.bounds_min.x; d.a[1] = c.bounds_max.x;
            d.a[2] = c.bounds_min.y; d.a[3] = c.bounds_max.y;
            d.b[0] = c.bounds_min.z; d.b[1] = c.bounds_max.z;
        } else {
            d.b[2] = c.bounds_min.x; d.b[3] = c.bounds_max.x;
            d.c[0] = c.bounds_min.y; d.c[1] = c.bounds_max.y;
            d.c[2] = c.bounds_min.z; d.c[3] = c.bounds_max.z;
        }
        if (c.links.y != 0) {
            d.d[side] = c.links.x;
            d.d[2 + side] = c.links.y;
        } else {
            d.d[side] = dev[child];
            d.d[2 + side] = 0;
        }
    };
    if (n[0].links.y != 0) {
        // Single-leaf tree: a synthetic root with the leaf on the left and an
        // empty box on the right.  The empty box is +inf on every bound: both
        // slab distances are +inf (or -inf) on each axis, so no ray enters it
        // (lo = +inf, hi = -inf would swap into an infinite interval).
        out.root_is_leaf = 1;
        DeviceNode d{};
        put_child(d, 0, 0);
        d.b[2] = INFINITY; d.b[3] = INFINITY;
        d.c[0] = INFINITY; d.c[1] = INFINITY; d.c[2] = INFINITY; d.c[3] = INFINITY;
        d.d[1] = 0; d.d[3] = 0;
        out.nodes.push_back(d);
        out.node_original = {0u, kInvalid};
        return;
    }
    out.nodes.resize(count);
    out.node_original.resize(size_t(count) * 2);
    for (size_t i = 0; i < n.size(); ++i) {
        if (n[i].links.y != 0) continue;
        DeviceNode& d = out.nodes[dev[i]];
        put_child(d, 0, n[i].links.x);
        put_child(d, 1, n[i].links.z);
        out.node_original[size_t(dev[i]) * 2 + 0] = n[i].links.x;
        out.node_original[size_t(dev[i]) * 2 + 1] = n[i].links.z;
    }
}

namespace {

float surface_area(const re_software_node& n) {
    const float dx = n.bounds_max.x - n.bounds_min.x, dy = n.bounds_max.y - n.bounds_min.y,
                dz = n.bounds_max.z - n.bounds_min.z;
    return dx * dy + dy * dz + dz * dx;
}

}  // namespace

void build_wide_layout(const FlatBvh& flat, WideLayout& out) {
    out = WideLayout{};
    const auto& n = flat.nodes;
    if (n.empty()) return;
    auto set_child = [&](WideNode& w, int c, uint32_t child) {
        const re_software_node& b = n[child];
        w.lo_x[c] = b.bounds_min.x; w.hi_x[c] = b.bounds_max.x;
        w.lo_y[c] = b.bounds_min.y; w.hi_y[c] = b.bounds_max.y;
        w.lo_z[c] = b.bounds_min.z; w.hi_z[c] = b.bounds_max.z;
    };
    auto clear = [](WideNode& w) {
        for (int c = 0; c < 4; ++c) {
            w.lo_x[c] = w.hi_x[c] = w.lo_y[c] = w.hi_y[c] = w.lo_z[c] = w.hi_z[c] = INFINITY;
            w.entry[c] = 0;
            w.count[c] = kWideEmpty;
        }
    };
    struct Item {
        uint32_t binary;  // binary interior node to collapse
        uint32_t wide;    // its wide node
        uint32_t depth;   // wide level (root 1)
        uint32_t stack;   // stack entries held by ancestors' pushed siblings
    };
    out.nodes.emplace_back();
    clear(out.nodes[0]);
    if (n[0].links.y != 0) {  // single leaf
        set_child(out.nodes[0], 0, 0);
        out.nodes[0].entry[0] = n[0].links.x | (n[0].links.y << kWideLeafShift);
        out.nodes[0].count[0] = n[0].links.y;
        out.max_depth = 1;
        out.stack_bound = 0;
        return;
    }
    std::vector<Item> todo{{0u, 0u, 1u, 0u}};
    while (!todo.empty()) {
        const Item it = todo.back();
        todo.pop_back();
        std::vector<uint32_t> kids{n[it.binary].links.x, n[it.binary].links.z};
        while (kids.size() < 4) {
            int pick = -1;
            float best = -1.0f;
            for (size_t k = 0; k < kids.size(); ++k) {
                if (n[kids[k]].links.y != 0) continue;
                const float a = surface_area(n[kids[k]]);
                if (a > best) {
                    best = a;
                    pick = int(k);
                }
            }
            if (pick < 0) break;
            const uint32_t open = kids[size_t(pick)];
            kids[size_t(pick)] = n[open].links.z;
            kids.insert(kids.begin() + pick, n[open].links.x);
        }
        // A traversal at this node pushes all but its nearest child.
        const uint32_t stack_here = it.stack + uint32_t(kids.size()) - 1u;
        out.max_depth = std::max(out.max_depth, it.depth);
        out.stack_bound = std::max(out.stack_bound, stack_here);
        std::vector<Item> next;
        for (size_t k = 0; k < kids.size(); ++k) {
            const uint32_t child = kids[k];
            set_child(out.nodes[it.wide], int(k), child);
            if (n[child].links.y != 0) {
                out.nodes[it.wide].entry[k] = n[child].links.x;
                out.nodes[it.wide].count[k] = n[child].links.y;
            } else {
                out.nodes[it.wide].count[k] = 0;
                next.push_back({child, 0u, it.depth + 1u, stack_here});
                next.back().wide = uint32_t(k);  // slot, resolved below
            }
        }
        // The interior children of a node get consecutive indices; they are
        // collapsed depth first, leftmost first.
        for (auto r = next.rbegin(); r != next.rend(); ++r) todo.push_back(*r);
        for (size_t j = todo.size() - next.size(); j < todo.size(); ++j) {
            Item& c = todo[j];
            const uint32_t slot = c.wide;
            const uint32_t idx = uint32_t(out.nodes.size());
            out.nodes.emplace_back();
            clear(out.nodes.back());
            out.nodes[it.wide].entry[slot] = idx;
            c.wide = idx;
        }
    }
    // Pack each child's leaf count above its reference (references stay
    // below 2^28: triangle counts are limited to that, wide nodes are fewer).
    for (WideNode& w : out.nodes)
        for (int c = 0; c < 4; ++c)
            w.entry[c] = w.count[c] == kWideEmpty ? kWideEmpty : (w.entry[c] | (w.count[c] << kWideLeafShift));
}

namespace {

// float(a + b) rounded toward -inf / +inf, as the device's __fadd_rd /
// __fadd_ru compute it: the sum of two floats is exact in double here (their
// exponents differ by far less than 29), then rounded once.
float add_down(float a, float b) {
    const double d = double(a) + double(b);
    float f = float(d);
    if (double(f) > d) f = std::nextafter(f, -INFINITY);
    return f;
}
float add_up(float a, float b) {
    const double d = double(a) + double(b);
    float f = float(d);
    if (double(f) < d) f = std::nextafter(f, INFINITY);
    return f;
}

// Quantises the children's boxes of one eight-wide node (see Wide8QNode).
void compress_wide8(const Wide8Node& w, Wide8QNode& q) {
    std::memset(&q, 0, sizeof(q));
    const float* lo[3] = {w.lo_x, w.lo_y, w.lo_z};
    const float* hi[3] = {w.hi_x, w.hi_y, w.hi_z};
    uint8_t* qlo[3] = {q.lo_x, q.lo_y, q.lo_z};
    uint8_t* qhi[3] = {q.hi_x, q.hi_y, q.hi_z};
    for (int c = 0; c < 8; ++c) q.entry[c] = w.entry[c];
    for (int a = 0; a < 3; ++a) {
        float org = INFINITY, top = -INFINITY;
        for (int c = 0; c < 8; ++c) {
            if (w.entry[c] == kWideEmpty) continue;
            org = std::min(org, lo[a][c]);
            top = std::max(top, hi[a][c]);
        }
        if (!(org <= top)) {  // no child at all: any origin, all slots inverted
            org = 0.0f;
            top = 0.0f;
        }
        // One float step of room below the lowest bound (q = 0 must decode
        // at least that far down).
        org = std::nextafter(std::nextafter(org, -INFINITY), -INFINITY);
        top = std::nextafter(std::nextafter(top, INFINITY), INFINITY);
        const double extent = double(top) - double(org);
        int e = extent > 0.0 ? int(std::ceil(std::log2(extent / 255.0))) : -126;
        e = std::max(e, -126);
        for (;; ++e) {
            const float scale = std::ldexp(1.0f, e);
            bool fits = true;
            for (int c = 0; c < 8 && fits; ++c) {
                if (w.entry[c] == kWideEmpty) {
                    qlo[a][c] = 255;
                    qhi[a][c] = 0;
                    continue;
                }
                // Largest lower bound whose decoded value stays below lo by
                // at least one float step, and the smallest upper bound whose
                // decoded value stays above hi by one (a margin for a sum the
                // double above could not hold exactly).
                const float lo_m = std::nextafter(lo[a][c], -INFINITY);
                const float hi_m = std::nextafter(hi[a][c], INFINITY);
                long ql = long(std::floor((double(lo_m) - double(org)) / double(scale)));
                ql = std::max(0L, std::min(255L, ql));
                while (ql > 0 && add_down(org, float(ql) * scale) > lo_m) --ql;
                long qh = long(std::ceil((double(hi_m) - double(org)) / double(scale)));
                qh = std::max(0L, qh);
                while (qh <= 255 && add_up(org, float(qh) * scale) < hi_m) ++qh;
                if (qh > 255 || add_down(org, float(ql) * scale) > lo_m) {
                    fits = false;
                    break;
                }
                qlo[a][c] = uint8_t(ql);
                qhi[a][c] = uint8_t(qh);
            }
            if (fits) break;
        }
        q.origin[a] = org;
        q.exponent[a] = uint8_t(e + 127);
    }
}

}  // namespace

void build_wide8_layout(const FlatBvh& flat, Wide8Layout& out) {
    out = Wide8Layout{};
    const auto& n = flat.nodes;
    if (n.empty()) return;
    auto clear = [](Wide8Node& w) {
        for (int c = 0; c < 8; ++c) {
            w.lo_x[c] = w.hi_x[c] = w.lo_y[c] = w.hi_y[c] = w.lo_z[c] = w.hi_z[c] = INFINITY;
            w.entry[c] = kWideEmpty;
            w.pad[c] = 0u;
        }
    };
    auto set_child = [&](Wide8Node& w, int c, uint32_t child) {
        const re_software_node& b = n[child];
        w.lo_x[c] = b.bounds_min.x; w.hi_x[c] = b.bounds_max.x;
        w.lo_y[c] = b.bounds_min.y; w.hi_y[c] = b.bounds_max.y;
        w.lo_z[c] = b.bounds_min.z; w.hi_z[c] = b.bounds_max.z;
    };
    out.nodes.emplace_back();
    clear(out.nodes[0]);
    if (n[0].links.y != 0) {  // single leaf
        set_child(out.nodes[0], 0, 0);
        out.nodes[0].entry[0] = n[0].links.x | (n[0].links.y << kWideLeafShift);
        out.max_depth = 1;
    } else {
        struct Item {
            uint32_t binary, wide, depth, stack;
        };
        std::vector<Item> todo{{0u, 0u, 1u, 0u}};
        while (!todo.empty()) {
            const Item it = todo.back();
            todo.pop_back();
            std::vector<uint32_t> kids{n[it.binary].links.x, n[it.binary].links.z};
            while (kids.size() < 8) {
                int pick = -1;
                float best = -1.0f;
                for (size_t k = 0; k < kids.size(); ++k) {
                    if (n[kids[k]].links.y != 0) continue;
                    const float a = surface_area(n[kids[k]]);
                    if (a > best) {
                        best = a;
                        pick = int(k);
                    }
                }
                if (pick < 0) break;
                const uint32_t open = kids[size_t(pick)];
                kids[size_t(pick)] = n[open].links.z;
                kids.insert(kids.begin() + pick, n[open].links.x);
            }
            const uint32_t stack_here = it.stack + uint32_t(kids.size()) - 1u;
            out.max_depth = std::max(out.max_depth, it.depth);
            out.stack_bound = std::max(out.stack_bound, stack_here);
            std::vector<std::pair<uint32_t, uint32_t>> interior;  // (slot, binary child)
            for (size_t k = 0; k < kids.size(); ++k) {
                const uint32_t child = kids[k];
                set_child(out.nodes[it.wide], int(k), child);
                if (n[child].links.y != 0)
                    out.nodes[it.wide].entry[k] = n[child].links.x | (n[child].links.y << kWideLeafShift);
                else
                    interior.emplace_back(uint32_t(k), child);
            }
            // Interior children get consecutive indices, collapsed depth
            // first, leftmost first.
            std::vector<Item> next;
            for (const auto& sc : interior) {
                const uint32_t idx = uint32_t(out.nodes.size());
                out.nodes.emplace_back();
                clear(out.nodes.back());
                out.nodes[it.wide].entry[sc.first] = idx;
                next.push_back({sc.second, idx, it.depth + 1u, stack_here});
            }
            for (auto r = next.rbegin(); r != next.rend(); ++r) todo.push_back(*r);
        }
    }
    out.qnodes.resize(out.nodes.size());
    for (size_t i = 0; i < out.nodes.size(); ++i) compress_wide8(out.nodes[i], out.qnodes[i]);
}

}  // namespace re
