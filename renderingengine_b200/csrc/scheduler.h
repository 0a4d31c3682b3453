// Host-side bookkeeping of the render server: the path-pool range allocator,
// the launch planner and the least-recently-used residency set of scenes.
// Plain C++ with no CUDA dependency (the CPU tests compile it on its own).
#pragma once

#include <algorithm>
#include <cstdint>
#include <iterator>
#include <limits>
#include <map>
#include <unordered_map>
#include <vector>

namespace re {

// First-fit allocator of contiguous path ranges in [0, capacity); freed
// ranges merge with their neighbours.
class PathAllocator {
public:
    explicit PathAllocator(uint32_t capacity = 0) { reset(capacity); }

    void reset(uint32_t capacity) {
        capacity_ = capacity;
        free_.clear();
        if (capacity > 0) free_[0] = capacity;
        used_ = 0;
    }

    bool allocate(uint32_t size, uint32_t& offset) {
        if (size == 0) return false;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < size) continue;
            offset = it->first;
            const uint32_t rest = it->second - size;
            free_.erase(it);
            if (rest > 0) free_[offset + size] = rest;
            used_ += size;
            return true;
        }
        return false;
    }

    void release(uint32_t offset, uint32_t size) {
        if (size == 0) return;
        used_ -= size;
        auto next = free_.lower_bound(offset);
        uint32_t start = offset, len = size;
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == offset) {
                start = prev->first;
                len += prev->second;
                free_.erase(prev);
            }
        }
        if (next != free_.end() && offset + size == next->first) {
            len += next->second;
            free_.erase(next);
        }
        free_[start] = len;
    }

    uint32_t largest_free() const {
        uint32_t m = 0;
        for (const auto& f : free_) m = f.second > m ? f.second : m;
        return m;
    }
    uint32_t used() const { return used_; }
    uint32_t capacity() const { return capacity_; }
    size_t fragments() const { return free_.size(); }

private:
    uint32_t capacity_ = 0, used_ = 0;
    std::map<uint32_t, uint32_t> free_;  // offset -> size
};

// Launch plan of one batch step.  The views of each scene are cut, in their
// given order, into chunks of at most `launch_paths` paths (a view larger
// than that is a chunk of its own); chunks are then placed first-fit into
// launches of at most `launch_paths` paths.  So a large scene fills
// launches of its own (its hierarchy stays hot in L2 through the launch)
// while small scenes share one, and a step takes few launches.  Scenes keep
// the order of their first view.  Returns the launch index of every view;
// `launches` gets the count.
inline std::vector<uint32_t> plan_launches(const uint32_t* slots, const uint32_t* pixels, size_t n,
                                           uint32_t launch_paths, uint32_t& launches) {
    std::vector<uint32_t> launch_of(n, 0);
    std::vector<uint32_t> scene_order;
    std::unordered_map<uint32_t, std::vector<size_t>> by_scene;
    for (size_t i = 0; i < n; ++i) {
        auto it = by_scene.find(slots[i]);
        if (it == by_scene.end()) {
            scene_order.push_back(slots[i]);
            it = by_scene.emplace(slots[i], std::vector<size_t>{}).first;
        }
        it->second.push_back(i);
    }
    std::vector<uint64_t> fill;  // paths per launch
    std::vector<size_t> chunk;
    uint64_t chunk_paths = 0;
    auto place = [&]() {
        if (chunk.empty()) return;
        size_t l = 0;
        while (l < fill.size() && fill[l] + chunk_paths > launch_paths) ++l;
        if (l == fill.size()) fill.push_back(0);
        fill[l] += chunk_paths;
        for (size_t i : chunk) launch_of[i] = uint32_t(l);
        chunk.clear();
        chunk_paths = 0;
    };
    for (uint32_t s : scene_order) {
        for (size_t i : by_scene[s]) {
            if (!chunk.empty() && chunk_paths + pixels[i] > launch_paths) place();
            chunk.push_back(i);
            chunk_paths += pixels[i];
        }
        place();
    }
    launches = uint32_t(fill.size());
    return launch_of;
}

// Residency set with least-recently-used eviction.  Pinned entries (in use
// by admitted requests) are never chosen as victims.
class LruResidency {
public:
    struct Entry {
        uint64_t bytes = 0;
        uint64_t last_use = 0;
        uint32_t pins = 0;
    };

    bool resident(uint64_t key) const { return entries_.count(key) != 0; }
    uint64_t bytes() const { return bytes_; }
    size_t size() const { return entries_.size(); }

    void insert(uint64_t key, uint64_t bytes, uint64_t stamp) {
        Entry& e = entries_[key];
        bytes_ += bytes - e.bytes;
        e.bytes = bytes;
        e.last_use = stamp;
    }
    void touch(uint64_t key, uint64_t stamp) {
        auto it = entries_.find(key);
        if (it != entries_.end()) it->second.last_use = stamp;
    }
    void pin(uint64_t key) { entries_.at(key).pins += 1; }
    void unpin(uint64_t key) {
        auto it = entries_.find(key);
        if (it != entries_.end() && it->second.pins > 0) it->second.pins -= 1;
    }
    uint32_t pins(uint64_t key) const {
        auto it = entries_.find(key);
        return it == entries_.end() ? 0u : it->second.pins;
    }
    void erase(uint64_t key) {
        auto it = entries_.find(key);
        if (it == entries_.end()) return;
        bytes_ -= it->second.bytes;
        entries_.erase(it);
    }

    // Unpinned entries, least recently used first, whose removal brings the
    // total to at most `target` bytes; empty when that is impossible.
    std::vector<uint64_t> victims(uint64_t target) const {
        std::vector<std::pair<uint64_t, uint64_t>> cand;  // (last_use, key)
        for (const auto& kv : entries_)
            if (kv.second.pins == 0) cand.emplace_back(kv.second.last_use, kv.first);
        std::sort(cand.begin(), cand.end());
        std::vector<uint64_t> out;
        uint64_t total = bytes_;
        for (const auto& c : cand) {
            if (total <= target) break;
            out.push_back(c.second);
            total -= entries_.at(c.second).bytes;
        }
        if (total > target) out.clear();
        return out;
    }

private:
    std::unordered_map<uint64_t, Entry> entries_;
    uint64_t bytes_ = 0;
};

}  // namespace re
