// Host-side bookkeeping of the render server: the path-pool range allocator
// and the least-recently-used residency set of scenes.  Plain C++ with no
// CUDA dependency (the CPU tests compile it on its own).
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
