// Test harness: exposes the render server's host bookkeeping
// (renderingengine_b200/csrc/scheduler.h) to the CPU tests through a few
// extern "C" calls.  Compiled by tests/test_scheduler.py with g++.
#include <cstdint>
#include <vector>

#include "scheduler.h"

extern "C" {

void* alloc_create(uint32_t capacity) { return new re::PathAllocator(capacity); }
void alloc_destroy(void* a) { delete static_cast<re::PathAllocator*>(a); }
int alloc_take(void* a, uint32_t size, uint32_t* offset) {
    return static_cast<re::PathAllocator*>(a)->allocate(size, *offset) ? 1 : 0;
}
void alloc_give(void* a, uint32_t offset, uint32_t size) { static_cast<re::PathAllocator*>(a)->release(offset, size); }
uint32_t alloc_used(void* a) { return static_cast<re::PathAllocator*>(a)->used(); }
uint32_t alloc_largest(void* a) { return static_cast<re::PathAllocator*>(a)->largest_free(); }
uint64_t alloc_fragments(void* a) { return static_cast<re::PathAllocator*>(a)->fragments(); }

void* lru_create() { return new re::LruResidency(); }
void lru_destroy(void* l) { delete static_cast<re::LruResidency*>(l); }
void lru_insert(void* l, uint64_t key, uint64_t bytes, uint64_t stamp) {
    static_cast<re::LruResidency*>(l)->insert(key, bytes, stamp);
}
void lru_touch(void* l, uint64_t key, uint64_t stamp) { static_cast<re::LruResidency*>(l)->touch(key, stamp); }
void lru_pin(void* l, uint64_t key) { static_cast<re::LruResidency*>(l)->pin(key); }
void lru_unpin(void* l, uint64_t key) { static_cast<re::LruResidency*>(l)->unpin(key); }
void lru_erase(void* l, uint64_t key) { static_cast<re::LruResidency*>(l)->erase(key); }
uint64_t lru_bytes(void* l) { return static_cast<re::LruResidency*>(l)->bytes(); }
// Writes up to `cap` victim keys; returns their count.
uint32_t lru_victims(void* l, uint64_t target, uint64_t* out, uint32_t cap) {
    const std::vector<uint64_t> v = static_cast<re::LruResidency*>(l)->victims(target);
    uint32_t n = 0;
    for (uint64_t k : v)
        if (n < cap) out[n++] = k;
    return n;
}

}  // extern "C"
