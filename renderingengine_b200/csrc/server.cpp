// Render server: continuous batching of render requests over one batched
// wavefront renderer.  The reference renders one request per
// Wave2Runtime::RecordFrame; here every step renders one sample of every
// admitted request in a single launch (re_renderer_render_views), requests
// join as soon as a path range and HBM budget are free, scenes are made
// resident on demand (GPU LBVH) and evicted least-recently-used.
//
// Timing: completion times come from CUDA events recorded after each
// request's result copy, placed on the host clock through a base event
// synchronised at creation; latency = completion - arrival.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <thread>
#include <unordered_map>
#include <vector>

#include "runtime.h"
#include "scheduler.h"

static_assert(sizeof(re_restir_config) == 44, "re_restir_config is 11 words");
static_assert(sizeof(re_server_desc) == 88, "re_server_desc layout");

using namespace re;

namespace {

struct SceneRecord {
    std::vector<re_canonical_triangle> tris;
    std::vector<re_material> materials;
    std::vector<re_light> lights;
    std::vector<re_float4> fixtures;
    uint32_t light_selection = 0;
    float radius = 1.0f;
    re_scene* scene = nullptr;  // resident build, or null
    int slot = -1;
    uint64_t bytes = 0;
};

struct Request {
    uint64_t id = 0, scene_key = 0;
    re_frame_constants frame{};
    uint32_t spp = 0, samples_done = 0, state = RE_REQUEST_WAITING, error = RE_SUCCESS;
    uint32_t offset = 0, pixels = 0;
    double arrival = 0.0, admitted = 0.0, completed = 0.0;
    uint32_t bypassed = 0;  // later requests admitted ahead of this one while it waited
    cudaEvent_t done = nullptr;
    void* result = nullptr;  // pinned, pixels x re_float4
    size_t result_bytes = 0;
};

// Device bytes a resident scene takes: BVH nodes, triangles and attributes
// (re_scene_info.device_bytes) plus the renderer's per-slot tables.
uint64_t scene_bytes(const SceneRecord& rec, const re_scene_info& info) {
    return info.device_bytes + uint64_t(rec.tris.size()) * 4u + rec.materials.size() * sizeof(re_material) +
           rec.lights.size() * (sizeof(re_light) + 24u) + rec.fixtures.size() * sizeof(re_float4);
}

// Charge of a scene before it is built: an upper bound of scene_bytes (a
// binary hierarchy has at most two nodes per triangle) plus 1 MiB for the
// builder's transient scratch.
uint64_t scene_charge(const SceneRecord& rec) {
    const uint64_t n = rec.tris.size();
    return n * (2u * sizeof(re::DeviceNode) + sizeof(re::DeviceTriangle) + sizeof(re::DeviceAttr) + 4u) +
           rec.materials.size() * sizeof(re_material) + rec.lights.size() * (sizeof(re_light) + 24u) +
           rec.fixtures.size() * sizeof(re_float4) + (1u << 20);
}

}  // namespace

struct re_server {
    re_server_desc desc{};
    re_renderer* renderer = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t base = nullptr;
    std::chrono::steady_clock::time_point t0;
    double base_host = 0.0;  // host clock of the base event
    std::unordered_map<uint64_t, SceneRecord> scenes;
    LruResidency lru;
    PathAllocator paths;
    bool slot_used[RE_MAX_SCENE_SLOTS] = {};
    std::unordered_map<uint64_t, Request> requests;
    std::multimap<double, uint64_t> future;  // arrival -> request
    std::deque<uint64_t> arrived;            // FIFO of arrived, not admitted
    std::vector<uint64_t> active, finishing;
    uint64_t next_id = 1, stamp = 0;
    uint64_t fixed_bytes = 0;
    std::unordered_map<size_t, std::vector<void*>> pinned_free;
    std::vector<double> latencies;
    re_server_stats stats{};

    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    ~re_server() {
        if (stream) cudaStreamSynchronize(stream);
        for (auto& kv : requests) {
            if (kv.second.done) cudaEventDestroy(kv.second.done);
            if (kv.second.result) cudaFreeHost(kv.second.result);
        }
        for (auto& kv : pinned_free)
            for (void* p : kv.second) cudaFreeHost(p);
        if (renderer) re_renderer_destroy(renderer);
        for (auto& kv : scenes)
            if (kv.second.scene) re_scene_destroy(kv.second.scene);
        if (base) cudaEventDestroy(base);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

void* pinned_get(re_server* s, size_t bytes) {
    auto& v = s->pinned_free[bytes];
    if (!v.empty()) {
        void* p = v.back();
        v.pop_back();
        return p;
    }
    void* p = nullptr;
    if (cudaMallocHost(&p, bytes) != cudaSuccess) return nullptr;
    return p;
}

void pinned_put(re_server* s, void* p, size_t bytes) {
    if (p != nullptr) s->pinned_free[bytes].push_back(p);
}

void evict(re_server* s, uint64_t key) {
    SceneRecord& rec = s->scenes.at(key);
    if (rec.slot >= 0) {
        re_renderer_unbind_scene(s->renderer, uint32_t(rec.slot));
        s->slot_used[rec.slot] = false;
    }
    if (rec.scene) re_scene_destroy(rec.scene);
    rec.scene = nullptr;
    rec.slot = -1;
    s->lru.erase(key);
    ++s->stats.evictions;
}

// Makes a registered scene resident (build + bind), evicting least recently
// used unpinned scenes for budget and slots (unless `may_evict` is false).
// RE_BUDGET_EXCEEDED when it cannot fit now.
re_status make_resident(re_server* s, uint64_t key, bool may_evict = true) {
    SceneRecord& rec = s->scenes.at(key);
    if (rec.scene != nullptr) return RE_SUCCESS;
    const uint64_t estimate = scene_charge(rec);
    const uint64_t budget = s->desc.hbm_budget_bytes;
    if (s->fixed_bytes + estimate > budget)
        return set_error(RE_BUDGET_EXCEEDED, "scene does not fit the HBM budget");
    if (s->fixed_bytes + s->lru.bytes() + estimate > budget) {
        if (!may_evict) return set_error(RE_BUDGET_EXCEEDED, "scene does not fit beside the resident ones");
        const auto vict = s->lru.victims(budget - s->fixed_bytes - estimate);
        if (vict.empty()) return set_error(RE_BUDGET_EXCEEDED, "no evictable scene frees enough of the budget");
        for (uint64_t v : vict) evict(s, v);
    }
    int slot = -1;
    for (int k = 0; k < int(RE_MAX_SCENE_SLOTS); ++k)
        if (!s->slot_used[k]) {
            slot = k;
            break;
        }
    if (slot < 0) {
        if (!may_evict) return set_error(RE_BUDGET_EXCEEDED, "every scene slot is in use");
        const auto vict = s->lru.victims(s->lru.bytes() > 0 ? s->lru.bytes() - 1 : 0);
        if (vict.empty()) return set_error(RE_BUDGET_EXCEEDED, "every scene slot is in use");
        evict(s, vict.front());
        for (int k = 0; k < int(RE_MAX_SCENE_SLOTS); ++k)
            if (!s->slot_used[k]) {
                slot = k;
                break;
            }
    }
    re_scene_desc d{};
    d.triangles = rec.tris.data();
    d.triangle_count = uint32_t(rec.tris.size());
    d.build_kind = s->desc.build_kind;
    d.sah_bins = 16;
    d.max_leaf_size = 4;
    d.fingerprint = key + 1u;
    d.generation = 1;
    d.device = s->desc.device;
    re_status st = re_scene_create(&d, &rec.scene);
    if (st != RE_SUCCESS) return st;
    st = re_renderer_bind_scene(s->renderer, uint32_t(slot), rec.scene, rec.materials.data(),
                                uint32_t(rec.materials.size()), rec.lights.empty() ? nullptr : rec.lights.data(),
                                uint32_t(rec.lights.size()), rec.fixtures.empty() ? nullptr : rec.fixtures.data(),
                                uint32_t(rec.fixtures.size() / 4), rec.light_selection, rec.radius);
    if (st != RE_SUCCESS) {
        re_scene_destroy(rec.scene);
        rec.scene = nullptr;
        return st;
    }
    re_scene_info info{};
    re_scene_info_get(rec.scene, &info);
    rec.bytes = scene_bytes(rec, info);
    rec.slot = slot;
    s->slot_used[slot] = true;
    s->lru.insert(key, rec.bytes, ++s->stamp);
    ++s->stats.scene_builds;
    return RE_SUCCESS;
}

void fail(re_server* s, Request& q, re_status code) {
    q.state = RE_REQUEST_FAILED;
    q.error = uint32_t(code);
    ++s->stats.failed;
}

// Completion events that have fired: latency bookkeeping.
void retire_finished(re_server* s, bool wait_first) {
    for (size_t i = 0; i < s->finishing.size();) {
        Request& q = s->requests.at(s->finishing[i]);
        cudaError_t e = (wait_first && i == 0) ? cudaEventSynchronize(q.done) : cudaEventQuery(q.done);
        if (e == cudaErrorNotReady) {
            ++i;
            continue;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, s->base, q.done);
        q.completed = s->base_host + double(ms) * 1e-3;
        q.state = RE_REQUEST_DONE;
        s->latencies.push_back(q.completed - q.arrival);
        s->stats.last_completion = std::max(s->stats.last_completion, q.completed);
        ++s->stats.completed;
        s->stats.samples += uint64_t(q.pixels) * q.spp;
        s->lru.unpin(q.scene_key);
        s->finishing.erase(s->finishing.begin() + long(i));
        wait_first = false;
    }
}

void admit(re_server* s, double now) {
    while (!s->future.empty() && s->future.begin()->first <= now) {
        s->arrived.push_back(s->future.begin()->second);
        s->future.erase(s->future.begin());
    }
    // Arrival order, with bounded backfilling: a request that cannot start
    // yet (its scene does not fit beside the running requests' scenes, or
    // no path range of its size is free) holds back the ones behind it,
    // except that a later request that fits now -- without evicting a scene
    // -- may start ahead of it, at most backfill_window times per waiting
    // request (so none waits behind an unbounded stream of small ones).
    auto it = s->arrived.begin();
    while (it != s->arrived.end() && s->active.size() < s->desc.max_batch_views) {
        const bool head = it == s->arrived.begin();
        Request& q = s->requests.at(*it);
        const bool alone = s->active.empty() && s->finishing.empty();
        bool started = false;
        re_status st = make_resident(s, q.scene_key, head);
        if (st != RE_SUCCESS && head && alone) {  // nothing will ever free budget for it
            fail(s, q, st);
            it = s->arrived.erase(it);
            continue;
        }
        if (st == RE_SUCCESS) {
            uint32_t off = 0;
            if (s->paths.allocate(q.pixels, off)) {
                q.offset = off;
                q.admitted = now;
                q.state = RE_REQUEST_RUNNING;
                s->lru.pin(q.scene_key);
                s->lru.touch(q.scene_key, ++s->stamp);
                s->active.push_back(q.id);
                started = true;
            } else if (head && alone && q.pixels > s->paths.capacity()) {
                fail(s, q, RE_BUDGET_EXCEEDED);
                it = s->arrived.erase(it);
                continue;
            }
        }
        if (started) {
            if (!head) {
                ++s->requests.at(s->arrived.front()).bypassed;
                ++s->stats.backfilled;
            }
            it = s->arrived.erase(it);
            continue;
        }
        const Request& first = s->requests.at(s->arrived.front());
        if (first.bypassed >= s->desc.backfill_window) break;
        ++it;
    }
}

// One step: one sample of every active request, in the launches of
// plan_launches (requests grouped by scene, under the path budget).
re_status step(re_server* s) {
    const size_t n = s->active.size();
    std::vector<re_view_desc> views(n);
    std::vector<re_frame_constants> frames(n);
    std::vector<uint32_t> slots(n), pixels(n);
    for (size_t k = 0; k < n; ++k) {
        Request& q = s->requests.at(s->active[k]);
        frames[k] = q.frame;
        frames[k].image.z = q.frame.image.z + q.samples_done;
        re_view_desc& v = views[k];
        v.frame = &frames[k];
        v.scene_slot = uint32_t(s->scenes.at(q.scene_key).slot);
        v.path_offset = q.offset;
        v.accumulate = q.samples_done > 0 ? 1u : 0u;
        v.view_key = q.id;
        slots[k] = v.scene_slot;
        pixels[k] = q.pixels;
    }
    uint32_t launches = 0;
    const std::vector<uint32_t> plan = plan_launches(slots.data(), pixels.data(), n, s->desc.launch_paths, launches);
    std::vector<re_view_desc> group;
    re_status st = RE_SUCCESS;
    for (uint32_t l = 0; l < launches; ++l) {
        group.clear();
        for (size_t k = 0; k < n; ++k)
            if (plan[k] == l) group.push_back(views[k]);
        st = re_renderer_render_views(s->renderer, group.data(), uint32_t(group.size()), s->stream);
        if (st != RE_SUCCESS) return st;
        ++s->stats.launches;
    }
    std::vector<uint64_t> still;
    for (uint64_t id : s->active) {
        Request& q = s->requests.at(id);
        if (++q.samples_done < q.spp) {
            still.push_back(id);
            continue;
        }
        // Result copy on the launch stream; the path range is reusable by the
        // next launch, which is stream-ordered after the copy.
        q.result_bytes = size_t(q.pixels) * sizeof(re_float4);
        q.result = pinned_get(s, q.result_bytes);
        if (q.result == nullptr) return set_error(RE_OUT_OF_MEMORY, "pinned result buffer allocation failed");
        st = renderer_copy_mean_async(s->renderer, q.offset, q.pixels, q.result, s->stream);
        if (st != RE_SUCCESS) return st;
        if (q.done == nullptr) RE_CUDA_TRY(cudaEventCreate(&q.done));
        RE_CUDA_TRY(cudaEventRecord(q.done, s->stream));
        s->paths.release(q.offset, q.pixels);
        re_renderer_release_view(s->renderer, q.id);
        s->finishing.push_back(id);
    }
    s->active.swap(still);
    return RE_SUCCESS;
}

}  // namespace

extern "C" {

RE_API re_status re_plan_launches(const uint32_t* scene_slots, const uint32_t* pixel_counts, uint32_t view_count,
                                  uint32_t launch_paths, uint32_t* launch_of_view, uint32_t* launch_count) {
    if (launch_count == nullptr || (view_count > 0 && (scene_slots == nullptr || pixel_counts == nullptr ||
                                                       launch_of_view == nullptr)))
        return set_error(RE_INVALID_ARGUMENT, "null argument");
    if (launch_paths == 0) return set_error(RE_INVALID_ARGUMENT, "launch path budget must be positive");
    uint32_t launches = 0;
    const std::vector<uint32_t> plan = plan_launches(scene_slots, pixel_counts, view_count, launch_paths, launches);
    std::copy(plan.begin(), plan.end(), launch_of_view);
    *launch_count = launches;
    return clear_error();
}

RE_API re_status re_server_create(const re_server_desc* desc, re_server** out) {
    if (desc == nullptr || out == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (desc->path_capacity == 0 || desc->max_batch_views == 0 || desc->max_batch_views > RE_MAX_BATCH_VIEWS ||
        (desc->build_kind != RE_BUILD_LBVH && desc->build_kind != RE_BUILD_FLATTENED_SAH))
        return set_error(RE_INVALID_ARGUMENT, "invalid server description");
    RE_CUDA_TRY(cudaSetDevice(int(desc->device)));
    auto s = new re_server();
    s->desc = *desc;
    if (s->desc.launch_paths == 0) s->desc.launch_paths = 16u << 20;
    if (s->desc.backfill_window == RE_BACKFILL_DEFAULT) s->desc.backfill_window = 64u;
    re_renderer_desc rd{16384u, (desc->path_capacity + 16383u) / 16384u, desc->max_depth, desc->device};
    re_status st = re_renderer_create(&rd, &s->renderer);
    if (st == RE_SUCCESS && desc->restir) {
        st = re_renderer_set_restir(s->renderer, &desc->restir_config);
        if (st == RE_SUCCESS) st = renderer_reserve_restir(s->renderer);
    }
    if (st != RE_SUCCESS) {
        delete s;
        return st;
    }
    uint32_t cap = 0;
    re_renderer_path_capacity(s->renderer, &cap);
    s->paths.reset(cap);
    s->fixed_bytes = renderer_device_bytes(s->renderer);
    if (s->fixed_bytes > desc->hbm_budget_bytes) {
        delete s;
        return set_error(RE_BUDGET_EXCEEDED, "the path pool alone exceeds the HBM budget");
    }
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&s->base) != cudaSuccess) {
        delete s;
        return set_error(RE_CUDA_ERROR, "stream / event creation failed");
    }
    s->t0 = std::chrono::steady_clock::now();
    cudaEventRecord(s->base, s->stream);
    cudaEventSynchronize(s->base);
    s->base_host = s->now();
    s->stats.budget_bytes = desc->hbm_budget_bytes;
    s->stats.first_arrival = -1.0;
    *out = s;
    return clear_error();
}

RE_API re_status re_server_destroy(re_server* s) {
    if (s != nullptr) cudaSetDevice(int(s->desc.device));
    delete s;
    return clear_error();
}

RE_API double re_server_clock(const re_server* s) { return s == nullptr ? 0.0 : s->now(); }

RE_API re_status re_server_register_scene(re_server* s, uint64_t key, const re_canonical_triangle* triangles,
                                          uint32_t triangle_count, const re_material* materials,
                                          uint32_t material_count, const re_light* lights, uint32_t light_count,
                                          const re_float4* fixtures, uint32_t fixture_count,
                                          uint32_t light_selection, float scene_radius) {
    if (s == nullptr || triangles == nullptr || triangle_count == 0 || materials == nullptr || material_count == 0)
        return set_error(RE_INVALID_ARGUMENT, "null argument or empty scene");
    if (s->scenes.count(key)) return set_error(RE_INVALID_ARGUMENT, "scene key already registered");
    SceneRecord rec;
    rec.tris.assign(triangles, triangles + triangle_count);
    rec.materials.assign(materials, materials + material_count);
    if (light_count) rec.lights.assign(lights, lights + light_count);
    if (fixture_count) rec.fixtures.assign(fixtures, fixtures + size_t(fixture_count) * 4);
    rec.light_selection = light_selection;
    rec.radius = scene_radius;
    s->scenes.emplace(key, std::move(rec));
    return clear_error();
}

RE_API re_status re_server_submit(re_server* s, const re_render_request* req, uint64_t* id) {
    if (s == nullptr || req == nullptr || id == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    if (!s->scenes.count(req->scene_key)) return set_error(RE_MISSING_SCENE, "unknown scene key");
    if (req->spp == 0) return set_error(RE_INVALID_ARGUMENT, "a request needs at least one sample");
    const uint64_t pixels = uint64_t(req->frame.image.x) * req->frame.image.y;
    if (pixels == 0 || pixels > s->paths.capacity())
        return set_error(RE_INVALID_ARGUMENT, "request extent exceeds the server's path capacity");
    if (req->frame.image.w > s->desc.max_depth) return set_error(RE_INVALID_ARGUMENT, "request depth too large");
    if (req->frame.sampling.w == RE_ESTIMATOR_RESTIR_PRIMARY && !s->desc.restir)
        return set_error(RE_UNSUPPORTED, "the server was created without ReSTIR state");
    Request q;
    q.id = s->next_id++;
    q.scene_key = req->scene_key;
    q.frame = req->frame;
    q.spp = req->spp;
    q.pixels = uint32_t(pixels);
    q.arrival = std::max(req->arrival_time, s->now());
    if (req->arrival_time > 0.0 && req->arrival_time > s->now()) q.arrival = req->arrival_time;
    s->future.emplace(q.arrival, q.id);
    if (s->stats.first_arrival < 0.0 || q.arrival < s->stats.first_arrival) s->stats.first_arrival = q.arrival;
    *id = q.id;
    s->requests.emplace(q.id, q);
    ++s->stats.submitted;
    return clear_error();
}

RE_API re_status re_server_pump(re_server* s, uint32_t max_steps, double max_wait, uint32_t* steps_out) {
    if (s == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    RE_CUDA_TRY(cudaSetDevice(int(s->desc.device)));
    uint32_t steps = 0;
    const double start = s->now();
    while (steps < max_steps) {
        retire_finished(s, false);
        admit(s, s->now());
        if (s->active.empty()) {
            if (!s->finishing.empty()) {
                retire_finished(s, true);
                continue;
            }
            if (s->future.empty() && s->arrived.empty()) break;
            if (!s->arrived.empty()) continue;  // admission failed a request; try the next
            const double next = s->future.begin()->first, now = s->now();
            if (next - start > max_wait) break;
            if (next > now) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(next - now, 0.05)));
            continue;
        }
        const re_status st = step(s);
        if (st != RE_SUCCESS) return st;
        ++steps;
    }
    if (steps_out) *steps_out = steps;
    return clear_error();
}

RE_API re_status re_server_drain(re_server* s) {
    if (s == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    while (!s->future.empty() || !s->arrived.empty() || !s->active.empty() || !s->finishing.empty()) {
        uint32_t steps = 0;
        const re_status st = re_server_pump(s, 1u << 30, 1.0e9, &steps);
        if (st != RE_SUCCESS) return st;
        if (steps == 0 && s->active.empty() && s->finishing.empty() && s->future.empty() && !s->arrived.empty())
            break;
    }
    RE_CUDA_TRY(cudaStreamSynchronize(s->stream));
    retire_finished(s, false);
    return clear_error();
}

RE_API re_status re_server_poll(re_server* s, uint64_t id, re_request_status* out) {
    if (s == nullptr || out == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    auto it = s->requests.find(id);
    if (it == s->requests.end()) return set_error(RE_INVALID_ARGUMENT, "unknown request");
    retire_finished(s, false);
    const Request& q = it->second;
    *out = re_request_status{q.state, q.samples_done, q.error, 0u, q.arrival, q.admitted, q.completed};
    return clear_error();
}

RE_API re_status re_server_read_result(re_server* s, uint64_t id, re_float4* out, uint32_t pixel_count) {
    if (s == nullptr || out == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    auto it = s->requests.find(id);
    if (it == s->requests.end()) return set_error(RE_INVALID_ARGUMENT, "unknown request");
    Request& q = it->second;
    if (q.state == RE_REQUEST_FAILED) return set_error(re_status(q.error), "request failed");
    if (q.state != RE_REQUEST_DONE) {
        if (q.done == nullptr) return set_error(RE_NOT_READY, "request still in flight");
        RE_CUDA_TRY(cudaEventSynchronize(q.done));
        retire_finished(s, false);
    }
    if (pixel_count < q.pixels) return set_error(RE_INVALID_ARGUMENT, "output smaller than the request's film");
    std::memcpy(out, q.result, q.result_bytes);
    return clear_error();
}

RE_API re_status re_server_release(re_server* s, uint64_t id) {
    if (s == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    auto it = s->requests.find(id);
    if (it == s->requests.end()) return set_error(RE_INVALID_ARGUMENT, "unknown request");
    Request& q = it->second;
    if (q.state != RE_REQUEST_DONE && q.state != RE_REQUEST_FAILED)
        return set_error(RE_NOT_READY, "request still in flight");
    pinned_put(s, q.result, q.result_bytes);
    if (q.done) cudaEventDestroy(q.done);
    s->requests.erase(it);
    return clear_error();
}

RE_API re_status re_server_stats_get(re_server* s, re_server_stats* out) {
    if (s == nullptr || out == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    RE_CUDA_TRY(cudaStreamSynchronize(s->stream));
    retire_finished(s, false);
    re_server_stats st = s->stats;
    renderer_ray_totals(s->renderer, &st.path_rays, &st.shadow_rays);
    st.resident_bytes = s->fixed_bytes + s->lru.bytes();
    if (!s->latencies.empty()) {
        std::vector<double> v = s->latencies;
        std::sort(v.begin(), v.end());
        auto pct = [&](double p) {
            const double idx = p * double(v.size() - 1);
            const size_t lo = size_t(std::floor(idx)), hi = std::min(lo + 1, v.size() - 1);
            return v[lo] + (v[hi] - v[lo]) * (idx - double(lo));
        };
        st.latency_p50 = pct(0.5);
        st.latency_p99 = pct(0.99);
        double sum = 0.0;
        for (double x : v) sum += x;
        st.latency_mean = sum / double(v.size());
    }
    *out = st;
    return clear_error();
}

}  // extern "C"
