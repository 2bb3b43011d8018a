// pdm1_pool.cu -- the plans' caching allocator.
//
// A plan holds ~20 device buffers (state, stage states, box ping-pong, tables,
// maps) and two small pinned host blocks.  cudaMalloc/cudaFree of hundreds of
// MB cost tens of ms per plan and cudaFree synchronises the device, which
// dominates a call that creates, marches and destroys a plan (energy_march,
// every wave of a field).  Freed blocks are kept per device in free lists
// keyed by their rounded size and handed to the next request of that size;
// on an allocation failure every cached block of the device is released and
// the request retried.  pdm1_pool_release() returns the cache to the driver.
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <unordered_map>

#include "pdm1_device.cuh"

namespace pdm1 {

namespace {

constexpr int kHostDevice = -1;   // the pinned host pool's key

struct Block {
    int device;
    size_t bytes;
};

struct State {
    std::mutex mu;
    std::map<int, std::multimap<size_t, void *>> free_blocks;   // device -> size -> block
    std::unordered_map<void *, Block> live;
    std::map<int, size_t> cached;                                // device -> bytes in free lists
};

State &state() {
    static State *s = new State();   // outlives every plan, including at process exit
    return *s;
}

size_t round_size(size_t bytes) {
    const size_t small = 512, large = size_t(2) << 20;
    if (bytes == 0) bytes = 1;
    return bytes <= (size_t(1) << 20) ? (bytes + small - 1) / small * small : (bytes + large - 1) / large * large;
}

void release_locked(State &s, int device) {
    auto it = s.free_blocks.find(device);
    if (it == s.free_blocks.end()) return;
    for (auto &kv : it->second) {
        if (device == kHostDevice) cudaFreeHost(kv.second);
        else cudaFree(kv.second);
    }
    it->second.clear();
    s.cached[device] = 0;
}

cudaError_t acquire(void **ptr, size_t bytes, int device) {
    State &s = state();
    const size_t r = round_size(bytes);
    {
        std::lock_guard<std::mutex> lk(s.mu);
        auto &fl = s.free_blocks[device];
        auto it = fl.find(r);
        if (it != fl.end()) {
            *ptr = it->second;
            fl.erase(it);
            s.cached[device] -= r;
            s.live[*ptr] = Block{device, r};
            return cudaSuccess;
        }
    }
    auto raw = [&](void **p) { return device == kHostDevice ? cudaMallocHost(p, r) : cudaMalloc(p, r); };
    cudaError_t e = raw(ptr);
    if (e == cudaErrorMemoryAllocation) {
        (void)cudaGetLastError();
        {
            std::lock_guard<std::mutex> lk(s.mu);
            release_locked(s, device);
        }
        e = raw(ptr);
    }
    if (e != cudaSuccess) {
        *ptr = nullptr;
        return e;
    }
    std::lock_guard<std::mutex> lk(s.mu);
    s.live[*ptr] = Block{device, r};
    return cudaSuccess;
}

void give_back(void *ptr) {
    if (!ptr) return;
    State &s = state();
    std::lock_guard<std::mutex> lk(s.mu);
    auto it = s.live.find(ptr);
    if (it == s.live.end()) return;   // not a pool block
    const Block b = it->second;
    s.live.erase(it);
    s.free_blocks[b.device].emplace(b.bytes, ptr);
    s.cached[b.device] += b.bytes;
}

}  // namespace

cudaError_t pool_malloc(void **ptr, size_t bytes) {
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    return acquire(ptr, bytes, device);
}

cudaError_t pool_malloc_host(void **ptr, size_t bytes) { return acquire(ptr, bytes, kHostDevice); }

void pool_free(void *ptr) { give_back(ptr); }

}  // namespace pdm1

extern "C" {

size_t pdm1_pool_cached_bytes(void) {
    pdm1::State &s = pdm1::state();
    std::lock_guard<std::mutex> lk(s.mu);
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return 0;
    auto it = s.cached.find(device);
    return it == s.cached.end() ? 0 : it->second;
}

int pdm1_pool_release(void) {
    pdm1::State &s = pdm1::state();
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return pdm1::report_error(PDM1_ERR_CUDA, "cudaGetDevice failed");
    if (cudaDeviceSynchronize() != cudaSuccess)
        return pdm1::report_error(PDM1_ERR_CUDA, "pdm1_pool_release: cudaDeviceSynchronize failed");
    std::lock_guard<std::mutex> lk(s.mu);
    pdm1::release_locked(s, device);
    pdm1::release_locked(s, pdm1::kHostDevice);
    return PDM1_OK;
}

}  // extern "C"
