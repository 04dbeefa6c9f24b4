// Device memory of the library's buffers (DBuf): cudaMalloc'd blocks kept,
// once freed, in a per-device cache and handed out again to requests of
// (nearly) the same size.
//
// A fresh workspace (a mesh, an AMG hierarchy, a Newton workspace) makes
// dozens of allocations; with plain cudaMalloc / cudaFree each one goes to
// the driver, and on a busy device such a call at times takes tens to
// hundreds of milliseconds.  Repeated set-ups of the same problem ask for
// the same sizes, so they are served from the cache instead.
//
// A freed block may still be read or written by work in flight on any
// stream, so dev_free waits for the device before it caches the block --
// the same synchronisation cudaFree implies.  The cache holds at most
// cap bytes per process (UP3D_POOL_CACHE_MB, default 4096; 0 turns caching
// off); past the cap the least recently freed blocks are released until
// three quarters of it remain (so that eviction, which costs what the
// deferred cudaFree calls cost, comes in few batches).  When
// cudaMalloc runs out of memory the device's cached blocks are released
// and the allocation is retried once.
#include <cstdint>
#include <cstdlib>
#include <map>
#include <mutex>
#include <unordered_map>

#include "internal.cuh"

namespace up3d {
namespace {

struct Block {
    int device;
    size_t size;
};

struct Cached {
    void* p;
    uint64_t seq;  // order of the frees (eviction takes the oldest first)
};

struct Pool {
    std::mutex mu;
    std::unordered_map<void*, Block> live;                   // handed out
    std::multimap<std::pair<int, size_t>, Cached> cached;    // (device, size) -> free block
    size_t cached_bytes = 0, live_bytes = 0;
    int64_t hits = 0, misses = 0;
    uint64_t seq = 0;
    size_t cap = size_t(4096) << 20;
    Pool() {
        if (const char* v = std::getenv("UP3D_POOL_CACHE_MB")) {
            char* end = nullptr;
            const long long mb = std::strtoll(v, &end, 10);
            if (end != v && mb >= 0) cap = size_t(mb) << 20;
        }
    }
};

// never destroyed: buffers released during process exit still find it
Pool& pool() {
    static Pool* p = new Pool();
    return *p;
}

// 512-byte steps up to 1 MiB, 2 MiB steps above
size_t round_size(size_t b) {
    if (b == 0) b = 1;
    if (b <= (size_t(1) << 20)) return (b + 511) & ~size_t(511);
    const size_t g = size_t(2) << 20;
    return (b + g - 1) / g * g;
}

// cudaFree of the device's cached blocks (all devices when device < 0);
// the caller holds the lock.  Returns the bytes released.
size_t release_locked(Pool& P, int device) {
    size_t freed = 0;
    int prev = -1;
    cudaGetDevice(&prev);
    for (auto it = P.cached.begin(); it != P.cached.end();) {
        if (device >= 0 && it->first.first != device) {
            ++it;
            continue;
        }
        if (it->first.first != prev) cudaSetDevice(it->first.first);
        cudaFree(it->second.p);
        freed += it->first.second;
        P.cached_bytes -= it->first.second;
        it = P.cached.erase(it);
    }
    if (prev >= 0) cudaSetDevice(prev);
    return freed;
}

}  // namespace

void* dev_alloc(size_t bytes) {
    int dev = 0;
    UP3D_CUDA(cudaGetDevice(&dev));
    const size_t sz = round_size(bytes);
    Pool& P = pool();
    {
        std::lock_guard<std::mutex> g(P.mu);
        // the smallest cached block of this device that fits, if it is at
        // most a quarter larger than asked
        auto it = P.cached.lower_bound({dev, sz});
        if (it != P.cached.end() && it->first.first == dev && it->first.second - sz <= sz / 4) {
            void* p = it->second.p;
            const size_t bsz = it->first.second;
            P.cached.erase(it);
            P.cached_bytes -= bsz;
            P.live[p] = {dev, bsz};
            P.live_bytes += bsz;
            ++P.hits;
            return p;
        }
        ++P.misses;
    }
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, sz);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();  // clear the failed call's error
        {
            std::lock_guard<std::mutex> g(P.mu);
            release_locked(P, dev);
        }
        e = cudaMalloc(&p, sz);
    }
    UP3D_CUDA(e);
    std::lock_guard<std::mutex> g(P.mu);
    P.live[p] = {dev, sz};
    P.live_bytes += sz;
    return p;
}

void dev_free(void* p) {
    if (!p) return;
    Pool& P = pool();
    Block b{};
    {
        std::lock_guard<std::mutex> g(P.mu);
        auto it = P.live.find(p);
        if (it == P.live.end()) {
            cudaFree(p);  // not one of ours
            return;
        }
        b = it->second;
        P.live.erase(it);
        P.live_bytes -= b.size;
    }
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != b.device) cudaSetDevice(b.device);
    // work in flight may still use the block: wait for it, as cudaFree does
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess || b.size > P.cap) {
        cudaFree(p);
        cudaGetLastError();
    } else {
        std::lock_guard<std::mutex> g(P.mu);
        P.cached.insert({{b.device, b.size}, Cached{p, P.seq++}});
        P.cached_bytes += b.size;
        // over the cap: release the least recently freed blocks down to
        // three quarters of it
        if (P.cached_bytes > P.cap) {
            const size_t low = P.cap - P.cap / 4;
            while (P.cached_bytes > low && !P.cached.empty()) {
                auto old = P.cached.begin();
                for (auto it = P.cached.begin(); it != P.cached.end(); ++it)
                    if (it->second.seq < old->second.seq) old = it;
                if (old->first.first != b.device) cudaSetDevice(old->first.first);
                cudaFree(old->second.p);
                if (old->first.first != b.device) cudaSetDevice(b.device);
                P.cached_bytes -= old->first.second;
                P.cached.erase(old);
            }
        }
    }
    if (prev >= 0 && prev != b.device) cudaSetDevice(prev);
}

}  // namespace up3d

using namespace up3d;

extern "C" {

int up3d_pool_stats(int64_t* cached_bytes, int64_t* live_bytes, int64_t* hits, int64_t* misses) {
    return guarded([&] {
        UP3D_REQUIRE(cached_bytes && live_bytes && hits && misses, UP3D_ERR_ARGUMENT,
                     "up3d_pool_stats: null argument");
        Pool& P = pool();
        std::lock_guard<std::mutex> g(P.mu);
        *cached_bytes = (int64_t)P.cached_bytes;
        *live_bytes = (int64_t)P.live_bytes;
        *hits = P.hits;
        *misses = P.misses;
    });
}

int up3d_pool_release(int64_t* released_bytes) {
    return guarded([&] {
        Pool& P = pool();
        std::lock_guard<std::mutex> g(P.mu);
        const size_t freed = release_locked(P, -1);
        if (released_bytes) *released_bytes = (int64_t)freed;
    });
}

}  // extern "C"
