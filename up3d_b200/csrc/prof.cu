// Launch accounting and per-phase CUDA-event timing of the up3d library.
//
// Every kernel launch site of the library bumps a process-wide counter
// (up3d_launch_count).  With profiling enabled, the phases of the fused
// evaluation and of the solvers record event pairs on their stream; the
// elapsed times are summed when read (which synchronises the events).

#include <atomic>
#include <mutex>
#include <vector>

#include "internal.cuh"
#include "prof.cuh"

namespace up3d {

std::atomic<long long> g_launches{0};

namespace {
struct Slot {
    std::vector<cudaEvent_t> start, stop;
    std::vector<cudaStream_t> open;
    long long launches = 0;
};
std::mutex g_mu;
bool g_on = false;
Slot g_slots[PROF_SLOTS];
std::vector<cudaEvent_t> g_pool;

cudaEvent_t take() {
    if (!g_pool.empty()) {
        cudaEvent_t e = g_pool.back();
        g_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    UP3D_CUDA(cudaEventCreate(&e));
    return e;
}
}  // namespace

void prof_begin(int slot, cudaStream_t s) {
    if (!g_on) return;
    std::lock_guard<std::mutex> lk(g_mu);
    cudaEvent_t e = take();
    UP3D_CUDA(cudaEventRecord(e, s));
    g_slots[slot].start.push_back(e);
}

void prof_end(int slot, cudaStream_t s, int launches) {
    if (!g_on) return;
    std::lock_guard<std::mutex> lk(g_mu);
    cudaEvent_t e = take();
    UP3D_CUDA(cudaEventRecord(e, s));
    g_slots[slot].stop.push_back(e);
    g_slots[slot].launches += launches;
}

}  // namespace up3d

using namespace up3d;

extern "C" {

int up3d_launch_count(int64_t* out) {
    return guarded([&] {
        UP3D_REQUIRE(out, UP3D_ERR_ARGUMENT, "up3d_launch_count: null argument");
        *out = g_launches.load();
    });
}

int up3d_profile(int enable) {
    return guarded([&] {
        std::lock_guard<std::mutex> lk(g_mu);
        for (auto& s : g_slots) {
            for (auto e : s.start) g_pool.push_back(e);
            for (auto e : s.stop) g_pool.push_back(e);
            s.start.clear();
            s.stop.clear();
            s.launches = 0;
        }
        g_on = enable != 0;
    });
}

int up3d_profile_read(double* ms, int64_t* calls, int64_t* launches, int n_slots) {
    return guarded([&] {
        UP3D_REQUIRE(ms && calls && launches && n_slots >= 0, UP3D_ERR_ARGUMENT,
                     "up3d_profile_read: bad argument");
        std::lock_guard<std::mutex> lk(g_mu);
        for (int k = 0; k < n_slots && k < PROF_SLOTS; ++k) {
            Slot& s = g_slots[k];
            double tot = 0.0;
            size_t n = std::min(s.start.size(), s.stop.size());
            for (size_t i = 0; i < n; ++i) {
                UP3D_CUDA(cudaEventSynchronize(s.stop[i]));
                float t = 0.f;
                UP3D_CUDA(cudaEventElapsedTime(&t, s.start[i], s.stop[i]));
                tot += t;
            }
            ms[k] = tot;
            calls[k] = (int64_t)n;
            launches[k] = s.launches;
        }
    });
}

}  // extern "C"
