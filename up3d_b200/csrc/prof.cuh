// Launch accounting and phase timing (see prof.cu).
#pragma once

#include <atomic>

#include <cuda_runtime.h>

namespace up3d {

// Phase slots reported by up3d_profile_read.
enum ProfSlot {
    PROF_ELEM = 0,    // element sweep (fused or per-call prep)
    PROF_ROW = 1,     // row gather (residual / matrix / Jacobian rows)
    PROF_TERM3 = 2,   // Term-3 build (flags, select, COO, sort, merge)
    PROF_SPMV = 3,    // sparse matrix-vector products
    PROF_KRYLOV = 4,  // Krylov vector kernels and preconditioner
    PROF_SLOTS = 8
};

extern std::atomic<long long> g_launches;

void prof_begin(int slot, cudaStream_t s);
void prof_end(int slot, cudaStream_t s, int launches);

// Counts one launch of a library kernel.
inline void count_launch(int n = 1) { g_launches.fetch_add(n, std::memory_order_relaxed); }

}  // namespace up3d
