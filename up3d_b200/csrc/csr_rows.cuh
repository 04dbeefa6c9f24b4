// CSR rows summed a warp at a time: the common core of the SpMV, the
// Jacobi smoother and the AMG transfer operators.
//
// One warp owns 32 consecutive rows.  Their entries are contiguous, so the
// lanes read them 32 at a time -- fully coalesced, CSR_ROWS_CHUNK / 32
// independent loads per lane in flight -- and stage the products in shared
// memory; each lane then adds its own row's products in entry order, the
// order of a sequential CSR product.  (Striding each row's ~15 entries over
// a few lanes instead leaves each lane a short chain of dependent index ->
// value loads and sectors shared between neighbouring rows.)
#pragma once

#include "internal.cuh"

namespace up3d {

constexpr int CSR_ROWS_CHUNK = 256;   // entries staged per pass of a warp
constexpr int CSR_ROWS_BLOCK = 256;   // threads per block (8 warps)

// Sum over row r0 + lane of prod(k), k over the row's entries, for the
// calling warp's rows [r0, min(r0 + 32, n)); 0 for lanes past n.  `sh`
// holds CSR_ROWS_CHUNK values private to the warp.  Every lane must call.
template <class T, class Prod>
__device__ __forceinline__ T warp_row_sum(const int32_t* __restrict__ Ap, int64_t r0, int64_t n, T* sh, Prod prod) {
    const int lane = threadIdx.x & 31;
    const int64_t r = r0 + lane;
    const int64_t rend = r0 + 32 < n ? r0 + 32 : n;
    const int32_t s = Ap[r0], e = Ap[rend];
    int32_t ms = 0, me = 0;
    if (r < n) {
        ms = Ap[r];
        me = Ap[r + 1];
    }
    T acc = T(0);
    for (int32_t c0 = s; c0 < e; c0 += CSR_ROWS_CHUNK) {
        T v[CSR_ROWS_CHUNK / 32];
#pragma unroll
        for (int j = 0; j < CSR_ROWS_CHUNK / 32; ++j) {
            const int32_t k = c0 + j * 32 + lane;
            v[j] = k < e ? prod(k) : T(0);
        }
#pragma unroll
        for (int j = 0; j < CSR_ROWS_CHUNK / 32; ++j) sh[j * 32 + lane] = v[j];
        __syncwarp();
        const int32_t a = ms > c0 ? ms : c0;
        const int32_t b = me < c0 + CSR_ROWS_CHUNK ? me : c0 + CSR_ROWS_CHUNK;
        for (int32_t k = a; k < b; ++k) acc += sh[k - c0];
        __syncwarp();
    }
    return acc;
}

// Sum over row r of prod(k) by TPR lanes striding the row's entries,
// reduced by a fixed shuffle tree; every lane of the warp must call (rows
// past n contribute 0).  For short matrices (few rows: the warp-rows form
// would leave most SMs idle) and long rows (AMG coarse levels, restriction).
template <class T, int TPR, class Prod>
__device__ __forceinline__ T lanes_row_sum(const int32_t* __restrict__ Ap, int64_t r, int64_t n, Prod prod) {
    const int sub = threadIdx.x % TPR;
    T acc = T(0);
    if (r < n)
        for (int32_t k = Ap[r] + sub; k < Ap[r + 1]; k += TPR) acc += prod(k);
#pragma unroll
    for (int o = TPR / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, TPR);
    return acc;
}

// The warp-rows form pays once a matrix has rows enough to give every SM
// a few warps of 32 rows and its rows are short (measured on B200: the
// 625 k-row P1 Jacobian 0.045 -> 0.034 ms; a 24 k-row AMG level with 26
// entries per row 2x slower than 16 lanes per row).
constexpr int64_t CSR_ROWS_MIN_ROWS = 148 * 16 * 32;
inline bool use_warp_rows(int64_t n, int64_t nnz) { return n >= CSR_ROWS_MIN_ROWS && nnz <= 24 * n; }

// Lanes per row from the mean row length (thresholds tuned on B200).
inline int lanes_per_row(int64_t nnz, int64_t n) {
    const double avg = n > 0 ? (double)nnz / (double)n : 0.0;
    return avg <= 16 ? 4 : avg <= 24 ? 8 : avg <= 96 ? 16 : 32;
}
inline unsigned lanes_grid(int64_t n, int tpr) { return grid_for(n, 256 / tpr, (int64_t)148 * 64); }

// Blocks for n rows at 32 rows per warp, capped at a persistent wave.
inline unsigned csr_rows_grid(int64_t n) {
    const int64_t groups = (n + 31) / 32;
    const int64_t blocks = (groups + CSR_ROWS_BLOCK / 32 - 1) / (CSR_ROWS_BLOCK / 32);
    const int64_t cap = (int64_t)148 * 8;
    return (unsigned)(blocks < 1 ? 1 : blocks > cap ? cap : blocks);
}

}  // namespace up3d
