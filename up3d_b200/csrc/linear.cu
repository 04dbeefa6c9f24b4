// CSR SpMV of the up3d library (the matrix-vector product inside the
// reference's spla.cg / spla.gmres calls, solve/picard.py:375-380,
// solve/linear.py:182, solve/newton.py:1029-1032).
//
// One warp per 32 rows with coalesced entry loads (csr_rows.cuh) on large
// matrices, 4 lanes per row on small ones; a fixed summation order either
// way (bit-reproducible).  The optional Dirichlet mask
// embeds the free-DOF operator A[free][:, free] (solve/linear.py:20-58) in
// full size: constrained rows act as identity, constrained columns are
// dropped.

#include "csr_rows.cuh"

namespace up3d {
namespace {

// y = A x (+ X x: a second CSR on the same rows, the Term-3 entries outside
// the P1 pattern, added after the row's P1 entries).  With the Dirichlet
// mask, constrained rows give y = x and constrained columns are dropped.
// TPR = 0: one warp per 32 rows; else TPR lanes per row.
template <class T, int TPR>
__global__ void __launch_bounds__(CSR_ROWS_BLOCK)
    k_spmv(int64_t n, const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices,
           const T* __restrict__ data, const int32_t* __restrict__ xptr, const int32_t* __restrict__ xidx,
           const T* __restrict__ xdata, const T* __restrict__ x, T* __restrict__ y, const uint8_t* __restrict__ dir) {
    auto p1 = [&](int32_t k) {
        const int32_t c = indices[k];
        const T v = data[k] * x[c];
        return (dir && dir[c]) ? T(0) : v;
    };
    auto p3 = [&](int32_t k) {
        const int32_t c = xidx[k];
        const T v = xdata[k] * x[c];
        return (dir && dir[c]) ? T(0) : v;
    };
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    if constexpr (TPR == 0) {
        __shared__ T sh[CSR_ROWS_BLOCK / 32][CSR_ROWS_CHUNK];
        T* my = sh[threadIdx.x >> 5];
        const int lane = threadIdx.x & 31;
        for (int64_t r0 = warp * 32; r0 < n; r0 += n_warps * 32) {   // warp-uniform
            T acc = warp_row_sum<T>(indptr, r0, n, my, p1);
            if (xptr) acc += warp_row_sum<T>(xptr, r0, n, my, p3);
            const int64_t r = r0 + lane;
            if (r < n) y[r] = (dir && dir[r]) ? x[r] : acc;
        }
    } else {
        constexpr int RPW = 32 / TPR;
        const int sub = threadIdx.x % TPR, group = (threadIdx.x & 31) / TPR;
        for (int64_t base = warp * RPW; base < n; base += n_warps * RPW) {   // warp-uniform
            const int64_t r = base + group;
            T acc = lanes_row_sum<T, TPR>(indptr, r, n, p1);
            if (xptr) acc += lanes_row_sum<T, TPR>(xptr, r, n, p3);
            if (sub == 0 && r < n) y[r] = (dir && dir[r]) ? x[r] : acc;
        }
    }
}

}  // namespace

// P1 rows hold ~15 entries: one warp per 32 rows when the matrix has rows
// enough to fill the GPU that way, else 4 lanes per row
template <class T>
void launch_spmv2(int64_t n, const int32_t* indptr, const int32_t* indices, const T* data, const int32_t* xptr,
                  const int32_t* xidx, const T* xdata, const T* x, T* y, const uint8_t* dir, cudaStream_t s) {
    if (n >= CSR_ROWS_MIN_ROWS)
        k_spmv<T, 0><<<csr_rows_grid(n), CSR_ROWS_BLOCK, 0, s>>>(n, indptr, indices, data, xptr, xidx, xdata, x, y,
                                                                 dir);
    else
        k_spmv<T, 4><<<lanes_grid(n, 4), CSR_ROWS_BLOCK, 0, s>>>(n, indptr, indices, data, xptr, xidx, xdata, x, y,
                                                                 dir);
    UP3D_CHECK_LAUNCH();
}

template <class T>
void launch_spmv(int64_t n, const int32_t* indptr, const int32_t* indices, const T* data, const T* x, T* y,
                 const uint8_t* dir, cudaStream_t s) {
    launch_spmv2<T>(n, indptr, indices, data, nullptr, nullptr, nullptr, x, y, dir, s);
}

template void launch_spmv<double>(int64_t, const int32_t*, const int32_t*, const double*, const double*, double*,
                                  const uint8_t*, cudaStream_t);
template void launch_spmv<float>(int64_t, const int32_t*, const int32_t*, const float*, const float*, float*,
                                 const uint8_t*, cudaStream_t);
template void launch_spmv2<double>(int64_t, const int32_t*, const int32_t*, const double*, const int32_t*,
                                   const int32_t*, const double*, const double*, double*, const uint8_t*,
                                   cudaStream_t);
template void launch_spmv2<float>(int64_t, const int32_t*, const int32_t*, const float*, const int32_t*,
                                  const int32_t*, const float*, const float*, float*, const uint8_t*, cudaStream_t);

}  // namespace up3d

using namespace up3d;

extern "C" {

int up3d_spmv(int64_t n, const int32_t* indptr, const int32_t* indices, const double* data, const double* x,
              double* y, const uint8_t* dir, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(indptr && indices && data && x && y && n >= 0, UP3D_ERR_ARGUMENT, "up3d_spmv: bad argument");
        if (n == 0) return;
        launch_spmv<double>(n, indptr, indices, data, x, y, dir, S(stream));
    });
}

int up3d_spmv_f32(int64_t n, const int32_t* indptr, const int32_t* indices, const float* data, const float* x,
                  float* y, const uint8_t* dir, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(indptr && indices && data && x && y && n >= 0, UP3D_ERR_ARGUMENT,
                     "up3d_spmv_f32: bad argument");
        if (n == 0) return;
        launch_spmv<float>(n, indptr, indices, data, x, y, dir, S(stream));
    });
}

}  // extern "C"
