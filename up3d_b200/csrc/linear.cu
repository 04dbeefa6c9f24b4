// CSR SpMV of the up3d library (the matrix-vector product inside the
// reference's spla.cg / spla.gmres calls, solve/picard.py:375-380,
// solve/linear.py:182, solve/newton.py:1029-1032).
//
// UP3D_SPMV_TPR lanes per row (4: P1 rows hold ~15 entries), fixed reduction
// tree (bit-reproducible).  The optional Dirichlet mask embeds the free-DOF
// operator A[free][:, free] (solve/linear.py:20-58) in full size:
// constrained rows act as identity, constrained columns are dropped.

#include "internal.cuh"

namespace up3d {
namespace {

// y = A x (+ X x: a second CSR on the same rows, the Term-3 entries outside
// the P1 pattern), TPR lanes per row.  With the Dirichlet mask, constrained
// rows give y = x and constrained columns are dropped.
template <class T, int TPR>
__global__ void __launch_bounds__(256)
    k_spmv(int64_t n, const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices,
           const T* __restrict__ data, const int32_t* __restrict__ xptr, const int32_t* __restrict__ xidx,
           const T* __restrict__ xdata, const T* __restrict__ x, T* __restrict__ y, const uint8_t* __restrict__ dir) {
    // warp-uniform loop: every lane reaches the shuffles
    const int sub = threadIdx.x % TPR;
    const int group = (threadIdx.x & 31) / TPR;
    constexpr int RPW = 32 / TPR;  // rows per warp
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = warp * RPW; base < n; base += n_warps * RPW) {
        const int64_t r = base + group;
        T acc = T(0);
        bool fixed = false;
        if (r < n) {
            fixed = dir && dir[r];
            if (!fixed) {
                const int32_t e = indptr[r + 1];
                for (int32_t k = indptr[r] + sub; k < e; k += TPR) {
                    int32_t c = indices[k];
                    if (!dir || !dir[c]) acc += data[k] * x[c];
                }
                if (xptr) {
                    const int32_t xe = xptr[r + 1];
                    for (int32_t k = xptr[r] + sub; k < xe; k += TPR) {
                        int32_t c = xidx[k];
                        if (!dir || !dir[c]) acc += xdata[k] * x[c];
                    }
                }
            }
        }
#pragma unroll
        for (int o = TPR / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, TPR);
        if (sub == 0 && r < n) y[r] = fixed ? x[r] : acc;
    }
}

}  // namespace

// P1 rows hold ~15 entries: 4 lanes per row measured fastest on B200
#ifndef UP3D_SPMV_TPR
#define UP3D_SPMV_TPR 4
#endif
template <class T>
void launch_spmv2(int64_t n, const int32_t* indptr, const int32_t* indices, const T* data, const int32_t* xptr,
                  const int32_t* xidx, const T* xdata, const T* x, T* y, const uint8_t* dir, cudaStream_t s) {
    constexpr int TPR = UP3D_SPMV_TPR;
    const int block = 256;
    const unsigned grid = grid_for(n * TPR, block, (int64_t)148 * 64);
    k_spmv<T, TPR><<<grid, block, 0, s>>>(n, indptr, indices, data, xptr, xidx, xdata, x, y, dir);
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
