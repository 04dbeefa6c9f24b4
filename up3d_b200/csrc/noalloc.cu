// CG with point-Jacobi preconditioning that allocates nothing.
//
// For callers that cannot let this library call cudaMalloc/cudaFree: a
// process whose device memory is already handed to another allocator (a
// framework's caching allocator, a fixed pre-reserved pool), where a
// library-side cudaMalloc would fail or fragment that pool, or a
// time-critical host loop that cannot afford the implicit device
// synchronisation of cudaMalloc/cudaFree.  All working vectors and the
// reduction partials live in one file-scope device array; the caller passes
// only its inputs and outputs.  The result equals up3d_cg with an
// up3d_precond_jacobi preconditioner (same kernels, same reduction order).
//
// The array holds UP3D_NOALLOC_MAX_ROWS rows (see up3d.h).  CUDA loads a
// library's device code lazily by default (CUDA_MODULE_LOADING=LAZY, CUDA
// 12.2 and later), so the driver commits the array's device memory on each
// device at the first use of this file's device code there -- the first
// call of this entry point on that device, which therefore makes one
// driver-side allocation (and can fail with out-of-memory once another
// allocator has reserved the device).  Callers make that first call, or run
// with CUDA_MODULE_LOADING=EAGER, before their pool reserves the device; from
// then on the array stays resident until the process exits and no call
// allocates.  All calls share it: calls that overlap on the GPU (other
// streams or threads) race on it and must be serialised by the caller.

#include <cmath>

#include "internal.cuh"

namespace up3d {

template <class T>
void launch_spmv(int64_t n, const int32_t* indptr, const int32_t* indices, const T* data, const T* x, T* y,
                 const uint8_t* dir, cudaStream_t s);

namespace {

constexpr int NA_RB = 256;     // reduction block (as in krylov.cu)
constexpr int NA_RGRID = 592;  // fixed partial count (as in krylov.cu)
constexpr int64_t NA_ROWS = UP3D_NOALLOC_MAX_ROWS;
// r, z, p, q, D^-1, then the reduction partials and the scalars
constexpr int64_t NA_DOUBLES = 5 * NA_ROWS + NA_RGRID + 8;

static __device__ __align__(256) double g_scratch[NA_DOUBLES];

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

// The two reduction passes of the allocating CG's dot products (krylov.cu
// k_multidot with one vector, k_finish): per block, warp butterflies then
// the block's warp sums in order; then one warp over the block partials.
__global__ void __launch_bounds__(NA_RB) k_na_dot(const double* __restrict__ x, const double* __restrict__ y,
                                                  int64_t n, double* __restrict__ partial) {
    __shared__ double sh[NA_RB / 32];
    double acc = 0.0;
    GRID_STRIDE(i, n) acc += x[i] * y[i];
    const double v = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
#pragma unroll
        for (int q = 0; q < NA_RB / 32; ++q) t += sh[q];
        partial[blockIdx.x] = t;
    }
}

__global__ void k_na_finish(const double* __restrict__ partial, int nb, double* __restrict__ out) {
    if (threadIdx.x >= 32) return;
    double acc = 0.0;
    for (int b = threadIdx.x; b < nb; b += 32) acc += partial[b];
    acc = warp_sum(acc);
    if (threadIdx.x == 0) *out = acc;
}

__global__ void k_na_diag(int64_t n, const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices,
                          const double* __restrict__ data, const uint8_t* __restrict__ dir,
                          double* __restrict__ dinv) {
    GRID_STRIDE(r, n) {
        double d = 0.0;
        for (int32_t k = indptr[r]; k < indptr[r + 1]; ++k)
            if (indices[k] == r) d = data[k];
        if (dir && dir[r]) d = 1.0;
        dinv[r] = d != 0.0 ? 1.0 / d : 1.0;
    }
}

__global__ void k_na_sub(const double* __restrict__ b, const double* __restrict__ ax, double* __restrict__ r,
                         int64_t n) {
    GRID_STRIDE(i, n) r[i] = b[i] - ax[i];
}

__global__ void k_na_mul(const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ out,
                         int64_t n) {
    GRID_STRIDE(i, n) out[i] = a[i] * b[i];
}

__global__ void k_na_update(const double* __restrict__ sc, double* __restrict__ x, double* __restrict__ r,
                            const double* __restrict__ p, const double* __restrict__ q, int64_t n) {
    const double alpha = sc[0] / sc[1];
    GRID_STRIDE(i, n) {
        x[i] += alpha * p[i];
        r[i] -= alpha * q[i];
    }
}

__global__ void k_na_dir(const double* __restrict__ sc, const double* __restrict__ z, double* __restrict__ p,
                         int64_t n) {
    const double beta = sc[2] / sc[0];
    GRID_STRIDE(i, n) p[i] = z[i] + beta * p[i];
}

__global__ void k_na_copy_scalar(const double* __restrict__ src, double* __restrict__ dst) { *dst = *src; }

// Device address of g_scratch on the current device.  The host-side name is
// only a stand-in, so the address is asked for on every call (cheap once the
// module is loaded): a pointer cached across a device reset could point at
// memory of a dead context.
double* scratch_for_current_device() {
    void* p = nullptr;
    UP3D_CUDA(cudaGetSymbolAddress(&p, g_scratch));
    return static_cast<double*>(p);
}

}  // namespace
}  // namespace up3d

using namespace up3d;

extern "C" int up3d_cg_jacobi_noalloc(const up3d_csr* A, const double* b, double* x, double rtol, double atol,
                                      int maxiter, int64_t* iters, double* resid, int* info,
                                      up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(A && A->indptr && A->indices && A->data && b && x && A->n >= 0 && maxiter >= 0,
                     UP3D_ERR_ARGUMENT, "up3d_cg_jacobi_noalloc: bad argument");
        UP3D_REQUIRE(A->n <= NA_ROWS, UP3D_ERR_VALUE,
                     "up3d_cg_jacobi_noalloc: " + std::to_string(A->n) + " rows exceed the static limit of " +
                         std::to_string(NA_ROWS) + " (UP3D_NOALLOC_MAX_ROWS); use up3d_cg");
        cudaStream_t s = S(stream);
        const int64_t n = A->n;
        double* base = scratch_for_current_device();
        double* r = base;
        double* z = base + NA_ROWS;
        double* p = base + 2 * NA_ROWS;
        double* q = base + 3 * NA_ROWS;
        double* dinv = base + 4 * NA_ROWS;
        double* partial = base + 5 * NA_ROWS;
        double* sc = partial + NA_RGRID;  // rz, pq, rz_new, norm
        // previous calls leave their values behind: start the scalars at 0
        UP3D_CUDA(cudaMemsetAsync(sc, 0, 8 * sizeof(double), s));
        auto dot = [&](const double* u, const double* v, double* out) {
            k_na_dot<<<NA_RGRID, NA_RB, 0, s>>>(u, v, n, partial);
            UP3D_CHECK_LAUNCH();
            k_na_finish<<<1, 1024, 0, s>>>(partial, NA_RGRID, out);
            UP3D_CHECK_LAUNCH();
        };
        auto nrm = [&](const double* u) {
            dot(u, u, sc + 3);
            double h = 0.0;
            UP3D_CUDA(cudaMemcpyAsync(&h, sc + 3, sizeof(double), cudaMemcpyDeviceToHost, s));
            UP3D_CUDA(cudaStreamSynchronize(s));
            return std::sqrt(h);
        };
        int64_t it = 0;
        double rn = 0.0;
        if (n > 0) {
            k_na_diag<<<grid_for(n, 256), 256, 0, s>>>(n, A->indptr, A->indices, A->data, A->dirichlet, dinv);
            UP3D_CHECK_LAUNCH();
            const double bnrm = nrm(b);
            const double tol = std::max(atol, rtol * bnrm);
            launch_spmv<double>(n, A->indptr, A->indices, A->data, x, q, A->dirichlet, s);
            k_na_sub<<<grid_for(n, 256), 256, 0, s>>>(b, q, r, n);
            UP3D_CHECK_LAUNCH();
            rn = nrm(r);
            if (bnrm == 0.0) {
                UP3D_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, s));
                rn = 0.0;
            }
            if (rn > tol) {
                k_na_mul<<<grid_for(n, 256), 256, 0, s>>>(dinv, r, z, n);
                UP3D_CHECK_LAUNCH();
                UP3D_CUDA(cudaMemcpyAsync(p, z, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
                dot(r, z, sc + 0);
                for (it = 1; it <= maxiter; ++it) {
                    launch_spmv<double>(n, A->indptr, A->indices, A->data, p, q, A->dirichlet, s);
                    dot(p, q, sc + 1);
                    k_na_update<<<grid_for(n, 256), 256, 0, s>>>(sc, x, r, p, q, n);
                    UP3D_CHECK_LAUNCH();
                    rn = nrm(r);
                    if (rn <= tol || !std::isfinite(rn)) break;
                    k_na_mul<<<grid_for(n, 256), 256, 0, s>>>(dinv, r, z, n);
                    UP3D_CHECK_LAUNCH();
                    dot(r, z, sc + 2);
                    k_na_dir<<<grid_for(n, 256), 256, 0, s>>>(sc, z, p, n);
                    UP3D_CHECK_LAUNCH();
                    k_na_copy_scalar<<<1, 1, 0, s>>>(sc + 2, sc + 0);
                    UP3D_CHECK_LAUNCH();
                }
                if (it > maxiter) it = maxiter;
            }
            // every path (b = 0 included) leaves x complete on return
            UP3D_CUDA(cudaStreamSynchronize(s));
            if (iters) *iters = it;
            if (resid) *resid = rn;
            if (info) *info = rn <= tol ? 0 : maxiter;
        } else {
            if (iters) *iters = 0;
            if (resid) *resid = 0.0;
            if (info) *info = 0;
        }
    });
}
