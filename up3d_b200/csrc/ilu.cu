// Incomplete-LU preconditioner on the device: ILU(0) on the matrix's own
// pattern (the B200 stand-in for the reference's threshold ILU,
// solve/linear.py:84-131, which scipy's serial spilu factors on the host).
//
// Factorisation: the fixed-point form of ILU(0) (Chow and Patel, "Fine-
// grained parallel incomplete LU factorization", SIAM J. Sci. Comput. 37,
// 2015): every entry (r, c) of the pattern is updated at once from the
// previous sweep's factors,
//     l_rc = (a_rc - sum_{k < c} l_rk u_kc) / u_cc     (r > c)
//     u_rc =  a_rc - sum_{k < r} l_rk u_kc             (r <= c),
// k over row r's pattern, u_kc found by binary search in row k; the
// iteration starts from L = strict lower part of A scaled by the diagonal,
// U = upper part, and a few sweeps reach the ILU(0) factors to rounding on
// the P1 matrices.  Application: z = U^-1 L^-1 r with each triangular solve
// done by a few Jacobi sweeps on its triangle (the iterative triangular
// solves of the same approach), every sweep a row pass over half the
// entries.  The Dirichlet mask embeds the free-DOF operator: constrained
// rows factor as identity rows, constrained columns are dropped.  A
// factorisation that yields a non-finite value is redone on A + eps I, eps
// = 1e-3 mean |a_ii| (the diagonal shift of the reference's fallback
// ladder).  All sums in a fixed order: bit-reproducible.

#include <cmath>

#include "csr_rows.cuh"
#include "internal.cuh"
#include "krylov.cuh"

namespace up3d {
namespace {

__global__ void k_row_of(int64_t n, const int32_t* __restrict__ p, int32_t* __restrict__ row) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
        for (int32_t e = p[r]; e < p[r + 1]; ++e) row[e] = (int32_t)r;
}

// position of the diagonal of each row (-1 when the pattern has none)
__global__ void k_diag_pos(int64_t n, const int32_t* __restrict__ p, const int32_t* __restrict__ ci,
                           int32_t* __restrict__ diag) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        int32_t d = -1;
        for (int32_t e = p[r]; e < p[r + 1]; ++e)
            if (ci[e] == r) d = e;
        diag[r] = d;
    }
}

__device__ __forceinline__ bool masked(const uint8_t* dir, int64_t r, int32_t c) {
    return dir && (dir[r] || dir[c]);
}

// The matrix entry the factorisation sees: identity rows and dropped
// columns under the mask, plus the diagonal shift.
__device__ __forceinline__ double a_entry(const double* a, const uint8_t* dir, int64_t r, int32_t c, int32_t e,
                                          double shift) {
    if (masked(dir, r, c)) return r == c ? 1.0 : 0.0;
    return r == c ? a[e] + shift : a[e];
}

__global__ void k_ilu_init(int64_t nnz, const int32_t* __restrict__ row, const int32_t* __restrict__ ci,
                           const double* __restrict__ a, const uint8_t* __restrict__ dir,
                           const int32_t* __restrict__ diag, double shift, double* __restrict__ lu) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = row[e];
        const int32_t c = ci[e];
        const double v = a_entry(a, dir, r, c, (int32_t)e, shift);
        if (r > c) {
            const int32_t dc = diag[c];
            const double ucc = dc < 0 ? 0.0 : a_entry(a, dir, c, c, dc, shift);
            lu[e] = v / ucc;
        } else {
            lu[e] = v;
        }
    }
}

__global__ void k_ilu_sweep(int64_t nnz, const int32_t* __restrict__ p, const int32_t* __restrict__ row,
                            const int32_t* __restrict__ ci, const double* __restrict__ a,
                            const uint8_t* __restrict__ dir, const int32_t* __restrict__ diag, double shift,
                            const double* __restrict__ lu_old, double* __restrict__ lu_new) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = row[e];
        const int32_t c = ci[e];
        double s = a_entry(a, dir, r, c, (int32_t)e, shift);
        if (!masked(dir, r, c)) {
            const int32_t m = (int32_t)(r < c ? r : c);
            for (int32_t q = p[r]; q < p[r + 1]; ++q) {
                const int32_t k = ci[q];
                if (k >= m) break;  // columns ascending
                // u_kc: entry (k, c) of row k
                int32_t lo = p[k], hi = p[k + 1] - 1;
                while (lo <= hi) {
                    const int32_t mid = (lo + hi) >> 1;
                    const int32_t cm = ci[mid];
                    if (cm == c) {
                        s -= lu_old[q] * lu_old[mid];
                        break;
                    }
                    if (cm < c) lo = mid + 1;
                    else hi = mid - 1;
                }
            }
        }
        if (r > c) {
            const int32_t dc = diag[c];
            lu_new[e] = s / (dc < 0 ? 0.0 : lu_old[dc]);
        } else {
            lu_new[e] = s;
        }
    }
}

__global__ void k_nonfinite(int64_t nnz, const double* __restrict__ lu, int* __restrict__ flag) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz; e += (int64_t)gridDim.x * blockDim.x)
        if (!isfinite(lu[e])) *flag = 1;
}

__global__ void k_abs_diag_sum(int64_t n, const double* __restrict__ a, const int32_t* __restrict__ diag,
                               const uint8_t* __restrict__ dir, double* __restrict__ out) {
    // one block, fixed order
    __shared__ double sh[256];
    double acc = 0.0;
    for (int64_t r = threadIdx.x; r < n; r += blockDim.x)
        if (diag[r] >= 0 && !(dir && dir[r])) acc += fabs(a[diag[r]]);
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = sh[0];
}

// One Jacobi sweep of a triangular solve, 4 lanes per row:
//   LOWER: y_new[r] = b[r] - sum_{c < r} l_rc y[c]           (unit diagonal)
//   upper: y_new[r] = (b[r] - sum_{c > r} u_rc y[c]) / u_rr
template <bool LOWER>
__global__ void __launch_bounds__(256)
    k_tri_sweep(int64_t n, const int32_t* __restrict__ p, const int32_t* __restrict__ ci, const double* __restrict__ lu,
                const int32_t* __restrict__ diag, const double* __restrict__ b, const double* __restrict__ y,
                double* __restrict__ y_new) {
    constexpr int TPR = 4, RPW = 32 / TPR;
    const int sub = threadIdx.x % TPR, group = (threadIdx.x & 31) / TPR;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = warp * RPW; base < n; base += n_warps * RPW) {   // warp-uniform
        const int64_t r = base + group;
        const double acc = lanes_row_sum<double, TPR>(p, r, n, [&](int32_t e) {
            const int32_t c = ci[e];
            return (LOWER ? c < r : c > r) ? lu[e] * y[c] : 0.0;
        });
        if (sub == 0 && r < n) y_new[r] = LOWER ? b[r] - acc : (b[r] - acc) / lu[diag[r]];
    }
}

__global__ void k_div_diag(int64_t n, const double* __restrict__ lu, const int32_t* __restrict__ diag,
                           const double* __restrict__ b, double* __restrict__ z) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
        z[r] = b[r] / lu[diag[r]];
}

}  // namespace

struct Ilu0 {
    int64_t n = 0, nnz = 0;
    int tri_sweeps = 3;
    DBuf<int32_t> p, ci, diag;
    DBuf<double> lu, y0, y1;
    double shift = 0.0;
};

void* ilu0_create(const up3d_csr* A, int sweeps, int tri_sweeps, cudaStream_t s) {
    UP3D_REQUIRE(A && A->indptr && A->indices && A->data && A->n > 0, UP3D_ERR_ARGUMENT, "up3d_precond_ilu0: bad CSR");
    UP3D_REQUIRE(sweeps >= 1 && sweeps <= 100 && tri_sweeps >= 1 && tri_sweeps <= 100, UP3D_ERR_VALUE,
                 "up3d_precond_ilu0: sweeps and tri_sweeps must be in [1, 100]");
    auto* F = new Ilu0();
    const int64_t n = A->n;
    int32_t nnz32 = 0;
    UP3D_CUDA(cudaMemcpyAsync(&nnz32, A->indptr + n, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    UP3D_CUDA(cudaStreamSynchronize(s));
    const int64_t nnz = nnz32;
    F->n = n;
    F->nnz = nnz;
    F->tri_sweeps = tri_sweeps;
    F->p.alloc(n + 1);
    F->ci.alloc(nnz);
    F->diag.alloc(n);
    F->lu.alloc(nnz);
    F->y0.alloc(n);
    F->y1.alloc(n);
    UP3D_CUDA(cudaMemcpyAsync(F->p.get(), A->indptr, sizeof(int32_t) * (n + 1), cudaMemcpyDeviceToDevice, s));
    UP3D_CUDA(cudaMemcpyAsync(F->ci.get(), A->indices, sizeof(int32_t) * nnz, cudaMemcpyDeviceToDevice, s));
    DBuf<int32_t> row;
    DBuf<double> other, scal;
    DBuf<int> flag;
    row.alloc(nnz);
    other.alloc(nnz);
    scal.alloc(1);
    flag.alloc(1);
    k_row_of<<<grid_for(n, 256), 256, 0, s>>>(n, A->indptr, row.get());
    k_diag_pos<<<grid_for(n, 256), 256, 0, s>>>(n, A->indptr, A->indices, F->diag.get());
    UP3D_CHECK_LAUNCH();
    // every row needs its diagonal in the pattern
    {
        std::vector<int32_t> d(n);
        UP3D_CUDA(cudaMemcpyAsync(d.data(), F->diag.get(), sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s));
        UP3D_CUDA(cudaStreamSynchronize(s));
        for (int64_t r = 0; r < n; ++r)
            UP3D_REQUIRE(d[r] >= 0, UP3D_ERR_VALUE, "up3d_precond_ilu0: a row has no diagonal entry");
    }
    for (int attempt = 0; attempt < 2; ++attempt) {
        double shift = 0.0;
        if (attempt == 1) {
            k_abs_diag_sum<<<1, 256, 0, s>>>(n, A->data, F->diag.get(), A->dirichlet, scal.get());
            UP3D_CHECK_LAUNCH();
            double sum = 0.0;
            UP3D_CUDA(cudaMemcpyAsync(&sum, scal.get(), sizeof(double), cudaMemcpyDeviceToHost, s));
            UP3D_CUDA(cudaStreamSynchronize(s));
            const double mean = sum / (double)n;
            shift = 1e-3 * (mean > 0.0 ? mean : 1.0);
        }
        double* cur = F->lu.get();
        double* nxt = other.get();
        k_ilu_init<<<grid_for(nnz, 256), 256, 0, s>>>(nnz, row.get(), A->indices, A->data, A->dirichlet,
                                                      F->diag.get(), shift, cur);
        UP3D_CHECK_LAUNCH();
        for (int k = 0; k < sweeps; ++k) {
            k_ilu_sweep<<<grid_for(nnz, 256), 256, 0, s>>>(nnz, A->indptr, row.get(), A->indices, A->data,
                                                           A->dirichlet, F->diag.get(), shift, cur, nxt);
            UP3D_CHECK_LAUNCH();
            std::swap(cur, nxt);
        }
        if (cur != F->lu.get())
            UP3D_CUDA(cudaMemcpyAsync(F->lu.get(), cur, sizeof(double) * nnz, cudaMemcpyDeviceToDevice, s));
        UP3D_CUDA(cudaMemsetAsync(flag.get(), 0, sizeof(int), s));
        k_nonfinite<<<grid_for(nnz, 256), 256, 0, s>>>(nnz, F->lu.get(), flag.get());
        UP3D_CHECK_LAUNCH();
        int bad = 0;
        UP3D_CUDA(cudaMemcpyAsync(&bad, flag.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
        UP3D_CUDA(cudaStreamSynchronize(s));
        F->shift = shift;
        if (!bad) return F;
    }
    delete F;
    UP3D_REQUIRE(false, UP3D_ERR_RUNTIME, "up3d_precond_ilu0: the factorisation is not finite, even shifted");
    return nullptr;
}

void ilu0_destroy(void* f) { delete static_cast<Ilu0*>(f); }

void ilu0_factors(const void* f, double* out, double* shift, cudaStream_t s) {
    auto* F = static_cast<const Ilu0*>(f);
    if (out) UP3D_CUDA(cudaMemcpyAsync(out, F->lu.get(), sizeof(double) * F->nnz, cudaMemcpyDeviceToDevice, s));
    if (shift) *shift = F->shift;
}

void ilu0_apply(void* f, const double* r, double* z, cudaStream_t s) {
    auto* F = static_cast<Ilu0*>(f);
    const int64_t n = F->n;
    const int m = F->tri_sweeps;
    const unsigned g4 = lanes_grid(n, 4);
    double* buf[2] = {F->y0.get(), F->y1.get()};
    // y = L^-1 r: iterates y_0 = r, y_j in buf[(j - 1) % 2]
    const double* y = r;
    for (int j = 1; j <= m; ++j) {
        double* out = buf[(j - 1) % 2];
        k_tri_sweep<true><<<g4, 256, 0, s>>>(n, F->p.get(), F->ci.get(), F->lu.get(), F->diag.get(), r, y, out);
        UP3D_CHECK_LAUNCH();
        y = out;
    }
    // z = U^-1 y: iterates x_0 = y / diag(U), x_j alternating between z and
    // the free buffer so that x_m lands in z
    double* spare = buf[m % 2];
    auto slot = [&](int j) { return ((m - j) % 2 == 0) ? z : spare; };
    k_div_diag<<<grid_for(n, 256), 256, 0, s>>>(n, F->lu.get(), F->diag.get(), y, slot(0));
    UP3D_CHECK_LAUNCH();
    for (int j = 1; j <= m; ++j) {
        k_tri_sweep<false><<<g4, 256, 0, s>>>(n, F->p.get(), F->ci.get(), F->lu.get(), F->diag.get(), y, slot(j - 1),
                                               slot(j));
        UP3D_CHECK_LAUNCH();
    }
}

}  // namespace up3d
