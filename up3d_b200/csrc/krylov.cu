// Krylov solvers of the up3d library: preconditioned CG for the SPD Picard
// systems and restarted, left-preconditioned GMRES for the nonsymmetric
// Newton Jacobian (reference: solve/linear.py:134-239, which calls
// scipy.sparse.linalg.cg / gmres).
//
// Vectors live on the device; each iteration's scalars (dots, norms) are
// reduced on the device with a fixed two-pass tree (bit-reproducible) and
// read back once per iteration for the convergence test.  GMRES follows
// scipy's algorithm (left preconditioning, Givens rotations, adaptive inner
// tolerance, true-residual test after every cycle) with classical
// Gram-Schmidt applied twice (CGS2) in place of modified Gram-Schmidt, so
// each Arnoldi step is two batched multi-dot / multi-axpy passes.

#include <cmath>
#include <mutex>
#include <vector>

#include "internal.cuh"
#include "krylov.cuh"

namespace up3d {

namespace {

constexpr int RB = 256;      // reduction block
constexpr int RGRID = 592;   // fixed partial count (4 x 148 SMs): reproducible sums

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

// Called by every thread of every block after the block has written its
// partials: the last block to arrive sums partial[b * K + k] over b for
// each k into out (lanes stride b, then a warp sum: a fixed order)
// and re-arms the counter for the next launch on the stream.
__device__ __forceinline__ void last_block_finish(const double* partial, int nb, int K, double* out,
                                                  unsigned int* counter) {
    __shared__ bool last;
    const unsigned int blocks = gridDim.x * gridDim.y;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == blocks - 1u;
    __syncthreads();
    if (!last) return;
    __threadfence();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int k = w; k < K; k += nw) {
        double acc = 0.0;
        for (int b = lane; b < nb; b += 32) acc += __ldcg(partial + (int64_t)b * K + k);
        acc = warp_sum(acc);
        if (lane == 0) out[k] = acc;
    }
    if (threadIdx.x == 0) *counter = 0u;
}

// partial[b*K + k] = sum over block column b's slice of x_k . y (K vectors
// of V), MD_KT dot products per block: blockIdx.y picks the group of MD_KT
// vectors, so the groups run side by side instead of one after another in
// each block (y, read once per group, stays in L2).  Products and sums in
// FP64 whatever the vector type.
constexpr int MD_KT = 8;
template <class T>
__global__ void __launch_bounds__(RB)
    k_multidot(const T* __restrict__ V, int64_t ldv, int Kv, int K, const T* __restrict__ y, int64_t n,
               double* __restrict__ partial, double* __restrict__ out, unsigned int* __restrict__ counter) {
    __shared__ double sh[MD_KT][RB / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int k0 = blockIdx.y * MD_KT;
    const int kt = min(MD_KT, K - k0);
    double acc[MD_KT];
#pragma unroll
    for (int j = 0; j < MD_KT; ++j) acc[j] = 0.0;
    GRID_STRIDE(i, n) {
        const double yi = (double)y[i];
#pragma unroll
        for (int j = 0; j < MD_KT; ++j)
            if (j < kt) {
                const T* v = (k0 + j < Kv) ? V + (int64_t)(k0 + j) * ldv : y;
                acc[j] += (double)v[i] * yi;
            }
    }
#pragma unroll
    for (int j = 0; j < MD_KT; ++j) {
        const double v = warp_sum(acc[j]);
        if (lane == 0) sh[j][w] = v;
    }
    __syncthreads();
    if (threadIdx.x < kt) {
        double t = 0.0;
#pragma unroll
        for (int q = 0; q < RB / 32; ++q) t += sh[threadIdx.x][q];
        partial[(int64_t)blockIdx.x * K + k0 + threadIdx.x] = t;
    }
    last_block_finish(partial, (int)gridDim.x, K, out, counter);
}


// y -= sum_k h[k] V_k  (h on the device, staged in shared memory 64 at a
// time; k ascending for every element)
template <class T>
__global__ void __launch_bounds__(256)
    k_multiaxpy(const T* __restrict__ V, int64_t ldv, int K, const double* __restrict__ h, T* __restrict__ y,
                int64_t n) {
    __shared__ double hs[64];
    for (int c0 = 0; c0 < K; c0 += 64) {
        const int kc = min(64, K - c0);
        __syncthreads();
        if (threadIdx.x < kc) hs[threadIdx.x] = h[c0 + threadIdx.x];
        __syncthreads();
        GRID_STRIDE(i, n) {
            double acc = (double)y[i];
            const T* v = V + (int64_t)c0 * ldv + i;
#pragma unroll 8
            for (int k = 0; k < kc; ++k) acc -= hs[k] * (double)v[(int64_t)k * ldv];
            y[i] = (T)acc;
        }
    }
}

// The second and third passes of a CGS2 Arnoldi step, each one sweep over
// the basis: y -= sum_k h[k] V_k (K <= 64 vectors) tile by tile (one row
// per thread, 256-row tiles), then over the same tile, whose V values the
// update has just brought into cache, the partial dots V_k . y (DOTS) or
// y . y (NORM) of the new y: partial[b * P + k] with P = K (DOTS) or 1,
// one block's tiles in ascending order (reproducible sums).
constexpr int CG_TILE = 256;
template <class T, bool DOTS>
__global__ void __launch_bounds__(CG_TILE)
    k_axpy_dots(const T* __restrict__ V, int64_t ldv, int K, const double* __restrict__ h, T* __restrict__ y,
                int64_t n, double* __restrict__ partial, double* __restrict__ out, unsigned int* __restrict__ counter) {
    __shared__ double hs[64];
    __shared__ double ys[CG_TILE];
    __shared__ double acc_blk[64];
    __shared__ double wsum[CG_TILE / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x < K) hs[threadIdx.x] = h[threadIdx.x];
    if (threadIdx.x < 64) acc_blk[threadIdx.x] = 0.0;
    __syncthreads();
    for (int64_t tile = blockIdx.x; tile * CG_TILE < n; tile += gridDim.x) {
        const int64_t i0 = tile * CG_TILE;
        const int64_t i = i0 + threadIdx.x;
        double yi = 0.0;
        if (i < n) {
            double a = (double)y[i];
            const T* v = V + i;
#pragma unroll 8
            for (int k = 0; k < K; ++k) a -= hs[k] * (double)v[(int64_t)k * ldv];
            const T r = (T)a;
            y[i] = r;
            yi = (double)r;
        }
        if (DOTS) {
            ys[threadIdx.x] = yi;
            __syncthreads();
            const int rows = n - i0 < CG_TILE ? (int)(n - i0) : CG_TILE;
            for (int k = warp; k < K; k += CG_TILE / 32) {
                const T* v = V + (int64_t)k * ldv + i0;
                double d = 0.0;
#pragma unroll
                for (int m = 0; m < CG_TILE / 32; ++m) {
                    const int r = lane + 32 * m;
                    if (r < rows) d += (double)v[r] * ys[r];
                }
                d = warp_sum(d);
                if (lane == 0) acc_blk[k] += d;
            }
            __syncthreads();
        } else {
            const double d = warp_sum(yi * yi);
            if (lane == 0) wsum[warp] = d;
            __syncthreads();
            if (threadIdx.x == 0) {
                double t = 0.0;
#pragma unroll
                for (int q = 0; q < CG_TILE / 32; ++q) t += wsum[q];
                acc_blk[0] += t;
            }
            __syncthreads();
        }
    }
    const int P = DOTS ? K : 1;
    if (threadIdx.x < P) partial[(int64_t)blockIdx.x * P + threadIdx.x] = acc_blk[threadIdx.x];
    last_block_finish(partial, (int)gridDim.x, P, out, counter);
}

__global__ void k_axpby(double a, const double* __restrict__ x, double b, double* __restrict__ y, int64_t n) {
    GRID_STRIDE(i, n) y[i] = a * x[i] + b * y[i];
}

template <class T>
__global__ void k_scale(T* __restrict__ x, double a, int64_t n) {
    GRID_STRIDE(i, n) x[i] = (T)((double)x[i] * a);
}

template <class T>
__global__ void k_sub(const T* __restrict__ b, const T* __restrict__ ax, T* __restrict__ r, int64_t n) {
    GRID_STRIDE(i, n) r[i] = b[i] - ax[i];
}

// a += b
template <class T>
__global__ void k_accumulate(T* __restrict__ a, const T* __restrict__ b, int64_t n) {
    GRID_STRIDE(i, n) a[i] += b[i];
}

// x += (double) d
__global__ void k_add_f32(double* __restrict__ x, const float* __restrict__ d, int64_t n) {
    GRID_STRIDE(i, n) x[i] += (double)d[i];
}

__global__ void k_to_f32(const double* __restrict__ a, float* __restrict__ b, int64_t n) {
    GRID_STRIDE(i, n) b[i] = (float)a[i];
}

// CG updates: x += alpha p, r -= alpha q (alpha = num/den from the device)
__global__ void k_cg_update(const double* __restrict__ sc, double* __restrict__ x, double* __restrict__ r,
                            const double* __restrict__ p, const double* __restrict__ q, int64_t n) {
    const double alpha = sc[0] / sc[1];
    GRID_STRIDE(i, n) {
        x[i] += alpha * p[i];
        r[i] -= alpha * q[i];
    }
}

// p = z + beta p (beta = rz_new / rz_old)
__global__ void k_cg_dir(const double* __restrict__ sc, const double* __restrict__ z, double* __restrict__ p,
                         int64_t n) {
    const double beta = sc[2] / sc[0];
    GRID_STRIDE(i, n) p[i] = z[i] + beta * p[i];
}

__global__ void k_jacobi_diag(int64_t n, const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices,
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

template <class T>
__global__ void k_mul(const double* __restrict__ a, const T* __restrict__ b, T* __restrict__ out, int64_t n) {
    GRID_STRIDE(i, n) out[i] = (T)(a[i] * (double)b[i]);
}

template <class T>
__global__ void k_mask(T* __restrict__ x, const uint8_t* __restrict__ dir, int64_t n) {
    GRID_STRIDE(i, n) if (dir[i]) x[i] = T(0);
}

__global__ void k_copy_scalar(const double* __restrict__ src, double* __restrict__ dst) { *dst = *src; }

}  // namespace

// ------------------------------------------------------------ Vec helper

Blas::Blas(cudaStream_t s) : s(s) {
    partial.alloc((size_t)std::max(RGRID, 148 * 8) * 64);
    scal.alloc(128);
    counter.alloc(1);
    UP3D_CUDA(cudaMemsetAsync(counter.get(), 0, sizeof(unsigned int), s));
    UP3D_CUDA(cudaMallocHost(&host, 128 * sizeof(double)));
}
Blas::~Blas() {
    if (host) cudaFreeHost(host);
}

template <class T>
void Blas::multidot(const T* V, int64_t ldv, int K, const T* y, int64_t n, double* out_dev, bool self_dot) {
    const int Ktot = K + (self_dot ? 1 : 0);
    for (int k0 = 0; k0 < Ktot; k0 += 64) {
        int kk = std::min(64, Ktot - k0);
        k_multidot<T><<<dim3(RGRID, (kk + MD_KT - 1) / MD_KT), RB, 0, s>>>(V + (int64_t)k0 * ldv, ldv, K - k0, kk, y,
                                                                          n, partial.get(), out_dev + k0,
                                                                          counter.get());
        UP3D_CHECK_LAUNCH();
    }
}

template <class T>
double Blas::dot(const T* x, const T* y, int64_t n) {
    multidot(x, 0, 1, y, n, scal.get());
    UP3D_CUDA(cudaMemcpyAsync(host, scal.get(), sizeof(double), cudaMemcpyDeviceToHost, s));
    UP3D_CUDA(cudaStreamSynchronize(s));
    return host[0];
}

template <class T>
double Blas::nrm2(const T* x, int64_t n) {
    return std::sqrt(dot(x, x, n));
}

void Blas::axpby(double a, const double* x, double b, double* y, int64_t n) {
    k_axpby<<<grid_for(n, 256), 256, 0, s>>>(a, x, b, y, n);
    UP3D_CHECK_LAUNCH();
}

template <class T>
void Blas::scale(T* x, double a, int64_t n) {
    k_scale<T><<<grid_for(n, 256), 256, 0, s>>>(x, a, n);
    UP3D_CHECK_LAUNCH();
}

template <class T>
void Blas::multiaxpy(const T* V, int64_t ldv, int K, const double* h_dev, T* y, int64_t n) {
    k_multiaxpy<T><<<grid_for(n, 256), 256, 0, s>>>(V, ldv, K, h_dev, y, n);
    UP3D_CHECK_LAUNCH();
}

template <class T>
void Blas::axpy_dots(const T* V, int64_t ldv, int K, const double* h_dev, T* y, int64_t n, bool dots,
                     double* out_dev) {
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + CG_TILE - 1) / CG_TILE, 148 * 8));
    if (dots)
        k_axpy_dots<T, true><<<grid, CG_TILE, 0, s>>>(V, ldv, K, h_dev, y, n, partial.get(), out_dev, counter.get());
    else
        k_axpy_dots<T, false><<<grid, CG_TILE, 0, s>>>(V, ldv, K, h_dev, y, n, partial.get(), out_dev, counter.get());
    UP3D_CHECK_LAUNCH();
}

#define UP3D_BLAS_INST(T)                                                                 \
    template void Blas::multidot<T>(const T*, int64_t, int, const T*, int64_t, double*, bool); \
    template double Blas::dot<T>(const T*, const T*, int64_t);                           \
    template double Blas::nrm2<T>(const T*, int64_t);                                    \
    template void Blas::scale<T>(T*, double, int64_t);                                   \
    template void Blas::multiaxpy<T>(const T*, int64_t, int, const double*, T*, int64_t); \
    template void Blas::axpy_dots<T>(const T*, int64_t, int, const double*, T*, int64_t, bool, double*);
UP3D_BLAS_INST(double)
UP3D_BLAS_INST(float)
#undef UP3D_BLAS_INST

// ------------------------------------------------------------ solver workspaces

// Per-device Krylov workspaces, kept between solves so that a solve makes
// no device or pinned allocation once the buffers have grown to its size
// (cudaMalloc / cudaFree would synchronise the device on every call).  A
// solve holds its device's lock for its whole duration: concurrent solves
// on one device run one after the other.
struct KrylovWs {
    std::recursive_mutex mu;
    Blas* bl = nullptr;
    DBuf<double> d[8];
    DBuf<float> f[8];
    double* pin = nullptr;
    size_t pin_n = 0;
    double* pinned(size_t n) {
        if (n > pin_n) {
            if (pin) cudaFreeHost(pin);
            pin = nullptr;
            pin_n = 0;
            UP3D_CUDA(cudaMallocHost(&pin, sizeof(double) * n));
            pin_n = n;
        }
        return pin;
    }
    template <class T>
    DBuf<T>* bufs();
};
template <>
DBuf<double>* KrylovWs::bufs<double>() {
    return d;
}
template <>
DBuf<float>* KrylovWs::bufs<float>() {
    return f;
}

KrylovWs& krylov_ws() {
    static KrylovWs ws[64];
    int dev = 0;
    UP3D_CUDA(cudaGetDevice(&dev));
    UP3D_REQUIRE(dev >= 0 && dev < 64, UP3D_ERR_RUNTIME, "device index out of range");
    return ws[dev];
}

Blas& ws_blas(KrylovWs& w, cudaStream_t s) {
    if (!w.bl) w.bl = new Blas(s);
    w.bl->s = s;
    return *w.bl;
}

// ------------------------------------------------------------ operators

void Operator::apply(const double* x, double* y, cudaStream_t s) const {
    if (coupled) {
        coupled_apply(coupled, A, extra, x, nullptr, y, nullptr, s);
        return;
    }
    // y = A x (+ extra x: the Term-3 entries outside the P1 pattern), one pass
    launch_spmv2<double>(A.n, A.indptr, A.indices, A.data, extra.indptr, extra.indices, extra.data, x, y,
                         A.dirichlet, s);
}

// FP32 operator: the FP32 copies of the values (data32, extra32).
void Operator::apply(const float* x, float* y, cudaStream_t s) const {
    UP3D_REQUIRE(!coupled, UP3D_ERR_ARGUMENT, "the coupled wake operator is FP64 only");
    UP3D_REQUIRE(data32 && (!extra.indptr || extra32), UP3D_ERR_ARGUMENT, "FP32 operator without FP32 values");
    launch_spmv2<float>(A.n, A.indptr, A.indices, data32, extra.indptr, extra.indices, extra32, x, y, A.dirichlet,
                        s);
}

}  // namespace up3d

// ------------------------------------------------------------ preconditioners

void up3d_precond::apply(const double* r, double* z, cudaStream_t s) {
    using namespace up3d;
    if (kind == 1) {
        k_mul<double><<<grid_for(n, 256), 256, 0, s>>>(dinv.get(), r, z, n);
        UP3D_CHECK_LAUNCH();
    } else if (kind == 2) {
        amg_apply(amg, r, z, s);
    } else if (kind == 3) {
        ilu0_apply(ilu, r, z, s);
    } else {
        UP3D_CUDA(cudaMemcpyAsync(z, r, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    }
}

void up3d_precond::apply(const float* r, float* z, cudaStream_t s) {
    using namespace up3d;
    if (kind == 1) {
        k_mul<float><<<grid_for(n, 256), 256, 0, s>>>(dinv.get(), r, z, n);
        UP3D_CHECK_LAUNCH();
    } else if (kind == 2) {
        amg_apply_f32(amg, r, z, s);
    } else if (kind == 3) {
        UP3D_REQUIRE(false, UP3D_ERR_NOT_IMPLEMENTED, "the ILU(0) preconditioner applies to FP64 vectors only");
    } else {
        UP3D_CUDA(cudaMemcpyAsync(z, r, sizeof(float) * n, cudaMemcpyDeviceToDevice, s));
    }
}

namespace up3d {

template <class T>
void precond_apply(up3d_precond* M, const T* r, T* z, int64_t n, cudaStream_t s) {
    if (M) {
        M->apply(r, z, s);
    } else {
        UP3D_CUDA(cudaMemcpyAsync(z, r, sizeof(T) * n, cudaMemcpyDeviceToDevice, s));
    }
}

// scipy-convention effective absolute tolerance: max(atol, rtol * ||b||)
static double eff_atol(double atol, double rtol, double bnrm) { return std::max(atol, rtol * bnrm); }

// ------------------------------------------------------------ CG

// scipy.sparse.linalg.cg (solve/linear.py:232, solve/picard.py:375-380):
// preconditioned CG, converged when ||r|| <= max(rtol ||b||, atol).
int cg_solve(const Operator& op, const double* b, double* x, double rtol, double atol, int maxiter, up3d_precond* M,
             int64_t* iters, double* resid, cudaStream_t s) {
    const int64_t n = op.rows();
    KrylovWs& W = krylov_ws();
    std::lock_guard<std::recursive_mutex> lock(W.mu);
    Blas& bl = ws_blas(W, s);
    DBuf<double>& r = W.d[0];
    DBuf<double>& z = W.d[1];
    DBuf<double>& p = W.d[2];
    DBuf<double>& q = W.d[3];
    DBuf<double>& sc = W.d[4];
    r.alloc(n);
    z.alloc(n);
    p.alloc(n);
    q.alloc(n);
    sc.alloc(4);
    const double bnrm = bl.nrm2(b, n);
    const double tol = eff_atol(atol, rtol, bnrm);
    op.apply(x, q.get(), s);
    k_sub<double><<<grid_for(n, 256), 256, 0, s>>>(b, q.get(), r.get(), n);
    UP3D_CHECK_LAUNCH();
    double rn = bl.nrm2(r.get(), n);
    int64_t it = 0;
    if (bnrm == 0.0) {
        UP3D_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, s));
        rn = 0.0;
    }
    if (rn > tol) {
        precond_apply(M, r.get(), z.get(), n, s);
        UP3D_CUDA(cudaMemcpyAsync(p.get(), z.get(), sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        bl.multidot(r.get(), 0, 1, z.get(), n, sc.get() + 0);  // rz
        for (it = 1; it <= maxiter; ++it) {
            op.apply(p.get(), q.get(), s);
            bl.multidot(p.get(), 0, 1, q.get(), n, sc.get() + 1);  // pq
            k_cg_update<<<grid_for(n, 256), 256, 0, s>>>(sc.get(), x, r.get(), p.get(), q.get(), n);
            UP3D_CHECK_LAUNCH();
            rn = bl.nrm2(r.get(), n);
            if (rn <= tol || !std::isfinite(rn)) break;
            precond_apply(M, r.get(), z.get(), n, s);
            bl.multidot(r.get(), 0, 1, z.get(), n, sc.get() + 2);  // rz_new
            k_cg_dir<<<grid_for(n, 256), 256, 0, s>>>(sc.get(), z.get(), p.get(), n);
            UP3D_CHECK_LAUNCH();
            k_copy_scalar<<<1, 1, 0, s>>>(sc.get() + 2, sc.get() + 0);
            UP3D_CHECK_LAUNCH();
        }
        if (it > maxiter) it = maxiter;
    }
    if (iters) *iters = it;
    if (resid) *resid = rn;
    return rn <= tol ? 0 : (int)maxiter;
}

// ------------------------------------------------------------ GMRES

// V_{col+1} *= 1 / |w| unless |w| <= eps |w_before| (Arnoldi breakdown);
// hn = (|w_before|^2, |w|^2)
template <class T>
__global__ void k_scale_unless_breakdown(const T* __restrict__ w, T* __restrict__ v, const double* __restrict__ hn,
                                         double eps, int64_t n) {
    const double h0 = sqrt(hn[0]), h1 = sqrt(hn[1]);
    const bool keep = h1 <= eps * h0;   // breakdown: the vector is copied unscaled
    const double f = keep ? 1.0 : 1.0 / h1;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        v[i] = keep ? w[i] : (T)((double)w[i] * f);
}

// Givens rotation as LAPACK xLARTG: c*f + s*g = r, -s*f + c*g = 0.
static void lartg(double f, double g, double& c, double& sn, double& r) {
    if (g == 0.0) {
        c = 1.0;
        sn = 0.0;
        r = f;
    } else if (f == 0.0) {
        c = 0.0;
        sn = g > 0 ? 1.0 : -1.0;
        r = std::fabs(g);
    } else {
        double d = std::sqrt(f * f + g * g);
        c = std::fabs(f) / d;
        r = f > 0 ? d : -d;
        sn = g / r;
    }
}

// scipy.sparse.linalg.gmres (solve/linear.py:182-201): restarted,
// left-preconditioned; `maxiter` counts restart cycles.
// T: the vector (and operator value) type -- double, or float for the inner
// solves of the mixed-precision refinement (dot products accumulate in
// FP64, the Hessenberg least-squares problem is FP64 on the host).
template <class T>
int gmres_solve(const Operator& op, const T* b, T* x, double rtol, double atol, int restart, int maxiter,
                up3d_precond* M, int64_t* inner, double* resid, cudaStream_t s) {
    const int64_t n = op.rows();
    KrylovWs& W = krylov_ws();
    std::lock_guard<std::recursive_mutex> lock(W.mu);
    Blas& bl = ws_blas(W, s);
    restart = (int)std::min<int64_t>(restart, n);
    DBuf<T>* B = W.bufs<T>();
    DBuf<T>& V = B[0];
    DBuf<T>& w = B[1];
    DBuf<T>& r = B[2];
    DBuf<T>& tmp = B[3];
    DBuf<double>& hdev = W.d[5];
    V.alloc((size_t)(restart + 1) * n);
    w.alloc(n);
    r.alloc(n);
    tmp.alloc(n);
    hdev.alloc(2 * restart + 6);
    double* hbuf = W.pinned(restart + 3);
    std::vector<double> H((size_t)restart * (restart + 1), 0.0), gc(restart), gs(restart), S(restart + 1);
    const double bnrm = bl.nrm2(b, n);
    double atol_eff = eff_atol(atol, rtol, bnrm);
    if (bnrm == 0.0) {
        UP3D_CUDA(cudaMemcpyAsync(x, b, sizeof(T) * n, cudaMemcpyDeviceToDevice, s));
        if (inner) *inner = 0;
        if (resid) *resid = 0.0;
        return 0;
    }
    const double eps = 2.220446049250313e-16;
    precond_apply(M, b, tmp.get(), n, s);
    const double Mb = bl.nrm2(tmp.get(), n);
    double ptol_max = 1.0;
    double ptol = Mb * std::min(ptol_max, atol_eff / bnrm);
    double presid = 0.0, rnorm = 0.0;
    int64_t total = 0;
    bool done = false;
    auto Hat = [&](int col, int k) -> double& { return H[(size_t)col * (restart + 1) + k]; };
    for (int cycle = 0; cycle < maxiter && !done; ++cycle) {
        if (cycle == 0) {
            op.apply(x, tmp.get(), s);
            k_sub<T><<<grid_for(n, 256), 256, 0, s>>>(b, tmp.get(), r.get(), n);
            UP3D_CHECK_LAUNCH();
            rnorm = bl.nrm2(r.get(), n);
            if (rnorm < atol_eff) {
                done = true;
                break;
            }
        }
        precond_apply(M, r.get(), V.get(), n, s);
        double beta = bl.nrm2(V.get(), n);
        bl.scale(V.get(), 1.0 / beta, n);
        std::fill(S.begin(), S.end(), 0.0);
        S[0] = beta;
        bool breakdown = false;
        int col = 0;
        for (col = 0; col < restart; ++col) {
            // one Arnoldi step on the device, one readback: the column
            // [h_0 .. h_col] (CGS2: two projections onto V_0..V_col, summed),
            // |w| before and after the projections
            // pass 1 takes V_0..V_col and the new vector itself in one
            // multidot (h and |w|^2), passes 2 and 3 are one sweep each
            // (update + the next pass's dots, update + |w|^2), and the
            // normalisation writes the vector into V[col + 1].  The
            // preconditioner's output stays the one buffer w, so its
            // captured V-cycle graph is replayed, not captured per column.
            double* hsum = hdev.get();                  // h_0..h_col, |w|^2 before, |w|^2 after
            double* hpass = hdev.get() + (restart + 3);
            double* hn = hsum + col + 1;
            T* wv = w.get();
            op.apply(V.get() + (size_t)col * n, tmp.get(), s);
            precond_apply(M, tmp.get(), wv, n, s);
            bl.multidot(V.get(), n, col + 1, wv, n, hsum, true);
            if (col + 1 <= 64) {
                bl.axpy_dots(V.get(), n, col + 1, hsum, wv, n, true, hpass);
                bl.axpy_dots(V.get(), n, col + 1, hpass, wv, n, false, hn + 1);
            } else {
                bl.multiaxpy(V.get(), n, col + 1, hsum, wv, n);
                bl.multidot(V.get(), n, col + 1, wv, n, hpass);
                bl.multiaxpy(V.get(), n, col + 1, hpass, wv, n);
                bl.multidot(wv, 0, 0, wv, n, hn + 1, true);
            }
            k_accumulate<double><<<1, 64, 0, s>>>(hsum, hpass, col + 1);
            UP3D_CHECK_LAUNCH();
            k_scale_unless_breakdown<T><<<grid_for(n, 256), 256, 0, s>>>(wv, V.get() + (size_t)(col + 1) * n, hn, eps, n);
            UP3D_CHECK_LAUNCH();
            UP3D_CUDA(cudaMemcpyAsync(hbuf, hsum, sizeof(double) * (col + 3), cudaMemcpyDeviceToHost, s));
            UP3D_CUDA(cudaStreamSynchronize(s));
            for (int k = 0; k <= col; ++k) Hat(col, k) = hbuf[k];
            const double h0 = std::sqrt(hbuf[col + 1]);
            const double h1 = std::sqrt(hbuf[col + 2]);
            Hat(col, col + 1) = h1;
            if (h1 <= eps * h0) {
                Hat(col, col + 1) = 0.0;
                breakdown = true;
            }
            for (int k = 0; k < col; ++k) {
                double c = gc[k], sn = gs[k];
                double n0 = Hat(col, k), n1 = Hat(col, k + 1);
                Hat(col, k) = c * n0 + sn * n1;
                Hat(col, k + 1) = -sn * n0 + c * n1;
            }
            double c, sn, mag;
            lartg(Hat(col, col), Hat(col, col + 1), c, sn, mag);
            gc[col] = c;
            gs[col] = sn;
            Hat(col, col) = mag;
            Hat(col, col + 1) = 0.0;
            double t = -sn * S[col];
            S[col] = c * S[col];
            S[col + 1] = t;
            presid = std::fabs(t);
            ++total;
            if (presid <= ptol || breakdown) break;
        }
        if (col == restart) col = restart - 1;
        if (Hat(col, col) == 0.0) S[col] = 0.0;
        std::vector<double> y(S.begin(), S.begin() + col + 1);
        for (int k = col; k > 0; --k) {
            if (y[k] != 0.0) {
                y[k] /= Hat(k, k);
                double tk = y[k];
                for (int j = 0; j < k; ++j) y[j] -= tk * Hat(k, j);
            }
        }
        if (y[0] != 0.0) y[0] /= Hat(0, 0);
        // x += V^T y  (as x -= V (-y))
        for (auto& v : y) v = -v;
        UP3D_CUDA(cudaMemcpyAsync(hdev.get(), y.data(), sizeof(double) * (col + 1), cudaMemcpyHostToDevice, s));
        bl.multiaxpy(V.get(), n, col + 1, hdev.get(), x, n);
        op.apply(x, tmp.get(), s);
        k_sub<T><<<grid_for(n, 256), 256, 0, s>>>(b, tmp.get(), r.get(), n);
        UP3D_CHECK_LAUNCH();
        rnorm = bl.nrm2(r.get(), n);
        if (rnorm <= atol_eff || breakdown || !std::isfinite(rnorm)) break;
        if (presid <= ptol) ptol_max = std::max(eps, 0.25 * ptol_max);
        else ptol_max = std::min(1.0, 1.5 * ptol_max);
        ptol = presid * std::min(ptol_max, atol_eff / rnorm);
    }
    if (inner) *inner = total;
    if (resid) *resid = rnorm;
    return rnorm <= atol_eff ? 0 : maxiter;
}

template int gmres_solve<double>(const Operator&, const double*, double*, double, double, int, int, up3d_precond*,
                                  int64_t*, double*, cudaStream_t);
template int gmres_solve<float>(const Operator&, const float*, float*, double, double, int, int, up3d_precond*,
                                 int64_t*, double*, cudaStream_t);

// Mixed-precision GMRES with FP64 iterative refinement.  The outer loop
// forms the true residual r = b - A x with the FP64 values and tests the
// criterion of gmres_solve: with a preconditioner, the preconditioned
// residual |M r| <= |M b| min(1, max(rtol, atol / |b|)) (M applied in FP32
// to r rounded to FP32), without one |r| <= max(rtol |b|, atol).  Each
// correction solves A d = r by restarted GMRES on the FP32 operator (data32,
// extra32) with FP32 vectors and M applied in FP32, to max(inner_rtol,
// tol / |M r|) relative, and is added to x in FP64.  A correction that fails
// to halve the tested residual hands the rest of the solve to FP64 GMRES
// from the current iterate.  The Arnoldi steps of all corrections (and of
// that FP64 finish) share one budget of restart x maxiter, the cap of one
// gmres_solve call, so a solve that cannot meet its tolerance costs what
// the FP64 solve would.  Returns 0 when converged; resid = |r|.
int gmres_ir_solve(const Operator& op, const double* b, double* x, double rtol, double atol, int restart,
                   int maxiter, int refine_max, double inner_rtol, up3d_precond* M, int64_t* inner, int64_t* outer,
                   double* resid, cudaStream_t s) {
    const int64_t n = op.rows();
    KrylovWs& W = krylov_ws();
    std::lock_guard<std::recursive_mutex> lock(W.mu);
    Blas& bl = ws_blas(W, s);
    DBuf<double>& r = W.d[6];
    DBuf<double>& tmp = W.d[7];
    DBuf<float>& r32 = W.f[6];
    DBuf<float>& d32 = W.f[7];
    r.alloc(n);
    tmp.alloc(n);
    r32.alloc(n);
    d32.alloc(n);
    restart = (int)std::max<int64_t>(1, std::min<int64_t>(restart, n));
    const int64_t budget = (int64_t)restart * maxiter;
    // |v| of an FP64 vector in the tested norm: preconditioned (through the
    // FP32 copy r32, which the correction then uses as its right-hand side)
    // or plain
    auto tested_norm = [&](const double* v) -> double {
        k_to_f32<<<grid_for(n, 256), 256, 0, s>>>(v, r32.get(), n);
        UP3D_CHECK_LAUNCH();
        if (!M) return bl.nrm2(v, n);
        precond_apply(M, r32.get(), d32.get(), n, s);
        return bl.nrm2(d32.get(), n);
    };
    const double bnrm = bl.nrm2(b, n);
    const double bt = tested_norm(b);
    const double tol = M ? bt * std::min(1.0, eff_atol(atol, rtol, bnrm) / std::max(bnrm, 1e-300))
                         : eff_atol(atol, rtol, bnrm);
    int64_t tot_inner = 0, it = 0;
    double rn = 0.0, rn_prev = 0.0, rtrue = 0.0;
    for (;; ++it) {
        op.apply(x, tmp.get(), s);
        k_sub<double><<<grid_for(n, 256), 256, 0, s>>>(b, tmp.get(), r.get(), n);
        UP3D_CHECK_LAUNCH();
        rn = tested_norm(r.get());
        rtrue = M ? bl.nrm2(r.get(), n) : rn;
        if (rn <= tol || !std::isfinite(rn) || it >= refine_max || tot_inner >= budget) break;
        const int cycles_left = (int)std::max<int64_t>(1, (budget - tot_inner + restart - 1) / restart);
        if (it > 0 && rn > 0.5 * rn_prev) {
            // the FP32 corrections stopped paying (a system too ill-conditioned
            // for FP32): finish with FP64 GMRES from the current iterate
            int64_t inn = 0;
            double r64 = 0.0;
            gmres_solve<double>(op, b, x, rtol, atol, restart, cycles_left, M, &inn, &r64, s);
            tot_inner += inn;
            ++it;
            op.apply(x, tmp.get(), s);
            k_sub<double><<<grid_for(n, 256), 256, 0, s>>>(b, tmp.get(), r.get(), n);
            UP3D_CHECK_LAUNCH();
            rn = tested_norm(r.get());
            rtrue = M ? bl.nrm2(r.get(), n) : rn;
            break;
        }
        rn_prev = rn;
        UP3D_CUDA(cudaMemsetAsync(d32.get(), 0, sizeof(float) * n, s));
        int64_t inn = 0;
        double ires = 0.0;
        gmres_solve<float>(op, r32.get(), d32.get(), std::max(inner_rtol, tol / rn), 0.0, restart, cycles_left, M,
                           &inn, &ires, s);
        tot_inner += inn;
        k_add_f32<<<grid_for(n, 256), 256, 0, s>>>(x, d32.get(), n);
        UP3D_CHECK_LAUNCH();
    }
    if (inner) *inner = tot_inner;
    if (outer) *outer = it;
    if (resid) *resid = rtrue;
    return rn <= tol ? 0 : maxiter;
}

}  // namespace up3d

using namespace up3d;

namespace {
void make_op(Operator& op, const up3d_csr* A, const up3d_csr* extra) {
    UP3D_REQUIRE(A && A->indptr && A->indices && A->data && A->n >= 0, UP3D_ERR_ARGUMENT, "bad CSR operand");
    op.A = *A;
    if (extra && extra->indptr) {
        UP3D_REQUIRE(extra->n == A->n, UP3D_ERR_ARGUMENT, "extra operand size mismatch");
        op.extra = *extra;
    }
}
}  // namespace

extern "C" {

int up3d_precond_ilu0(const up3d_csr* A, int sweeps, int tri_sweeps, up3d_precond** out, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(A && out, UP3D_ERR_ARGUMENT, "up3d_precond_ilu0: null argument");
        auto* M = new up3d_precond();
        M->kind = 3;
        M->n = A->n;
        try {
            M->ilu = ilu0_create(A, sweeps, tri_sweeps, S(stream));
        } catch (...) {
            delete M;
            throw;
        }
        *out = M;
    });
}

int up3d_precond_ilu0_factors(const up3d_precond* M, double* lu, double* shift, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(M && M->kind == 3 && M->ilu, UP3D_ERR_ARGUMENT, "up3d_precond_ilu0_factors: not an ILU(0) handle");
        ilu0_factors(M->ilu, lu, shift, S(stream));
    });
}

int up3d_precond_jacobi(const up3d_csr* A, up3d_precond** out, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(A && out, UP3D_ERR_ARGUMENT, "up3d_precond_jacobi: null argument");
        auto* M = new up3d_precond();
        M->kind = 1;
        M->n = A->n;
        M->dinv.alloc(A->n);
        k_jacobi_diag<<<grid_for(A->n, 256), 256, 0, S(stream)>>>(A->n, A->indptr, A->indices, A->data, A->dirichlet,
                                                                 M->dinv.get());
        UP3D_CHECK_LAUNCH();
        *out = M;
    });
}

int up3d_precond_apply(up3d_precond* M, const double* r, double* z, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(M && r && z, UP3D_ERR_ARGUMENT, "up3d_precond_apply: null argument");
        M->apply(r, z, S(stream));
    });
}

int up3d_amg_vcycle(up3d_precond* M, const double* r, double* z, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(M && r && z, UP3D_ERR_ARGUMENT, "up3d_amg_vcycle: null argument");
        UP3D_REQUIRE(M->kind == 2, UP3D_ERR_VALUE, "up3d_amg_vcycle: not an AMG hierarchy");
        M->apply(r, z, S(stream));
    });
}

int up3d_amg_vcycle_f32(up3d_precond* M, const float* r, float* z, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(M && r && z, UP3D_ERR_ARGUMENT, "up3d_amg_vcycle_f32: null argument");
        UP3D_REQUIRE(M->kind == 2, UP3D_ERR_VALUE, "up3d_amg_vcycle_f32: not an AMG hierarchy");
        M->apply(r, z, S(stream));
    });
}

int up3d_precond_destroy(up3d_precond* M) {
    return guarded([&] { delete M; });
}

int up3d_cg(const up3d_csr* A, const double* b, double* x, double rtol, double atol, int maxiter, up3d_precond* M,
            int64_t* iters, double* resid, int* info, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(b && x, UP3D_ERR_ARGUMENT, "up3d_cg: null argument");
        Operator op;
        make_op(op, A, nullptr);
        int inf = cg_solve(op, b, x, rtol, atol, maxiter, M, iters, resid, S(stream));
        if (info) *info = inf;
    });
}

int up3d_gmres_ir(const up3d_csr* A, const up3d_csr* extra, const float* data32, const float* extra32,
                  const double* b, double* x, double rtol, double atol, int restart, int maxiter, int refine_max,
                  double inner_rtol, up3d_precond* M, int64_t* inner, int64_t* outer, double* resid, int* info,
                  up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(b && x && data32 && restart > 0 && maxiter > 0 && refine_max >= 0, UP3D_ERR_ARGUMENT,
                     "up3d_gmres_ir: bad argument");
        Operator op;
        make_op(op, A, extra);
        UP3D_REQUIRE(!op.extra.indptr || extra32, UP3D_ERR_ARGUMENT,
                     "up3d_gmres_ir: extra operand without FP32 values");
        op.data32 = data32;
        op.extra32 = extra32;
        int inf = gmres_ir_solve(op, b, x, rtol, atol, restart, maxiter, refine_max, inner_rtol, M, inner, outer,
                                 resid, S(stream));
        if (info) *info = inf;
    });
}

int up3d_gmres(const up3d_csr* A, const up3d_csr* extra, const double* b, double* x, double rtol, double atol,
               int restart, int maxiter, up3d_precond* M, int64_t* inner, double* resid, int* info,
               up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(b && x && restart > 0 && maxiter > 0, UP3D_ERR_ARGUMENT, "up3d_gmres: bad argument");
        Operator op;
        make_op(op, A, extra);
        int inf = gmres_solve(op, b, x, rtol, atol, restart, maxiter, M, inner, resid, S(stream));
        if (info) *info = inf;
    });
}

int up3d_gmres_coupled(const up3d_coupled* c, const up3d_csr* J, const up3d_csr* extra, const double* b,
                       double* x, double rtol, double atol, int restart, int maxiter, up3d_precond* M,
                       int64_t* inner, double* resid, int* info, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(c && b && x && restart > 0 && maxiter > 0, UP3D_ERR_ARGUMENT, "up3d_gmres_coupled: bad argument");
        Operator op;
        make_op(op, J, extra);
        op.coupled = c;
        UP3D_REQUIRE(!M || M->n == coupled_rows(c), UP3D_ERR_ARGUMENT,
                     "up3d_gmres_coupled: preconditioner size differs from the reduced system");
        int inf = gmres_solve(op, b, x, rtol, atol, restart, maxiter, M, inner, resid, S(stream));
        if (info) *info = inf;
    });
}

}  // extern "C"
