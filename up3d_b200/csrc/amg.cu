// Smoothed-aggregation AMG preconditioner of the up3d library (the
// reference's build_amg_preconditioner, solve/linear.py:61-81, which wraps
// pyamg.smoothed_aggregation_solver with its defaults).
//
// Setup (host, OpenMP): all off-diagonal connections strong (theta = 0),
// the three-pass standard aggregation, tentative prolongator T for the
// constant near-null-space vector, smoothed prolongator
// P = (I - omega D^-1 A) T with omega = (4/3) / rho(D^-1 A), Galerkin
// coarse operators R A P with R = P^T, down to at most `max_coarse`
// unknowns, where the operator is inverted densely in FP64.
//
// Cycle (device): V-cycle with damped-Jacobi pre/post smoothing
// (omega_s = (4/3) / rho(D^-1 A) per level), in FP64 or FP32 (mixed
// precision: level operators, smoothing, restriction and prolongation in
// FP32, the coarsest solve in FP64).  No atomics: bit-reproducible.
// Constrained (Dirichlet) rows of the finest operator are identity rows and
// belong to no aggregate.

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "internal.cuh"
#include "krylov.cuh"

namespace up3d {

namespace {

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

struct HostCSR {
    int64_t n = 0, m = 0;  // rows, cols
    std::vector<int32_t> p, i;
    std::vector<double> x;
};

// ------------------------------------------------------------ host setup

// Standard aggregation (three passes, node order).  agg[i] = -1 for nodes
// without strong connections (isolated / constrained).
int64_t standard_aggregation(const HostCSR& A, const std::vector<uint8_t>& skip, std::vector<int32_t>& agg) {
    const int64_t n = A.n;
    agg.assign(n, -1);
    int64_t na = 0;
    auto strong = [&](int64_t r, int32_t c) { return c != r && !skip[c]; };
    // pass 1: node whose strong neighbours are all free seeds an aggregate
    for (int64_t r = 0; r < n; ++r) {
        if (skip[r] || agg[r] >= 0) continue;
        bool free_nbhd = true, has_nbr = false;
        for (int32_t k = A.p[r]; k < A.p[r + 1]; ++k) {
            int32_t c = A.i[k];
            if (!strong(r, c)) continue;
            has_nbr = true;
            if (agg[c] >= 0) {
                free_nbhd = false;
                break;
            }
        }
        if (!has_nbr || !free_nbhd) continue;
        agg[r] = (int32_t)na;
        for (int32_t k = A.p[r]; k < A.p[r + 1]; ++k) {
            int32_t c = A.i[k];
            if (strong(r, c)) agg[c] = (int32_t)na;
        }
        ++na;
    }
    // pass 2: join an aggregated strong neighbour (first in row order)
    std::vector<int32_t> agg1 = agg;
    for (int64_t r = 0; r < n; ++r) {
        if (skip[r] || agg[r] >= 0) continue;
        for (int32_t k = A.p[r]; k < A.p[r + 1]; ++k) {
            int32_t c = A.i[k];
            if (strong(r, c) && agg1[c] >= 0) {
                agg[r] = agg1[c];
                break;
            }
        }
    }
    // pass 3: leftovers seed aggregates with their free strong neighbours
    for (int64_t r = 0; r < n; ++r) {
        if (skip[r] || agg[r] >= 0) continue;
        bool has_nbr = false;
        for (int32_t k = A.p[r]; k < A.p[r + 1]; ++k)
            if (strong(r, A.i[k])) has_nbr = true;
        if (!has_nbr) continue;
        agg[r] = (int32_t)na;
        for (int32_t k = A.p[r]; k < A.p[r + 1]; ++k) {
            int32_t c = A.i[k];
            if (strong(r, c) && agg[c] < 0) agg[c] = (int32_t)na;
        }
        ++na;
    }
    return na;
}

void host_spmv(const HostCSR& A, const std::vector<double>& x, std::vector<double>& y) {
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < A.n; ++r) {
        double s = 0.0;
        for (int32_t k = A.p[r]; k < A.p[r + 1]; ++k) s += A.x[k] * x[A.i[k]];
        y[r] = s;
    }
}

// rho(D^-1 A) by power iteration on the symmetric scaling D^-1/2 A D^-1/2.
double spectral_radius(const HostCSR& A, const std::vector<double>& dinv, const std::vector<uint8_t>& skip) {
    const int64_t n = A.n;
    std::vector<double> x(n), y(n), s(n);
    for (int64_t r = 0; r < n; ++r) s[r] = std::sqrt(std::fabs(dinv[r]));
    uint64_t h = 0x9E3779B97F4A7C15ull;
    for (int64_t r = 0; r < n; ++r) {
        h ^= h << 13;
        h ^= h >> 7;
        h ^= h << 17;
        x[r] = skip[r] ? 0.0 : 0.5 + (double)(h % 1000003) / 1000003.0;
    }
    double lam = 0.0;
    for (int it = 0; it < 20; ++it) {
        std::vector<double> xs(n);
        for (int64_t r = 0; r < n; ++r) xs[r] = s[r] * x[r];
        host_spmv(A, xs, y);
        double num = 0.0, den = 0.0;
        for (int64_t r = 0; r < n; ++r) {
            y[r] = skip[r] ? 0.0 : s[r] * y[r];
            num += y[r] * x[r];
            den += x[r] * x[r];
        }
        lam = den > 0 ? num / den : 0.0;
        double nrm = 0.0;
        for (int64_t r = 0; r < n; ++r) nrm += y[r] * y[r];
        nrm = std::sqrt(nrm);
        if (nrm == 0.0) break;
        for (int64_t r = 0; r < n; ++r) x[r] = y[r] / nrm;
    }
    return lam > 0 ? 1.05 * lam : 2.0;  // small safety margin on the Rayleigh quotient
}

// Smoothed prolongator P = (I - omega D^-1 A) T.
HostCSR smoothed_prolongator(const HostCSR& A, const std::vector<double>& dinv, const std::vector<int32_t>& agg,
                             int64_t na, double omega) {
    const int64_t n = A.n;
    std::vector<int32_t> size(na, 0);
    for (int64_t r = 0; r < n; ++r)
        if (agg[r] >= 0) size[agg[r]]++;
    std::vector<double> t(n, 0.0);
    for (int64_t r = 0; r < n; ++r)
        if (agg[r] >= 0) t[r] = 1.0 / std::sqrt((double)size[agg[r]]);
    HostCSR P;
    P.n = n;
    P.m = na;
    P.p.assign(n + 1, 0);
    std::vector<std::vector<std::pair<int32_t, double>>> rows(n);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t r = 0; r < n; ++r) {
        auto& row = rows[r];
        if (agg[r] >= 0) row.emplace_back(agg[r], t[r]);
        const double f = omega * dinv[r];
        for (int32_t k = A.p[r]; k < A.p[r + 1]; ++k) {
            int32_t c = A.i[k];
            if (agg[c] < 0) continue;
            row.emplace_back(agg[c], -f * A.x[k] * t[c]);
        }
        std::sort(row.begin(), row.end(),
                  [](const auto& a, const auto& b) { return a.first < b.first; });
        size_t w = 0;
        for (size_t q = 0; q < row.size(); ++q) {
            if (w > 0 && row[w - 1].first == row[q].first) row[w - 1].second += row[q].second;
            else row[w++] = row[q];
        }
        row.resize(w);
    }
    for (int64_t r = 0; r < n; ++r) P.p[r + 1] = P.p[r] + (int32_t)rows[r].size();
    P.i.resize(P.p[n]);
    P.x.resize(P.p[n]);
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n; ++r) {
        int32_t o = P.p[r];
        for (auto& e : rows[r]) {
            P.i[o] = e.first;
            P.x[o] = e.second;
            ++o;
        }
    }
    return P;
}

HostCSR transpose(const HostCSR& P) {
    HostCSR R;
    R.n = P.m;
    R.m = P.n;
    R.p.assign(R.n + 1, 0);
    for (int32_t c : P.i) R.p[c + 1]++;
    for (int64_t r = 0; r < R.n; ++r) R.p[r + 1] += R.p[r];
    R.i.resize(P.i.size());
    R.x.resize(P.x.size());
    std::vector<int32_t> cur(R.p.begin(), R.p.end() - 1);
    for (int64_t r = 0; r < P.n; ++r)
        for (int32_t k = P.p[r]; k < P.p[r + 1]; ++k) {
            int32_t c = P.i[k];
            R.i[cur[c]] = (int32_t)r;
            R.x[cur[c]] = P.x[k];
            ++cur[c];
        }
    return R;
}

// C = A B (Gustavson, sorted columns, OpenMP over rows).
HostCSR spgemm(const HostCSR& A, const HostCSR& B) {
    HostCSR C;
    C.n = A.n;
    C.m = B.m;
    C.p.assign(A.n + 1, 0);
    std::vector<std::vector<int32_t>> ci(A.n);
    std::vector<std::vector<double>> cx(A.n);
#pragma omp parallel
    {
        std::vector<double> acc(B.m, 0.0);
        std::vector<int32_t> mark(B.m, -1), cols;
#pragma omp for schedule(dynamic, 512)
        for (int64_t r = 0; r < A.n; ++r) {
            cols.clear();
            for (int32_t k = A.p[r]; k < A.p[r + 1]; ++k) {
                const int32_t a = A.i[k];
                const double av = A.x[k];
                for (int32_t q = B.p[a]; q < B.p[a + 1]; ++q) {
                    const int32_t c = B.i[q];
                    if (mark[c] != (int32_t)r) {
                        mark[c] = (int32_t)r;
                        acc[c] = 0.0;
                        cols.push_back(c);
                    }
                    acc[c] += av * B.x[q];
                }
            }
            std::sort(cols.begin(), cols.end());
            ci[r] = cols;
            cx[r].resize(cols.size());
            for (size_t q = 0; q < cols.size(); ++q) cx[r][q] = acc[cols[q]];
        }
    }
    for (int64_t r = 0; r < A.n; ++r) C.p[r + 1] = C.p[r] + (int32_t)ci[r].size();
    C.i.resize(C.p[A.n]);
    C.x.resize(C.p[A.n]);
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < A.n; ++r) {
        std::copy(ci[r].begin(), ci[r].end(), C.i.begin() + C.p[r]);
        std::copy(cx[r].begin(), cx[r].end(), C.x.begin() + C.p[r]);
    }
    return C;
}

// Dense inverse by Gauss-Jordan with partial pivoting (coarsest level).
bool dense_inverse(std::vector<double>& a, int64_t n, std::vector<double>& inv) {
    inv.assign(n * n, 0.0);
    for (int64_t r = 0; r < n; ++r) inv[r * n + r] = 1.0;
    for (int64_t c = 0; c < n; ++c) {
        int64_t piv = c;
        for (int64_t r = c + 1; r < n; ++r)
            if (std::fabs(a[r * n + c]) > std::fabs(a[piv * n + c])) piv = r;
        if (a[piv * n + c] == 0.0) return false;
        if (piv != c)
            for (int64_t k = 0; k < n; ++k) {
                std::swap(a[c * n + k], a[piv * n + k]);
                std::swap(inv[c * n + k], inv[piv * n + k]);
            }
        const double d = 1.0 / a[c * n + c];
        for (int64_t k = 0; k < n; ++k) {
            a[c * n + k] *= d;
            inv[c * n + k] *= d;
        }
#pragma omp parallel for schedule(static)
        for (int64_t r = 0; r < n; ++r) {
            if (r == c) continue;
            const double f = a[r * n + c];
            if (f == 0.0) continue;
            for (int64_t k = 0; k < n; ++k) {
                a[r * n + k] -= f * a[c * n + k];
                inv[r * n + k] -= f * inv[c * n + k];
            }
        }
    }
    return true;
}

// ------------------------------------------------------------ device kernels

template <class T>
__global__ void k_jacobi_first(const T* __restrict__ dinv, const T* __restrict__ b, T* __restrict__ x, T w,
                               int64_t n) {
    GRID_STRIDE(i, n) x[i] = w * dinv[i] * b[i];
}

// out = x + w D^-1 (b - A x)   (or, with RESID, out = b - A x)
template <class T, bool RESID>
__global__ void __launch_bounds__(256)
    k_jacobi_sweep(int64_t n, const int32_t* __restrict__ Ap, const int32_t* __restrict__ Ai,
                   const T* __restrict__ Ax, const T* __restrict__ dinv, const T* __restrict__ b,
                   const T* __restrict__ x, T* __restrict__ out, T w, const uint8_t* __restrict__ dir) {
    constexpr int TPR = 8, RPW = 32 / TPR;
    const int sub = threadIdx.x % TPR, group = (threadIdx.x & 31) / TPR;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = warp * RPW; base < n; base += n_warps * RPW) {
        const int64_t r = base + group;
        T acc = T(0);
        bool fixed = false;
        if (r < n) {
            fixed = dir && dir[r];
            if (!fixed)
                for (int32_t k = Ap[r] + sub; k < Ap[r + 1]; k += TPR) {
                    int32_t c = Ai[k];
                    if (!dir || !dir[c]) acc += Ax[k] * x[c];
                }
        }
#pragma unroll
        for (int o = TPR / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, TPR);
        if (sub == 0 && r < n) {
            T ax = fixed ? x[r] : acc;
            T res = b[r] - ax;
            out[r] = RESID ? res : x[r] + w * dinv[r] * res;
        }
    }
}

// y (+)= A x, rectangular (restriction / prolongation)
template <class T, bool ADD>
__global__ void __launch_bounds__(256)
    k_spmv_rect(int64_t n, const int32_t* __restrict__ Ap, const int32_t* __restrict__ Ai, const T* __restrict__ Ax,
                const T* __restrict__ x, T* __restrict__ y) {
    constexpr int TPR = 8, RPW = 32 / TPR;
    const int sub = threadIdx.x % TPR, group = (threadIdx.x & 31) / TPR;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = warp * RPW; base < n; base += n_warps * RPW) {
        const int64_t r = base + group;
        T acc = T(0);
        if (r < n)
            for (int32_t k = Ap[r] + sub; k < Ap[r + 1]; k += TPR) acc += Ax[k] * x[Ai[k]];
#pragma unroll
        for (int o = TPR / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, TPR);
        if (sub == 0 && r < n) y[r] = ADD ? y[r] + acc : acc;
    }
}

// x = Cinv b (dense, one warp per row), FP64, inputs/outputs of type T
template <class T>
__global__ void k_dense_solve(const double* __restrict__ Cinv, int64_t n, const T* __restrict__ b,
                              T* __restrict__ x) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = warp; r < n; r += n_warps) {
        double acc = 0.0;
        for (int64_t c = lane; c < n; c += 32) acc += Cinv[r * n + c] * (double)b[c];
        acc = warp_sum(acc);
        if (lane == 0) x[r] = (T)acc;
    }
}

__global__ void k_d2f(const double* __restrict__ a, float* __restrict__ b, int64_t n) {
    GRID_STRIDE(i, n) b[i] = (float)a[i];
}
__global__ void k_f2d(const float* __restrict__ a, double* __restrict__ b, int64_t n) {
    GRID_STRIDE(i, n) b[i] = (double)a[i];
}

template <class T>
struct DevCSR {
    int64_t n = 0, m = 0, nnz = 0;
    DBuf<int32_t> p, i;
    DBuf<T> x;
    void upload(const HostCSR& h, cudaStream_t s) {
        n = h.n;
        m = h.m;
        nnz = (int64_t)h.i.size();
        p.alloc(n + 1);
        i.alloc(std::max<int64_t>(nnz, 1));
        x.alloc(std::max<int64_t>(nnz, 1));
        UP3D_CUDA(cudaMemcpyAsync(p.get(), h.p.data(), sizeof(int32_t) * (n + 1), cudaMemcpyHostToDevice, s));
        if (nnz) {
            UP3D_CUDA(cudaMemcpyAsync(i.get(), h.i.data(), sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, s));
            std::vector<T> v(h.x.begin(), h.x.end());
            UP3D_CUDA(cudaMemcpyAsync(x.get(), v.data(), sizeof(T) * nnz, cudaMemcpyHostToDevice, s));
            UP3D_CUDA(cudaStreamSynchronize(s));
        }
    }
};

template <class T>
struct Level {
    DevCSR<T> A, P, R;
    DBuf<T> dinv, x, b, r;
    T w_smooth = T(0);
    const uint8_t* dir = nullptr;  // finest level only
};

}  // namespace

struct Amg {
    bool fp32 = false;
    int pre = 2, post = 2;
    int64_t n_coarse = 0;
    DBuf<double> cinv;
    std::vector<Level<double>*> Ld;
    std::vector<Level<float>*> Lf;
    DBuf<float> in_f, out_f;
    DBuf<double> bc_d, xc_d;
    up3d_amg_info info{};
    ~Amg() {
        for (auto* l : Ld) delete l;
        for (auto* l : Lf) delete l;
    }
};

namespace {

template <class T>
void vcycle(Amg& a, std::vector<Level<T>*>& L, size_t l, cudaStream_t s) {
    Level<T>& lv = *L[l];
    const int64_t n = lv.A.n;
    if (l + 1 == L.size()) {
        // coarsest: dense FP64 solve
        if (std::is_same<T, double>::value) {
            k_dense_solve<T><<<grid_for(32 * n, 256), 256, 0, s>>>(a.cinv.get(), n, lv.b.get(), lv.x.get());
        } else {
            k_dense_solve<T><<<grid_for(32 * n, 256), 256, 0, s>>>(a.cinv.get(), n, lv.b.get(), lv.x.get());
        }
        UP3D_CHECK_LAUNCH();
        return;
    }
    const unsigned g1 = grid_for(n, 256), g8 = grid_for(8 * n, 256, (int64_t)148 * 64);
    // pre-smoothing from x = 0
    k_jacobi_first<T><<<g1, 256, 0, s>>>(lv.dinv.get(), lv.b.get(), lv.x.get(), lv.w_smooth, n);
    UP3D_CHECK_LAUNCH();
    for (int k = 1; k < a.pre; ++k) {
        k_jacobi_sweep<T, false><<<g8, 256, 0, s>>>(n, lv.A.p.get(), lv.A.i.get(), lv.A.x.get(), lv.dinv.get(),
                                                    lv.b.get(), lv.x.get(), lv.r.get(), lv.w_smooth, lv.dir);
        UP3D_CHECK_LAUNCH();
        std::swap(lv.x.p, lv.r.p);
    }
    // residual, restriction
    k_jacobi_sweep<T, true><<<g8, 256, 0, s>>>(n, lv.A.p.get(), lv.A.i.get(), lv.A.x.get(), lv.dinv.get(),
                                               lv.b.get(), lv.x.get(), lv.r.get(), lv.w_smooth, lv.dir);
    UP3D_CHECK_LAUNCH();
    Level<T>& cv = *L[l + 1];
    k_spmv_rect<T, false><<<grid_for(8 * cv.A.n, 256, (int64_t)148 * 64), 256, 0, s>>>(
        lv.R.n, lv.R.p.get(), lv.R.i.get(), lv.R.x.get(), lv.r.get(), cv.b.get());
    UP3D_CHECK_LAUNCH();
    vcycle<T>(a, L, l + 1, s);
    // prolongation
    k_spmv_rect<T, true><<<g8, 256, 0, s>>>(lv.P.n, lv.P.p.get(), lv.P.i.get(), lv.P.x.get(), cv.x.get(),
                                            lv.x.get());
    UP3D_CHECK_LAUNCH();
    for (int k = 0; k < a.post; ++k) {
        k_jacobi_sweep<T, false><<<g8, 256, 0, s>>>(n, lv.A.p.get(), lv.A.i.get(), lv.A.x.get(), lv.dinv.get(),
                                                    lv.b.get(), lv.x.get(), lv.r.get(), lv.w_smooth, lv.dir);
        UP3D_CHECK_LAUNCH();
        std::swap(lv.x.p, lv.r.p);
    }
}

template <class T>
void upload_levels(Amg& a, std::vector<Level<T>*>& L, const std::vector<HostCSR>& As, const std::vector<HostCSR>& Ps,
                   const std::vector<std::vector<double>>& dinvs, const std::vector<double>& wsm,
                   const uint8_t* dir_dev, cudaStream_t s) {
    for (size_t l = 0; l < As.size(); ++l) {
        auto* lv = new Level<T>();
        lv->A.upload(As[l], s);
        const int64_t n = As[l].n;
        lv->x.alloc(n);
        lv->b.alloc(n);
        lv->r.alloc(n);
        if (l < Ps.size()) {
            lv->P.upload(Ps[l], s);
            lv->R.upload(transpose(Ps[l]), s);
            lv->dinv.alloc(n);
            std::vector<T> d(dinvs[l].begin(), dinvs[l].end());
            UP3D_CUDA(cudaMemcpyAsync(lv->dinv.get(), d.data(), sizeof(T) * n, cudaMemcpyHostToDevice, s));
            UP3D_CUDA(cudaStreamSynchronize(s));
            lv->w_smooth = (T)wsm[l];
        }
        if (l == 0) lv->dir = dir_dev;
        L.push_back(lv);
    }
}

}  // namespace

void amg_apply(void* p, const double* r, double* z, cudaStream_t s) {
    Amg& a = *static_cast<Amg*>(p);
    if (!a.fp32) {
        Level<double>& f = *a.Ld[0];
        const int64_t n = f.A.n;
        UP3D_CUDA(cudaMemcpyAsync(f.b.get(), r, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        vcycle<double>(a, a.Ld, 0, s);
        UP3D_CUDA(cudaMemcpyAsync(z, f.x.get(), sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    } else {
        Level<float>& f = *a.Lf[0];
        const int64_t n = f.A.n;
        k_d2f<<<grid_for(n, 256), 256, 0, s>>>(r, f.b.get(), n);
        UP3D_CHECK_LAUNCH();
        vcycle<float>(a, a.Lf, 0, s);
        k_f2d<<<grid_for(n, 256), 256, 0, s>>>(f.x.get(), z, n);
        UP3D_CHECK_LAUNCH();
    }
}

void amg_destroy(void* p) { delete static_cast<Amg*>(p); }

// Builds the hierarchy for `A` (device CSR); the finest operator's
// constrained rows (A->dirichlet) are identity rows.
void* amg_setup(const up3d_csr& A, const up3d_amg_options& opt, cudaStream_t s) {
    auto* a = new Amg();
    try {
        a->fp32 = opt.fp32 != 0;
        a->pre = std::max(1, opt.presmooth);
        a->post = std::max(0, opt.postsmooth);
        const int64_t n = A.n;
        HostCSR h;
        h.n = h.m = n;
        h.p.resize(n + 1);
        UP3D_CUDA(cudaMemcpyAsync(h.p.data(), A.indptr, sizeof(int32_t) * (n + 1), cudaMemcpyDeviceToHost, s));
        UP3D_CUDA(cudaStreamSynchronize(s));
        const int64_t nnz = h.p[n];
        h.i.resize(nnz);
        h.x.resize(nnz);
        UP3D_CUDA(cudaMemcpyAsync(h.i.data(), A.indices, sizeof(int32_t) * nnz, cudaMemcpyDeviceToHost, s));
        UP3D_CUDA(cudaMemcpyAsync(h.x.data(), A.data, sizeof(double) * nnz, cudaMemcpyDeviceToHost, s));
        std::vector<uint8_t> skip(n, 0);
        if (A.dirichlet)
            UP3D_CUDA(cudaMemcpyAsync(skip.data(), A.dirichlet, n, cudaMemcpyDeviceToHost, s));
        UP3D_CUDA(cudaStreamSynchronize(s));
        // finest operator as the embedded free-DOF system: identity rows,
        // constrained columns dropped
        if (A.dirichlet) {
            HostCSR e;
            e.n = e.m = n;
            e.p.assign(n + 1, 0);
            for (int64_t r = 0; r < n; ++r) {
                int32_t cnt = 0;
                if (skip[r]) cnt = 1;
                else
                    for (int32_t k = h.p[r]; k < h.p[r + 1]; ++k) cnt += !skip[h.i[k]];
                e.p[r + 1] = e.p[r] + cnt;
            }
            e.i.resize(e.p[n]);
            e.x.resize(e.p[n]);
            for (int64_t r = 0; r < n; ++r) {
                int32_t o = e.p[r];
                if (skip[r]) {
                    e.i[o] = (int32_t)r;
                    e.x[o] = 1.0;
                    continue;
                }
                for (int32_t k = h.p[r]; k < h.p[r + 1]; ++k)
                    if (!skip[h.i[k]]) {
                        e.i[o] = h.i[k];
                        e.x[o] = h.x[k];
                        ++o;
                    }
            }
            h = std::move(e);
        }
        std::vector<HostCSR> As, Ps;
        std::vector<std::vector<double>> dinvs;
        std::vector<double> wsm;
        As.push_back(std::move(h));
        std::vector<uint8_t> cur_skip = skip;
        const int64_t max_coarse = std::max<int64_t>(opt.max_coarse, 1);
        while (As.back().n > max_coarse && (int)As.size() < std::max(2, opt.max_levels)) {
            const HostCSR& Al = As.back();
            std::vector<double> dinv(Al.n, 1.0);
            for (int64_t r = 0; r < Al.n; ++r)
                for (int32_t k = Al.p[r]; k < Al.p[r + 1]; ++k)
                    if (Al.i[k] == r && Al.x[k] != 0.0) dinv[r] = 1.0 / Al.x[k];
            const double rho = spectral_radius(Al, dinv, cur_skip);
            std::vector<int32_t> agg;
            const int64_t na = standard_aggregation(Al, cur_skip, agg);
            if (na == 0 || na >= Al.n) break;
            HostCSR P = smoothed_prolongator(Al, dinv, agg, na, (4.0 / 3.0) / rho);
            HostCSR AP = spgemm(Al, P);
            HostCSR Ac = spgemm(transpose(P), AP);
            dinvs.push_back(std::move(dinv));
            wsm.push_back((4.0 / 3.0) / rho);
            Ps.push_back(std::move(P));
            As.push_back(std::move(Ac));
            cur_skip.assign(As.back().n, 0);
        }
        // coarsest dense inverse (FP64)
        const HostCSR& Ac = As.back();
        const int64_t nc = Ac.n;
        UP3D_REQUIRE(nc <= 8192, UP3D_ERR_RUNTIME, "AMG coarsest level too large for the dense solve");
        std::vector<double> dense(nc * nc, 0.0), inv;
        for (int64_t r = 0; r < nc; ++r)
            for (int32_t k = Ac.p[r]; k < Ac.p[r + 1]; ++k) dense[r * nc + Ac.i[k]] = Ac.x[k];
        if (!dense_inverse(dense, nc, inv)) {
            // singular coarse operator (e.g. pure-Neumann): regularise the diagonal
            dense.assign(nc * nc, 0.0);
            double dmax = 0.0;
            for (int64_t r = 0; r < nc; ++r)
                for (int32_t k = Ac.p[r]; k < Ac.p[r + 1]; ++k) {
                    dense[r * nc + Ac.i[k]] = Ac.x[k];
                    if (Ac.i[k] == r) dmax = std::max(dmax, std::fabs(Ac.x[k]));
                }
            for (int64_t r = 0; r < nc; ++r) dense[r * nc + r] += 1e-12 * (dmax > 0 ? dmax : 1.0);
            UP3D_REQUIRE(dense_inverse(dense, nc, inv), UP3D_ERR_RUNTIME, "AMG coarsest operator is singular");
        }
        a->n_coarse = nc;
        a->cinv.alloc(nc * nc);
        UP3D_CUDA(cudaMemcpyAsync(a->cinv.get(), inv.data(), sizeof(double) * nc * nc, cudaMemcpyHostToDevice, s));
        UP3D_CUDA(cudaStreamSynchronize(s));
        if (a->fp32) upload_levels<float>(*a, a->Lf, As, Ps, dinvs, wsm, A.dirichlet, s);
        else upload_levels<double>(*a, a->Ld, As, Ps, dinvs, wsm, A.dirichlet, s);
        a->info.n_levels = (int32_t)As.size();
        int64_t tot = 0;
        for (auto& M : As) tot += (int64_t)M.i.size();
        a->info.operator_complexity = (double)tot / (double)std::max<size_t>(As[0].i.size(), 1);
        a->info.n_coarse = nc;
        for (size_t l = 0; l < As.size() && l < 16; ++l) a->info.level_rows[l] = As[l].n;
    } catch (...) {
        delete a;
        throw;
    }
    return a;
}

const up3d_amg_info* amg_info(void* p) { return &static_cast<Amg*>(p)->info; }

}  // namespace up3d

using namespace up3d;

extern "C" {

int up3d_amg_setup(const up3d_csr* A, const up3d_amg_options* opt, up3d_precond** out, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(A && out && A->indptr && A->indices && A->data, UP3D_ERR_ARGUMENT,
                     "up3d_amg_setup: null argument");
        up3d_amg_options o{10, 500, 2, 2, 0};
        if (opt) o = *opt;
        auto* M = new up3d_precond();
        M->kind = 2;
        M->n = A->n;
        try {
            M->amg = amg_setup(*A, o, S(stream));
        } catch (...) {
            delete M;
            throw;
        }
        *out = M;
    });
}

int up3d_amg_get_info(const up3d_precond* M, up3d_amg_info* info) {
    return guarded([&] {
        UP3D_REQUIRE(M && info && M->kind == 2 && M->amg, UP3D_ERR_ARGUMENT, "up3d_amg_get_info: not an AMG handle");
        *info = *amg_info(M->amg);
    });
}

}  // extern "C"
