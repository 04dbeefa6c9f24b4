// Smoothed-aggregation AMG preconditioner of the up3d library (the
// reference's build_amg_preconditioner, solve/linear.py:61-81, which wraps
// pyamg.smoothed_aggregation_solver with its defaults).
//
// Setup, symbolic (host, once per sparsity pattern): all off-diagonal
// connections strong (theta = 0), the three-pass standard aggregation, and
// the patterns of the tentative prolongator T (constant near-null-space
// vector), the smoothed prolongator P = (I - omega D^-1 A) T, A P and the
// Galerkin operator R A P with R = P^T, down to at most `max_coarse`
// unknowns.  With every connection strong the aggregates and all patterns
// depend on the fine pattern alone.
//
// Setup, numeric (device, on every setup and refresh): D^-1, rho(D^-1 A) by
// power iteration, omega = (4/3) / rho, the values of P, A P and R A P in a
// fixed per-row order, and the dense FP64 inverse of the coarsest operator
// (Gauss-Jordan with partial pivoting).  A refresh with a new matrix of the
// same pattern therefore reproduces a fresh setup bit for bit.
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
#include <cstring>
#include <memory>
#include <mutex>
#include <numeric>
#include <vector>

#include "csr_rows.cuh"
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

// Host <-> device copies of the setup through one process-wide page-locked
// staging buffer (grown once, kept): pageable copies of the level patterns
// were a large part of the setup time.
struct Stage {
    std::mutex mu;
    unsigned char* p = nullptr;
    size_t n = 0;
};
Stage& stage() {
    static Stage st;
    return st;
}
constexpr size_t STAGE_CHUNK = size_t(32) << 20;
unsigned char* stage_buffer(Stage& st) {
    if (!st.p) {
        UP3D_CUDA(cudaMallocHost(&st.p, STAGE_CHUNK));
        st.n = STAGE_CHUNK;
    }
    return st.p;
}
// host memcpy spread over the OpenMP threads (1 MiB pieces): a single
// thread copies pageable memory at a fraction of the link's rate
void par_memcpy(unsigned char* dst, const unsigned char* src, size_t bytes) {
    constexpr size_t PIECE = size_t(1) << 20;
    const int64_t pieces = (int64_t)((bytes + PIECE - 1) / PIECE);
#pragma omp parallel for schedule(static) if (pieces > 1)
    for (int64_t k = 0; k < pieces; ++k) {
        const size_t o = (size_t)k * PIECE;
        std::memcpy(dst + o, src + o, std::min(PIECE, bytes - o));
    }
}
void h2d(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    Stage& st = stage();
    std::lock_guard<std::mutex> g(st.mu);
    unsigned char* buf = stage_buffer(st);
    for (size_t o = 0; o < bytes; o += STAGE_CHUNK) {
        const size_t b = std::min(STAGE_CHUNK, bytes - o);
        par_memcpy(buf, static_cast<const unsigned char*>(src) + o, b);
        UP3D_CUDA(cudaMemcpyAsync(static_cast<unsigned char*>(dst) + o, buf, b, cudaMemcpyHostToDevice, s));
        UP3D_CUDA(cudaStreamSynchronize(s));
    }
}
void d2h(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    Stage& st = stage();
    std::lock_guard<std::mutex> g(st.mu);
    unsigned char* buf = stage_buffer(st);
    for (size_t o = 0; o < bytes; o += STAGE_CHUNK) {
        const size_t b = std::min(STAGE_CHUNK, bytes - o);
        UP3D_CUDA(cudaMemcpyAsync(buf, static_cast<const unsigned char*>(src) + o, b, cudaMemcpyDeviceToHost, s));
        UP3D_CUDA(cudaStreamSynchronize(s));
        par_memcpy(static_cast<unsigned char*>(dst) + o, buf, b);
    }
}

// ------------------------------------------------------------ host symbolic setup

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

int32_t find_col(const HostCSR& P, int64_t r, int32_t c) {
    auto b = P.i.begin() + P.p[r], e = P.i.begin() + P.p[r + 1];
    auto it = std::lower_bound(b, e, c);
    return (it != e && *it == c) ? (int32_t)(it - P.i.begin()) : -1;
}

// Pattern of P = (I - omega D^-1 A) T: row r holds agg[r] and agg[c] of its
// aggregated neighbours.  amap[k] = slot of A entry k's contribution (-1 when
// its column is unaggregated), self[r] = slot of agg[r] (-1 when none).
// Two passes (count, fill) with a per-thread marker array: no per-row
// allocation.
HostCSR prolongator_pattern(const HostCSR& A, const std::vector<int32_t>& agg, int64_t na,
                            std::vector<int32_t>& amap, std::vector<int32_t>& self) {
    const int64_t n = A.n;
    HostCSR P;
    P.n = n;
    P.m = na;
    P.p.assign(n + 1, 0);
#pragma omp parallel
    {
        std::vector<int32_t> mark(na, -1);
#pragma omp for schedule(static)
        for (int64_t r = 0; r < n; ++r) {
            int32_t cnt = 0;
            if (agg[r] >= 0) {
                mark[agg[r]] = (int32_t)r;
                ++cnt;
            }
            for (int32_t k = A.p[r]; k < A.p[r + 1]; ++k) {
                const int32_t a = agg[A.i[k]];
                if (a >= 0 && mark[a] != (int32_t)r) {
                    mark[a] = (int32_t)r;
                    ++cnt;
                }
            }
            P.p[r + 1] = cnt;
        }
    }
    for (int64_t r = 0; r < n; ++r) P.p[r + 1] += P.p[r];
    P.i.resize(P.p[n]);
    amap.assign(A.i.size(), -1);
    self.assign(n, -1);
#pragma omp parallel
    {
        std::vector<int32_t> mark(na, -1);
#pragma omp for schedule(static)
        for (int64_t r = 0; r < n; ++r) {
            int32_t o = P.p[r];
            if (agg[r] >= 0) {
                mark[agg[r]] = (int32_t)r;
                P.i[o++] = agg[r];
            }
            for (int32_t k = A.p[r]; k < A.p[r + 1]; ++k) {
                const int32_t a = agg[A.i[k]];
                if (a >= 0 && mark[a] != (int32_t)r) {
                    mark[a] = (int32_t)r;
                    P.i[o++] = a;
                }
            }
            std::sort(P.i.begin() + P.p[r], P.i.begin() + P.p[r + 1]);
            if (agg[r] >= 0) self[r] = find_col(P, r, agg[r]);
            for (int32_t k = A.p[r]; k < A.p[r + 1]; ++k)
                if (agg[A.i[k]] >= 0) amap[k] = find_col(P, r, agg[A.i[k]]);
        }
    }
    return P;
}

// R = P^T pattern; R entry t takes the value of P entry tperm[t].  Each
// R row lists its P rows in ascending order: the P rows are cut into one
// contiguous range per thread, each thread counts its range's entries per
// column, and the column-major prefix over (column, thread) gives every
// thread its own slots, filled in row order.
HostCSR transpose_pattern(const HostCSR& P, std::vector<int32_t>& tperm) {
    HostCSR R;
    R.n = P.m;
    R.m = P.n;
    R.p.assign(R.n + 1, 0);
    R.i.resize(P.i.size());
    tperm.resize(P.i.size());
    const int T = std::max(1, std::min(omp_get_max_threads(), 64));
    const int64_t nc = R.n;
    std::vector<int64_t> cnt((size_t)T * (nc + 1), 0);  // (thread, column) counts, then offsets
    auto lo = [&](int t) { return P.n * t / T; };
#pragma omp parallel for schedule(static, 1) num_threads(T)
    for (int t = 0; t < T; ++t) {
        int64_t* c_t = cnt.data() + (size_t)t * (nc + 1);
        for (int64_t r = lo(t); r < lo(t + 1); ++r)
            for (int32_t k = P.p[r]; k < P.p[r + 1]; ++k) c_t[P.i[k]]++;
    }
    int64_t run = 0;
    for (int64_t c = 0; c < nc; ++c) {
        R.p[c] = (int32_t)run;
        for (int t = 0; t < T; ++t) {
            int64_t& v = cnt[(size_t)t * (nc + 1) + c];
            const int64_t n_tc = v;
            v = run;
            run += n_tc;
        }
    }
    R.p[nc] = (int32_t)run;
#pragma omp parallel for schedule(static, 1) num_threads(T)
    for (int t = 0; t < T; ++t) {
        int64_t* c_t = cnt.data() + (size_t)t * (nc + 1);
        for (int64_t r = lo(t); r < lo(t + 1); ++r)
            for (int32_t k = P.p[r]; k < P.p[r + 1]; ++k) {
                const int32_t c = P.i[k];
                const int64_t o = c_t[c]++;
                R.i[o] = (int32_t)r;
                tperm[o] = k;
            }
    }
    return R;
}

// Pattern of C = A B (sorted columns, OpenMP over rows; count and fill
// passes with a per-thread marker array, no per-row allocation).
HostCSR spgemm_pattern(const HostCSR& A, const HostCSR& B) {
    HostCSR C;
    C.n = A.n;
    C.m = B.m;
    C.p.assign(A.n + 1, 0);
#pragma omp parallel
    {
        std::vector<int32_t> mark(B.m, -1);
#pragma omp for schedule(dynamic, 1024)
        for (int64_t r = 0; r < A.n; ++r) {
            int32_t cnt = 0;
            for (int32_t k = A.p[r]; k < A.p[r + 1]; ++k) {
                const int32_t a = A.i[k];
                for (int32_t q = B.p[a]; q < B.p[a + 1]; ++q) {
                    const int32_t c = B.i[q];
                    if (mark[c] != (int32_t)r) {
                        mark[c] = (int32_t)r;
                        ++cnt;
                    }
                }
            }
            C.p[r + 1] = cnt;
        }
    }
    for (int64_t r = 0; r < A.n; ++r) C.p[r + 1] += C.p[r];
    C.i.resize(C.p[A.n]);
#pragma omp parallel
    {
        std::vector<int32_t> mark(B.m, -1);
#pragma omp for schedule(dynamic, 1024)
        for (int64_t r = 0; r < A.n; ++r) {
            int32_t o = C.p[r];
            for (int32_t k = A.p[r]; k < A.p[r + 1]; ++k) {
                const int32_t a = A.i[k];
                for (int32_t q = B.p[a]; q < B.p[a + 1]; ++q) {
                    const int32_t c = B.i[q];
                    if (mark[c] != (int32_t)r) {
                        mark[c] = (int32_t)r;
                        C.i[o++] = c;
                    }
                }
            }
            std::sort(C.i.begin() + C.p[r], C.i.begin() + C.p[r + 1]);
        }
    }
    return C;
}

// Dense inverse by Gauss-Jordan with partial pivoting: the host fallback
// for a singular coarsest operator, inverted after diagonal regularisation.
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

// Power-iteration start vector (deterministic xorshift sequence; 0 on
// skipped rows).
std::vector<double> power_start(int64_t n, const std::vector<uint8_t>& skip) {
    std::vector<double> x(n);
    uint64_t h = 0x9E3779B97F4A7C15ull;
    for (int64_t r = 0; r < n; ++r) {
        h ^= h << 13;
        h ^= h >> 7;
        h ^= h << 17;
        x[r] = skip[r] ? 0.0 : 0.5 + (double)(h % 1000003) / 1000003.0;
    }
    return x;
}

// ------------------------------------------------------------ device numeric setup

__device__ __forceinline__ int32_t dev_lower_bound(const int32_t* __restrict__ a, int32_t len, int32_t v) {
    int32_t lo = 0, hi = len;
    while (lo < hi) {
        const int32_t mid = (lo + hi) >> 1;
        if (a[mid] < v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// finest operator from the caller's matrix: src[k] = caller entry, or -1
// for the identity entry of a constrained row
__global__ void k_embed(int64_t nnz, const int32_t* __restrict__ src, const double* __restrict__ data,
                        double* __restrict__ out) {
    GRID_STRIDE(k, nnz) out[k] = src[k] >= 0 ? data[src[k]] : 1.0;
}

__global__ void k_dinv(int64_t n, const int32_t* __restrict__ diag, const double* __restrict__ Ax,
                       double* __restrict__ dinv, double* __restrict__ s, const double* __restrict__ x0,
                       double* __restrict__ x) {
    GRID_STRIDE(r, n) {
        const double d = diag[r] >= 0 ? Ax[diag[r]] : 0.0;
        const double di = d != 0.0 ? __ddiv_rn(1.0, d) : 1.0;
        dinv[r] = di;
        s[r] = sqrt(fabs(di));
        x[r] = x0[r];
    }
}

// y = skip ? 0 : s * (A (s * x))   (rows of 8 lanes)
__global__ void __launch_bounds__(256)
    k_pw_apply(int64_t n, const int32_t* __restrict__ Ap, const int32_t* __restrict__ Ai,
               const double* __restrict__ Ax, const double* __restrict__ s, const double* __restrict__ x,
               const uint8_t* __restrict__ skip, double* __restrict__ y, const int* __restrict__ done) {
    if (*done) return;
    constexpr int TPR = 8, RPW = 32 / TPR;
    const int sub = threadIdx.x % TPR, group = (threadIdx.x & 31) / TPR;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = warp * RPW; base < n; base += n_warps * RPW) {
        const int64_t r = base + group;
        double acc = 0.0;
        if (r < n)
            for (int32_t k = Ap[r] + sub; k < Ap[r + 1]; k += TPR) {
                const int32_t c = Ai[k];
                acc += Ax[k] * (s[c] * x[c]);
            }
#pragma unroll
        for (int o = TPR / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, TPR);
        if (sub == 0 && r < n) y[r] = (skip && skip[r]) ? 0.0 : s[r] * acc;
    }
}

// dots = (x.y, y.y, x.x): lambda = x.y / x.x (Rayleigh quotient), stop when
// y == 0, else normalise (dots[3] = |y|)
__global__ void k_pw_update(double* __restrict__ dots, double* __restrict__ lam, int* __restrict__ done) {
    if (*done) return;
    *lam = dots[2] > 0.0 ? dots[0] / dots[2] : 0.0;
    if (dots[1] == 0.0) *done = 1;
    else dots[3] = sqrt(dots[1]);
}

__global__ void k_pw_norm(int64_t n, const double* __restrict__ y, double* __restrict__ x,
                          const double* __restrict__ dots, const int* __restrict__ done) {
    if (*done) return;
    const double nrm = dots[3];
    GRID_STRIDE(r, n) x[r] = y[r] / nrm;
}

// omega = (4/3) / rho with rho = 1.05 lambda (small safety margin on the
// Rayleigh quotient), 2 when lambda <= 0
__global__ void k_pw_finish(const double* __restrict__ lam, double* __restrict__ omega) {
    const double l = *lam;
    const double rho = l > 0.0 ? 1.05 * l : 2.0;
    *omega = (4.0 / 3.0) / rho;
}

// P = (I - omega D^-1 A) T, one row per thread, contributions in the
// order (T entry, then A's entries in row order)
__global__ void k_prolong(int64_t n, const int32_t* __restrict__ Ap, const int32_t* __restrict__ Ai,
                          const double* __restrict__ Ax, const int32_t* __restrict__ amap,
                          const int32_t* __restrict__ self, const double* __restrict__ t,
                          const double* __restrict__ dinv, const double* __restrict__ omega,
                          const int32_t* __restrict__ Pp, double* __restrict__ Px) {
    GRID_STRIDE(r, n) {
        for (int32_t q = Pp[r]; q < Pp[r + 1]; ++q) Px[q] = 0.0;
        if (self[r] >= 0) Px[self[r]] = t[r];
        const double f = __dmul_rn(*omega, dinv[r]);
        for (int32_t k = Ap[r]; k < Ap[r + 1]; ++k) {
            const int32_t q = amap[k];
            if (q < 0) continue;
            Px[q] = __dadd_rn(Px[q], __dmul_rn(__dmul_rn(-f, Ax[k]), t[Ai[k]]));
        }
    }
}

__global__ void k_gather_vals(int64_t m, const int32_t* __restrict__ perm, const double* __restrict__ src,
                              double* __restrict__ dst) {
    GRID_STRIDE(k, m) dst[k] = src[perm[k]];
}

// C = A B on C's precomputed pattern, one row per thread, products added in
// (A entry, B entry) order
__global__ void k_spgemm_num(int64_t n, const int32_t* __restrict__ Ap, const int32_t* __restrict__ Ai,
                             const double* __restrict__ Ax, const int32_t* __restrict__ Bp,
                             const int32_t* __restrict__ Bi, const double* __restrict__ Bx,
                             const int32_t* __restrict__ Cp, const int32_t* __restrict__ Ci,
                             double* __restrict__ Cx) {
    GRID_STRIDE(r, n) {
        const int32_t cb = Cp[r], cl = Cp[r + 1] - cb;
        for (int32_t q = 0; q < cl; ++q) Cx[cb + q] = 0.0;
        for (int32_t k = Ap[r]; k < Ap[r + 1]; ++k) {
            const double a = Ax[k];
            const int32_t j = Ai[k];
            for (int32_t q = Bp[j]; q < Bp[j + 1]; ++q) {
                const int32_t pos = cb + dev_lower_bound(Ci + cb, cl, Bi[q]);
                Cx[pos] = __dadd_rn(Cx[pos], __dmul_rn(a, Bx[q]));
            }
        }
    }
}

__global__ void k_densify(int64_t n, const int32_t* __restrict__ Cp, const int32_t* __restrict__ Ci,
                          const double* __restrict__ Cx, double* __restrict__ a, double* __restrict__ inv) {
    GRID_STRIDE(r, n) {
        for (int64_t c = 0; c < n; ++c) {
            a[r * n + c] = 0.0;
            inv[r * n + c] = (c == r) ? 1.0 : 0.0;
        }
        for (int32_t k = Cp[r]; k < Cp[r + 1]; ++k) a[r * n + Ci[k]] = Cx[k];
    }
}

// Gauss-Jordan column step c (one block): pivot = first row of largest
// |a[r][c]|, r >= c; swap; scale row c; fcol[r] = a[r][c] for r != c.
__global__ void __launch_bounds__(1024)
    k_gj_pivot(double* __restrict__ a, double* __restrict__ inv, int64_t n, int64_t c, double* __restrict__ fcol,
               int* __restrict__ singular) {
    __shared__ double sv[32];
    __shared__ int64_t si[32];
    __shared__ double sd;
    __shared__ int64_t spiv;
    if (*singular) return;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    double best = -1.0;
    int64_t bi = n;
    for (int64_t r = c + tid; r < n; r += blockDim.x) {
        const double v = fabs(a[r * n + c]);
        if (v > best) {
            best = v;
            bi = r;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, best, o);
        const int64_t oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ov > best || (ov == best && oi < bi)) {
            best = ov;
            bi = oi;
        }
    }
    if (lane == 0) {
        sv[w] = best;
        si[w] = bi;
    }
    __syncthreads();
    if (tid == 0) {
        double b = -1.0;
        int64_t p = n;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k)
            if (sv[k] > b || (sv[k] == b && si[k] < p)) {
                b = sv[k];
                p = si[k];
            }
        spiv = p;
    }
    __syncthreads();
    const int64_t piv = spiv;
    if (piv >= n || a[piv * n + c] == 0.0) {
        if (tid == 0) *singular = 1;
        return;
    }
    if (piv != c)
        for (int64_t k = tid; k < n; k += blockDim.x) {
            double t0 = a[c * n + k];
            a[c * n + k] = a[piv * n + k];
            a[piv * n + k] = t0;
            t0 = inv[c * n + k];
            inv[c * n + k] = inv[piv * n + k];
            inv[piv * n + k] = t0;
        }
    __syncthreads();
    if (tid == 0) sd = __ddiv_rn(1.0, a[c * n + c]);
    __syncthreads();
    const double d = sd;
    for (int64_t k = tid; k < n; k += blockDim.x) {
        a[c * n + k] = __dmul_rn(a[c * n + k], d);
        inv[c * n + k] = __dmul_rn(inv[c * n + k], d);
    }
    __syncthreads();
    for (int64_t r = tid; r < n; r += blockDim.x) fcol[r] = r == c ? 0.0 : a[r * n + c];
}

// Gauss-Jordan elimination of column c from every other row.
__global__ void k_gj_elim(double* __restrict__ a, double* __restrict__ inv, int64_t n, int64_t c,
                          const double* __restrict__ fcol, const int* __restrict__ singular) {
    if (*singular) return;
    GRID_STRIDE(idx, n * 2 * n) {
        const int64_t r = idx / (2 * n), k = idx % (2 * n);
        const double f = fcol[r];
        if (r == c || f == 0.0) continue;
        if (k < n) a[r * n + k] = __dsub_rn(a[r * n + k], __dmul_rn(f, a[c * n + k]));
        else inv[r * n + k - n] = __dsub_rn(inv[r * n + k - n], __dmul_rn(f, inv[c * n + k - n]));
    }
}

// ------------------------------------------------------------ device kernels

template <class T>
__global__ void k_jacobi_first(const T* __restrict__ dinv, const T* __restrict__ b, T* __restrict__ x, T w,
                               int64_t n) {
    GRID_STRIDE(i, n) x[i] = w * dinv[i] * b[i];
}

// Row loop shared by the CSR kernels below: TPR = 0 is one warp per 32
// rows (csr_rows.cuh warp_row_sum), else TPR lanes per row; epi(r, acc)
// writes row r (called once per row, by one lane).
template <class T, int TPR, class Prod, class Epi>
__device__ __forceinline__ void csr_rows_loop(int64_t n, const int32_t* __restrict__ Ap, T* sh, Prod prod, Epi epi) {
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    if constexpr (TPR == 0) {
        const int lane = threadIdx.x & 31;
        for (int64_t r0 = warp * 32; r0 < n; r0 += n_warps * 32) {   // warp-uniform
            const T acc = warp_row_sum<T>(Ap, r0, n, sh, prod);
            if (r0 + lane < n) epi(r0 + lane, acc);
        }
    } else {
        constexpr int RPW = 32 / TPR;
        const int sub = threadIdx.x % TPR, group = (threadIdx.x & 31) / TPR;
        for (int64_t base = warp * RPW; base < n; base += n_warps * RPW) {   // warp-uniform
            const int64_t r = base + group;
            const T acc = lanes_row_sum<T, TPR>(Ap, r, n, prod);
            if (sub == 0 && r < n) epi(r, acc);
        }
    }
}

// out = x + w D^-1 (b - A x)   (or, with RESID, out = b - A x).  The finest
// operator is the embedded one (identity rows, no constrained columns): no
// mask.
template <class T, bool RESID, int TPR>
__global__ void __launch_bounds__(256)
    k_jacobi_sweep(int64_t n, const int32_t* __restrict__ Ap, const int32_t* __restrict__ Ai,
                   const T* __restrict__ Ax, const T* __restrict__ dinv, const T* __restrict__ b,
                   const T* __restrict__ x, T* __restrict__ out, T w) {
    __shared__ T sh[TPR == 0 ? 256 / 32 : 1][TPR == 0 ? CSR_ROWS_CHUNK : 1];
    csr_rows_loop<T, TPR>(
        n, Ap, sh[TPR == 0 ? threadIdx.x >> 5 : 0], [&](int32_t k) { return Ax[k] * x[Ai[k]]; },
        [&](int64_t r, T acc) {
            const T res = b[r] - acc;
            out[r] = RESID ? res : x[r] + w * dinv[r] * res;
        });
}

// y (+)= A x, rectangular (restriction / prolongation)
template <class T, bool ADD, int TPR>
__global__ void __launch_bounds__(256)
    k_spmv_rect(int64_t n, const int32_t* __restrict__ Ap, const int32_t* __restrict__ Ai, const T* __restrict__ Ax,
                const T* __restrict__ x, T* __restrict__ y) {
    __shared__ T sh[TPR == 0 ? 256 / 32 : 1][TPR == 0 ? CSR_ROWS_CHUNK : 1];
    csr_rows_loop<T, TPR>(
        n, Ap, sh[TPR == 0 ? threadIdx.x >> 5 : 0], [&](int32_t k) { return Ax[k] * x[Ai[k]]; },
        [&](int64_t r, T acc) { y[r] = ADD ? y[r] + acc : acc; });
}

template <class T, bool RESID>
void launch_sweep(int64_t n, int64_t nnz, const int32_t* Ap, const int32_t* Ai, const T* Ax, const T* dinv,
                  const T* b, const T* x, T* out, T w, cudaStream_t s) {
    if (use_warp_rows(n, nnz)) {
        k_jacobi_sweep<T, RESID, 0><<<csr_rows_grid(n), 256, 0, s>>>(n, Ap, Ai, Ax, dinv, b, x, out, w);
    } else {
        switch (lanes_per_row(nnz, n)) {
            case 4: k_jacobi_sweep<T, RESID, 4><<<lanes_grid(n, 4), 256, 0, s>>>(n, Ap, Ai, Ax, dinv, b, x, out, w); break;
            case 8: k_jacobi_sweep<T, RESID, 8><<<lanes_grid(n, 8), 256, 0, s>>>(n, Ap, Ai, Ax, dinv, b, x, out, w); break;
            case 16:
                k_jacobi_sweep<T, RESID, 16><<<lanes_grid(n, 16), 256, 0, s>>>(n, Ap, Ai, Ax, dinv, b, x, out, w);
                break;
            default:
                k_jacobi_sweep<T, RESID, 32><<<lanes_grid(n, 32), 256, 0, s>>>(n, Ap, Ai, Ax, dinv, b, x, out, w);
        }
    }
    UP3D_CHECK_LAUNCH();
}

template <class T, bool ADD>
void launch_rect(int64_t n, int64_t nnz, const int32_t* Ap, const int32_t* Ai, const T* Ax, const T* x, T* y,
                 cudaStream_t s) {
    if (use_warp_rows(n, nnz)) {
        k_spmv_rect<T, ADD, 0><<<csr_rows_grid(n), 256, 0, s>>>(n, Ap, Ai, Ax, x, y);
    } else {
        switch (lanes_per_row(nnz, n)) {
            case 4: k_spmv_rect<T, ADD, 4><<<lanes_grid(n, 4), 256, 0, s>>>(n, Ap, Ai, Ax, x, y); break;
            case 8: k_spmv_rect<T, ADD, 8><<<lanes_grid(n, 8), 256, 0, s>>>(n, Ap, Ai, Ax, x, y); break;
            case 16: k_spmv_rect<T, ADD, 16><<<lanes_grid(n, 16), 256, 0, s>>>(n, Ap, Ai, Ax, x, y); break;
            default: k_spmv_rect<T, ADD, 32><<<lanes_grid(n, 32), 256, 0, s>>>(n, Ap, Ai, Ax, x, y);
        }
    }
    UP3D_CHECK_LAUNCH();
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
    void upload_pattern(const HostCSR& h, cudaStream_t s) {
        n = h.n;
        m = h.m;
        nnz = (int64_t)h.i.size();
        p.alloc(n + 1);
        i.alloc(std::max<int64_t>(nnz, 1));
        x.alloc(std::max<int64_t>(nnz, 1));
        h2d(p.get(), h.p.data(), sizeof(int32_t) * (n + 1), s);
        if (nnz) h2d(i.get(), h.i.data(), sizeof(int32_t) * nnz, s);
    }
    template <class U>
    void copy_pattern(const DevCSR<U>& o, cudaStream_t s) {
        n = o.n;
        m = o.m;
        nnz = o.nnz;
        p.alloc(n + 1);
        i.alloc(std::max<int64_t>(nnz, 1));
        x.alloc(std::max<int64_t>(nnz, 1));
        UP3D_CUDA(cudaMemcpyAsync(p.get(), o.p.get(), sizeof(int32_t) * (n + 1), cudaMemcpyDeviceToDevice, s));
        if (nnz)
            UP3D_CUDA(cudaMemcpyAsync(i.get(), o.i.get(), sizeof(int32_t) * nnz, cudaMemcpyDeviceToDevice, s));
    }
};

template <class T>
void upload(DBuf<T>& d, const std::vector<T>& h, cudaStream_t s) {
    d.alloc(std::max<size_t>(h.size(), 1));
    if (!h.empty()) h2d(d.get(), h.data(), sizeof(T) * h.size(), s);
}

// values of type T from FP64 (copy or narrowing)
template <class T>
void convert(const double* src, T* dst, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    if constexpr (std::is_same<T, double>::value) {
        UP3D_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    } else {
        k_d2f<<<grid_for(n, 256), 256, 0, s>>>(src, dst, n);
        UP3D_CHECK_LAUNCH();
    }
}

template <class T>
struct Ref {  // non-owning device pointer with the DBuf accessor
    T* v = nullptr;
    T* get() const { return v; }
};
template <class T>
struct CsrRef {
    int64_t n = 0, m = 0, nnz = 0;
    Ref<const int32_t> p, i;
    Ref<T> x;
};

// One level of the cycle: views of the symbolic level's patterns and, for
// the FP64 cycle, of its FP64 values; the FP32 cycle owns FP32 copies.
template <class T>
struct Level {
    CsrRef<T> A, P, R;
    Ref<T> dinv;
    DBuf<T> own_A, own_P, own_R, own_dinv;  // FP32 values (unused for FP64)
    DBuf<T> x, b, r;
    T w_smooth = T(0);
};

// Symbolic structure and FP64 values of one level.
struct SymLevel {
    DevCSR<double> A;            // level operator
    DBuf<int32_t> diag;          // (n) slot of the diagonal, -1 when absent
    DBuf<uint8_t> skip;          // (n) constrained rows (finest level only)
    DBuf<double> x0, dinv, sq;   // power-iteration start, D^-1, sqrt|D^-1|
    // to the next level (absent on the coarsest)
    DBuf<int32_t> amap, self;    // A entry / row -> P slot
    DBuf<double> t;              // tentative prolongator value of each row
    DevCSR<double> P, R, AP;     // prolongator, restriction (P^T), A P
    DBuf<int32_t> tperm;         // R entry -> P entry
    bool has_skip = false;
};

}  // namespace

struct Amg {
    bool fp32 = false;  // an FP32 cycle exists (Lf)
    bool fp64 = true;   // an FP64 cycle exists (Ld)
    int pre = 2, post = 2;
    int64_t n_coarse = 0;
    // the caller's finest pattern (refresh checks) and its embedding
    int64_t n_in = 0, nnz_in = 0;
    bool has_dir = false;
    DBuf<int32_t> in_p, in_i, emb_src;
    DBuf<uint8_t> in_dir;
    std::vector<SymLevel*> sym;
    // numeric scratch
    DBuf<double> pw_xy, pw_scal, omega_dev, dense_a, fcol;
    DBuf<int> flags;
    std::vector<double> omega;
    DBuf<double> cinv;
    std::vector<Level<double>*> Ld;
    std::vector<Level<float>*> Lf;
    up3d_amg_info info{};
    // one V-cycle as a CUDA graph per (input, output) pair: captured on a
    // private stream at first use, replayed on the caller's stream
    struct Graph {
        const void* r;
        void* z;
        bool f32;  // FP32 input and output
        cudaGraphExec_t exec;
        long long launches;
    };
    DBuf<double> io64_in, io64_out;  // FP32 input/output through an FP64 hierarchy
    std::vector<Graph> graphs;
    cudaStream_t capture_stream = nullptr;
    int device = 0;
    // the numeric phase's vector kernels (kept: set-up and every refresh
    // would otherwise allocate and free its scratch and pinned readback)
    std::unique_ptr<Blas> blas;
    void drop_graphs() {
        for (auto& g : graphs) cudaGraphExecDestroy(g.exec);
        graphs.clear();
    }
    ~Amg() {
        drop_graphs();
        if (capture_stream) cudaStreamDestroy(capture_stream);
        for (auto* l : Ld) delete l;
        for (auto* l : Lf) delete l;
        for (auto* l : sym) delete l;
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
    const unsigned g1 = grid_for(n, 256);
    const int64_t nnz = lv.A.nnz;
    // pre-smoothing from x = 0
    k_jacobi_first<T><<<g1, 256, 0, s>>>(lv.dinv.get(), lv.b.get(), lv.x.get(), lv.w_smooth, n);
    UP3D_CHECK_LAUNCH();
    for (int k = 1; k < a.pre; ++k) {
        launch_sweep<T, false>(n, nnz, lv.A.p.get(), lv.A.i.get(), lv.A.x.get(), lv.dinv.get(), lv.b.get(),
                               lv.x.get(), lv.r.get(), lv.w_smooth, s);
        std::swap(lv.x.p, lv.r.p);
    }
    // residual, restriction
    launch_sweep<T, true>(n, nnz, lv.A.p.get(), lv.A.i.get(), lv.A.x.get(), lv.dinv.get(), lv.b.get(), lv.x.get(),
                          lv.r.get(), lv.w_smooth, s);
    Level<T>& cv = *L[l + 1];
    launch_rect<T, false>(lv.R.n, lv.R.nnz, lv.R.p.get(), lv.R.i.get(), lv.R.x.get(), lv.r.get(), cv.b.get(), s);
    vcycle<T>(a, L, l + 1, s);
    // prolongation
    launch_rect<T, true>(lv.P.n, lv.P.nnz, lv.P.p.get(), lv.P.i.get(), lv.P.x.get(), cv.x.get(), lv.x.get(), s);
    for (int k = 0; k < a.post; ++k) {
        launch_sweep<T, false>(n, nnz, lv.A.p.get(), lv.A.i.get(), lv.A.x.get(), lv.dinv.get(), lv.b.get(),
                               lv.x.get(), lv.r.get(), lv.w_smooth, s);
        std::swap(lv.x.p, lv.r.p);
    }
}

// Diagonal slot of each row of a pattern.
std::vector<int32_t> diag_slots(const HostCSR& A) {
    std::vector<int32_t> d(A.n, -1);
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < A.n; ++r)
        for (int32_t k = A.p[r]; k < A.p[r + 1]; ++k)
            if (A.i[k] == r) d[r] = k;
    return d;
}

// Device numeric phase: every level's D^-1, omega, P, R, A P and coarser
// operator, then the coarsest inverse; fills the cycle's levels.
void numeric(Amg& a, cudaStream_t s) {
    const size_t L = a.sym.size();
    if (!a.blas) a.blas.reset(new Blas(s));
    Blas& blas = *a.blas;
    blas.s = s;
    double* dots = a.pw_scal.get();       // x.y, y.y, x.x, |y|
    double* lam = a.pw_scal.get() + 4;
    int* done = a.flags.get();
    int* singular = a.flags.get() + 1;
    for (size_t l = 0; l + 1 < L; ++l) {
        SymLevel& F = *a.sym[l];
        SymLevel& C = *a.sym[l + 1];
        const int64_t n = F.A.n;
        double* x = a.pw_xy.get();
        double* y = a.pw_xy.get() + n;
        k_dinv<<<grid_for(n, 256), 256, 0, s>>>(n, F.diag.get(), F.A.x.get(), F.dinv.get(), F.sq.get(),
                                                F.x0.get(), x);
        UP3D_CHECK_LAUNCH();
        UP3D_CUDA(cudaMemsetAsync(done, 0, sizeof(int), s));
        UP3D_CUDA(cudaMemsetAsync(lam, 0, sizeof(double), s));
        const unsigned g8 = grid_for(8 * n, 256, (int64_t)148 * 64);
        for (int it = 0; it < 20; ++it) {
            k_pw_apply<<<g8, 256, 0, s>>>(n, F.A.p.get(), F.A.i.get(), F.A.x.get(), F.sq.get(), x,
                                          F.has_skip ? F.skip.get() : nullptr, y, done);
            UP3D_CHECK_LAUNCH();
            blas.multidot(x, n, 2, y, n, dots);   // (x.y, y.y)
            blas.multidot(x, 0, 1, x, n, dots + 2);
            k_pw_update<<<1, 1, 0, s>>>(dots, lam, done);
            UP3D_CHECK_LAUNCH();
            k_pw_norm<<<grid_for(n, 256), 256, 0, s>>>(n, y, x, dots, done);
            UP3D_CHECK_LAUNCH();
        }
        k_pw_finish<<<1, 1, 0, s>>>(lam, a.omega_dev.get() + l);
        UP3D_CHECK_LAUNCH();
        k_prolong<<<grid_for(n, 128), 128, 0, s>>>(n, F.A.p.get(), F.A.i.get(), F.A.x.get(), F.amap.get(),
                                                   F.self.get(), F.t.get(), F.dinv.get(), a.omega_dev.get() + l,
                                                   F.P.p.get(), F.P.x.get());
        UP3D_CHECK_LAUNCH();
        k_gather_vals<<<grid_for(F.R.nnz, 256), 256, 0, s>>>(F.R.nnz, F.tperm.get(), F.P.x.get(), F.R.x.get());
        UP3D_CHECK_LAUNCH();
        k_spgemm_num<<<grid_for(n, 128), 128, 0, s>>>(n, F.A.p.get(), F.A.i.get(), F.A.x.get(), F.P.p.get(),
                                                      F.P.i.get(), F.P.x.get(), F.AP.p.get(), F.AP.i.get(),
                                                      F.AP.x.get());
        UP3D_CHECK_LAUNCH();
        k_spgemm_num<<<grid_for(F.R.n, 128), 128, 0, s>>>(F.R.n, F.R.p.get(), F.R.i.get(), F.R.x.get(),
                                                          F.AP.p.get(), F.AP.i.get(), F.AP.x.get(), C.A.p.get(),
                                                          C.A.i.get(), C.A.x.get());
        UP3D_CHECK_LAUNCH();
    }
    // coarsest dense inverse
    const SymLevel& Cl = *a.sym.back();
    const int64_t nc = Cl.A.n;
    UP3D_CUDA(cudaMemsetAsync(singular, 0, sizeof(int), s));
    k_densify<<<grid_for(nc, 128), 128, 0, s>>>(nc, Cl.A.p.get(), Cl.A.i.get(), Cl.A.x.get(), a.dense_a.get(),
                                                a.cinv.get());
    UP3D_CHECK_LAUNCH();
    for (int64_t c = 0; c < nc; ++c) {
        k_gj_pivot<<<1, 1024, 0, s>>>(a.dense_a.get(), a.cinv.get(), nc, c, a.fcol.get(), singular);
        UP3D_CHECK_LAUNCH();
        k_gj_elim<<<grid_for(2 * nc * nc, 256), 256, 0, s>>>(a.dense_a.get(), a.cinv.get(), nc, c, a.fcol.get(),
                                                             singular);
        UP3D_CHECK_LAUNCH();
    }
    int sing = 0;
    a.omega.assign(L > 1 ? L - 1 : 0, 0.0);
    if (L > 1)
        UP3D_CUDA(cudaMemcpyAsync(a.omega.data(), a.omega_dev.get(), sizeof(double) * (L - 1),
                                  cudaMemcpyDeviceToHost, s));
    UP3D_CUDA(cudaMemcpyAsync(&sing, singular, sizeof(int), cudaMemcpyDeviceToHost, s));
    UP3D_CUDA(cudaStreamSynchronize(s));
    if (sing) {
        // singular coarse operator (e.g. pure-Neumann): regularise the
        // diagonal and invert on the host
        HostCSR h;
        h.n = h.m = nc;
        h.p.resize(nc + 1);
        h.i.resize(Cl.A.nnz);
        h.x.resize(Cl.A.nnz);
        UP3D_CUDA(cudaMemcpyAsync(h.p.data(), Cl.A.p.get(), sizeof(int32_t) * (nc + 1), cudaMemcpyDeviceToHost, s));
        UP3D_CUDA(cudaMemcpyAsync(h.i.data(), Cl.A.i.get(), sizeof(int32_t) * Cl.A.nnz, cudaMemcpyDeviceToHost, s));
        UP3D_CUDA(cudaMemcpyAsync(h.x.data(), Cl.A.x.get(), sizeof(double) * Cl.A.nnz, cudaMemcpyDeviceToHost, s));
        UP3D_CUDA(cudaStreamSynchronize(s));
        std::vector<double> dense(nc * nc, 0.0), inv;
        double dmax = 0.0;
        for (int64_t r = 0; r < nc; ++r)
            for (int32_t k = h.p[r]; k < h.p[r + 1]; ++k) {
                dense[r * nc + h.i[k]] = h.x[k];
                if (h.i[k] == r) dmax = std::max(dmax, std::fabs(h.x[k]));
            }
        for (int64_t r = 0; r < nc; ++r) dense[r * nc + r] += 1e-12 * (dmax > 0 ? dmax : 1.0);
        UP3D_REQUIRE(dense_inverse(dense, nc, inv), UP3D_ERR_RUNTIME, "AMG coarsest operator is singular");
        UP3D_CUDA(cudaMemcpyAsync(a.cinv.get(), inv.data(), sizeof(double) * nc * nc, cudaMemcpyHostToDevice, s));
        UP3D_CUDA(cudaStreamSynchronize(s));
    }
}

// Narrows the FP64 level values into the FP32 cycle (the FP64 cycle views
// them in place) and sets the smoothing weights.
template <class T>
void fill_levels(Amg& a, std::vector<Level<T>*>& Lv, cudaStream_t s) {
    for (size_t l = 0; l < a.sym.size(); ++l) {
        SymLevel& F = *a.sym[l];
        Level<T>& lv = *Lv[l];
        if constexpr (!std::is_same<T, double>::value) convert<T>(F.A.x.get(), lv.A.x.get(), F.A.nnz, s);
        if (l + 1 < a.sym.size()) {
            if constexpr (!std::is_same<T, double>::value) {
                convert<T>(F.P.x.get(), lv.P.x.get(), F.P.nnz, s);
                convert<T>(F.R.x.get(), lv.R.x.get(), F.R.nnz, s);
                convert<T>(F.dinv.get(), lv.dinv.get(), F.A.n, s);
            }
            lv.w_smooth = (T)a.omega[l];
        }
    }
}

template <class T>
void view(CsrRef<T>& r, const DevCSR<double>& F, DBuf<T>& own) {
    r.n = F.n;
    r.m = F.m;
    r.nnz = F.nnz;
    r.p.v = F.p.get();
    r.i.v = F.i.get();
    if constexpr (std::is_same<T, double>::value) {
        r.x.v = F.x.get();
    } else {
        own.alloc(std::max<int64_t>(F.nnz, 1));
        r.x.v = own.get();
    }
}

template <class T>
void make_levels(Amg& a, std::vector<Level<T>*>& Lv, cudaStream_t s) {
    for (size_t l = 0; l < a.sym.size(); ++l) {
        SymLevel& F = *a.sym[l];
        auto* lv = new Level<T>();
        Lv.push_back(lv);
        view(lv->A, F.A, lv->own_A);
        const int64_t n = F.A.n;
        lv->x.alloc(n);
        lv->b.alloc(n);
        lv->r.alloc(n);
        if (l + 1 < a.sym.size()) {
            view(lv->P, F.P, lv->own_P);
            view(lv->R, F.R, lv->own_R);
            if constexpr (std::is_same<T, double>::value) {
                lv->dinv.v = F.dinv.get();
            } else {
                lv->own_dinv.alloc(n);
                lv->dinv.v = lv->own_dinv.get();
            }
        }
    }
}

__global__ void k_diff_i32(int64_t n, const int32_t* __restrict__ a, const int32_t* __restrict__ b,
                           int* __restrict__ flag) {
    GRID_STRIDE(i, n) if (a[i] != b[i]) *flag = 1;
}
__global__ void k_diff_u8(int64_t n, const uint8_t* __restrict__ a, const uint8_t* __restrict__ b,
                          int* __restrict__ flag) {
    GRID_STRIDE(i, n) if ((a[i] != 0) != (b[i] != 0)) *flag = 1;
}

}  // namespace

// One V-cycle z = M r as a sequence of launches on stream s.
void amg_cycle(Amg& a, const double* r, double* z, cudaStream_t s) {
    if (a.fp64) {
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

// The cycle's level buffers swap between sweeps; restoring them after each
// cycle keeps every cycle (and every captured graph) on the same buffers.
template <class T>
std::vector<std::pair<T*, T*>> save_buffers(std::vector<Level<T>*>& L) {
    std::vector<std::pair<T*, T*>> v;
    for (auto* l : L) v.emplace_back(l->x.p, l->r.p);
    return v;
}
template <class T>
void restore_buffers(std::vector<Level<T>*>& L, const std::vector<std::pair<T*, T*>>& v) {
    for (size_t i = 0; i < L.size(); ++i) {
        L[i]->x.p = v[i].first;
        L[i]->r.p = v[i].second;
    }
}

// One V-cycle with FP32 input and output.
void amg_cycle_f32(Amg& a, const float* r, float* z, cudaStream_t s) {
    if (a.fp32) {
        Level<float>& f = *a.Lf[0];
        const int64_t n = f.A.n;
        UP3D_CUDA(cudaMemcpyAsync(f.b.get(), r, sizeof(float) * n, cudaMemcpyDeviceToDevice, s));
        vcycle<float>(a, a.Lf, 0, s);
        UP3D_CUDA(cudaMemcpyAsync(z, f.x.get(), sizeof(float) * n, cudaMemcpyDeviceToDevice, s));
    } else {
        const int64_t n = a.Ld[0]->A.n;
        k_f2d<<<grid_for(n, 256), 256, 0, s>>>(r, a.io64_in.get(), n);
        UP3D_CHECK_LAUNCH();
        amg_cycle(a, a.io64_in.get(), a.io64_out.get(), s);
        k_d2f<<<grid_for(n, 256), 256, 0, s>>>(a.io64_out.get(), z, n);
        UP3D_CHECK_LAUNCH();
    }
}

// Replays the cached graph of one V-cycle for (r, z), capturing it first.
void apply_graph(Amg& a, const void* r, void* z, bool f32, cudaStream_t s) {
    for (auto& g : a.graphs)
        if (g.r == r && g.z == z && g.f32 == f32) {
            UP3D_CUDA(cudaGraphLaunch(g.exec, s));
            count_launch((int)g.launches);
            return;
        }
    if (f32 && !a.fp32) {
        const int64_t n = a.Ld[0]->A.n;
        a.io64_in.alloc(n);  // before the capture
        a.io64_out.alloc(n);
    }
    if (!a.capture_stream) UP3D_CUDA(cudaStreamCreateWithFlags(&a.capture_stream, cudaStreamNonBlocking));
    auto sd = save_buffers(a.Ld);
    auto sf = save_buffers(a.Lf);
    const long long l0 = g_launches.load();
    cudaGraph_t graph = nullptr;
    UP3D_CUDA(cudaStreamBeginCapture(a.capture_stream, cudaStreamCaptureModeThreadLocal));
    try {
        if (f32) amg_cycle_f32(a, static_cast<const float*>(r), static_cast<float*>(z), a.capture_stream);
        else amg_cycle(a, static_cast<const double*>(r), static_cast<double*>(z), a.capture_stream);
    } catch (...) {
        cudaStreamEndCapture(a.capture_stream, &graph);
        if (graph) cudaGraphDestroy(graph);
        restore_buffers(a.Ld, sd);
        restore_buffers(a.Lf, sf);
        throw;
    }
    UP3D_CUDA(cudaStreamEndCapture(a.capture_stream, &graph));
    restore_buffers(a.Ld, sd);
    restore_buffers(a.Lf, sf);
    const long long launches = g_launches.load() - l0;
    g_launches.fetch_sub(launches);  // counted at each replay instead
    cudaGraphExec_t exec = nullptr;
    const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    UP3D_CUDA(e);
    if (a.graphs.size() >= 16) {
        cudaGraphExecDestroy(a.graphs.front().exec);
        a.graphs.erase(a.graphs.begin());
    }
    a.graphs.push_back({r, z, f32, exec, launches});
    UP3D_CUDA(cudaGraphLaunch(exec, s));
    count_launch((int)launches);
}

void amg_apply(void* p, const double* r, double* z, cudaStream_t s) {
    apply_graph(*static_cast<Amg*>(p), r, z, false, s);
}

void amg_apply_f32(void* p, const float* r, float* z, cudaStream_t s) {
    apply_graph(*static_cast<Amg*>(p), r, z, true, s);
}

void amg_destroy(void* p) { delete static_cast<Amg*>(p); }

// Builds the hierarchy for `A` (device CSR); the finest operator's
// constrained rows (A->dirichlet) are identity rows.
void* amg_setup(const up3d_csr& A, const up3d_amg_options& opt, cudaStream_t s) {
    auto* a = new Amg();
    try {
        // 0: FP64 cycle, 1: FP32 cycle, 2: both (each vector type gets its own)
        UP3D_REQUIRE(opt.fp32 >= 0 && opt.fp32 <= 2, UP3D_ERR_VALUE, "AMG setup: fp32 must be 0, 1 or 2");
        a->fp32 = opt.fp32 != 0;
        a->fp64 = opt.fp32 != 1;
        a->pre = std::max(1, opt.presmooth);
        a->post = std::max(0, opt.postsmooth);
        const int64_t n = A.n;
        UP3D_REQUIRE(n > 0, UP3D_ERR_VALUE, "AMG setup: empty matrix");
        HostCSR h;
        h.n = h.m = n;
        h.p.resize(n + 1);
        d2h(h.p.data(), A.indptr, sizeof(int32_t) * (n + 1), s);
        const int64_t nnz = h.p[n];
        h.i.resize(nnz);
        d2h(h.i.data(), A.indices, sizeof(int32_t) * nnz, s);
        std::vector<uint8_t> skip(n, 0);
        if (A.dirichlet)
            UP3D_CUDA(cudaMemcpyAsync(skip.data(), A.dirichlet, n, cudaMemcpyDeviceToHost, s));
        UP3D_CUDA(cudaStreamSynchronize(s));
        for (auto& v : skip) v = v != 0;
        // the caller's pattern, kept for refresh checks
        a->n_in = n;
        a->nnz_in = nnz;
        a->has_dir = A.dirichlet != nullptr;
        a->in_p.alloc(n + 1);
        a->in_i.alloc(std::max<int64_t>(nnz, 1));
        UP3D_CUDA(cudaMemcpyAsync(a->in_p.get(), A.indptr, sizeof(int32_t) * (n + 1), cudaMemcpyDeviceToDevice, s));
        if (nnz)
            UP3D_CUDA(cudaMemcpyAsync(a->in_i.get(), A.indices, sizeof(int32_t) * nnz, cudaMemcpyDeviceToDevice, s));
        if (a->has_dir) upload(a->in_dir, skip, s);
        // finest operator as the embedded free-DOF system: identity rows,
        // constrained columns dropped; src = caller entry (-1: identity)
        HostCSR e;
        std::vector<int32_t> src;
        e.n = e.m = n;
        e.p.assign(n + 1, 0);
#pragma omp parallel for schedule(static)
        for (int64_t r = 0; r < n; ++r) {
            int32_t cnt = 0;
            if (skip[r]) cnt = 1;
            else
                for (int32_t k = h.p[r]; k < h.p[r + 1]; ++k) cnt += !skip[h.i[k]];
            e.p[r + 1] = cnt;
        }
        for (int64_t r = 0; r < n; ++r) e.p[r + 1] += e.p[r];
        e.i.resize(e.p[n]);
        src.resize(e.p[n]);
#pragma omp parallel for schedule(static)
        for (int64_t r = 0; r < n; ++r) {
            int32_t o = e.p[r];
            if (skip[r]) {
                e.i[o] = (int32_t)r;
                src[o] = -1;
                continue;
            }
            for (int32_t k = h.p[r]; k < h.p[r + 1]; ++k)
                if (!skip[h.i[k]]) {
                    e.i[o] = h.i[k];
                    src[o] = k;
                    ++o;
                }
        }
        upload(a->emb_src, src, s);
        // symbolic levels
        std::vector<HostCSR> As;
        As.push_back(std::move(e));
        std::vector<uint8_t> cur_skip = skip;
        const int64_t max_coarse = std::max<int64_t>(opt.max_coarse, 1);
        int64_t nmax = n;
        while (true) {
            const HostCSR& Al = As.back();
            auto* F = new SymLevel();
            a->sym.push_back(F);
            F->A.upload_pattern(Al, s);
            upload(F->diag, diag_slots(Al), s);
            F->has_skip = a->sym.size() == 1 && a->has_dir;
            if (F->has_skip) upload(F->skip, cur_skip, s);
            F->dinv.alloc(Al.n);
            F->sq.alloc(Al.n);
            if (Al.n <= max_coarse || (int)As.size() >= std::max(2, opt.max_levels)) break;
            std::vector<int32_t> agg;
            const int64_t na = standard_aggregation(Al, cur_skip, agg);
            if (na == 0 || na >= Al.n) break;
            upload(F->x0, power_start(Al.n, cur_skip), s);
            std::vector<int32_t> amap, self, tperm;
            HostCSR P = prolongator_pattern(Al, agg, na, amap, self);
            std::vector<int32_t> size(na, 0);
            for (int64_t r = 0; r < Al.n; ++r)
                if (agg[r] >= 0) size[agg[r]]++;
            std::vector<double> t(Al.n, 0.0);
            for (int64_t r = 0; r < Al.n; ++r)
                if (agg[r] >= 0) t[r] = 1.0 / std::sqrt((double)size[agg[r]]);
            HostCSR R = transpose_pattern(P, tperm);
            HostCSR AP = spgemm_pattern(Al, P);
            HostCSR Ac = spgemm_pattern(R, AP);
            upload(F->amap, amap, s);
            upload(F->self, self, s);
            upload(F->t, t, s);
            upload(F->tperm, tperm, s);
            F->P.upload_pattern(P, s);
            F->R.upload_pattern(R, s);
            F->AP.upload_pattern(AP, s);
            UP3D_CUDA(cudaStreamSynchronize(s));  // host vectors above go out of scope
            As.push_back(std::move(Ac));
            cur_skip.assign(As.back().n, 0);
        }
        // a level that stopped early without a start vector is the coarsest
        const int64_t nc = As.back().n;
        UP3D_REQUIRE(nc <= 8192, UP3D_ERR_RUNTIME, "AMG coarsest level too large for the dense solve");
        a->n_coarse = nc;
        a->pw_xy.alloc(2 * nmax);
        a->pw_scal.alloc(8);
        a->omega_dev.alloc(std::max<size_t>(a->sym.size(), 1));
        a->flags.alloc(2);
        a->dense_a.alloc(nc * nc);
        a->cinv.alloc(nc * nc);
        a->fcol.alloc(nc);
        k_embed<<<grid_for(a->sym[0]->A.nnz, 256), 256, 0, s>>>(a->sym[0]->A.nnz, a->emb_src.get(), A.data,
                                                                a->sym[0]->A.x.get());
        UP3D_CHECK_LAUNCH();
        numeric(*a, s);
        if (a->fp32) {
            make_levels<float>(*a, a->Lf, s);
            fill_levels<float>(*a, a->Lf, s);
        }
        if (a->fp64) {
            make_levels<double>(*a, a->Ld, s);
            fill_levels<double>(*a, a->Ld, s);
        }
        UP3D_CUDA(cudaStreamSynchronize(s));
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

// New values for the hierarchy: `A` must have the pattern and Dirichlet
// mask of the matrix the hierarchy was set up from.
void amg_refresh(void* p, const up3d_csr& A, cudaStream_t s) {
    Amg& a = *static_cast<Amg*>(p);
    UP3D_REQUIRE(A.n == a.n_in, UP3D_ERR_VALUE, "AMG refresh: matrix size differs from the setup matrix");
    UP3D_REQUIRE((A.dirichlet != nullptr) == a.has_dir, UP3D_ERR_VALUE,
                 "AMG refresh: Dirichlet mask presence differs from the setup matrix");
    int* flag = a.flags.get();
    UP3D_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), s));
    k_diff_i32<<<grid_for(a.n_in + 1, 256), 256, 0, s>>>(a.n_in + 1, A.indptr, a.in_p.get(), flag);
    UP3D_CHECK_LAUNCH();
    int diff = 0;
    UP3D_CUDA(cudaMemcpyAsync(&diff, flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    UP3D_CUDA(cudaStreamSynchronize(s));
    UP3D_REQUIRE(!diff, UP3D_ERR_VALUE, "AMG refresh: sparsity pattern differs from the setup matrix");
    k_diff_i32<<<grid_for(a.nnz_in, 256), 256, 0, s>>>(a.nnz_in, A.indices, a.in_i.get(), flag);
    UP3D_CHECK_LAUNCH();
    if (a.has_dir) {
        k_diff_u8<<<grid_for(a.n_in, 256), 256, 0, s>>>(a.n_in, A.dirichlet, a.in_dir.get(), flag);
        UP3D_CHECK_LAUNCH();
    }
    UP3D_CUDA(cudaMemcpyAsync(&diff, flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    UP3D_CUDA(cudaStreamSynchronize(s));
    UP3D_REQUIRE(!diff, UP3D_ERR_VALUE, "AMG refresh: sparsity pattern or Dirichlet mask differs from the setup matrix");
    k_embed<<<grid_for(a.sym[0]->A.nnz, 256), 256, 0, s>>>(a.sym[0]->A.nnz, a.emb_src.get(), A.data,
                                                           a.sym[0]->A.x.get());
    UP3D_CHECK_LAUNCH();
    numeric(a, s);
    if (a.fp32) fill_levels<float>(a, a.Lf, s);
    if (a.fp64) fill_levels<double>(a, a.Ld, s);
    a.drop_graphs();  // the smoothing weights are launch arguments of the graphs
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

int up3d_amg_refresh(up3d_precond* M, const up3d_csr* A, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(M && A && M->kind == 2 && M->amg && A->indptr && A->indices && A->data, UP3D_ERR_ARGUMENT,
                     "up3d_amg_refresh: null argument or not an AMG handle");
        amg_refresh(M->amg, *A, S(stream));
    });
}

int up3d_amg_get_info(const up3d_precond* M, up3d_amg_info* info) {
    return guarded([&] {
        UP3D_REQUIRE(M && info && M->kind == 2 && M->amg, UP3D_ERR_ARGUMENT, "up3d_amg_get_info: not an AMG handle");
        *info = *amg_info(M->amg);
    });
}

}  // extern "C"
