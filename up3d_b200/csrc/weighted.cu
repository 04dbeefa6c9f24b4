// The weighted upwind modes of the up3d library (kernels/upwind.py:128-454):
// outward face normals, the BFS face-neighbour neighbourhoods, and the two
// differentiable upwinded densities -- the streamline-Gaussian "kernel"
// sample over the neighbourhood and the face-ring "blend" with reach
// compensation.  The reference uses them in Picard when upwind_weighted is
// set (solve/picard.py:440-446, :596-602); its Newton path keeps the walk.
//
// One thread per element; every sum runs in the reference's order (the
// neighbourhood ascending, faces 0..3) with IEEE-rounded products and sums
// (no contraction), like the oracle.

#include <algorithm>
#include <vector>

#include <cub/cub.cuh>

#include "elem.cuh"
#include "internal.cuh"

namespace up3d {
namespace {

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

// Deepest neighbourhood built on the device: 4 hops (at most
// 4 + 12 + 36 + 108 elements besides e on a tet mesh).
constexpr int NB_MAX_DEPTH = 4;
constexpr int NB_MAX = 1 + 4 + 12 + 36 + 108;

struct WMon {
    double nu_max = 0.0;
    unsigned long long sup = 0, flo = 0;
};

__device__ __forceinline__ void flush(WMon a, up3d_monitors* mon) {
    const double nm = warp_max(a.nu_max);
    const unsigned long long s = warp_sum_u64(a.sup), f = warp_sum_u64(a.flo);
    if ((threadIdx.x & 31) == 0) {
        if (nm > 0.0) atomic_max_nonneg(&mon->nu_max, nm);
        if (s) atomicAdd(reinterpret_cast<unsigned long long*>(&mon->n_supersonic), s);
        if (f) atomicAdd(reinterpret_cast<unsigned long long*>(&mon->n_floored), f);
    }
}

// compute_face_normals (kernels/upwind.py:128-172): face f opposite local
// node f, normal (b - a) x (c - a) normalised, flipped to point away from
// the apex.  out (E, 4, 3).
__global__ void k_face_normals(const int4* __restrict__ conn, const double4* __restrict__ X, int64_t E,
                               double* __restrict__ out) {
    constexpr int FD[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};
    GRID_STRIDE(e, E) {
        const int4 c = conn[e];
        const int nd[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            const double4 a = X[nd[FD[f][0]]], b = X[nd[FD[f][1]]], cc = X[nd[FD[f][2]]], p = X[nd[f]];
            const double e1x = rsub(b.x, a.x), e1y = rsub(b.y, a.y), e1z = rsub(b.z, a.z);
            const double e2x = rsub(cc.x, a.x), e2y = rsub(cc.y, a.y), e2z = rsub(cc.z, a.z);
            double nx = rsub(rmul(e1y, e2z), rmul(e1z, e2y));
            double ny = rsub(rmul(e1z, e2x), rmul(e1x, e2z));
            double nz = rsub(rmul(e1x, e2y), rmul(e1y, e2x));
            const double nn = sqrt(dot3r(nx, ny, nz, nx, ny, nz));
            if (nn > 0.0) {
                nx = __ddiv_rn(nx, nn);
                ny = __ddiv_rn(ny, nn);
                nz = __ddiv_rn(nz, nn);
            }
            const double ox = rsub(__ddiv_rn(radd(radd(a.x, b.x), cc.x), 3.0), p.x);
            const double oy = rsub(__ddiv_rn(radd(radd(a.y, b.y), cc.y), 3.0), p.y);
            const double oz = rsub(__ddiv_rn(radd(radd(a.z, b.z), cc.z), 3.0), p.z);
            if (dot3r(nx, ny, nz, ox, oy, oz) < 0.0) {
                nx = -nx;
                ny = -ny;
                nz = -nz;
            }
            out[12 * e + 3 * f] = nx;
            out[12 * e + 3 * f + 1] = ny;
            out[12 * e + 3 * f + 2] = nz;
        }
    }
}

// build_upstream_neighborhoods (kernels/upwind.py:313-341): the elements
// within `depth` face hops of e, e excluded, ascending.  Breadth-first in
// a per-thread list whose levels are its own frontiers; the list is then
// insertion-sorted.  Count pass (cnt[e]) or fill pass (idx from off).
template <bool FILL>
__global__ void __launch_bounds__(128)
    k_neighborhoods(const int4* __restrict__ fn, int64_t E, int depth, int64_t* __restrict__ cnt,
                    const int64_t* __restrict__ off, int32_t* __restrict__ idx) {
    GRID_STRIDE(e, E) {
        int32_t seen[NB_MAX];
        int ns = 1, lo = 0, hi = 1;
        seen[0] = (int32_t)e;
        for (int d = 0; d < depth; ++d) {
            for (int i = lo; i < hi; ++i) {
                const int4 f = fn[seen[i]];
                const int32_t nb[4] = {f.x, f.y, f.z, f.w};
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if (nb[k] < 0 || nb[k] >= E) continue;
                    bool found = false;
                    for (int j = 0; j < ns && !found; ++j) found = seen[j] == nb[k];
                    if (!found && ns < NB_MAX) seen[ns++] = nb[k];
                }
            }
            lo = hi;
            hi = ns;
        }
        if constexpr (!FILL) {
            cnt[e] = ns - 1;
        } else {
            for (int i = 2; i < ns; ++i) {
                const int32_t v = seen[i];
                int j = i - 1;
                while (j >= 1 && seen[j] > v) {
                    seen[j + 1] = seen[j];
                    --j;
                }
                seen[j + 1] = v;
            }
            int32_t* out = idx + off[e];
            for (int i = 1; i < ns; ++i) out[i - 1] = seen[i];
        }
    }
}

// The unit streamwise direction and the element's extent along it
// (kernels/upwind.py:243-253, :389-403).
__device__ __forceinline__ void stream_extent(const int4 c, const double4* __restrict__ X, double vx, double vy,
                                              double vz, double& pmin, double& pmax) {
    const int nd[4] = {c.x, c.y, c.z, c.w};
    pmin = 1e300;
    pmax = -1e300;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double4 x = X[nd[k]];
        const double pr = dot3r(x.x, x.y, x.z, vx, vy, vz);
        if (pr < pmin) pmin = pr;
        if (pr > pmax) pmax = pr;
    }
}

// rho_tilde_kernel_sweep (kernels/upwind.py:345-454).
__global__ void k_rho_tilde_kernel(const int4* __restrict__ conn, const double4* __restrict__ X,
                                   const double4* __restrict__ cen, const int64_t* __restrict__ nb_off,
                                   const int32_t* __restrict__ nb_idx, const double* __restrict__ grad,
                                   const double* __restrict__ q2, const double* __restrict__ rho, int64_t E, Flow F,
                                   double reach_frac, double sig_s, double sig_p, double* __restrict__ nu_out,
                                   double* __restrict__ rt_out, up3d_monitors* mon) {
    WMon acc;
    GRID_STRIDE(e, E) {
        const double gx = grad[3 * e], gy = grad[3 * e + 1], gz = grad[3 * e + 2];
        const double gmag = sqrt(dot3r(gx, gy, gz, gx, gy, gz));
        const double nu_e = switch_of(mach2_of(q2[e], F), F);
        const double re = rho[e];
        double nu = nu_e, rt = re;
        if (gmag > 0.0) {
            const double vx = __ddiv_rn(gx, gmag), vy = __ddiv_rn(gy, gmag), vz = __ddiv_rn(gz, gmag);
            double pmin, pmax;
            stream_extent(conn[e], X, vx, vy, vz, pmin, pmax);
            const double extent = rsub(pmax, pmin);
            const double target = rmul(reach_frac, extent);
            const double ss = rmul(sig_s, extent), sp = rmul(sig_p, extent);
            const double inv2ss = __ddiv_rn(1.0, radd(rmul(2.0, rmul(ss, ss)), 1e-300));
            const double inv2sp = __ddiv_rn(1.0, radd(rmul(2.0, rmul(sp, sp)), 1e-300));
            const double4 ce = cen[e];
            double w_sum = 0.0, rho_acc = 0.0, m2_acc = 0.0;
            const int64_t j1 = nb_off[e + 1];
            for (int64_t j = nb_off[e]; j < j1; ++j) {
                const int32_t c = nb_idx[j];
                const double4 cc = cen[c];
                const double dx = rsub(cc.x, ce.x), dy = rsub(cc.y, ce.y), dz = rsub(cc.z, ce.z);
                const double up = -dot3r(vx, vy, vz, dx, dy, dz);
                if (up <= 0.0) continue;
                const double d2 = dot3r(dx, dy, dz, dx, dy, dz);
                double perp2 = rsub(d2, rmul(up, up));
                if (perp2 < 0.0) perp2 = 0.0;
                const double du = rsub(up, target);
                const double w = exp(-radd(rmul(rmul(du, du), inv2ss), rmul(perp2, inv2sp)));
                w_sum = radd(w_sum, w);
                rho_acc = radd(rho_acc, rmul(w, rho[c]));
                m2_acc = radd(m2_acc, rmul(w, mach2_of(q2[c], F)));
            }
            if (w_sum > 0.0) {
                const double rho_up = __ddiv_rn(rho_acc, w_sum), m2_up = __ddiv_rn(m2_acc, w_sum);
                const double nu_u = switch_of(m2_up, F);
                nu = nu_e > nu_u ? nu_e : nu_u;
                if (nu > 0.0) {
                    rt = rsub(re, rmul(nu, rsub(re, rho_up)));
                    rt = rt > F.floor_ ? rt : F.floor_;
                }
            }
        }
        nu_out[e] = nu;
        rt_out[e] = rt;
        acc.nu_max = fmax(acc.nu_max, nu);
        acc.sup += (nu > 0.0);
        acc.flo += (rt == F.floor_);
    }
    if (mon) flush(acc, mon);
}

// rho_tilde_weighted_sweep, the face-ring "blend" (kernels/upwind.py:176-309).
__global__ void k_rho_tilde_blend(const int4* __restrict__ conn, const double4* __restrict__ X,
                                  const double4* __restrict__ cen, const int4* __restrict__ fn,
                                  const double* __restrict__ grad, const double* __restrict__ q2,
                                  const double* __restrict__ rho, int64_t E, Flow F, double p_weight,
                                  double reach_frac, double gain_max, double* __restrict__ nu_out,
                                  double* __restrict__ rt_out, up3d_monitors* mon) {
    WMon acc;
    GRID_STRIDE(e, E) {
        const double gx = grad[3 * e], gy = grad[3 * e + 1], gz = grad[3 * e + 2];
        const double gmag = sqrt(dot3r(gx, gy, gz, gx, gy, gz));
        const double nu_e = switch_of(mach2_of(q2[e], F), F);
        const double re = rho[e];
        double nu = nu_e, rt = re;
        if (gmag > 0.0) {
            const double vx = __ddiv_rn(gx, gmag), vy = __ddiv_rn(gy, gmag), vz = __ddiv_rn(gz, gmag);
            const double4 ce = cen[e];
            const int4 f4 = fn[e];
            const int32_t nbs[4] = {f4.x, f4.y, f4.z, f4.w};
            double w_sum = 0.0, rho_acc = 0.0, m2_acc = 0.0, reach_acc = 0.0;
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                const int32_t nb = nbs[f];
                if (nb < 0 || nb >= E) continue;
                const double4 cc = cen[nb];
                const double dx = rsub(cc.x, ce.x), dy = rsub(cc.y, ce.y), dz = rsub(cc.z, ce.z);
                const double dlen = sqrt(dot3r(dx, dy, dz, dx, dy, dz));
                if (dlen <= 0.0) continue;
                const double up = -dot3r(vx, vy, vz, dx, dy, dz);
                const double a = __ddiv_rn(up, dlen);
                if (a <= 0.0) continue;
                const double w = pow(a, p_weight);
                w_sum = radd(w_sum, w);
                rho_acc = radd(rho_acc, rmul(w, rho[nb]));
                m2_acc = radd(m2_acc, rmul(w, mach2_of(q2[nb], F)));
                reach_acc = radd(reach_acc, rmul(w, up));
            }
            if (w_sum > 0.0) {
                const double rho_up = __ddiv_rn(rho_acc, w_sum), m2_up = __ddiv_rn(m2_acc, w_sum);
                const double reach = __ddiv_rn(reach_acc, w_sum);
                const double nu_u = switch_of(m2_up, F);
                nu = nu_e > nu_u ? nu_e : nu_u;
                if (nu > 0.0) {
                    double pmin, pmax;
                    stream_extent(conn[e], X, vx, vy, vz, pmin, pmax);
                    const double reach_target = rmul(reach_frac, rsub(pmax, pmin));
                    double g = __ddiv_rn(reach_target, reach > 1e-30 ? reach : 1e-30);
                    if (g < 1.0) g = 1.0;
                    else if (g > gain_max) g = gain_max;
                    rt = rsub(re, rmul(rmul(nu, g), rsub(re, rho_up)));
                    rt = rt > F.floor_ ? rt : F.floor_;
                }
            }
        }
        nu_out[e] = nu;
        rt_out[e] = rt;
        acc.nu_max = fmax(acc.nu_max, nu);
        acc.sup += (nu > 0.0);
        acc.flo += (rt == F.floor_);
    }
    if (mon) flush(acc, mon);
}

}  // namespace

// Neighbourhoods deeper than NB_MAX_DEPTH hops grow past what one
// thread's list holds; they are built on the host from a copy of the face
// table (OpenMP over elements; one mark array per thread makes each BFS
// linear in the neighbourhood's size) and uploaded.  Same lists: the
// elements within `depth` hops, the element excluded, ascending.
// Synchronises the stream.
static int64_t neighborhoods_host(const int4* fn_dev, int64_t E, int depth, int64_t* off_dev, DBuf<int32_t>* idx_out,
                                  int32_t* idx_dev, cudaStream_t s) {
    std::vector<int4> fn(E);
    if (E) UP3D_CUDA(cudaMemcpyAsync(fn.data(), fn_dev, sizeof(int4) * E, cudaMemcpyDeviceToHost, s));
    UP3D_CUDA(cudaStreamSynchronize(s));
    std::vector<std::vector<int32_t>> lists(E);
#pragma omp parallel
    {
        std::vector<int64_t> mark(E, -1);
        std::vector<int32_t> seen;
#pragma omp for schedule(dynamic, 1024)
        for (int64_t e = 0; e < E; ++e) {
            seen.clear();
            seen.push_back((int32_t)e);
            mark[e] = e;
            size_t lo = 0, hi = 1;
            for (int d = 0; d < depth && lo < hi; ++d) {
                for (size_t i = lo; i < hi; ++i) {
                    const int4 f = fn[seen[i]];
                    const int32_t nb[4] = {f.x, f.y, f.z, f.w};
                    for (int k = 0; k < 4; ++k) {
                        if (nb[k] < 0 || nb[k] >= E || mark[nb[k]] == e) continue;
                        mark[nb[k]] = e;
                        seen.push_back(nb[k]);
                    }
                }
                lo = hi;
                hi = seen.size();
            }
            lists[e].assign(seen.begin() + 1, seen.end());
            std::sort(lists[e].begin(), lists[e].end());
        }
    }
    std::vector<int64_t> off(E + 1, 0);
    for (int64_t e = 0; e < E; ++e) off[e + 1] = off[e] + (int64_t)lists[e].size();
    const int64_t total = off[E];
    std::vector<int32_t> idx(total > 0 ? total : 1);
    for (int64_t e = 0; e < E; ++e) std::copy(lists[e].begin(), lists[e].end(), idx.begin() + off[e]);
    UP3D_CUDA(cudaMemcpyAsync(off_dev, off.data(), sizeof(int64_t) * (E + 1), cudaMemcpyHostToDevice, s));
    int32_t* dst = idx_dev;
    if (idx_out) {
        idx_out->alloc(total > 0 ? total : 1);
        dst = idx_out->get();
    }
    if (dst && total) UP3D_CUDA(cudaMemcpyAsync(dst, idx.data(), sizeof(int32_t) * total, cudaMemcpyHostToDevice, s));
    UP3D_CUDA(cudaStreamSynchronize(s));
    return total;
}

// Offsets (n + 1) of the depth-hop neighbourhoods of the face-neighbour
// table fn; returns the total.  Synchronises the stream.
static int64_t neighborhood_offsets(const int4* fn, int64_t E, int depth, int64_t* off, DBuf<unsigned char>& tmp,
                                    cudaStream_t s) {
    DBuf<int64_t> cnt;
    cnt.alloc(E);
    k_neighborhoods<false><<<grid_for(E, 128), 128, 0, s>>>(fn, E, depth, cnt.get(), nullptr, nullptr);
    UP3D_CHECK_LAUNCH();
    UP3D_CUDA(cudaMemsetAsync(off, 0, sizeof(int64_t), s));
    size_t bytes = 0;
    UP3D_CUDA(cub::DeviceScan::InclusiveSum(nullptr, bytes, cnt.get(), off + 1, E, s));
    tmp.alloc(bytes);
    UP3D_CUDA(cub::DeviceScan::InclusiveSum(tmp.get(), bytes, cnt.get(), off + 1, E, s));
    int64_t total = 0;
    UP3D_CUDA(cudaMemcpyAsync(&total, off + E, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    UP3D_CUDA(cudaStreamSynchronize(s));
    return total;
}

// Builds (or reuses) the mesh's neighbourhood CSR of the given depth.
// Synchronises the stream (the total sizes the index array).
void ensure_neighborhoods(up3d_mesh* m, int depth, cudaStream_t s) {
    if (m->nb_depth == depth) return;
    const int64_t E = m->E;
    m->nb_depth = 0;
    m->nb_off.alloc(E + 1);
    if (depth > NB_MAX_DEPTH) {
        m->nb_total = neighborhoods_host(m->fnbr.get(), E, depth, m->nb_off.get(), &m->nb_idx, nullptr, s);
        m->nb_depth = depth;
        return;
    }
    DBuf<unsigned char> tmp;
    const int64_t total = neighborhood_offsets(m->fnbr.get(), E, depth, m->nb_off.get(), tmp, s);
    m->nb_idx.alloc(total > 0 ? total : 1);
    k_neighborhoods<true><<<grid_for(E, 128), 128, 0, s>>>(m->fnbr.get(), E, depth, nullptr, m->nb_off.get(),
                                                          m->nb_idx.get());
    UP3D_CHECK_LAUNCH();
    m->nb_total = total;
    m->nb_depth = depth;
}

}  // namespace up3d

using namespace up3d;

extern "C" {

int up3d_face_normals(const up3d_mesh* m, double* out, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(m && out, UP3D_ERR_ARGUMENT, "up3d_face_normals: null argument");
        k_face_normals<<<grid_for(m->E, 256), 256, 0, S(stream)>>>(m->conn.get(), m->nodes4.get(), m->E, out);
        UP3D_CHECK_LAUNCH();
    });
}

int up3d_mesh_neighborhoods(up3d_mesh* m, int depth, const int64_t** offsets, const int32_t** indices,
                            int64_t* total, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(m, UP3D_ERR_ARGUMENT, "up3d_mesh_neighborhoods: null argument");
        UP3D_REQUIRE(depth >= 1, UP3D_ERR_VALUE, "up3d_mesh_neighborhoods: depth must be >= 1");
        ensure_neighborhoods(m, depth, S(stream));
        if (offsets) *offsets = m->nb_off.get();
        if (indices) *indices = m->nb_idx.get();
        if (total) *total = m->nb_total;
    });
}

int up3d_face_neighborhoods(const int32_t* fn, int64_t n, int depth, int64_t* offsets, int32_t* indices,
                            int64_t* total, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(fn && offsets && n >= 0, UP3D_ERR_ARGUMENT, "up3d_face_neighborhoods: null argument");
        UP3D_REQUIRE(depth >= 1, UP3D_ERR_VALUE, "up3d_face_neighborhoods: depth must be >= 1");
        cudaStream_t s = S(stream);
        const int4* f4 = reinterpret_cast<const int4*>(fn);
        if (!indices) {
            UP3D_REQUIRE(total, UP3D_ERR_ARGUMENT, "up3d_face_neighborhoods: total is needed with offsets only");
            if (n == 0) {
                UP3D_CUDA(cudaMemsetAsync(offsets, 0, sizeof(int64_t), s));
                *total = 0;
                return;
            }
            if (depth > NB_MAX_DEPTH) {
                *total = neighborhoods_host(f4, n, depth, offsets, nullptr, nullptr, s);
                return;
            }
            DBuf<unsigned char> tmp;
            *total = neighborhood_offsets(f4, n, depth, offsets, tmp, s);
            return;
        }
        if (n == 0) return;
        if (depth > NB_MAX_DEPTH) {
            neighborhoods_host(f4, n, depth, offsets, nullptr, indices, s);
            return;
        }
        k_neighborhoods<true><<<grid_for(n, 128), 128, 0, s>>>(f4, n, depth, nullptr, offsets, indices);
        UP3D_CHECK_LAUNCH();
    });
}

int up3d_rho_tilde_kernel(up3d_mesh* m, const double* grad, const double* q2, const double* rho,
                          const up3d_flow* flow, int depth, double reach_frac, double sigma_s_frac,
                          double sigma_p_frac, double* nu, double* rho_tilde, up3d_monitors* mon,
                          up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(m && grad && q2 && rho && flow && nu && rho_tilde, UP3D_ERR_ARGUMENT,
                     "up3d_rho_tilde_kernel: null argument");
        UP3D_REQUIRE(depth >= 1, UP3D_ERR_VALUE, "up3d_rho_tilde_kernel: depth must be >= 1");
        cudaStream_t s = S(stream);
        ensure_neighborhoods(m, depth, s);
        if (mon) UP3D_CUDA(cudaMemsetAsync(mon, 0, sizeof(up3d_monitors), s));
        k_rho_tilde_kernel<<<grid_for(m->E, 256), 256, 0, s>>>(
            m->conn.get(), m->nodes4.get(), m->cen.get(), m->nb_off.get(), m->nb_idx.get(), grad, q2, rho, m->E,
            make_flow(*flow), reach_frac, sigma_s_frac, sigma_p_frac, nu, rho_tilde, mon);
        UP3D_CHECK_LAUNCH();
    });
}

int up3d_rho_tilde_blend(const up3d_mesh* m, const double* grad, const double* q2, const double* rho,
                         const up3d_flow* flow, double p_weight, double reach_frac, double reach_gain_max,
                         double* nu, double* rho_tilde, up3d_monitors* mon, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(m && grad && q2 && rho && flow && nu && rho_tilde, UP3D_ERR_ARGUMENT,
                     "up3d_rho_tilde_blend: null argument");
        cudaStream_t s = S(stream);
        if (mon) UP3D_CUDA(cudaMemsetAsync(mon, 0, sizeof(up3d_monitors), s));
        k_rho_tilde_blend<<<grid_for(m->E, 256), 256, 0, s>>>(m->conn.get(), m->nodes4.get(), m->cen.get(),
                                                              m->fnbr.get(), grad, q2, rho, m->E, make_flow(*flow),
                                                              p_weight, reach_frac, reach_gain_max, nu,
                                                              rho_tilde, mon);
        UP3D_CHECK_LAUNCH();
    });
}

}  // extern "C"
