// Discrete adjoint building blocks of the up3d library: the vector-Jacobian
// product of the residual with respect to the node coordinates and the
// free-stream Mach number, and the transpose of the Newton Jacobian's
// values on the symmetric P1 pattern.
//
// The residual (kernels/jacobian.py:361-375, kernels/residual.py:44-76) is
//   R_i = sum_e rho~_e V_e (g_e . B_e,i),   g_e = sum_j phi_j B_e,j,
// with rho~_e a function of q2_e = |g_e|^2 / u_inf^2, of q2 of the upstream
// element u(e) and of M_inf (upstream and branch held fixed: the
// linearisation the Newton Jacobian uses).  For L = lam^T R + sum_e w_e q2_e
// (w: an objective's weights on the element speeds) the product is formed
// element-locally, with no stored per-element intermediates beyond scalars:
//   pass 1 (per element e): c_e = V_e (g_e . h_e), h_e = sum_i lam_i B_e,i;
//     t_e = c_e s_e + w_e (weight on q2_e), a_e = c_e s_u (weight on q2 of
//     u(e)), and c_e d rho~_e / dM by forward-mode differentiation;
//   the a_e are summed per upstream element in ascending e (stable sort);
//   pass 2 (per element k): dL/dB_k,j = rho~ V (phi_j h + lam_j g)
//     + Q_k (2/u^2) phi_j g with Q_k = t_k + sum a, dL/dV_k = rho~ (g . h),
//     then through B = D^-1 (rows), V = |det D| / 6 with D = [x1-x0, x2-x0,
//     x3-x0]:  dL/dD = -B^T G B^T + dL/dV V B^T;
//   node gathers over the node -> element entries (fixed order).
// Everything is deterministic (no atomics on values).

#include <cub/cub.cuh>

#include "elem.cuh"
#include "internal.cuh"

namespace up3d {

namespace {

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

// ------------------------------------------------------------ forward-mode dual numbers

struct Dual {
    double v, d;
};
__device__ __forceinline__ Dual dconst(double v) { return {v, 0.0}; }
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
    const double q = a.v / b.v;
    return {q, (a.d - q * b.d) / b.v};
}
__device__ __forceinline__ Dual dpow(Dual a, double p) {
    const double v = pow(a.v, p);
    return {v, p * pow(a.v, p - 1.0) * a.d};
}

struct FlowM {  // the Mach-independent flow constants
    double gamma, hgm, expo, mc2, C, floor_, mcap2;
};

// density of the limited speed, as a function of M (q2n fixed): the
// limiter cap q2(M_cap) moves with M (physics/isentropic.py:262-314)
__device__ Dual rho_dual(double q2n, Dual m2, const FlowM& F, Dual& q2l, Dual& b) {
    const Dual cap = (dconst(F.mcap2) * (dconst(1.0) + dconst(F.hgm) * m2)) /
                     (m2 * dconst(1.0 + F.hgm * F.mcap2));
    q2l = q2n < cap.v ? dconst(q2n) : cap;
    b = dconst(1.0) + dconst(F.hgm) * m2 * (dconst(1.0) - q2l);
    if (b.v < 1e-10) b = dconst(1e-10);
    return dpow(b, F.expo);
}

// nu = C max(0, 1 - M_c^2 / max(M^2, M_c^2)) of the local Mach number
__device__ Dual nu_dual(Dual q2l, Dual b, Dual m2, const FlowM& F) {
    const Dual ml2 = q2l * m2 / b;
    if (ml2.v > F.mc2) return dconst(F.C) * (dconst(1.0) - dconst(F.mc2) / ml2);
    return dconst(0.0);
}

// d rho~ / dM at fixed speeds, upstream and (frozen) branch; br < 0: live
__device__ double drho_tilde_dM(double q2n_e, double q2n_u, bool self_up, int br, double m_inf, const FlowM& F) {
    const Dual M = {m_inf, 1.0};
    const Dual m2 = M * M;
    Dual q2e, be, q2u, bu;
    const Dual rho_e = rho_dual(q2n_e, m2, F, q2e, be);
    if (br == 3) return 0.0;
    if (br == 0) return rho_e.d;
    const Dual rho_u = self_up ? rho_e : rho_dual(q2n_u, m2, F, q2u, bu);
    if (self_up) {
        q2u = q2e;
        bu = be;
    }
    Dual rt;
    if (br == 1 || br == 2) {
        const Dual nu = br == 1 ? nu_dual(q2e, be, m2, F) : nu_dual(q2u, bu, m2, F);
        rt = rho_e - nu * (rho_e - rho_u);
        return rt.d;
    }
    // live: nu = max(nu_e, nu_u), floored result
    const Dual nu_e = nu_dual(q2e, be, m2, F), nu_u = nu_dual(q2u, bu, m2, F);
    const Dual nu = nu_e.v >= nu_u.v ? nu_e : nu_u;
    rt = rho_e - nu * (rho_e - rho_u);
    return rt.v > F.floor_ ? rt.d : 0.0;
}

// ------------------------------------------------------------ passes

__device__ __forceinline__ void lam_grad(const int4 c, const double* b, const double* __restrict__ lam, double h[3]) {
    const double l0 = lam[c.x], l1 = lam[c.y], l2 = lam[c.z], l3 = lam[c.w];
#pragma unroll
    for (int d = 0; d < 3; ++d) h[d] = l0 * b[d] + l1 * b[3 + d] + l2 * b[6 + d] + l3 * b[9 + d];
}

// Pass 1: per element, the weights on its own speed (t), on its upstream
// element's speed (a), rho~, and c_e d rho~/dM summed per block.
__global__ void __launch_bounds__(256)
    k_vjp_elem(const int4* __restrict__ conn, const double* __restrict__ B, const double* __restrict__ V,
               const double* __restrict__ phi, Flow F, FlowM FM, double m_inf, double u2,
               const int64_t* __restrict__ up, const int8_t* __restrict__ br, int64_t E,
               const double* __restrict__ lam, const double* __restrict__ w, double* __restrict__ t_out,
               double* __restrict__ a_out, double* __restrict__ rt_out, int32_t* __restrict__ key,
               int32_t* __restrict__ val, double* __restrict__ partial) {
    __shared__ double sh[8];
    double dm = 0.0;
    GRID_STRIDE(e, E) {
        double g[3], b[12];
        int4 c;
        elem_grad_B(conn, B, phi, e, g, b, c);
        const double q2n = __ddiv_rn(dot3r(g[0], g[1], g[2], g[0], g[1], g[2]), u2);
        const double q2l = q2n < F.q2cap ? q2n : F.q2cap;
        const bool lim_e = q2l == q2n;
        double rho_e, drho_e;
        rho_drho(q2l, F, rho_e, drho_e);
        const int64_t u = safe_up(up[e], e, E);
        double q2nu = q2n, q2lu = q2l, rho_u = rho_e;
        bool lim_u = lim_e;
        if (u != e) {
            double gu[3];
            elem_grad(conn, B, phi, u, gu);
            q2nu = __ddiv_rn(dot3r(gu[0], gu[1], gu[2], gu[0], gu[1], gu[2]), u2);
            q2lu = q2nu < F.q2cap ? q2nu : F.q2cap;
            lim_u = q2lu == q2nu;
            rho_u = rho_of(q2lu, F);
        }
        double rt, se = 0.0, su = 0.0;
        int bb = -1;
        if (br) {
            bb = br[e];
            if (bb == 3) rt = F.floor_;
            else if (bb == 0) rt = rho_e;
            else rt = rho_e - switch_of(mach2_of(bb == 1 ? q2l : q2lu, F), F) * (rho_e - rho_u);
            frozen_sensitivities(bb, q2l, rho_e, q2lu, rho_u, F, se, su);
        } else {
            const double nu = fmax(switch_of(mach2_of(q2l, F), F), switch_of(mach2_of(q2lu, F), F));
            rt = rho_e - nu * (rho_e - rho_u);
            rt = rt > F.floor_ ? rt : F.floor_;
            live_sensitivities(q2l, rho_e, q2lu, rho_u, u == e, F, se, su);
        }
        se *= lim_e ? 1.0 : 0.0;
        su *= lim_u ? 1.0 : 0.0;
        double cval = 0.0;
        if (lam) {
            double h[3];
            lam_grad(c, b, lam, h);
            cval = V[e] * (g[0] * h[0] + g[1] * h[1] + g[2] * h[2]);
            if (cval != 0.0) dm += cval * drho_tilde_dM(q2n, q2nu, u == e, bb, m_inf, FM);
        }
        t_out[e] = cval * se + (w ? w[e] : 0.0);
        a_out[e] = u != e ? cval * su : 0.0;
        rt_out[e] = rt;
        key[e] = (int32_t)u;
        val[e] = (int32_t)e;
    }
    dm = warp_sum(dm);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = dm;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) s += sh[q];
        partial[blockIdx.x] = s;
    }
}

__global__ void k_vjp_sum_partials(const double* __restrict__ partial, int nb, double* __restrict__ out) {
    if (threadIdx.x >= 32) return;
    double s = 0.0;
    for (int b = threadIdx.x; b < nb; b += 32) s += partial[b];
    s = warp_sum(s);
    if (threadIdx.x == 0) *out = s;
}

// A[k] = sum of a_e over the elements e (ascending) whose upstream is k.
__global__ void k_vjp_upstream_sums(const int32_t* __restrict__ key, const int32_t* __restrict__ val,
                                    const double* __restrict__ a, int64_t E, double* __restrict__ A) {
    GRID_STRIDE(i, E) {
        const int32_t k = key[i];
        if (i > 0 && key[i - 1] == k) continue;
        double s = 0.0;
        for (int64_t j = i; j < E && key[j] == k; ++j) s += a[val[j]];
        A[k] = s;
    }
}

// Pass 2: per element, dL/dB and dL/dV through the inverse edge matrix to
// the four nodes (dx, 12 values) and the objective's phi gradient (dphi).
__global__ void __launch_bounds__(256)
    k_vjp_geom(const int4* __restrict__ conn, const double* __restrict__ B, const double* __restrict__ V,
               const double* __restrict__ phi, double u2, int64_t E, const double* __restrict__ lam,
               const double* __restrict__ w, const double* __restrict__ t, const double* __restrict__ A,
               const double* __restrict__ rt, double* __restrict__ dx, double* __restrict__ dphi) {
    GRID_STRIDE(e, E) {
        double g[3], b[12];
        int4 c;
        elem_grad_B(conn, B, phi, e, g, b, c);
        const double p[4] = {phi[c.x], phi[c.y], phi[c.z], phi[c.w]};
        double h[3] = {0.0, 0.0, 0.0}, l[4] = {0.0, 0.0, 0.0, 0.0};
        if (lam) {
            lam_grad(c, b, lam, h);
            l[0] = lam[c.x];
            l[1] = lam[c.y];
            l[2] = lam[c.z];
            l[3] = lam[c.w];
        }
        const double Ve = V[e], r = rt[e];
        const double Q = t[e] + A[e];
        const double q2w = 2.0 * Q / u2;
        double G[4][3];
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int d = 0; d < 3; ++d) G[j][d] = r * Ve * (p[j] * h[d] + l[j] * g[d]) + q2w * p[j] * g[d];
        const double GV = r * (g[0] * h[0] + g[1] * h[1] + g[2] * h[2]);
        // B_0 = -(B_1 + B_2 + B_3): fold its gradient into the three rows of D^-1
        double Gm[3][3], Bm[3][3];
#pragma unroll
        for (int m = 0; m < 3; ++m)
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                Gm[m][d] = G[m + 1][d] - G[0][d];
                Bm[m][d] = b[3 * (m + 1) + d];
            }
        // T = Gm Bm^T, then dD = -Bm^T T + GV V Bm^T
        double T[3][3];
#pragma unroll
        for (int m = 0; m < 3; ++m)
#pragma unroll
            for (int cc = 0; cc < 3; ++cc)
                T[m][cc] = Gm[m][0] * Bm[cc][0] + Gm[m][1] * Bm[cc][1] + Gm[m][2] * Bm[cc][2];
        double out[12];
#pragma unroll
        for (int r0 = 0; r0 < 3; ++r0) {
            double col_sum = 0.0;
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) {
                const double dD = -(Bm[0][r0] * T[0][cc] + Bm[1][r0] * T[1][cc] + Bm[2][r0] * T[2][cc]) +
                                  GV * Ve * Bm[cc][r0];
                out[3 * (cc + 1) + r0] = dD;  // node cc+1, component r0
                col_sum += dD;
            }
            out[r0] = -col_sum;
        }
        double2* o2 = reinterpret_cast<double2*>(dx + 12 * e);
#pragma unroll
        for (int k = 0; k < 6; ++k) o2[k] = make_double2(out[2 * k], out[2 * k + 1]);
        if (dphi) {
            const double we = w ? 2.0 * w[e] / u2 : 0.0;
#pragma unroll
            for (int j = 0; j < 4; ++j)
                dphi[4 * e + j] = we * (g[0] * b[3 * j] + g[1] * b[3 * j + 1] + g[2] * b[3 * j + 2]);
        }
    }
}

// Node sums over the node -> element entries in their fixed order.
__global__ void k_vjp_gather(int64_t N, const int32_t* __restrict__ ent_off, const uint32_t* __restrict__ ent,
                             const double* __restrict__ dx, const double* __restrict__ dphi_e,
                             double* __restrict__ dX, double* __restrict__ dphi) {
    GRID_STRIDE(n, N) {
        double sx = 0.0, sy = 0.0, sz = 0.0, sp = 0.0;
        for (int32_t k = ent_off[n]; k < ent_off[n + 1]; ++k) {
            const uint32_t x = ent[k];
            const int64_t e = x >> 2;
            const int i = x & 3;
            sx += dx[12 * e + 3 * i];
            sy += dx[12 * e + 3 * i + 1];
            sz += dx[12 * e + 3 * i + 2];
            if (dphi) sp += dphi_e[4 * e + i];
        }
        if (dX) {
            dX[3 * n] = sx;
            dX[3 * n + 1] = sy;
            dX[3 * n + 2] = sz;
        }
        if (dphi) dphi[n] = sp;
    }
}

// J^T on the symmetric pattern: out[z] = data[transposed slot of z].
__global__ void k_transpose_values(int64_t nnz, const int32_t* __restrict__ zt, const double* __restrict__ data,
                                   double* __restrict__ out) {
    GRID_STRIDE(z, nnz) out[z] = data[zt[z]];
}

}  // namespace

}  // namespace up3d

using namespace up3d;

extern "C" {

int up3d_residual_vjp(up3d_mesh* m, const double* phi, const up3d_flow* flow, const int64_t* upstream,
                      const int8_t* branch, const double* lam, const double* w_q2, double* dphi, double* dX,
                      double* dM, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(m && phi && flow && upstream, UP3D_ERR_ARGUMENT, "up3d_residual_vjp: null argument");
        UP3D_REQUIRE(!dphi || w_q2, UP3D_ERR_ARGUMENT, "up3d_residual_vjp: dphi needs w_q2");
        cudaStream_t s = S(stream);
        const int64_t E = m->E, N = m->N;
        const Flow F = make_flow(*flow);
        FlowM FM{flow->gamma, 0.5 * (flow->gamma - 1.0), 1.0 / (flow->gamma - 1.0),
                 flow->m_crit * flow->m_crit, flow->upwind_c, flow->rho_floor, flow->m_cap * flow->m_cap};
        const double u2 = flow->u_inf * flow->u_inf;
        m->adj_t.alloc(E);
        m->adj_a.alloc(E);
        m->adj_rt.alloc(E);
        m->adj_A.alloc(E);
        m->adj_dx.alloc(12 * E);
        m->adj_dphi.alloc(4 * E);
        m->adj_key.alloc(E);
        m->adj_key_s.alloc(E);
        m->adj_val.alloc(E);
        m->adj_val_s.alloc(E);
        const unsigned grid = grid_for(E, 256, (int64_t)148 * 8);
        m->adj_part.alloc(grid + 1);
        k_vjp_elem<<<grid, 256, 0, s>>>(m->conn.get(), m->B.get(), m->V.get(), phi, F, FM, flow->m_inf, u2,
                                        upstream, branch, E, lam, w_q2, m->adj_t.get(), m->adj_a.get(),
                                        m->adj_rt.get(), m->adj_key.get(), m->adj_val.get(), m->adj_part.get());
        UP3D_CHECK_LAUNCH();
        if (dM) {
            k_vjp_sum_partials<<<1, 32, 0, s>>>(m->adj_part.get(), (int)grid, dM);
            UP3D_CHECK_LAUNCH();
        }
        // upstream sums: stable sort by upstream element, then per-key runs
        int end_bit = 1;
        while ((1ll << end_bit) < E) ++end_bit;
        size_t bytes = 0;
        UP3D_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, m->adj_key.get(), m->adj_key_s.get(),
                                                  m->adj_val.get(), m->adj_val_s.get(), E, 0, end_bit, s));
        m->cub_tmp.alloc(bytes);
        UP3D_CUDA(cub::DeviceRadixSort::SortPairs(m->cub_tmp.get(), bytes, m->adj_key.get(), m->adj_key_s.get(),
                                                  m->adj_val.get(), m->adj_val_s.get(), E, 0, end_bit, s));
        UP3D_CUDA(cudaMemsetAsync(m->adj_A.get(), 0, sizeof(double) * E, s));
        k_vjp_upstream_sums<<<grid_for(E, 256), 256, 0, s>>>(m->adj_key_s.get(), m->adj_val_s.get(),
                                                             m->adj_a.get(), E, m->adj_A.get());
        UP3D_CHECK_LAUNCH();
        k_vjp_geom<<<grid_for(E, 256), 256, 0, s>>>(m->conn.get(), m->B.get(), m->V.get(), phi, u2, E, lam, w_q2,
                                                    m->adj_t.get(), m->adj_A.get(), m->adj_rt.get(),
                                                    m->adj_dx.get(), dphi ? m->adj_dphi.get() : nullptr);
        UP3D_CHECK_LAUNCH();
        if (dX || dphi) {
            k_vjp_gather<<<grid_for(N, 256), 256, 0, s>>>(N, m->ent_off.get(), m->ent.get(), m->adj_dx.get(),
                                                          m->adj_dphi.get(), dX, dphi);
            UP3D_CHECK_LAUNCH();
        }
    });
}

int up3d_jacobian_transpose(up3d_mesh* m, const double* data, double* data_t, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(m && data && data_t && data != data_t, UP3D_ERR_ARGUMENT,
                     "up3d_jacobian_transpose: null or aliased argument");
        k_transpose_values<<<grid_for(m->nnz, 256), 256, 0, S(stream)>>>(m->nnz, m->zt.get(), data, data_t);
        UP3D_CHECK_LAUNCH();
    });
}

}  // extern "C"
