// Device building blocks of the element sweeps, shared by the single-purpose
// kernels (elem.cu) and the fused residual/Jacobian sweep (assemble.cu).
#pragma once

#include "internal.cuh"

namespace up3d {

// grad(phi)_e = sum_i phi_i B_e[i,:] in the reference's order
// (kernels/gradient.py:52-60), IEEE-rounded.
// 32-byte read-only global load (one 256-bit request on sm_100 instead of
// two 128-bit ones: every per-element record here -- B (96 bytes), the face
// displacements (96 bytes), a node's (x, y, z, 0) (32 bytes) -- starts on a
// 32-byte boundary, and the L1 request count is what bounds the sweep).
__device__ __forceinline__ void ld4(const double* p, double& a, double& b, double& c, double& d) {
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(a), "=d"(b), "=d"(c), "=d"(d) : "l"(p));
}
// The 12 B values of an element (global memory, 32-byte aligned).
__device__ __forceinline__ void ld_B(const double* __restrict__ be, double b[12]) {
    ld4(be, b[0], b[1], b[2], b[3]);
    ld4(be + 4, b[4], b[5], b[6], b[7]);
    ld4(be + 8, b[8], b[9], b[10], b[11]);
}

// B_e (12 values) and V_e from the four node positions, with the operations
// of the mesh set-up's geometry kernel, k_geometry (identical bits for every
// element that passed its degeneracy check).
__device__ __forceinline__ void geom_B_pts(double x0x, double x0y, double x0z, double x1x, double x1y, double x1z,
                                           double x2x, double x2y, double x2z, double x3x, double x3y, double x3z,
                                           double b[12], double& V) {
    const double v1x = rsub(x1x, x0x), v1y = rsub(x1y, x0y), v1z = rsub(x1z, x0z);
    const double v2x = rsub(x2x, x0x), v2y = rsub(x2y, x0y), v2z = rsub(x2z, x0z);
    const double v3x = rsub(x3x, x0x), v3y = rsub(x3y, x0y), v3z = rsub(x3z, x0z);
    const double c23x = rsub(rmul(v2y, v3z), rmul(v2z, v3y));
    const double c23y = rsub(rmul(v2z, v3x), rmul(v2x, v3z));
    const double c23z = rsub(rmul(v2x, v3y), rmul(v2y, v3x));
    const double c31x = rsub(rmul(v3y, v1z), rmul(v3z, v1y));
    const double c31y = rsub(rmul(v3z, v1x), rmul(v3x, v1z));
    const double c31z = rsub(rmul(v3x, v1y), rmul(v3y, v1x));
    const double c12x = rsub(rmul(v1y, v2z), rmul(v1z, v2y));
    const double c12y = rsub(rmul(v1z, v2x), rmul(v1x, v2z));
    const double c12z = rsub(rmul(v1x, v2y), rmul(v1y, v2x));
    const double det = dot3r(v1x, v1y, v1z, c23x, c23y, c23z);
    V = __ddiv_rn(fabs(det), 6.0);
    const double inv = __ddiv_rn(1.0, det);
    b[3] = rmul(c23x, inv); b[4] = rmul(c23y, inv); b[5] = rmul(c23z, inv);
    b[6] = rmul(c31x, inv); b[7] = rmul(c31y, inv); b[8] = rmul(c31z, inv);
    b[9] = rmul(c12x, inv); b[10] = rmul(c12y, inv); b[11] = rmul(c12z, inv);
#pragma unroll
    for (int d = 0; d < 3; ++d) b[d] = -radd(radd(b[3 + d], b[6 + d]), b[9 + d]);
}
// The same from the node table (global memory).
__device__ __forceinline__ void geom_B(const double4* __restrict__ X, int4 c, double b[12], double& V) {
    double x0x, x0y, x0z, w, x1x, x1y, x1z, x2x, x2y, x2z, x3x, x3y, x3z;
    ld4(reinterpret_cast<const double*>(X + c.x), x0x, x0y, x0z, w);
    ld4(reinterpret_cast<const double*>(X + c.y), x1x, x1y, x1z, w);
    ld4(reinterpret_cast<const double*>(X + c.z), x2x, x2y, x2z, w);
    ld4(reinterpret_cast<const double*>(X + c.w), x3x, x3y, x3z, w);
    geom_B_pts(x0x, x0y, x0z, x1x, x1y, x1z, x2x, x2y, x2z, x3x, x3y, x3z, b, V);
}
__device__ __forceinline__ void grad_from_B(int4 c, const double b[12], const double* __restrict__ phi, double g[3]) {
    const double p0 = phi[c.x], p1 = phi[c.y], p2 = phi[c.z], p3 = phi[c.w];
#pragma unroll
    for (int d = 0; d < 3; ++d)
        g[d] = radd(radd(radd(rmul(p0, b[d]), rmul(p1, b[3 + d])), rmul(p2, b[6 + d])), rmul(p3, b[9 + d]));
}

// From the element's nodes c and its 12 B values at `be` (global memory).
__device__ __forceinline__ void elem_grad_rec(int4 c, const double* __restrict__ be, const double* __restrict__ phi,
                                              double g[3]) {
    double b[12];
    ld_B(be, b);
    double p0 = phi[c.x], p1 = phi[c.y], p2 = phi[c.z], p3 = phi[c.w];
    g[0] = radd(radd(radd(rmul(p0, b[0]), rmul(p1, b[3])), rmul(p2, b[6])), rmul(p3, b[9]));
    g[1] = radd(radd(radd(rmul(p0, b[1]), rmul(p1, b[4])), rmul(p2, b[7])), rmul(p3, b[10]));
    g[2] = radd(radd(radd(rmul(p0, b[2]), rmul(p1, b[5])), rmul(p2, b[8])), rmul(p3, b[11]));
}
__device__ __forceinline__ void elem_grad(const int4* __restrict__ conn, const double* __restrict__ B,
                                          const double* __restrict__ phi, int64_t e, double g[3]) {
    elem_grad_rec(conn[e], B + 12 * e, phi, g);
}

// Same, also returning B_e (12 values) for reuse.
__device__ __forceinline__ void elem_grad_B(const int4* __restrict__ conn, const double* __restrict__ B,
                                            const double* __restrict__ phi, int64_t e, double g[3],
                                            double b[12], int4& c) {
    c = conn[e];
    ld_B(B + 12 * e, b);
    double p0 = phi[c.x], p1 = phi[c.y], p2 = phi[c.z], p3 = phi[c.w];
#pragma unroll
    for (int d = 0; d < 3; ++d)
        g[d] = radd(radd(radd(rmul(p0, b[d]), rmul(p1, b[3 + d])), rmul(p2, b[6 + d])), rmul(p3, b[9 + d]));
}

// upstream_elements (kernels/upwind.py:69-125): hop to the face neighbour
// with the most negative centroid displacement along grad until the reach
// covers 0.8 of the element's streamwise extent, at most 4 hops; u(e) = e
// when nothing is upstream.  The displacements cen(nbr) - cen(cur) come
// precomputed per element and face (IEEE-rounded like every other walk
// operation), so a hop is one dependent load of (fn, disp)[cur] instead of
// fn[cur] followed by four centroid gathers.  Neighbour entries outside
// [0, E) count as boundary faces.
__device__ __forceinline__ int64_t upstream_walk(const int4* __restrict__ fn, const double* __restrict__ disp,
                                                 const double4* __restrict__ X, const int4* __restrict__ conn,
                                                 int64_t e, int64_t E, const double g[3]) {
    const double gx = g[0], gy = g[1], gz = g[2];
    int4 c = conn[e];
    int nd[4] = {c.x, c.y, c.z, c.w};
    double pmin = 1e300, pmax = -1e300;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        double x, y, z, w;
        ld4(reinterpret_cast<const double*>(X + nd[k]), x, y, z, w);
        double p = dot3r(x, y, z, gx, gy, gz);
        if (p < pmin) pmin = p;
        if (p > pmax) pmax = p;
    }
    const double target = rmul(0.8, rsub(pmax, pmin));
    int64_t cur = e;
    double reach = 0.0;
    for (int hops = 0; hops < 4 && reach < target; ++hops) {
        const int4 f = fn[cur];
        double a[12];
        ld_B(disp + 12 * cur, a);  // the face displacements: the same 96-byte record shape
        const int nb[4] = {f.x, f.y, f.z, f.w};
        const double d[4] = {dot3r(a[0], a[1], a[2], gx, gy, gz), dot3r(a[3], a[4], a[5], gx, gy, gz),
                             dot3r(a[6], a[7], a[8], gx, gy, gz), dot3r(a[9], a[10], a[11], gx, gy, gz)};
        int64_t best = -1;
        double best_disp = 0.0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (nb[k] >= 0 && nb[k] < E && d[k] < best_disp) {
                best_disp = d[k];
                best = nb[k];
            }
        }
        if (best < 0) break;
        cur = best;
        reach = radd(reach, -best_disp);
    }
    return cur;
}

// rho_tilde_sensitivities_sweep, one element (kernels/upwind.py:687-730).
__device__ __forceinline__ void live_sensitivities(double q2e, double rho_e, double q2u, double rho_u, bool self_up,
                                                   const Flow& F, double& se, double& su) {
    double r_tmp, drho_e;
    rho_drho(q2e, F, r_tmp, drho_e);
    if (self_up) {
        se = rho_e <= F.floor_ ? 0.0 : drho_e;
        su = 0.0;
        return;
    }
    double m2 = mach2_of(q2e, F), m2u = mach2_of(q2u, F);
    double nu_e = switch_of(m2, F), nu_u = switch_of(m2u, F);
    double nu = fmax(nu_e, nu_u);
    double rt = rho_e - nu * (rho_e - rho_u);
    if (rt <= F.floor_) {
        se = 0.0;
        su = 0.0;
        return;
    }
    if (nu == 0.0) {
        se = drho_e;
        su = 0.0;
        return;
    }
    double drho_u;
    rho_drho(q2u, F, r_tmp, drho_u);
    double djump = rho_e - rho_u;
    if (nu_e >= nu_u) {
        double dnu_e = m2 > F.mc2 ? dswitch_of(q2e, m2, F) : 0.0;
        se = drho_e * (1.0 - nu) - djump * dnu_e;
        su = nu * drho_u;
    } else {
        double dnu_u = dswitch_of(q2u, m2u, F);
        se = drho_e * (1.0 - nu);
        su = nu * drho_u - djump * dnu_u;
    }
}

// rho_tilde_frozen_sensitivities_sweep, one element (kernels/upwind.py:616-643).
__device__ __forceinline__ void frozen_sensitivities(int b, double q2e, double rho_e, double q2u, double rho_u,
                                                     const Flow& F, double& se, double& su) {
    if (b == 3) {
        se = 0.0;
        su = 0.0;
        return;
    }
    double r_tmp, drho_e;
    rho_drho(q2e, F, r_tmp, drho_e);
    if (b == 0) {
        se = drho_e;
        su = 0.0;
        return;
    }
    double drho_u;
    rho_drho(q2u, F, r_tmp, drho_u);
    double djump = rho_e - rho_u;
    if (b == 1) {
        double m2 = mach2_of(q2e, F);
        double nu = switch_of(m2, F);
        double dnu_e = m2 > F.mc2 ? dswitch_of(q2e, m2, F) : 0.0;
        se = drho_e * (1.0 - nu) - djump * dnu_e;
        su = nu * drho_u;
    } else {
        double m2u = mach2_of(q2u, F);
        double nu = switch_of(m2u, F);
        double dnu_u = m2u > F.mc2 ? dswitch_of(q2u, m2u, F) : 0.0;
        se = drho_e * (1.0 - nu);
        su = nu * drho_u - djump * dnu_u;
    }
}

void launch_velocities(const up3d_mesh* m, const double* phi, double* grad, double* q2, cudaStream_t s);
void launch_walk32(const up3d_mesh* m, const double* grad, int32_t* up, cudaStream_t s);

}  // namespace up3d
