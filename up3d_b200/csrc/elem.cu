// Element sweeps of the up3d library: velocities, the isentropic field
// functions, the multi-hop upstream walk, the upwinded density (live and
// frozen), branch classification and the exact flux sensitivities.
//
// Reference: kernels/gradient.py:33-64, physics/isentropic.py:236-374,
// kernels/upwind.py:69-125, :457-730.

#include <cmath>

#include "elem.cuh"
#include "internal.cuh"

namespace up3d {

Flow make_flow(const up3d_flow& f) {
    Flow F;
    F.m2inf = f.m_inf * f.m_inf;
    F.hgm = 0.5 * (f.gamma - 1.0);
    F.expo = 1.0 / (f.gamma - 1.0);
    F.gamma = f.gamma;
    F.two_m_g = 2.0 - f.gamma;
    F.mc2 = f.m_crit * f.m_crit;
    F.C = f.upwind_c;
    F.floor_ = f.rho_floor;
    double u2 = f.u_inf * f.u_inf;
    F.inv_u2 = 1.0 / u2;
    // q2_at_mach (physics/isentropic.py:283-289): +inf at M_inf == 0
    if (f.m_inf == 0.0) {
        F.q2cap = INFINITY;
    } else {
        double mc = f.m_cap * f.m_cap;
        F.q2cap = mc * (1.0 + 0.5 * (f.gamma - 1.0) * F.m2inf) / (F.m2inf * (1.0 + 0.5 * (f.gamma - 1.0) * mc));
    }
    F.air = (f.gamma == 1.4);
    return F;
}

namespace {

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

__global__ void k_velocities(const int4* __restrict__ conn, const double* __restrict__ B,
                             const double* __restrict__ phi, int64_t E, double* __restrict__ grad,
                             double* __restrict__ q2) {
    GRID_STRIDE(e, E) {
        double g[3];
        elem_grad(conn, B, phi, e, g);
        grad[3 * e] = g[0];
        grad[3 * e + 1] = g[1];
        grad[3 * e + 2] = g[2];
        q2[e] = dot3r(g[0], g[1], g[2], g[0], g[1], g[2]);
    }
}

__global__ void k_limit(const double* __restrict__ q2, int64_t n, double cap, double* __restrict__ out,
                        unsigned long long* n_lim) {
    unsigned long long cnt = 0;
    GRID_STRIDE(i, n) {
        double q = q2[i];
        double o = q < cap ? q : cap;
        out[i] = o;
        cnt += (o != q);
    }
    if (n_lim) {
        cnt = warp_sum_u64(cnt);
        if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(n_lim, cnt);
    }
}

template <int WHAT>
__global__ void k_field(const double* __restrict__ q2, int64_t n, Flow F, double* __restrict__ out) {
    GRID_STRIDE(i, n) {
        double q = q2[i];
        double v;
        if (WHAT == 0) {
            v = rho_of(q, F);
        } else if (WHAT == 1) {
            v = mach2_of(q, F);
        } else if (WHAT == 2) {
            double r, d;
            rho_drho(q, F, r, d);
            v = d;
        } else if (WHAT == 3) {
            v = dmach2_of(q, F);
        } else {
            // Cp = 2 / (gamma M^2) (rho^gamma - 1)   (physics/isentropic.py:141-143)
            double r = rho_of(q, F);
            v = 2.0 / (F.gamma * F.m2inf) * (pow(r, F.gamma) - 1.0);
        }
        out[i] = v;
    }
}

template <class IDX>
__global__ void k_walk(const int4* __restrict__ fn, const double* __restrict__ disp,
                       const double4* __restrict__ X, const int4* __restrict__ conn,
                       const double* __restrict__ grad, int64_t E, IDX* __restrict__ out) {
    GRID_STRIDE(e, E) {
        double g[3] = {grad[3 * e], grad[3 * e + 1], grad[3 * e + 2]};
        out[e] = (IDX)upstream_walk(fn, disp, X, conn, e, E, g);
    }
}

struct MonAcc {
    double nu_max = 0.0;
    unsigned long long sup = 0, flo = 0;
};

__device__ __forceinline__ void flush_monitors(MonAcc a, up3d_monitors* mon) {
    double nm = warp_max(a.nu_max);
    unsigned long long s = warp_sum_u64(a.sup), f = warp_sum_u64(a.flo);
    if ((threadIdx.x & 31) == 0) {
        if (nm > 0.0) atomic_max_nonneg(&mon->nu_max, nm);
        if (s) atomicAdd(reinterpret_cast<unsigned long long*>(&mon->n_supersonic), s);
        if (f) atomicAdd(reinterpret_cast<unsigned long long*>(&mon->n_floored), f);
    }
}

// rho_tilde_sweep (kernels/upwind.py:457-500)
__global__ void k_rho_tilde(const double* __restrict__ q2, const double* __restrict__ rho,
                            const int64_t* __restrict__ up, int64_t n, Flow F, double* __restrict__ nu_out,
                            double* __restrict__ rt_out, up3d_monitors* mon) {
    MonAcc acc;
    GRID_STRIDE(e, n) {
        int64_t u = safe_up(up[e], e, n);
        double nu = fmax(switch_of(mach2_of(q2[e], F), F), switch_of(mach2_of(q2[u], F), F));
        double re = rho[e];
        double rt = re - nu * (re - rho[u]);
        rt = rt > F.floor_ ? rt : F.floor_;
        nu_out[e] = nu;
        rt_out[e] = rt;
        acc.nu_max = fmax(acc.nu_max, nu);
        acc.sup += (nu > 0.0);
        acc.flo += (rt == F.floor_);
    }
    if (mon) flush_monitors(acc, mon);
}

// classify_upwind_branches (kernels/upwind.py:504-541)
__global__ void k_classify(const double* __restrict__ q2, const double* __restrict__ rho,
                           const int64_t* __restrict__ up, int64_t n, Flow F, int8_t* __restrict__ br) {
    GRID_STRIDE(e, n) {
        int64_t u = safe_up(up[e], e, n);
        if (u == e) {
            br[e] = rho[e] <= F.floor_ ? 3 : 0;
            continue;
        }
        double nu_e = switch_of(mach2_of(q2[e], F), F);
        double nu_u = switch_of(mach2_of(q2[u], F), F);
        double nu = fmax(nu_e, nu_u);
        double rt = rho[e] - nu * (rho[e] - rho[u]);
        br[e] = rt <= F.floor_ ? 3 : (nu == 0.0 ? 0 : (nu_e >= nu_u ? 1 : 2));
    }
}

// rho_tilde_frozen_sweep (kernels/upwind.py:545-593)
__global__ void k_rho_tilde_frozen(const double* __restrict__ q2, const double* __restrict__ rho,
                                   const int64_t* __restrict__ up, const int8_t* __restrict__ br, int64_t n,
                                   Flow F, double* __restrict__ nu_out, double* __restrict__ rt_out,
                                   up3d_monitors* mon) {
    MonAcc acc;
    GRID_STRIDE(e, n) {
        int b = br[e];
        double nu = 0.0, rt;
        if (b == 3) {
            rt = F.floor_;
            acc.flo += 1;
        } else if (b == 0) {
            rt = rho[e];
        } else {
            int64_t u = safe_up(up[e], e, n);
            nu = switch_of(mach2_of(q2[b == 1 ? e : u], F), F);
            rt = rho[e] - nu * (rho[e] - rho[u]);
        }
        nu_out[e] = nu;
        rt_out[e] = rt;
        acc.nu_max = fmax(acc.nu_max, nu);
        acc.sup += (nu > 0.0);
    }
    if (mon) flush_monitors(acc, mon);
}

__global__ void k_sens(const double* __restrict__ q2, const double* __restrict__ rho,
                       const int64_t* __restrict__ up, int64_t n, Flow F, double* __restrict__ se,
                       double* __restrict__ su) {
    GRID_STRIDE(e, n) {
        int64_t u = safe_up(up[e], e, n);
        double s_e, s_u;
        live_sensitivities(q2[e], rho[e], q2[u], rho[u], u == e, F, s_e, s_u);
        se[e] = s_e;
        su[e] = s_u;
    }
}

__global__ void k_sens_frozen(const double* __restrict__ q2, const double* __restrict__ rho,
                              const int64_t* __restrict__ up, const int8_t* __restrict__ br, int64_t n,
                              Flow F, double* __restrict__ se, double* __restrict__ su) {
    GRID_STRIDE(e, n) {
        int64_t u = safe_up(up[e], e, n);
        double s_e, s_u;
        frozen_sensitivities(br[e], q2[e], rho[e], q2[u], rho[u], F, s_e, s_u);
        se[e] = s_e;
        su[e] = s_u;
    }
}

}  // namespace

// ------------------------------------------------------------ launchers

void launch_velocities(const up3d_mesh* m, const double* phi, double* grad, double* q2, cudaStream_t s) {
    k_velocities<<<grid_for(m->E, 256), 256, 0, s>>>(m->conn.get(), m->B.get(), phi, m->E, grad, q2);
    UP3D_CHECK_LAUNCH();
}

void launch_walk32(const up3d_mesh* m, const double* grad, int32_t* up, cudaStream_t s) {
    k_walk<int32_t><<<grid_for(m->E, 256), 256, 0, s>>>(m->fnbr.get(), m->disp.get(), m->nodes4.get(),
                                                       m->conn.get(), grad, m->E, up);
    UP3D_CHECK_LAUNCH();
}

}  // namespace up3d

using namespace up3d;

namespace {
inline Flow flow_from(double m_inf, double gamma) {
    up3d_flow f{m_inf, gamma, 1.0, 3.0, 0.95, 1.5, 0.05};
    return make_flow(f);
}
}  // namespace

extern "C" {

int up3d_velocities(const up3d_mesh* m, const double* phi, double* grad, double* q2, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(m && phi && grad && q2, UP3D_ERR_ARGUMENT, "up3d_velocities: null argument");
        launch_velocities(m, phi, grad, q2, S(stream));
    });
}

int up3d_limit_q2(const double* q2, int64_t n, double m_inf, double m_cap, double gamma, double* out,
                  int64_t* n_limited, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(q2 && out && n >= 0, UP3D_ERR_ARGUMENT, "up3d_limit_q2: bad argument");
        up3d_flow f{m_inf, gamma, 1.0, m_cap, 0.95, 1.5, 0.05};
        Flow F = make_flow(f);
        if (n_limited) UP3D_CUDA(cudaMemsetAsync(n_limited, 0, sizeof(int64_t), S(stream)));
        if (n == 0) return;
        k_limit<<<grid_for(n, 256), 256, 0, S(stream)>>>(q2, n, F.q2cap, out,
                                                        reinterpret_cast<unsigned long long*>(n_limited));
        UP3D_CHECK_LAUNCH();
    });
}

#define FIELD_ENTRY(NAME, WHAT)                                                                           \
    int NAME(const double* q2, int64_t n, double m_inf, double gamma, double* out, up3d_stream stream) { \
        return guarded([&] {                                                                              \
            UP3D_REQUIRE(q2 && out && n >= 0, UP3D_ERR_ARGUMENT, #NAME ": bad argument");                 \
            if (n == 0) return;                                                                           \
            k_field<WHAT><<<grid_for(n, 256), 256, 0, S(stream)>>>(q2, n, flow_from(m_inf, gamma), out);  \
            UP3D_CHECK_LAUNCH();                                                                          \
        });                                                                                               \
    }

FIELD_ENTRY(up3d_density, 0)
FIELD_ENTRY(up3d_mach_squared, 1)
FIELD_ENTRY(up3d_density_derivative, 2)
FIELD_ENTRY(up3d_mach_squared_derivative, 3)
FIELD_ENTRY(up3d_pressure_coefficient, 4)

int up3d_upwind_walk(const up3d_mesh* m, const double* grad, int64_t* upstream, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(m && grad && upstream, UP3D_ERR_ARGUMENT, "up3d_upwind_walk: null argument");
        k_walk<int64_t><<<grid_for(m->E, 256), 256, 0, S(stream)>>>(m->fnbr.get(), m->disp.get(), m->nodes4.get(),
                                                                   m->conn.get(), grad, m->E, upstream);
        UP3D_CHECK_LAUNCH();
    });
}

int up3d_rho_tilde(const double* q2, const double* rho, const int64_t* upstream, int64_t n, const up3d_flow* flow,
                   double* nu, double* rho_tilde, up3d_monitors* mon, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(q2 && rho && upstream && flow && nu && rho_tilde, UP3D_ERR_ARGUMENT,
                     "up3d_rho_tilde: null argument");
        if (mon) UP3D_CUDA(cudaMemsetAsync(mon, 0, sizeof(up3d_monitors), S(stream)));
        if (n == 0) return;
        k_rho_tilde<<<grid_for(n, 256), 256, 0, S(stream)>>>(q2, rho, upstream, n, make_flow(*flow), nu, rho_tilde,
                                                            mon);
        UP3D_CHECK_LAUNCH();
    });
}

int up3d_classify_branches(const double* q2, const double* rho, const int64_t* upstream, int64_t n,
                           const up3d_flow* flow, int8_t* branch, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(q2 && rho && upstream && flow && branch, UP3D_ERR_ARGUMENT,
                     "up3d_classify_branches: null argument");
        if (n == 0) return;
        k_classify<<<grid_for(n, 256), 256, 0, S(stream)>>>(q2, rho, upstream, n, make_flow(*flow), branch);
        UP3D_CHECK_LAUNCH();
    });
}

int up3d_rho_tilde_frozen(const double* q2, const double* rho, const int64_t* upstream, const int8_t* branch,
                          int64_t n, const up3d_flow* flow, double* nu, double* rho_tilde, up3d_monitors* mon,
                          up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(q2 && rho && upstream && branch && flow && nu && rho_tilde, UP3D_ERR_ARGUMENT,
                     "up3d_rho_tilde_frozen: null argument");
        if (mon) UP3D_CUDA(cudaMemsetAsync(mon, 0, sizeof(up3d_monitors), S(stream)));
        if (n == 0) return;
        k_rho_tilde_frozen<<<grid_for(n, 256), 256, 0, S(stream)>>>(q2, rho, upstream, branch, n, make_flow(*flow),
                                                                   nu, rho_tilde, mon);
        UP3D_CHECK_LAUNCH();
    });
}

int up3d_rho_tilde_sens(const double* q2, const double* rho, const int64_t* upstream, int64_t n,
                        const up3d_flow* flow, double* s_e, double* s_u, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(q2 && rho && upstream && flow && s_e && s_u, UP3D_ERR_ARGUMENT,
                     "up3d_rho_tilde_sens: null argument");
        if (n == 0) return;
        k_sens<<<grid_for(n, 256), 256, 0, S(stream)>>>(q2, rho, upstream, n, make_flow(*flow), s_e, s_u);
        UP3D_CHECK_LAUNCH();
    });
}

int up3d_rho_tilde_frozen_sens(const double* q2, const double* rho, const int64_t* upstream, const int8_t* branch,
                               int64_t n, const up3d_flow* flow, double* s_e, double* s_u, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(q2 && rho && upstream && branch && flow && s_e && s_u, UP3D_ERR_ARGUMENT,
                     "up3d_rho_tilde_frozen_sens: null argument");
        if (n == 0) return;
        k_sens_frozen<<<grid_for(n, 256), 256, 0, S(stream)>>>(q2, rho, upstream, branch, n, make_flow(*flow), s_e,
                                                              s_u);
        UP3D_CHECK_LAUNCH();
    });
}

}  // extern "C"

namespace up3d { void launch_velocities_raw(const int4* c, const double* B, const double* phi, int64_t E, double* g, double* q, cudaStream_t s) {
    k_velocities<<<grid_for(E, 256), 256, 0, s>>>(c, B, phi, E, g, q);
} }

extern "C" int up3d_element_velocity_q2(const int32_t* elements, const double* B, const double* phi, int64_t n_tets,
                                        double* grad, double* q2, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(elements && B && phi && grad && q2 && n_tets >= 0, UP3D_ERR_ARGUMENT,
                     "up3d_element_velocity_q2: bad argument");
        if (n_tets == 0) return;
        launch_velocities_raw(reinterpret_cast<const int4*>(elements), B, phi, n_tets, grad, q2, S(stream));
        UP3D_CHECK_LAUNCH();
    });
}
