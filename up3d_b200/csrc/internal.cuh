// Internal definitions of the up3d CUDA library: the mesh handle, error
// plumbing and the device-side physics shared by every kernel.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <memory>
#include <string>
#include <vector>

#include "../../include/up3d.h"
#include "prof.cuh"

namespace up3d {

// ------------------------------------------------------------ errors

void set_error(const std::string& msg);
int fail(int status, const std::string& msg);

struct Error {
    int status;
    std::string msg;
};

#define UP3D_CUDA(call)                                                              \
    do {                                                                             \
        cudaError_t _e = (call);                                                     \
        if (_e != cudaSuccess)                                                       \
            throw ::up3d::Error{UP3D_ERR_RUNTIME,                                    \
                                std::string(#call) + ": " + cudaGetErrorString(_e)}; \
    } while (0)

// Follows every launch of a library kernel: counts it and checks the launch.
#define UP3D_CHECK_LAUNCH()          \
    do {                             \
        ::up3d::count_launch();      \
        UP3D_CUDA(cudaGetLastError()); \
    } while (0)

#define UP3D_REQUIRE(cond, status, msg)                   \
    do {                                                  \
        if (!(cond)) throw ::up3d::Error{(status), (msg)}; \
    } while (0)

// Runs `body` and converts exceptions into a status code + message.
template <class F>
int guarded(F&& body) {
    try {
        body();
        return UP3D_OK;
    } catch (const Error& e) {
        return fail(e.status, e.msg);
    } catch (const std::exception& e) {
        return fail(UP3D_ERR_RUNTIME, e.what());
    }
}

inline cudaStream_t S(up3d_stream s) { return reinterpret_cast<cudaStream_t>(s); }

// Grid of at most `cap` blocks covering n items with `block` threads.
inline unsigned grid_for(int64_t n, int block, int64_t cap = 148 * 32) {
    int64_t g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (unsigned)g;
}

// ------------------------------------------------------------ device buffer

// Device blocks of the library's buffers (pool.cu): cudaMalloc'd, cached
// per device once freed (after the device has finished with them) and
// reused by later requests of nearly the same size.
void* dev_alloc(size_t bytes);
void dev_free(void* p);

template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    void release() {
        if (p) dev_free(p);
        p = nullptr;
        n = 0;
    }
    void alloc(size_t count) {
        if (count <= n && p) return;
        release();
        if (count == 0) count = 1;
        p = static_cast<T*>(dev_alloc(count * sizeof(T)));
        n = count;
    }
    T* get() const { return p; }
};

// ------------------------------------------------------------ mesh handle

// Local element data written by the element sweeps and gathered by rows:
//   LOC (E, 14): [R_0, J_00, R_1, J_11, R_2, J_22, R_3, J_33,
//                 J_01, J_02, J_03, J_12, J_13, J_23]
//     R_i  = rho~_e V_e (grad . B_i)                   residual contribution
//     J_ij = rho~_e V_e (B_i . B_j) [+ w2 gB_i gB_j]   Terms 1 + 2 (symmetric)
//   RES (E, 4): R_i only (residual-only evaluations)
//   T3V (E, 8): a_i = w3 gB_i, b_k = grad_u . B_u,k (Term-3 active elements)
constexpr int LOC_STRIDE = 14;
constexpr int PLAN8 = 8;
constexpr uint32_t PLAN8_END = 0xFFFFFFFFu;

struct Flow;      // physics constants of one flow (below)
struct TilePlan;  // tiled assembly plan (tiles.cuh)

}  // namespace up3d

struct up3d_mesh {
    int device = 0;
    int64_t N = 0, E = 0, nnz = 0;
    int32_t max_row_len = 0, max_deg = 0;
    int32_t n_colors = -1;
    int32_t n_sms = 148;                       // multiprocessors of the mesh's device
    up3d_tuning tune = {0, 512, 8, 0, 0, 256, 1, 0, 0.0, 0.0};  // launch shapes of the fused evaluation
    std::shared_ptr<up3d::TilePlan> tiles;     // tiled assembly plan (built on first use)
    int32_t batch_cases = 0;                   // cases of the flow table in flows_ws (0 = none)
    // face-hop neighbourhoods of the weighted "kernel" upwind mode (built on
    // request; nb_depth 0 = none)
    up3d::DBuf<int64_t> nb_off;  // (E+1)
    up3d::DBuf<int32_t> nb_idx;  // (nb_total) ascending per element
    int32_t nb_depth = 0;
    int64_t nb_total = 0;
    up3d_flow batch_flow0 = {};                // its case 0

    // geometry (device)
    up3d::DBuf<double4> nodes4;  // (N) x, y, z, 0
    up3d::DBuf<int4> conn;       // (E)
    up3d::DBuf<double> B;        // (E, 12) AoS
    up3d::DBuf<double> V;        // (E)
    up3d::DBuf<int4> fnbr;       // (E) face neighbours (-1 = boundary)
    up3d::DBuf<double4> cen;     // (E) centroids
    up3d::DBuf<double> disp;     // (E, 12) cen(face neighbour k) - cen(e), k = 0..3 (0 at boundary faces)

    // pattern + row-gather maps (device)
    up3d::DBuf<int32_t> indptr;   // (N+1)
    up3d::DBuf<int32_t> indices;  // (nnz)
    up3d::DBuf<int32_t> ent_off;  // (N+1) node -> incident entries
    up3d::DBuf<uint32_t> ent;     // (4E) (e << 2) | local i, ascending e per node
    up3d::DBuf<int32_t> plan_off; // (nnz+1) contributor list offset per nnz
    up3d::DBuf<uint32_t> plan;    // (6E) upper-slot contributors (e << 3) | pair index
    up3d::DBuf<int32_t> diag;     // (N) slot of the diagonal within its row
    up3d::DBuf<int32_t> zt;       // (nnz) slot of the transposed entry
    // the same upper-slot contributors in fixed-width records (PLAN8 per
    // slot, padded with PLAN8_END), indexed by upper-slot ordinal
    // up_off[n] + (s - diag[n] - 1); built when no slot has more
    up3d::DBuf<int32_t> up_off;   // (N+1)
    up3d::DBuf<uint32_t> plan8;   // (n_upper, PLAN8)
    bool has_plan8 = false;

    // workspaces (device)
    up3d::DBuf<double> loc;            // (E, LOC_STRIDE) local matrices + residual
    up3d::DBuf<double> res;            // (E, 4) residual contributions
    up3d::DBuf<double> t3v;            // (E, 8) Term-3 vectors of active elements
    up3d::DBuf<int32_t> up32;          // (E) upstream elements (workspace of the fused evaluation)
    up3d::DBuf<double> grad_ws;        // (E, 3)
    up3d::DBuf<double> q2_ws;          // (E)
    up3d::DBuf<int32_t> extra_cnt;     // (N+1) Term-3 extras per row
    up3d::DBuf<unsigned char> cub_tmp;
    // Term 3 (grown on demand)
    up3d::DBuf<uint8_t> t3_flag;       // (E) active elements
    up3d::DBuf<int32_t> x_col;         // (16E) per-row extras scratch at 4 ent_off[n]
    up3d::DBuf<double> x_val;
    up3d::DBuf<int32_t> x_ptr;         // (N+1) extras row pointer
    up3d::DBuf<int32_t> x_row_c, x_col_c;  // extras, (row, col) order
    up3d::DBuf<double> x_val_c;
    // Term-3 symbolic cache: while the active set and the active elements'
    // upstream repeat, Term 3 is a values-only sum per destination
    // (t3c_state 0: nothing recorded, 1: signature only, 2: cache valid)
    int t3c_state = 0;
    int64_t t3c_active = 0, t3c_extra = 0, t3c_nseg = 0;
    int64_t t3c_hits = 0;                   // values-only rebuilds since creation
    up3d::DBuf<uint8_t> t3c_flag;           // (E) recorded active flags
    up3d::DBuf<int32_t> t3c_up;             // (E) recorded upstream
    up3d::DBuf<uint32_t> t3c_code, t3c_code_tmp;  // (16E) contributor codes, by destination
    up3d::DBuf<int32_t> t3c_key, t3c_key_tmp;     // (16E) destinations (sorted: run keys)
    up3d::DBuf<int32_t> t3c_seg, t3c_cnt;   // segment offsets / lengths
    up3d::DBuf<int64_t> t3c_nruns;
    // adjoint (residual vector-Jacobian products), grown on demand
    up3d::DBuf<double> adj_t, adj_a, adj_rt, adj_A;   // (E) each
    up3d::DBuf<double> adj_dx;                        // (E, 12) per-element node gradients
    up3d::DBuf<double> adj_dphi;                      // (E, 4)
    up3d::DBuf<double> adj_part;                      // reduction partials
    up3d::DBuf<int32_t> adj_key, adj_key_s, adj_val, adj_val_s;  // (E) upstream -> element sort
    up3d::DBuf<up3d::Flow> flows_ws;   // per-case flows of batched evaluations
    up3d::DBuf<up3d_monitors> mon_ws;  // (1)
    up3d::DBuf<int64_t> i64_ws;        // small scalars
    int64_t last_extra = 0;            // extras of the last Jacobian
    int64_t last_active = 0;
    bool last_drop_zeros = false;
};

namespace up3d {

// ------------------------------------------------------------ IEEE helpers
// Explicitly rounded operations (no FMA contraction) for the arithmetic
// whose comparisons steer discrete decisions: geometry, gradients, q^2, the
// limiter, the walk and the Mach switch.  Kept bit-identical to the CPU
// restatement so that upstream selections and branch flags agree exactly.

__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dot3r(double ax, double ay, double az, double bx, double by,
                                        double bz) {
    return radd(radd(rmul(ax, bx), rmul(ay, by)), rmul(az, bz));
}

// ------------------------------------------------------------ physics
// physics/isentropic.py: density (:30-58), Mach^2 (:80-97), derivatives
// (:164-206), speed limiter (:262-314).  gamma == 1.4 (air) takes the exact
// algebraic shortcut base^2.5 = base^2 sqrt(base), rho^0.6 = base^1.5.

struct Flow {
    double m2inf;     // M_inf^2
    double hgm;       // 0.5 (gamma - 1)
    double expo;      // 1 / (gamma - 1)
    double gamma;
    double two_m_g;   // 2 - gamma
    double mc2;       // M_crit^2
    double C;
    double floor_;
    double inv_u2;
    double q2cap;     // q^2 at M_cap (+inf when M_inf == 0)
    bool air;         // gamma == 1.4
};

Flow make_flow(const up3d_flow& f);

__device__ __forceinline__ double base_of(double q2, const Flow& F) {
    // 1 + 0.5 (gamma - 1) M^2 (1 - q^2), evaluated left to right
    return radd(1.0, rmul(rmul(F.hgm, F.m2inf), rsub(1.0, q2)));
}

__device__ __forceinline__ double rho_of(double q2, const Flow& F) {
    double b = base_of(q2, F);
    if (b < 1e-10) b = 1e-10;
    if (F.air) return b * b * sqrt(b);
    return pow(b, F.expo);
}

// rho and d rho / d q^2 from one base evaluation.
__device__ __forceinline__ void rho_drho(double q2, const Flow& F, double& rho, double& drho) {
    double b = base_of(q2, F);
    if (b < 1e-10) b = 1e-10;
    if (F.air) {
        double sb = sqrt(b);
        rho = b * b * sb;
        drho = -0.5 * F.m2inf * (b * sb);
    } else {
        rho = pow(b, F.expo);
        drho = -0.5 * F.m2inf * pow(rho, F.two_m_g);
    }
}

__device__ __forceinline__ double mach2_of(double q2, const Flow& F) {
    return __ddiv_rn(rmul(q2, F.m2inf), base_of(q2, F));
}

__device__ __forceinline__ double dmach2_of(double q2, const Flow& F) {
    double D = base_of(q2, F);
    return F.m2inf * (1.0 + F.hgm * F.m2inf) / (D * D);
}

// nu = C max(0, 1 - M_c^2 / max(M^2, M_c^2))   (kernels/upwind.py:487-488)
__device__ __forceinline__ double switch_of(double m2, const Flow& F) {
    double m = m2 > F.mc2 ? m2 : F.mc2;
    double v = rsub(1.0, __ddiv_rn(F.mc2, m));
    return rmul(F.C, v > 0.0 ? v : 0.0);
}

// nu' on the active branch: C (M_c^2 / M^4) dM^2/dq^2 (kernels/upwind.py:720-728)
__device__ __forceinline__ double dswitch_of(double q2, double m2, const Flow& F) {
    return F.C * (F.mc2 / (m2 * m2)) * dmach2_of(q2, F);
}

// Caller-supplied upstream indices outside [0, n) are treated as
// self-upstream (u(e) = e) so that no sweep can read out of bounds.
__device__ __forceinline__ int64_t safe_up(int64_t u, int64_t e, int64_t n) {
    return (u >= 0 && u < n) ? u : e;
}

// ------------------------------------------------------------ reductions

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Non-negative doubles order like their bit patterns.
__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
    atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

// ------------------------------------------------------------ launchers
// (defined in the .cu files; host side)

void ensure_workspaces(up3d_mesh* m);

}  // namespace up3d
