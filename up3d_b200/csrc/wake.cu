// Wake master-slave elimination of the up3d library (constraints/wake.py:
// 32-127): the "+"-side copies of the wake-sheet nodes ("slaves", appended
// after the original nodes) fold onto their originals ("masters"),
//   phi_cut = T phi_red + g(Gamma),   T[i, i] = 1 (i < n_red),  T[s_k, m_k] = 1,
// so a cut-mesh operator A reduces to A_red = T^T A T and the Gamma columns
// H = T^T A G (G[s_k, station_k] = 1).  Both are gathers over A's values:
// the host works out, once per A pattern, which A slots land in which
// reduced slot (the symbolic phase); the device sums them (the numeric
// phase, one thread per output slot).
//
// Summation order: the reference forms A T first (for row k, the entries
// whose columns fold to the same reduced column, in stored order) and then
// T^T (A T) (for reduced row r, the rows k folding onto it, ascending: r
// itself, then its slaves).  The plan keeps that grouping: contributors are
// listed k-major, with a flag where a new row k starts, and the kernel sums
// within a group before adding the group to the total.

#include <algorithm>
#include <memory>
#include <string>
#include <vector>

#include "internal.cuh"
#include "krylov.cuh"

struct up3d_wake {
    int device = 0;
    int64_t n_cut = 0, n_red = 0, n_dup = 0, nnz_a = 0;
    int32_t n_st = 0;
    int64_t nnz_red = 0, nnz_h = 0;
    up3d::DBuf<int32_t> red_ptr, red_idx;  // A_red pattern (n_red + 1, nnz_red)
    up3d::DBuf<int64_t> red_poff, red_plan;
    up3d::DBuf<int32_t> h_ptr, h_idx;      // H pattern (n_red + 1, nnz_h), columns = stations
    up3d::DBuf<int64_t> h_poff, h_plan;
    up3d::DBuf<int32_t> t_ptr, t_idx;      // reduced row r -> its slaves, ascending
    up3d::DBuf<int32_t> slave, master, station;  // per duplicated node
};

namespace up3d {
namespace {

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

// out[z] = sum over groups of (sum over the group's A slots), plan entries
// (slot << 1) | (starts a new source row).
__global__ void k_wake_gather(int64_t n_slots, const int64_t* __restrict__ poff, const int64_t* __restrict__ plan,
                              const double* __restrict__ a, double* __restrict__ out) {
    GRID_STRIDE(z, n_slots) {
        const int64_t q0 = poff[z], q1 = poff[z + 1];
        double tot = 0.0, part = 0.0;
        for (int64_t q = q0; q < q1; ++q) {
            const int64_t e = plan[q];
            if ((e & 1) && q != q0) {
                tot = radd(tot, part);
                part = 0.0;
            }
            part = radd(part, a[e >> 1]);
        }
        out[z] = radd(tot, part);
    }
}

// reduced_rhs (constraints/wake.py:99-102): T^T b - sum_j Gamma_j h_j, with
// h_j the station-j column of H.
__global__ void k_wake_rhs(int64_t n_red, const int32_t* __restrict__ t_ptr, const int32_t* __restrict__ t_idx,
                           const int32_t* __restrict__ h_ptr, const int32_t* __restrict__ h_idx,
                           const double* __restrict__ h, const double* __restrict__ b,
                           const double* __restrict__ gamma, double* __restrict__ out) {
    GRID_STRIDE(r, n_red) {
        double tb = radd(0.0, b[r]);
        for (int32_t q = t_ptr[r]; q < t_ptr[r + 1]; ++q) tb = radd(tb, b[t_idx[q]]);
        double gh = 0.0;
        for (int32_t q = h_ptr[r]; q < h_ptr[r + 1]; ++q) gh = radd(gh, rmul(gamma[h_idx[q]], h[q]));
        out[r] = rsub(tb, gh);
    }
}

// expand (constraints/wake.py:104-112): masters copied to the slaves plus
// the station's jump.
__global__ void k_wake_expand(int64_t n_red, int64_t n_dup, const int32_t* __restrict__ slave,
                              const int32_t* __restrict__ master, const int32_t* __restrict__ station,
                              const double* __restrict__ phi_red, const double* __restrict__ gamma,
                              double* __restrict__ phi_cut) {
    GRID_STRIDE(i, n_red + n_dup) {
        if (i < n_red) {
            phi_cut[i] = phi_red[i];
        } else {
            const int64_t k = i - n_red;
            phi_cut[slave[k]] = radd(phi_red[master[k]], gamma[station[k]]);
        }
    }
}

template <class T>
void upload(DBuf<T>& d, const std::vector<T>& h) {
    d.alloc(h.size());
    if (!h.empty()) UP3D_CUDA(cudaMemcpy(d.get(), h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
}

// One contribution of an A slot to a reduced slot: the reduced column, the
// ordinal of the source row among those folding onto the reduced row.
struct Entry {
    int32_t col;
    int32_t group;
    int64_t slot;
};

}  // namespace
}  // namespace up3d

using namespace up3d;

extern "C" {

int up3d_wake_create(int64_t n_cut, int64_t n_red, int64_t n_dup, const int64_t* masters, const int64_t* slaves,
                     const int64_t* node_station, int32_t n_stations, const int64_t* a_indptr,
                     const int32_t* a_indices, int device, up3d_wake** out) {
    return guarded([&] {
        UP3D_REQUIRE(out && a_indptr && (n_dup == 0 || (masters && slaves && node_station)), UP3D_ERR_ARGUMENT,
                     "up3d_wake_create: null argument");
        UP3D_REQUIRE(n_cut == n_red + n_dup && n_red > 0 && n_dup >= 0, UP3D_ERR_VALUE,
                     "up3d_wake_create: A is " + std::to_string(n_cut) + "x" + std::to_string(n_cut) +
                         " but the wake cut implies " + std::to_string(n_red) + " + " + std::to_string(n_dup) +
                         " nodes");
        UP3D_REQUIRE(n_cut < (1ll << 31) && n_stations >= 0, UP3D_ERR_VALUE, "up3d_wake_create: bad sizes");
        // fold map and station of every cut node
        std::vector<int32_t> red_of(n_cut), station_of(n_cut, -1);
        for (int64_t i = 0; i < n_red; ++i) red_of[i] = (int32_t)i;
        std::vector<int32_t> seen(n_cut, 0);
        std::vector<int32_t> h_slave(n_dup), h_master(n_dup), h_station(n_dup);
        std::vector<int32_t> t_cnt(n_red + 1, 0);
        for (int64_t k = 0; k < n_dup; ++k) {
            const int64_t s = slaves[k], m = masters[k], st = node_station[k];
            UP3D_REQUIRE(s >= n_red && s < n_cut && !seen[s], UP3D_ERR_VALUE,
                         "up3d_wake_create: slave nodes must be distinct ids in [n_red, n_cut)");
            UP3D_REQUIRE(m >= 0 && m < n_red, UP3D_ERR_VALUE, "up3d_wake_create: master node out of range");
            UP3D_REQUIRE(st >= 0 && st < n_stations, UP3D_ERR_VALUE, "up3d_wake_create: station out of range");
            seen[s] = 1;
            red_of[s] = (int32_t)m;
            station_of[s] = (int32_t)st;
            h_slave[k] = (int32_t)s;
            h_master[k] = (int32_t)m;
            h_station[k] = (int32_t)st;
            ++t_cnt[m + 1];
        }
        UP3D_REQUIRE(a_indptr[0] == 0, UP3D_ERR_VALUE, "up3d_wake_create: indptr[0] must be 0");
        for (int64_t i = 0; i < n_cut; ++i)
            UP3D_REQUIRE(a_indptr[i + 1] >= a_indptr[i], UP3D_ERR_VALUE, "up3d_wake_create: indptr not monotone");
        const int64_t nnz_a = a_indptr[n_cut];
        for (int64_t p = 0; p < nnz_a; ++p)
            UP3D_REQUIRE(a_indices[p] >= 0 && a_indices[p] < n_cut, UP3D_ERR_VALUE,
                         "up3d_wake_create: column index out of range");
        // rows folding onto each reduced row: r, then its slaves ascending
        for (int64_t r = 0; r < n_red; ++r) t_cnt[r + 1] += t_cnt[r];
        std::vector<int32_t> t_idx(n_dup), t_fill(t_cnt.begin(), t_cnt.end() - 1);
        for (int64_t s = n_red; s < n_cut; ++s) t_idx[t_fill[red_of[s]]++] = (int32_t)s;
        // symbolic phase
        std::vector<int32_t> red_ptr(n_red + 1, 0), red_idx, h_ptr(n_red + 1, 0), h_idx;
        std::vector<int64_t> red_poff(1, 0), red_plan, h_poff(1, 0), h_plan;
        std::vector<Entry> ent, hent;
        // a column's contributors in encounter order (source rows k-major,
        // each row's entries in stored order); a group starts where the
        // source row changes
        auto emit = [](std::vector<Entry>& v, std::vector<int32_t>& idx, std::vector<int64_t>& poff,
                       std::vector<int64_t>& plan) {
            std::stable_sort(v.begin(), v.end(), [](const Entry& a, const Entry& b) { return a.col < b.col; });
            size_t i = 0;
            while (i < v.size()) {
                idx.push_back(v[i].col);
                int32_t last = -1;
                size_t j = i;
                for (; j < v.size() && v[j].col == v[i].col; ++j) {
                    plan.push_back((v[j].slot << 1) | (v[j].group != last ? 1 : 0));
                    last = v[j].group;
                }
                poff.push_back((int64_t)plan.size());
                i = j;
            }
        };
        for (int64_t r = 0; r < n_red; ++r) {
            ent.clear();
            hent.clear();
            const int32_t n_src = 1 + t_cnt[r + 1] - t_cnt[r];
            for (int32_t g = 0; g < n_src; ++g) {
                const int64_t k = g == 0 ? r : t_idx[t_cnt[r] + g - 1];
                for (int64_t p = a_indptr[k]; p < a_indptr[k + 1]; ++p) {
                    const int32_t j = a_indices[p];
                    ent.push_back({red_of[j], g, p});
                    if (station_of[j] >= 0) hent.push_back({station_of[j], g, p});
                }
            }
            emit(ent, red_idx, red_poff, red_plan);
            red_ptr[r + 1] = (int32_t)red_idx.size();
            emit(hent, h_idx, h_poff, h_plan);
            h_ptr[r + 1] = (int32_t)h_idx.size();
        }
        int cur = 0;
        UP3D_CUDA(cudaGetDevice(&cur));
        UP3D_CUDA(cudaSetDevice(device));
        auto* w = new up3d_wake();
        try {
            w->device = device;
            w->n_cut = n_cut;
            w->n_red = n_red;
            w->n_dup = n_dup;
            w->nnz_a = nnz_a;
            w->n_st = n_stations;
            w->nnz_red = (int64_t)red_idx.size();
            w->nnz_h = (int64_t)h_idx.size();
            upload(w->red_ptr, red_ptr);
            upload(w->red_idx, red_idx);
            upload(w->red_poff, red_poff);
            upload(w->red_plan, red_plan);
            upload(w->h_ptr, h_ptr);
            upload(w->h_idx, h_idx);
            upload(w->h_poff, h_poff);
            upload(w->h_plan, h_plan);
            std::vector<int32_t> tp(t_cnt.begin(), t_cnt.end());
            upload(w->t_ptr, tp);
            upload(w->t_idx, t_idx);
            upload(w->slave, h_slave);
            upload(w->master, h_master);
            upload(w->station, h_station);
        } catch (...) {
            delete w;
            cudaSetDevice(cur);
            throw;
        }
        UP3D_CUDA(cudaSetDevice(cur));
        *out = w;
    });
}

int up3d_wake_destroy(up3d_wake* w) {
    return guarded([&] { delete w; });
}

int up3d_wake_info(const up3d_wake* w, int64_t* n_red, int64_t* nnz_red, int64_t* nnz_h, int32_t* n_stations) {
    return guarded([&] {
        UP3D_REQUIRE(w, UP3D_ERR_ARGUMENT, "up3d_wake_info: null argument");
        if (n_red) *n_red = w->n_red;
        if (nnz_red) *nnz_red = w->nnz_red;
        if (nnz_h) *nnz_h = w->nnz_h;
        if (n_stations) *n_stations = w->n_st;
    });
}

int up3d_wake_patterns(const up3d_wake* w, const int32_t** red_indptr, const int32_t** red_indices,
                       const int32_t** h_indptr, const int32_t** h_indices) {
    return guarded([&] {
        UP3D_REQUIRE(w, UP3D_ERR_ARGUMENT, "up3d_wake_patterns: null argument");
        if (red_indptr) *red_indptr = w->red_ptr.get();
        if (red_indices) *red_indices = w->red_idx.get();
        if (h_indptr) *h_indptr = w->h_ptr.get();
        if (h_indices) *h_indices = w->h_idx.get();
    });
}

int up3d_wake_reduce(const up3d_wake* w, const double* a_data, double* red_data, double* h_data,
                     up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(w && a_data && red_data, UP3D_ERR_ARGUMENT, "up3d_wake_reduce: null argument");
        cudaStream_t s = S(stream);
        if (w->nnz_red) {
            k_wake_gather<<<grid_for(w->nnz_red, 256, (int64_t)148 * 32), 256, 0, s>>>(
                w->nnz_red, w->red_poff.get(), w->red_plan.get(), a_data, red_data);
            UP3D_CHECK_LAUNCH();
        }
        if (h_data && w->nnz_h) {
            k_wake_gather<<<grid_for(w->nnz_h, 256, (int64_t)148 * 32), 256, 0, s>>>(
                w->nnz_h, w->h_poff.get(), w->h_plan.get(), a_data, h_data);
            UP3D_CHECK_LAUNCH();
        }
    });
}

int up3d_wake_reduced_rhs(const up3d_wake* w, const double* b, const double* gamma, const double* h_data,
                          double* out, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(w && b && out && (w->n_st == 0 || (gamma && h_data)), UP3D_ERR_ARGUMENT,
                     "up3d_wake_reduced_rhs: null argument");
        k_wake_rhs<<<grid_for(w->n_red, 256, (int64_t)148 * 32), 256, 0, S(stream)>>>(
            w->n_red, w->t_ptr.get(), w->t_idx.get(), w->h_ptr.get(), w->h_idx.get(), h_data, b, gamma, out);
        UP3D_CHECK_LAUNCH();
    });
}

int up3d_wake_expand(const up3d_wake* w, const double* phi_red, const double* gamma, double* phi_cut,
                     up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(w && phi_red && phi_cut && (w->n_dup == 0 || gamma), UP3D_ERR_ARGUMENT,
                     "up3d_wake_expand: null argument");
        k_wake_expand<<<grid_for(w->n_red + w->n_dup, 256, (int64_t)148 * 32), 256, 0, S(stream)>>>(
            w->n_red, w->n_dup, w->slave.get(), w->master.get(), w->station.get(), phi_red, gamma, phi_cut);
        UP3D_CHECK_LAUNCH();
    });
}

}  // extern "C"

// ===================================================== the coupled (phi, Gamma) system
//
// NewtonWorkspace (solve/newton.py:97-502) solves for the free reduced
// potentials phi_f and the station circulations Gamma together:
//   phi_red = phi_f on free rows, vals0 + V Gamma on the far-field rows,
//   phi_cut = T phi_red + G Gamma,
//   R_f = (T^T R(phi_cut))[free],  F = taper * kutta(phi_cut) - Gamma.
// Its eliminated Newton step (kutta_blocks, :459-502, probe estimator)
// solves (J_ff + B K) dphi = -R_f - B F with B = J_red[free, dir] V +
// H_J[free] and dGamma = K dphi + F.  The operator here applies that
// linearisation without forming J_red, J_ff or B:
//   t = K x + g,  u_red = x on free rows, V t on far-field rows,
//   y = (T^T J (T u_red + G t))[free],  y = x on far-field rows,
// i.e. J_ff x + B (K x + g): one expand, one SpMV of the cut-mesh Jacobian
// (Term-3 entries included), one fold.  Vectors are full reduced size with
// the far-field rows carried as identity rows (the up3d_csr Dirichlet
// convention), so the solvers and the AMG of the reduced Picard block take
// them unchanged.

struct up3d_coupled {
    const up3d_wake* wake = nullptr;
    int64_t n_red = 0, n_cut = 0, n_dir = 0;
    int32_t n_st = 0;
    up3d::DBuf<int32_t> dir;                  // far-field reduced rows (n_dir)
    up3d::DBuf<uint8_t> mask;                 // n_red, 1 on far-field rows
    up3d::DBuf<int32_t> k_ptr, k_idx;         // K = dF/dphi_f (n_st rows, reduced columns)
    up3d::DBuf<double> k_val;
    up3d::DBuf<int32_t> te_ptr, te_up, te_lo; // Kutta probes per station, TE order
    up3d::DBuf<double> taper;                 // n_st
    up3d::DBuf<double> vals0, V;              // far-field basis (n_dir, n_dir x n_st row-major)
    bool has_farfield = false;
    mutable up3d::DBuf<double> u_red, u_cut, y_cut, t;
};

namespace up3d {
namespace {

// t[s] = sum_q K[s, q] x[col q] (+ g[s]), one thread per station
__global__ void k_kutta_rows(int32_t n_st, const int32_t* __restrict__ kp, const int32_t* __restrict__ ki,
                             const double* __restrict__ kv, const double* __restrict__ x,
                             const double* __restrict__ g, double* __restrict__ t) {
    for (int32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n_st; s += gridDim.x * blockDim.x) {
        double a = 0.0;
        for (int32_t q = kp[s]; q < kp[s + 1]; ++q) a = radd(a, rmul(kv[q], x[ki[q]]));
        t[s] = g ? radd(a, g[s]) : a;
    }
}

// u[i] = x[i] on free rows; on far-field row dir[k]: (vals0[k] +) V[k, :] t
__global__ void k_farfield_fill(int64_t n_red, int64_t n_dir, int32_t n_st, const int32_t* __restrict__ dir,
                                const uint8_t* __restrict__ mask, const double* __restrict__ vals0,
                                const double* __restrict__ V, const double* __restrict__ t,
                                const double* __restrict__ x, double* __restrict__ u) {
    GRID_STRIDE(i, n_red + n_dir) {
        if (i < n_red) {
            if (!mask[i]) u[i] = x[i];
        } else {
            const int64_t k = i - n_red;
            double a = 0.0;
            for (int32_t j = 0; j < n_st; ++j) a = radd(a, rmul(V[k * n_st + j], t[j]));
            u[dir[k]] = vals0 ? radd(vals0[k], a) : a;
        }
    }
}

// y = T^T b on free rows (the row itself, then its slaves ascending: the
// order of the reference's T.T @ b); far-field rows take xdir (0 if NULL)
__global__ void k_wake_fold(int64_t n_red, const int32_t* __restrict__ t_ptr, const int32_t* __restrict__ t_idx,
                            const uint8_t* __restrict__ mask, const double* __restrict__ b,
                            const double* __restrict__ xdir, double* __restrict__ y) {
    GRID_STRIDE(r, n_red) {
        if (mask[r]) {
            y[r] = xdir ? xdir[r] : 0.0;
        } else {
            double a = radd(0.0, b[r]);
            for (int32_t q = t_ptr[r]; q < t_ptr[r + 1]; ++q) a = radd(a, b[t_idx[q]]);
            y[r] = a;
        }
    }
}

// F[s] = taper[s] * (sum over the station's TE probes of phi[up] - phi[lo])
//        / count - Gamma[s]   (kutta_targets, constraints/wake.py:196-212,
// as used by eval_residual, solve/newton.py:417-419)
__global__ void k_kutta_residual(int32_t n_st, const int32_t* __restrict__ te_ptr, const int32_t* __restrict__ up,
                                 const int32_t* __restrict__ lo, const double* __restrict__ taper,
                                 const double* __restrict__ phi, const double* __restrict__ gamma,
                                 double* __restrict__ F) {
    for (int32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n_st; s += gridDim.x * blockDim.x) {
        double a = 0.0;
        for (int32_t q = te_ptr[s]; q < te_ptr[s + 1]; ++q) a = radd(a, rsub(phi[up[q]], phi[lo[q]]));
        const double mean = __ddiv_rn(a, (double)(te_ptr[s + 1] - te_ptr[s]));
        F[s] = rsub(rmul(taper[s], mean), gamma[s]);
    }
}

}  // namespace

int64_t coupled_rows(const up3d_coupled* c) { return c->n_red; }

void coupled_apply(const up3d_coupled* c, const up3d_csr& J, const up3d_csr& extra, const double* x,
                   const double* g, double* y, double* t_out, cudaStream_t s) {
    UP3D_REQUIRE(c->has_farfield, UP3D_ERR_VALUE, "coupled operator: far-field basis not set");
    UP3D_REQUIRE(J.n == c->n_cut && J.indptr && J.indices && J.data, UP3D_ERR_ARGUMENT,
                 "coupled operator: J must be the cut-mesh operator (n_cut rows)");
    const up3d_wake* w = c->wake;
    double* t = t_out ? t_out : c->t.get();
    if (c->n_st > 0) {
        k_kutta_rows<<<1, 128, 0, s>>>(c->n_st, c->k_ptr.get(), c->k_idx.get(), c->k_val.get(), x, g, t);
        UP3D_CHECK_LAUNCH();
    }
    k_farfield_fill<<<grid_for(c->n_red + c->n_dir, 256), 256, 0, s>>>(
        c->n_red, c->n_dir, c->n_st, c->dir.get(), c->mask.get(), nullptr, c->V.get(), t, x, c->u_red.get());
    UP3D_CHECK_LAUNCH();
    k_wake_expand<<<grid_for(w->n_red + w->n_dup, 256), 256, 0, s>>>(w->n_red, w->n_dup, w->slave.get(),
                                                                     w->master.get(), w->station.get(),
                                                                     c->u_red.get(), t, c->u_cut.get());
    UP3D_CHECK_LAUNCH();
    launch_spmv2<double>(J.n, J.indptr, J.indices, J.data, extra.indptr, extra.indices, extra.data, c->u_cut.get(),
                         c->y_cut.get(), nullptr, s);
    k_wake_fold<<<grid_for(c->n_red, 256), 256, 0, s>>>(c->n_red, w->t_ptr.get(), w->t_idx.get(), c->mask.get(),
                                                        c->y_cut.get(), x, y);
    UP3D_CHECK_LAUNCH();
}

}  // namespace up3d

extern "C" {

int up3d_coupled_create(const up3d_wake* w, int64_t n_dir, const int64_t* dir_nodes, const int64_t* k_indptr,
                        const int64_t* k_cols, const double* k_vals, int64_t n_te, const int64_t* te_station,
                        const int64_t* kutta_upper, const int64_t* kutta_lower, const double* taper,
                        up3d_coupled** out) {
    return guarded([&] {
        UP3D_REQUIRE(w && out && (n_dir == 0 || dir_nodes) && k_indptr && (n_te == 0 || (te_station && kutta_upper
                     && kutta_lower)) && (w->n_st == 0 || taper), UP3D_ERR_ARGUMENT,
                     "up3d_coupled_create: null argument");
        UP3D_REQUIRE(n_dir >= 0 && n_dir <= w->n_red && n_te >= 0, UP3D_ERR_VALUE, "up3d_coupled_create: bad sizes");
        UP3D_CUDA(cudaSetDevice(w->device));
        auto c = std::make_unique<up3d_coupled>();
        c->wake = w;
        c->n_red = w->n_red;
        c->n_cut = w->n_cut;
        c->n_dir = n_dir;
        c->n_st = w->n_st;
        const int32_t n_st = w->n_st;
        std::vector<uint8_t> mask(w->n_red, 0);
        std::vector<int32_t> dir(n_dir);
        for (int64_t k = 0; k < n_dir; ++k) {
            UP3D_REQUIRE(dir_nodes[k] >= 0 && dir_nodes[k] < w->n_red && !mask[dir_nodes[k]], UP3D_ERR_VALUE,
                         "up3d_coupled_create: far-field rows must be distinct reduced ids");
            mask[dir_nodes[k]] = 1;
            dir[k] = (int32_t)dir_nodes[k];
        }
        UP3D_REQUIRE(k_indptr[0] == 0, UP3D_ERR_VALUE, "up3d_coupled_create: K indptr[0] must be 0");
        for (int32_t s = 0; s < n_st; ++s)
            UP3D_REQUIRE(k_indptr[s + 1] >= k_indptr[s], UP3D_ERR_VALUE, "up3d_coupled_create: K indptr not monotone");
        const int64_t k_nnz = k_indptr[n_st];
        UP3D_REQUIRE(k_nnz == 0 || (k_cols && k_vals), UP3D_ERR_ARGUMENT, "up3d_coupled_create: null K");
        std::vector<int32_t> kp(n_st + 1), ki(k_nnz);
        for (int32_t s = 0; s <= n_st; ++s) kp[s] = (int32_t)k_indptr[s];
        for (int64_t q = 0; q < k_nnz; ++q) {
            UP3D_REQUIRE(k_cols[q] >= 0 && k_cols[q] < w->n_red && !mask[k_cols[q]], UP3D_ERR_VALUE,
                         "up3d_coupled_create: K columns must be free reduced ids");
            ki[q] = (int32_t)k_cols[q];
        }
        // TE probes grouped by station, each group in TE order
        std::vector<int32_t> tp(n_st + 1, 0), tu(n_te), tl(n_te);
        for (int64_t q = 0; q < n_te; ++q) {
            UP3D_REQUIRE(te_station[q] >= 0 && te_station[q] < n_st, UP3D_ERR_VALUE,
                         "up3d_coupled_create: TE station out of range");
            UP3D_REQUIRE(kutta_upper[q] >= 0 && kutta_upper[q] < w->n_red && kutta_lower[q] >= 0 &&
                             kutta_lower[q] < w->n_red,
                         UP3D_ERR_VALUE, "up3d_coupled_create: Kutta probes must be original nodes");
            ++tp[te_station[q] + 1];
        }
        for (int32_t s = 0; s < n_st; ++s) {
            UP3D_REQUIRE(tp[s + 1] > 0, UP3D_ERR_VALUE, "up3d_coupled_create: a station without TE probes");
            tp[s + 1] += tp[s];
        }
        std::vector<int32_t> fill(tp.begin(), tp.end() - 1);
        for (int64_t q = 0; q < n_te; ++q) {
            const int32_t at = fill[te_station[q]]++;
            tu[at] = (int32_t)kutta_upper[q];
            tl[at] = (int32_t)kutta_lower[q];
        }
        upload(c->dir, dir);
        upload(c->mask, mask);
        upload(c->k_ptr, kp);
        upload(c->k_idx, ki);
        upload(c->k_val, std::vector<double>(k_vals, k_vals + k_nnz));
        upload(c->te_ptr, tp);
        upload(c->te_up, tu);
        upload(c->te_lo, tl);
        upload(c->taper, std::vector<double>(taper, taper + n_st));
        c->u_red.alloc(c->n_red);
        c->u_cut.alloc(c->n_cut);
        c->y_cut.alloc(c->n_cut);
        c->t.alloc(std::max<int64_t>(n_st, 1));
        *out = c.release();
    });
}

int up3d_coupled_set_kutta_row(up3d_coupled* c, const int64_t* k_indptr, const int64_t* k_cols,
                               const double* k_vals) {
    return guarded([&] {
        UP3D_REQUIRE(c && k_indptr, UP3D_ERR_ARGUMENT, "up3d_coupled_set_kutta_row: null argument");
        UP3D_CUDA(cudaSetDevice(c->wake->device));
        const int32_t n_st = c->n_st;
        UP3D_REQUIRE(k_indptr[0] == 0, UP3D_ERR_VALUE, "up3d_coupled_set_kutta_row: indptr[0] must be 0");
        for (int32_t s = 0; s < n_st; ++s)
            UP3D_REQUIRE(k_indptr[s + 1] >= k_indptr[s], UP3D_ERR_VALUE,
                         "up3d_coupled_set_kutta_row: indptr not monotone");
        const int64_t nnz = k_indptr[n_st];
        UP3D_REQUIRE(nnz == 0 || (k_cols && k_vals), UP3D_ERR_ARGUMENT, "up3d_coupled_set_kutta_row: null K");
        std::vector<uint8_t> mask(c->n_red);
        UP3D_CUDA(cudaMemcpy(mask.data(), c->mask.get(), c->n_red, cudaMemcpyDeviceToHost));
        std::vector<int32_t> kp(n_st + 1), ki(nnz);
        for (int32_t s = 0; s <= n_st; ++s) kp[s] = (int32_t)k_indptr[s];
        for (int64_t q = 0; q < nnz; ++q) {
            UP3D_REQUIRE(k_cols[q] >= 0 && k_cols[q] < c->n_red && !mask[k_cols[q]], UP3D_ERR_VALUE,
                         "up3d_coupled_set_kutta_row: K columns must be free reduced ids");
            ki[q] = (int32_t)k_cols[q];
        }
        upload(c->k_ptr, kp);
        upload(c->k_idx, ki);
        upload(c->k_val, std::vector<double>(k_vals, k_vals + nnz));
    });
}

int up3d_coupled_destroy(up3d_coupled* c) {
    return guarded([&] { delete c; });
}

int up3d_coupled_set_farfield(up3d_coupled* c, const double* vals0, const double* V) {
    return guarded([&] {
        UP3D_REQUIRE(c && (c->n_dir == 0 || vals0) && (c->n_dir * c->n_st == 0 || V), UP3D_ERR_ARGUMENT,
                     "up3d_coupled_set_farfield: null argument");
        UP3D_CUDA(cudaSetDevice(c->wake->device));
        upload(c->vals0, std::vector<double>(vals0, vals0 + c->n_dir));
        upload(c->V, std::vector<double>(V, V + c->n_dir * c->n_st));
        c->has_farfield = true;
    });
}

int up3d_coupled_dirichlet(const up3d_coupled* c, const uint8_t** mask) {
    return guarded([&] {
        UP3D_REQUIRE(c && mask, UP3D_ERR_ARGUMENT, "up3d_coupled_dirichlet: null argument");
        *mask = c->mask.get();
    });
}

int up3d_coupled_state(const up3d_coupled* c, const double* phi_f, const double* gamma, double* phi_red,
                       double* phi_cut, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(c && phi_f && phi_red && phi_cut && (c->n_st == 0 || gamma), UP3D_ERR_ARGUMENT,
                     "up3d_coupled_state: null argument");
        UP3D_REQUIRE(c->has_farfield, UP3D_ERR_VALUE, "up3d_coupled_state: far-field basis not set");
        cudaStream_t s = S(stream);
        const up3d_wake* w = c->wake;
        k_farfield_fill<<<grid_for(c->n_red + c->n_dir, 256), 256, 0, s>>>(c->n_red, c->n_dir, c->n_st,
                                                                           c->dir.get(), c->mask.get(),
                                                                           c->vals0.get(), c->V.get(), gamma,
                                                                           phi_f, phi_red);
        UP3D_CHECK_LAUNCH();
        k_wake_expand<<<grid_for(w->n_red + w->n_dup, 256), 256, 0, s>>>(
            w->n_red, w->n_dup, w->slave.get(), w->master.get(), w->station.get(), phi_red, gamma, phi_cut);
        UP3D_CHECK_LAUNCH();
    });
}

int up3d_coupled_residual(const up3d_coupled* c, const double* R_cut, const double* phi_cut, const double* gamma,
                          double* R_red, double* F, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(c && R_cut && R_red && (!F || c->n_st == 0 || (phi_cut && gamma)), UP3D_ERR_ARGUMENT,
                     "up3d_coupled_residual: null argument");
        cudaStream_t s = S(stream);
        const up3d_wake* w = c->wake;
        k_wake_fold<<<grid_for(c->n_red, 256), 256, 0, s>>>(c->n_red, w->t_ptr.get(), w->t_idx.get(),
                                                            c->mask.get(), R_cut, nullptr, R_red);
        UP3D_CHECK_LAUNCH();
        if (F && c->n_st > 0) {
            k_kutta_residual<<<1, 128, 0, s>>>(c->n_st, c->te_ptr.get(), c->te_up.get(), c->te_lo.get(),
                                               c->taper.get(), phi_cut, gamma, F);
            UP3D_CHECK_LAUNCH();
        }
    });
}

int up3d_coupled_apply(const up3d_coupled* c, const up3d_csr* J, const up3d_csr* extra, const double* x,
                       const double* g, double* y, double* t, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(c && J && x && y, UP3D_ERR_ARGUMENT, "up3d_coupled_apply: null argument");
        up3d_csr none{};
        coupled_apply(c, *J, extra && extra->indptr ? *extra : none, x, g, y, t, S(stream));
    });
}

}  // extern "C"
