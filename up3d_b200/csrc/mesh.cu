// Per-mesh setup of the up3d library: element geometry, face adjacency,
// centroids, the P1 CSR pattern and the row-gather maps, built on the
// device; the reference's greedy colouring (host, on request).
//
// Reference: PicardOperator.__init__ (pyfp3d/kernels/jacobian.py:246-262),
// UpwindOperator.__init__ (pyfp3d/kernels/upwind.py:744-781),
// mesh/metrics.py:177-278, mesh/coloring.py:66-145.

#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "internal.cuh"
#include "tiles.cuh"

namespace up3d {

namespace {

thread_local std::string g_last_error;

// Restores the caller's current device on scope exit.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        UP3D_CUDA(cudaGetDevice(&prev));
        if (prev != dev) UP3D_CUDA(cudaSetDevice(dev));
    }
    ~DeviceGuard() {
        int cur = -1;
        if (cudaGetDevice(&cur) == cudaSuccess && cur != prev && prev >= 0) cudaSetDevice(prev);
    }
};

// ------------------------------------------------------------ kernels

__global__ void k_pad_nodes(const double* __restrict__ nodes, int64_t N, double4* __restrict__ out) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < N;
         n += (int64_t)gridDim.x * blockDim.x)
        out[n] = make_double4(nodes[3 * n], nodes[3 * n + 1], nodes[3 * n + 2], 0.0);
}

// B_e, V_e and centroids (mesh/metrics.py:27-70, :130-204;
// kernels/upwind.py:750).  Rows of J^{-1} are the cross products of J's
// columns over det J; B_0 = -(B_1 + B_2 + B_3).  `bad` receives the smallest
// degenerate element index (|det J| < 1e-12 * |v1||v2||v3|).  The fused
// element sweep recomputes B_e and V_e with the same operations (geom_B,
// elem.cuh); the two must stay in step.
__global__ void k_geometry(const double4* __restrict__ X, const int4* __restrict__ conn, int64_t E,
                           double* __restrict__ B, double* __restrict__ V, double4* __restrict__ cen,
                           unsigned long long* bad) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E;
         e += (int64_t)gridDim.x * blockDim.x) {
        int4 c = conn[e];
        double4 x0 = X[c.x], x1 = X[c.y], x2 = X[c.z], x3 = X[c.w];
        double v1x = rsub(x1.x, x0.x), v1y = rsub(x1.y, x0.y), v1z = rsub(x1.z, x0.z);
        double v2x = rsub(x2.x, x0.x), v2y = rsub(x2.y, x0.y), v2z = rsub(x2.z, x0.z);
        double v3x = rsub(x3.x, x0.x), v3y = rsub(x3.y, x0.y), v3z = rsub(x3.z, x0.z);
        double c23x = rsub(rmul(v2y, v3z), rmul(v2z, v3y));
        double c23y = rsub(rmul(v2z, v3x), rmul(v2x, v3z));
        double c23z = rsub(rmul(v2x, v3y), rmul(v2y, v3x));
        double c31x = rsub(rmul(v3y, v1z), rmul(v3z, v1y));
        double c31y = rsub(rmul(v3z, v1x), rmul(v3x, v1z));
        double c31z = rsub(rmul(v3x, v1y), rmul(v3y, v1x));
        double c12x = rsub(rmul(v1y, v2z), rmul(v1z, v2y));
        double c12y = rsub(rmul(v1z, v2x), rmul(v1x, v2z));
        double c12z = rsub(rmul(v1x, v2y), rmul(v1y, v2x));
        double det = dot3r(v1x, v1y, v1z, c23x, c23y, c23z);
        V[e] = __ddiv_rn(fabs(det), 6.0);
        double s1 = __dsqrt_rn(dot3r(v1x, v1y, v1z, v1x, v1y, v1z));
        double s2 = __dsqrt_rn(dot3r(v2x, v2y, v2z, v2x, v2y, v2z));
        double s3 = __dsqrt_rn(dot3r(v3x, v3y, v3z, v3x, v3y, v3z));
        double scale = rmul(rmul(s1, s2), s3);
        double b[12];
        if (scale == 0.0 || fabs(det) < rmul(1e-12, scale)) {
            atomicMin(bad, (unsigned long long)e);
            for (int k = 0; k < 12; ++k) b[k] = 0.0;
        } else {
            double inv = __ddiv_rn(1.0, det);
            b[3] = rmul(c23x, inv); b[4] = rmul(c23y, inv); b[5] = rmul(c23z, inv);
            b[6] = rmul(c31x, inv); b[7] = rmul(c31y, inv); b[8] = rmul(c31z, inv);
            b[9] = rmul(c12x, inv); b[10] = rmul(c12y, inv); b[11] = rmul(c12z, inv);
            for (int d = 0; d < 3; ++d) b[d] = -radd(radd(b[3 + d], b[6 + d]), b[9 + d]);
        }
        for (int k = 0; k < 12; ++k) B[12 * e + k] = b[k];
        double cx = radd(radd(radd(x0.x, x1.x), x2.x), x3.x);
        double cy = radd(radd(radd(x0.y, x1.y), x2.y), x3.y);
        double cz = radd(radd(radd(x0.z, x1.z), x2.z), x3.z);
        cen[e] = make_double4(cx * 0.25, cy * 0.25, cz * 0.25, 0.0);
    }
}

__global__ void k_node_keys(const int4* __restrict__ conn, int64_t E, int32_t* __restrict__ keys,
                            uint32_t* __restrict__ vals, int32_t* __restrict__ count) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E;
         e += (int64_t)gridDim.x * blockDim.x) {
        int4 c = conn[e];
        int n[4] = {c.x, c.y, c.z, c.w};
        for (int i = 0; i < 4; ++i) {
            keys[4 * e + i] = n[i];
            vals[4 * e + i] = (uint32_t)((e << 2) | i);
            atomicAdd(&count[n[i]], 1);
        }
    }
}

__global__ void k_pair_keys(const int4* __restrict__ conn, int64_t E, uint64_t* __restrict__ keys) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E;
         e += (int64_t)gridDim.x * blockDim.x) {
        int4 c = conn[e];
        uint64_t n[4] = {(uint64_t)c.x, (uint64_t)c.y, (uint64_t)c.z, (uint64_t)c.w};
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) keys[16 * e + 4 * i + j] = (n[i] << 32) | n[j];
    }
}

__global__ void k_pattern_from_keys(const uint64_t* __restrict__ keys, const int64_t* num,
                                    int32_t* __restrict__ indices, int32_t* __restrict__ rowcnt) {
    int64_t Z = *num;
    for (int64_t z = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; z < Z;
         z += (int64_t)gridDim.x * blockDim.x) {
        uint64_t k = keys[z];
        indices[z] = (int32_t)(k & 0xffffffffu);
        atomicAdd(&rowcnt[(int32_t)(k >> 32)], 1);
    }
}

__device__ __forceinline__ int32_t lower_bound(const int32_t* __restrict__ a, int32_t len, int32_t v) {
    int32_t lo = 0, hi = len;
    while (lo < hi) {
        int32_t mid = (lo + hi) >> 1;
        if (a[mid] < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Index of the off-diagonal pair (a, b), a < b, in (01,02,03,12,13,23).
__device__ __forceinline__ int pair_index(int a, int b) { return a * (7 - a) / 2 - 1 + b - a; }

// Row-gather plan, pass 1 (count) / pass 2 (fill).  The P1 element
// matrices are symmetric, so only upper-triangle slots (col > row) get a
// contributor list: for slot (n, m), the elements holding edge (n, m) in
// ascending element order, each as (e << 3) | (pair index of its local
// (i, j)).  Also the slot of the diagonal.
template <bool FILL>
__global__ void k_plan(int64_t N, const int4* __restrict__ conn, const int32_t* __restrict__ ent_off,
                       const uint32_t* __restrict__ ent, const int32_t* __restrict__ indptr,
                       const int32_t* __restrict__ indices, int32_t* __restrict__ cursor,
                       const int32_t* __restrict__ plan_off, uint32_t* __restrict__ plan,
                       int32_t* __restrict__ diag) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < N;
         n += (int64_t)gridDim.x * blockDim.x) {
        int32_t rb = indptr[n], L = indptr[n + 1] - rb;
        const int32_t* cols = indices + rb;
        int32_t eb = ent_off[n], deg = ent_off[n + 1] - eb;
        if (!FILL) diag[n] = lower_bound(cols, L, (int32_t)n);
        for (int32_t k = 0; k < deg; ++k) {
            uint32_t x = ent[eb + k];
            int64_t e = x >> 2;
            int i = x & 3;
            int4 c = conn[e];
            int nd[4] = {c.x, c.y, c.z, c.w};
            for (int j = 0; j < 4; ++j) {
                if (j == i || nd[j] <= n) continue;
                int32_t s = lower_bound(cols, L, nd[j]);
                if (FILL) {
                    int32_t pos = plan_off[rb + s] + cursor[rb + s]++;
                    const int q = i < j ? pair_index(i, j) : pair_index(j, i);
                    plan[pos] = (uint32_t)((e << 3) | q);
                } else {
                    cursor[rb + s]++;
                }
            }
        }
    }
}

// Upper-slot counts per row (slots right of the diagonal) and the largest
// contributor count of any upper slot.
__global__ void k_upper_counts(int64_t N, const int32_t* __restrict__ indptr, const int32_t* __restrict__ diag,
                               const int32_t* __restrict__ plan_off, int32_t* __restrict__ cnt,
                               int32_t* __restrict__ most) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < N;
         n += (int64_t)gridDim.x * blockDim.x) {
        const int32_t rb = indptr[n], L = indptr[n + 1] - rb, ds = diag[n];
        const int32_t u = L - ds - 1;
        cnt[n] = u > 0 ? u : 0;
        int32_t mx = 0;
        for (int32_t s = ds + 1; s < L; ++s) mx = max(mx, plan_off[rb + s + 1] - plan_off[rb + s]);
        most[n] = mx;
    }
}

// The fixed-width contributor records of every upper slot, in plan order.
__global__ void k_plan8(int64_t N, const int32_t* __restrict__ indptr, const int32_t* __restrict__ diag,
                        const int32_t* __restrict__ up_off, const int32_t* __restrict__ plan_off,
                        const uint32_t* __restrict__ plan, uint32_t* __restrict__ plan8) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < N;
         n += (int64_t)gridDim.x * blockDim.x) {
        const int32_t rb = indptr[n], L = indptr[n + 1] - rb, ds = diag[n];
        for (int32_t s = ds + 1; s < L; ++s) {
            uint32_t* out = plan8 + (size_t)PLAN8 * (up_off[n] + (s - ds - 1));
            const int32_t p0 = plan_off[rb + s], p1 = plan_off[rb + s + 1];
            for (int k = 0; k < PLAN8; ++k) out[k] = p0 + k < p1 ? plan[p0 + k] : PLAN8_END;
        }
    }
}

// Transposed slot of every non-zero: for (n, m) at z, the position of (m, n).
__global__ void k_transpose_slots(int64_t N, const int32_t* __restrict__ indptr,
                                  const int32_t* __restrict__ indices, int32_t* __restrict__ zt) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < N;
         n += (int64_t)gridDim.x * blockDim.x) {
        for (int32_t z = indptr[n]; z < indptr[n + 1]; ++z) {
            const int32_t m = indices[z];
            const int32_t mb = indptr[m], mL = indptr[m + 1] - mb;
            zt[z] = mb + lower_bound(indices + mb, mL, (int32_t)n);
        }
    }
}

// Face f of e is opposite local node f (mesh/metrics.py:224-232); its
// neighbour is the other element holding all three face nodes.
__global__ void k_face_neighbors(const int4* __restrict__ conn, int64_t E,
                                 const int32_t* __restrict__ ent_off, const uint32_t* __restrict__ ent,
                                 int4* __restrict__ fn) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E;
         e += (int64_t)gridDim.x * blockDim.x) {
        int4 c = conn[e];
        int nd[4] = {c.x, c.y, c.z, c.w};
        int out[4];
        for (int f = 0; f < 4; ++f) {
            int a = nd[f == 0 ? 1 : 0];
            int b = nd[f <= 1 ? 2 : 1];
            int d = nd[f <= 2 ? 3 : 2];
            int found = -1;
            for (int32_t k = ent_off[a]; k < ent_off[a + 1] && found < 0; ++k) {
                int64_t o = ent[k] >> 2;
                if (o == e) continue;
                int4 oc = conn[o];
                bool hb = oc.x == b || oc.y == b || oc.z == b || oc.w == b;
                bool hd = oc.x == d || oc.y == d || oc.z == d || oc.w == d;
                if (hb && hd) found = (int)o;
            }
            out[f] = found;
        }
        fn[e] = make_int4(out[0], out[1], out[2], out[3]);
    }
}

// Walk displacements: for every element and face k, cen(fn[k]) - cen(e)
// (IEEE-rounded), zero at boundary faces and out-of-range entries.
__global__ void k_face_disp(const int4* __restrict__ fn, const double4* __restrict__ cen, int64_t E,
                            double* __restrict__ disp) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int4 f = fn[e];
        const int nb[4] = {f.x, f.y, f.z, f.w};
        const double4 c = cen[e];
        for (int k = 0; k < 4; ++k) {
            double dx = 0.0, dy = 0.0, dz = 0.0;
            if (nb[k] >= 0 && nb[k] < E) {
                const double4 cn = cen[nb[k]];
                dx = __dsub_rn(cn.x, c.x);
                dy = __dsub_rn(cn.y, c.y);
                dz = __dsub_rn(cn.z, c.z);
            }
            disp[12 * e + 3 * k] = dx;
            disp[12 * e + 3 * k + 1] = dy;
            disp[12 * e + 3 * k + 2] = dz;
        }
    }
}

void refresh_disp(up3d_mesh* m, cudaStream_t s) {
    m->disp.alloc(12 * m->E);
    k_face_disp<<<grid_for(m->E, 256), 256, 0, s>>>(m->fnbr.get(), m->cen.get(), m->E, m->disp.get());
    UP3D_CHECK_LAUNCH();
}

__global__ void k_elem_to_csr(const int4* __restrict__ conn, int64_t E, const int32_t* __restrict__ indptr,
                              const int32_t* __restrict__ indices, int64_t* __restrict__ out) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E;
         e += (int64_t)gridDim.x * blockDim.x) {
        int4 c = conn[e];
        int nd[4] = {c.x, c.y, c.z, c.w};
        for (int i = 0; i < 4; ++i) {
            int32_t rb = indptr[nd[i]], L = indptr[nd[i] + 1] - rb;
            for (int j = 0; j < 4; ++j) out[16 * e + 4 * i + j] = rb + lower_bound(indices + rb, L, nd[j]);
        }
    }
}

__global__ void k_export_geometry(const double* __restrict__ B12, const double* __restrict__ V, int64_t E,
                                  double* __restrict__ B, double* __restrict__ Vout) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E;
         e += (int64_t)gridDim.x * blockDim.x) {
        for (int k = 0; k < 12; ++k) B[12 * e + k] = B12[12 * e + k];
        Vout[e] = V[e];
    }
}

__global__ void k_export_centroids(const double4* __restrict__ cen, int64_t E, double* __restrict__ out) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E;
         e += (int64_t)gridDim.x * blockDim.x) {
        double4 c = cen[e];
        out[3 * e] = c.x;
        out[3 * e + 1] = c.y;
        out[3 * e + 2] = c.z;
    }
}

template <class T>
void cub_exclusive_scan(up3d_mesh* m, const T* in, T* out, int64_t n, cudaStream_t s) {
    size_t bytes = 0;
    UP3D_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, s));
    m->cub_tmp.alloc(bytes);
    UP3D_CUDA(cub::DeviceScan::ExclusiveSum(m->cub_tmp.get(), bytes, in, out, n, s));
}

int32_t device_max(up3d_mesh* m, const int32_t* in, int64_t n, cudaStream_t s) {
    DBuf<int32_t> out;
    out.alloc(1);
    size_t bytes = 0;
    UP3D_CUDA(cub::DeviceReduce::Max(nullptr, bytes, in, out.get(), n, s));
    m->cub_tmp.alloc(bytes);
    UP3D_CUDA(cub::DeviceReduce::Max(m->cub_tmp.get(), bytes, in, out.get(), n, s));
    int32_t h = 0;
    UP3D_CUDA(cudaMemcpyAsync(&h, out.get(), sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    UP3D_CUDA(cudaStreamSynchronize(s));
    return h;
}

}  // namespace

void set_error(const std::string& msg) { g_last_error = msg; }
int fail(int status, const std::string& msg) {
    g_last_error = msg;
    return status;
}

// Host copies of the connectivity are kept for the (serial, reference-
// identical) greedy colouring, computed on request only.
struct HostMeshExtra {
    std::vector<int32_t> elements;
    std::vector<int64_t> color_offsets, color_elems;
};
static std::mutex g_extra_mu;
static std::vector<std::pair<const up3d_mesh*, HostMeshExtra*>> g_extra;

static HostMeshExtra* extra_of(const up3d_mesh* m, bool create) {
    std::lock_guard<std::mutex> lk(g_extra_mu);
    for (auto& p : g_extra)
        if (p.first == m) return p.second;
    if (!create) return nullptr;
    auto* x = new HostMeshExtra();
    g_extra.emplace_back(m, x);
    return x;
}
static void drop_extra(const up3d_mesh* m) {
    std::lock_guard<std::mutex> lk(g_extra_mu);
    for (size_t i = 0; i < g_extra.size(); ++i)
        if (g_extra[i].first == m) {
            delete g_extra[i].second;
            g_extra.erase(g_extra.begin() + i);
            return;
        }
}

static void build_mesh(up3d_mesh* m, const double* nodes, const int32_t* elements, cudaStream_t s) {
    const int64_t N = m->N, E = m->E;
    const int block = 256;
    // upload
    {
        DBuf<double> tmp;
        tmp.alloc(3 * N);
        UP3D_CUDA(cudaMemcpyAsync(tmp.get(), nodes, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, s));
        m->nodes4.alloc(N);
        k_pad_nodes<<<grid_for(N, block), block, 0, s>>>(tmp.get(), N, m->nodes4.get());
        UP3D_CHECK_LAUNCH();
        m->conn.alloc(E);
        UP3D_CUDA(cudaMemcpyAsync(m->conn.get(), elements, sizeof(int4) * E, cudaMemcpyHostToDevice, s));
        UP3D_CUDA(cudaStreamSynchronize(s));
    }
    // geometry
    m->B.alloc(12 * E);
    m->V.alloc(E);
    m->cen.alloc(E);
    {
        DBuf<unsigned long long> bad;
        bad.alloc(1);
        unsigned long long init = ~0ull;
        UP3D_CUDA(cudaMemcpyAsync(bad.get(), &init, sizeof(init), cudaMemcpyHostToDevice, s));
        k_geometry<<<grid_for(E, block), block, 0, s>>>(m->nodes4.get(), m->conn.get(), E, m->B.get(),
                                                         m->V.get(), m->cen.get(), bad.get());
        UP3D_CHECK_LAUNCH();
        unsigned long long hbad = 0;
        UP3D_CUDA(cudaMemcpyAsync(&hbad, bad.get(), sizeof(hbad), cudaMemcpyDeviceToHost, s));
        UP3D_CUDA(cudaStreamSynchronize(s));
        UP3D_REQUIRE(hbad == ~0ull, UP3D_ERR_VALUE,
                     "element_gradients: degenerate tetrahedron (|det J| < 1e-12 x edge-length^3 "
                     "scale) at element " + std::to_string(hbad) + " -- fix the mesh");
    }
    // node -> incident entries, ascending element per node (stable sort)
    m->ent_off.alloc(N + 1);
    m->ent.alloc(4 * E);
    {
        DBuf<int32_t> keys, keys_out, count;
        DBuf<uint32_t> vals;
        keys.alloc(4 * E);
        keys_out.alloc(4 * E);
        vals.alloc(4 * E);
        count.alloc(N + 1);
        UP3D_CUDA(cudaMemsetAsync(count.get(), 0, sizeof(int32_t) * (N + 1), s));
        k_node_keys<<<grid_for(E, block), block, 0, s>>>(m->conn.get(), E, keys.get(), vals.get(), count.get());
        UP3D_CHECK_LAUNCH();
        int end_bit = 1;
        while ((1ll << end_bit) < N) ++end_bit;
        size_t bytes = 0;
        UP3D_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, keys.get(), keys_out.get(), vals.get(),
                                                  m->ent.get(), 4 * E, 0, end_bit, s));
        m->cub_tmp.alloc(bytes);
        UP3D_CUDA(cub::DeviceRadixSort::SortPairs(m->cub_tmp.get(), bytes, keys.get(), keys_out.get(),
                                                  vals.get(), m->ent.get(), 4 * E, 0, end_bit, s));
        cub_exclusive_scan(m, count.get(), m->ent_off.get(), N + 1, s);
        m->max_deg = device_max(m, count.get(), N, s);
        UP3D_REQUIRE(m->max_deg < 16384, UP3D_ERR_VALUE,
                     "a node is shared by more than 16383 elements; unsupported connectivity");
    }
    // P1 pattern: sorted unique (row, col) pairs of every element
    m->indptr.alloc(N + 1);
    {
        DBuf<uint64_t> keys, sorted, uniq;
        DBuf<int64_t> num;
        DBuf<int32_t> rowcnt;
        keys.alloc(16 * E);
        sorted.alloc(16 * E);
        uniq.alloc(16 * E);
        num.alloc(1);
        rowcnt.alloc(N + 1);
        k_pair_keys<<<grid_for(E, block), block, 0, s>>>(m->conn.get(), E, keys.get());
        UP3D_CHECK_LAUNCH();
        int end_bit = 32;
        { int b = 1; while ((1ll << b) < N) ++b; end_bit = 32 + b; }
        size_t bytes = 0;
        UP3D_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, bytes, keys.get(), sorted.get(), 16 * E, 0, end_bit, s));
        m->cub_tmp.alloc(bytes);
        UP3D_CUDA(cub::DeviceRadixSort::SortKeys(m->cub_tmp.get(), bytes, keys.get(), sorted.get(), 16 * E, 0,
                                                 end_bit, s));
        bytes = 0;
        UP3D_CUDA(cub::DeviceSelect::Unique(nullptr, bytes, sorted.get(), uniq.get(), num.get(), 16 * E, s));
        m->cub_tmp.alloc(bytes);
        UP3D_CUDA(cub::DeviceSelect::Unique(m->cub_tmp.get(), bytes, sorted.get(), uniq.get(), num.get(), 16 * E, s));
        int64_t Z = 0;
        UP3D_CUDA(cudaMemcpyAsync(&Z, num.get(), sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        UP3D_CUDA(cudaStreamSynchronize(s));
        UP3D_REQUIRE(Z < (1ll << 31), UP3D_ERR_VALUE, "pattern exceeds 2^31 non-zeros");
        m->nnz = Z;
        m->indices.alloc(Z);
        UP3D_CUDA(cudaMemsetAsync(rowcnt.get(), 0, sizeof(int32_t) * (N + 1), s));
        k_pattern_from_keys<<<grid_for(Z, block), block, 0, s>>>(uniq.get(), num.get(), m->indices.get(),
                                                                  rowcnt.get());
        UP3D_CHECK_LAUNCH();
        cub_exclusive_scan(m, rowcnt.get(), m->indptr.get(), N + 1, s);
        m->max_row_len = device_max(m, rowcnt.get(), N, s);
    }
    // row-gather plan
    m->plan_off.alloc(m->nnz + 1);
    m->plan.alloc(6 * E);
    m->diag.alloc(N);
    m->zt.alloc(m->nnz);
    k_transpose_slots<<<grid_for(N, 128), 128, 0, s>>>(N, m->indptr.get(), m->indices.get(), m->zt.get());
    UP3D_CHECK_LAUNCH();
    {
        DBuf<int32_t> cursor;
        cursor.alloc(m->nnz + 1);
        UP3D_CUDA(cudaMemsetAsync(cursor.get(), 0, sizeof(int32_t) * (m->nnz + 1), s));
        k_plan<false><<<grid_for(N, 128), 128, 0, s>>>(N, m->conn.get(), m->ent_off.get(), m->ent.get(),
                                                      m->indptr.get(), m->indices.get(), cursor.get(),
                                                      nullptr, nullptr, m->diag.get());
        UP3D_CHECK_LAUNCH();
        cub_exclusive_scan(m, cursor.get(), m->plan_off.get(), m->nnz + 1, s);
        UP3D_CUDA(cudaMemsetAsync(cursor.get(), 0, sizeof(int32_t) * (m->nnz + 1), s));
        k_plan<true><<<grid_for(N, 128), 128, 0, s>>>(N, m->conn.get(), m->ent_off.get(), m->ent.get(),
                                                     m->indptr.get(), m->indices.get(), cursor.get(),
                                                     m->plan_off.get(), m->plan.get(), m->diag.get());
        UP3D_CHECK_LAUNCH();
        // fixed-width records when every upper slot has at most PLAN8
        // contributors
        DBuf<int32_t> most, ucnt;
        most.alloc(N);
        ucnt.alloc(N + 1);
        m->up_off.alloc(N + 1);
        UP3D_CUDA(cudaMemsetAsync(ucnt.get() + N, 0, sizeof(int32_t), s));
        k_upper_counts<<<grid_for(N, 128), 128, 0, s>>>(N, m->indptr.get(), m->diag.get(), m->plan_off.get(),
                                                       ucnt.get(), most.get());
        UP3D_CHECK_LAUNCH();
        cub_exclusive_scan(m, ucnt.get(), m->up_off.get(), N + 1, s);
        int32_t n_upper = 0;
        UP3D_CUDA(cudaMemcpyAsync(&n_upper, m->up_off.get() + N, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        const int32_t widest = device_max(m, most.get(), N, s);
        m->has_plan8 = false;
        if (widest <= PLAN8 && n_upper > 0) {
            m->plan8.alloc((size_t)PLAN8 * n_upper);
            k_plan8<<<grid_for(N, 128), 128, 0, s>>>(N, m->indptr.get(), m->diag.get(), m->up_off.get(),
                                                    m->plan_off.get(), m->plan.get(), m->plan8.get());
            UP3D_CHECK_LAUNCH();
            m->has_plan8 = true;
        }
    }
    // face adjacency
    m->fnbr.alloc(E);
    k_face_neighbors<<<grid_for(E, block), block, 0, s>>>(m->conn.get(), E, m->ent_off.get(), m->ent.get(),
                                                          m->fnbr.get());
    UP3D_CHECK_LAUNCH();
    refresh_disp(m, s);
    UP3D_CUDA(cudaStreamSynchronize(s));
}

void ensure_workspaces(up3d_mesh* m) {
    m->loc.alloc((size_t)LOC_STRIDE * m->E);
    m->res.alloc(4 * m->E);
    m->up32.alloc(m->E);
    m->t3v.alloc(8 * m->E);
    m->t3_flag.alloc(m->E);
    m->mon_ws.alloc(1);
    m->i64_ws.alloc(8);
}

}  // namespace up3d

using namespace up3d;

extern "C" {

const char* up3d_last_error(void) { return g_last_error.c_str(); }
int up3d_version(void) { return 1; }

int up3d_mesh_create(const double* nodes, const int32_t* elements, int64_t n_nodes, int64_t n_tets,
                     int device, up3d_stream stream, up3d_mesh** out) {
    return guarded([&] {
        UP3D_REQUIRE(nodes && elements && out, UP3D_ERR_ARGUMENT, "up3d_mesh_create: null argument");
        UP3D_REQUIRE(n_nodes > 0 && n_tets > 0, UP3D_ERR_VALUE, "up3d_mesh_create: empty mesh");
        UP3D_REQUIRE(n_nodes < (1ll << 31) && n_tets < (1ll << 29), UP3D_ERR_VALUE,
                     "up3d_mesh_create: mesh exceeds int32 connectivity");
        for (int64_t k = 0; k < 4 * n_tets; ++k)
            UP3D_REQUIRE(elements[k] >= 0 && elements[k] < n_nodes, UP3D_ERR_VALUE,
                         "up3d_mesh_create: element " + std::to_string(k / 4) +
                             " references node " + std::to_string(elements[k]) + " out of range");
        DeviceGuard g(device);
        auto* m = new up3d_mesh();
        m->device = device;
        m->N = n_nodes;
        m->E = n_tets;
        try {
            UP3D_CUDA(cudaDeviceGetAttribute(&m->n_sms, cudaDevAttrMultiProcessorCount, device));
            build_mesh(m, nodes, elements, S(stream));
            ensure_workspaces(m);
            auto* x = extra_of(m, true);
            x->elements.assign(elements, elements + 4 * n_tets);
        } catch (...) {
            drop_extra(m);
            delete m;
            throw;
        }
        *out = m;
    });
}

int up3d_mesh_destroy(up3d_mesh* m) {
    return guarded([&] {
        if (!m) return;
        DeviceGuard g(m->device);
        cudaDeviceSynchronize();
        drop_extra(m);
        delete m;
    });
}

int up3d_mesh_get_info(const up3d_mesh* m, up3d_mesh_info* info) {
    return guarded([&] {
        UP3D_REQUIRE(m && info, UP3D_ERR_ARGUMENT, "up3d_mesh_get_info: null argument");
        info->n_nodes = m->N;
        info->n_tets = m->E;
        info->nnz = m->nnz;
        info->max_row_len = m->max_row_len;
        info->max_node_degree = m->max_deg;
        info->n_colors = m->n_colors;
        info->device = m->device;
    });
}

int up3d_mesh_pattern(const up3d_mesh* m, const int32_t** indptr, const int32_t** indices) {
    return guarded([&] {
        UP3D_REQUIRE(m && indptr && indices, UP3D_ERR_ARGUMENT, "up3d_mesh_pattern: null argument");
        *indptr = m->indptr.get();
        *indices = m->indices.get();
    });
}

int up3d_mesh_geometry(const up3d_mesh* m, double* B, double* V, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(m && B && V, UP3D_ERR_ARGUMENT, "up3d_mesh_geometry: null argument");
        DeviceGuard g(m->device);
        k_export_geometry<<<grid_for(m->E, 256), 256, 0, S(stream)>>>(m->B.get(), m->V.get(), m->E, B, V);
        UP3D_CHECK_LAUNCH();
    });
}

int up3d_mesh_centroids(const up3d_mesh* m, double* out, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(m && out, UP3D_ERR_ARGUMENT, "up3d_mesh_centroids: null argument");
        DeviceGuard g(m->device);
        k_export_centroids<<<grid_for(m->E, 256), 256, 0, S(stream)>>>(m->cen.get(), m->E, out);
        UP3D_CHECK_LAUNCH();
    });
}

int up3d_mesh_face_neighbors(const up3d_mesh* m, int32_t* out, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(m && out, UP3D_ERR_ARGUMENT, "up3d_mesh_face_neighbors: null argument");
        DeviceGuard g(m->device);
        UP3D_CUDA(cudaMemcpyAsync(out, m->fnbr.get(), sizeof(int4) * m->E, cudaMemcpyDeviceToDevice, S(stream)));
    });
}

int up3d_mesh_set_face_neighbors(up3d_mesh* m, const int32_t* in, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(m && in, UP3D_ERR_ARGUMENT, "up3d_mesh_set_face_neighbors: null argument");
        DeviceGuard g(m->device);
        UP3D_CUDA(cudaMemcpyAsync(m->fnbr.get(), in, sizeof(int4) * m->E, cudaMemcpyDeviceToDevice, S(stream)));
        refresh_disp(m, S(stream));
        m->nb_depth = 0;  // the neighbourhoods follow the face neighbours
        m->tiles.reset();  // so does the tile plan (its neighbour table and components)
    });
}

int up3d_mesh_elem_to_csr(const up3d_mesh* m, int64_t* out, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(m && out, UP3D_ERR_ARGUMENT, "up3d_mesh_elem_to_csr: null argument");
        DeviceGuard g(m->device);
        k_elem_to_csr<<<grid_for(m->E, 256), 256, 0, S(stream)>>>(m->conn.get(), m->E, m->indptr.get(),
                                                                  m->indices.get(), out);
        UP3D_CHECK_LAUNCH();
    });
}

// greedy_coloring (mesh/coloring.py:66-126) + color_partition_csr (:129-145):
// elements visited in order, smallest colour unused by any element sharing a
// node; colour classes listed in ascending element order.
int up3d_mesh_coloring(up3d_mesh* m, int64_t* color_offsets, int64_t* color_elems, int32_t* n_colors) {
    return guarded([&] {
        UP3D_REQUIRE(m, UP3D_ERR_ARGUMENT, "up3d_mesh_coloring: null mesh");
        HostMeshExtra* x = extra_of(m, false);
        UP3D_REQUIRE(x, UP3D_ERR_ARGUMENT, "up3d_mesh_coloring: unknown mesh");
        if (x->color_offsets.empty()) {
            const int64_t E = m->E, N = m->N;
            const int32_t* el = x->elements.data();
            std::vector<int64_t> off(N + 1, 0), inc(4 * E);
            for (int64_t k = 0; k < 4 * E; ++k) off[el[k] + 1]++;
            for (int64_t n = 0; n < N; ++n) off[n + 1] += off[n];
            std::vector<int64_t> fill(off.begin(), off.end() - 1);
            for (int64_t k = 0; k < 4 * E; ++k) inc[fill[el[k]]++] = k / 4;
            std::vector<int32_t> colors(E, -1);
            int64_t mark[256];
            for (int c = 0; c < 256; ++c) mark[c] = -1;
            int32_t nc = 0;
            for (int64_t e = 0; e < E; ++e) {
                for (int i = 0; i < 4; ++i) {
                    int32_t node = el[4 * e + i];
                    for (int64_t k = off[node]; k < off[node + 1]; ++k) {
                        int32_t c = colors[inc[k]];
                        if (c >= 0) mark[c] = e;
                    }
                }
                int c = 0;
                while (c < 256 && mark[c] == e) ++c;
                UP3D_REQUIRE(c < 256, UP3D_ERR_VALUE,
                             "greedy coloring exceeded 256 colors -- pathological mesh connectivity "
                             "(a node shared by >255 elements)");
                colors[e] = c;
                nc = std::max(nc, c + 1);
            }
            x->color_offsets.assign(nc + 1, 0);
            for (int64_t e = 0; e < E; ++e) x->color_offsets[colors[e] + 1]++;
            for (int c = 0; c < nc; ++c) x->color_offsets[c + 1] += x->color_offsets[c];
            x->color_elems.resize(E);
            std::vector<int64_t> cur(x->color_offsets.begin(), x->color_offsets.end() - 1);
            for (int64_t e = 0; e < E; ++e) x->color_elems[cur[colors[e]]++] = e;
            m->n_colors = nc;
        }
        if (n_colors) *n_colors = m->n_colors;
        if (color_offsets)
            std::memcpy(color_offsets, x->color_offsets.data(), sizeof(int64_t) * x->color_offsets.size());
        if (color_elems) std::memcpy(color_elems, x->color_elems.data(), sizeof(int64_t) * x->color_elems.size());
    });
}

}  // extern "C"
