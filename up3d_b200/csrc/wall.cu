// Wall post-processing of the up3d library (post/surface.py:80-363): the
// in-plane P1 gradient of phi on every wall triangle (the wall velocity
// under the natural boundary condition), the triangle's outward normal
// (toward its owning tet), the optional normal-gated edge-neighbour
// smoothing of the gradients, the isentropic (or Bernoulli) Cp and the
// pressure-integrated force coefficient
//   cf = -sum_t Cp_t A_t n_t / S_ref.
// The owning tets and the edge adjacency are found once on the host
// (up3d_wall_create); each evaluation is three kernels and a fixed-order
// reduction on the device.

#include <algorithm>
#include <array>
#include <string>
#include <vector>

#include "internal.cuh"

struct up3d_wall {
    int device = 0;
    int64_t n_w = 0, n_nodes = 0;
    up3d::DBuf<int4> tri;       // (n_w) nodes a, b, c (stored winding), owning tet
    up3d::DBuf<int32_t> adj;    // (n_w, 3) neighbour across edges (0,1), (1,2), (2,0), or -1
    up3d::DBuf<double> g0, g1;  // (n_w, 3) gradients (smoothing ping-pong)
    up3d::DBuf<double> area;    // (n_w)
    up3d::DBuf<double> nout;    // (n_w, 3)
    up3d::DBuf<double> part;    // (blocks, 3) force partial sums
    up3d::DBuf<double> cf;      // (3)
};

namespace up3d {
namespace {

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

constexpr int WALL_BLOCK = 256;
constexpr int WALL_GRID = 148;

__device__ __forceinline__ void cross3(double ax, double ay, double az, double bx, double by, double bz, double& cx,
                                       double& cy, double& cz) {
    cx = rsub(rmul(ay, bz), rmul(az, by));
    cy = rsub(rmul(az, bx), rmul(ax, bz));
    cz = rsub(rmul(ax, by), rmul(ay, bx));
}

// triangle_tangential_gradients (post/surface.py:80-118) and
// wall_outward_normals (:192-231), per triangle.
__global__ void k_wall_tri(int64_t n_w, const int4* __restrict__ tri, const double4* __restrict__ X,
                           const int4* __restrict__ conn, const double* __restrict__ phi, double* __restrict__ g,
                           double* __restrict__ area, double* __restrict__ nout, double* __restrict__ nstored) {
    GRID_STRIDE(t, n_w) {
        const int4 f = tri[t];
        const double4 p0 = X[f.x], p1 = X[f.y], p2 = X[f.z];
        const double ax = rsub(p1.x, p0.x), ay = rsub(p1.y, p0.y), az = rsub(p1.z, p0.z);
        const double bx = rsub(p2.x, p0.x), by = rsub(p2.y, p0.y), bz = rsub(p2.z, p0.z);
        double vx, vy, vz;
        cross3(ax, ay, az, bx, by, bz, vx, vy, vz);
        const double ta = sqrt(dot3r(vx, vy, vz, vx, vy, vz));
        const double nx = __ddiv_rn(vx, ta), ny = __ddiv_rn(vy, ta), nz = __ddiv_rn(vz, ta);
        const double la = sqrt(dot3r(ax, ay, az, ax, ay, az));
        const double e1x = __ddiv_rn(ax, la), e1y = __ddiv_rn(ay, la), e1z = __ddiv_rn(az, la);
        double e2x, e2y, e2z;
        cross3(nx, ny, nz, e1x, e1y, e1z, e2x, e2y, e2z);
        const double u1 = dot3r(ax, ay, az, e1x, e1y, e1z), v1 = dot3r(ax, ay, az, e2x, e2y, e2z);
        const double u2 = dot3r(bx, by, bz, e1x, e1y, e1z), v2 = dot3r(bx, by, bz, e2x, e2y, e2z);
        const double df1 = rsub(phi[f.y], phi[f.x]), df2 = rsub(phi[f.z], phi[f.x]);
        const double det = rsub(rmul(u1, v2), rmul(v1, u2));
        const double du = __ddiv_rn(rsub(rmul(v2, df1), rmul(v1, df2)), det);
        const double dv = __ddiv_rn(radd(rmul(-u2, df1), rmul(u1, df2)), det);
        g[3 * t] = radd(rmul(du, e1x), rmul(dv, e2x));
        g[3 * t + 1] = radd(rmul(du, e1y), rmul(dv, e2y));
        g[3 * t + 2] = radd(rmul(du, e1z), rmul(dv, e2z));
        area[t] = rmul(0.5, ta);
        if (nstored) {
            nstored[3 * t] = nx;
            nstored[3 * t + 1] = ny;
            nstored[3 * t + 2] = nz;
        }
        // toward the owning tet's centroid
        const int4 c = conn[f.w];
        const double4 q0 = X[c.x], q1 = X[c.y], q2 = X[c.z], q3 = X[c.w];
        const double fx = __ddiv_rn(radd(radd(p0.x, p1.x), p2.x), 3.0);
        const double fy = __ddiv_rn(radd(radd(p0.y, p1.y), p2.y), 3.0);
        const double fz = __ddiv_rn(radd(radd(p0.z, p1.z), p2.z), 3.0);
        const double ox = __ddiv_rn(radd(radd(radd(q0.x, q1.x), q2.x), q3.x), 4.0);
        const double oy = __ddiv_rn(radd(radd(radd(q0.y, q1.y), q2.y), q3.y), 4.0);
        const double oz = __ddiv_rn(radd(radd(radd(q0.z, q1.z), q2.z), q3.z), 4.0);
        const double s = dot3r(nx, ny, nz, rsub(ox, fx), rsub(oy, fy), rsub(oz, fz)) < 0.0 ? -1.0 : 1.0;
        nout[3 * t] = s * nx;
        nout[3 * t + 1] = s * ny;
        nout[3 * t + 2] = s * nz;
    }
}

// smooth_wall_tangential_gradients, one pass (post/surface.py:147-189):
// the area-weighted mean of the triangle and its edge neighbours whose
// outward normals agree (n . n_nb > cos_thresh), neighbours in edge order.
__global__ void k_wall_smooth(int64_t n_w, const int32_t* __restrict__ adj, const double* __restrict__ area,
                              const double* __restrict__ nout, double cos_thresh, const double* __restrict__ g,
                              double* __restrict__ out) {
    GRID_STRIDE(t, n_w) {
        const double at = area[t];
        double sx = rmul(g[3 * t], at), sy = rmul(g[3 * t + 1], at), sz = rmul(g[3 * t + 2], at), w = at;
        for (int k = 0; k < 3; ++k) {
            const int32_t nb = adj[3 * t + k];
            if (nb < 0) continue;
            if (!(dot3r(nout[3 * t], nout[3 * t + 1], nout[3 * t + 2], nout[3 * nb], nout[3 * nb + 1],
                        nout[3 * nb + 2]) > cos_thresh))
                continue;
            const double an = area[nb];
            sx = radd(sx, rmul(g[3 * nb], an));
            sy = radd(sy, rmul(g[3 * nb + 1], an));
            sz = radd(sz, rmul(g[3 * nb + 2], an));
            w = radd(w, an);
        }
        out[3 * t] = __ddiv_rn(sx, w);
        out[3 * t + 1] = __ddiv_rn(sy, w);
        out[3 * t + 2] = __ddiv_rn(sz, w);
    }
}

// Cp per triangle (physics/isentropic.py:122-160: the exact isentropic law
// for M_inf > 0, Bernoulli at M_inf = 0) and block sums of Cp A n, summed
// in a fixed tree per block.
__global__ void __launch_bounds__(WALL_BLOCK)
    k_wall_cp(int64_t n_w, const double* __restrict__ g, const double* __restrict__ area,
              const double* __restrict__ nout, double u2, double m_inf, double gamma, double* __restrict__ cp,
              double* __restrict__ part) {
    __shared__ double sh[3][WALL_BLOCK];
    double fx = 0.0, fy = 0.0, fz = 0.0;
    GRID_STRIDE(t, n_w) {
        const double q2 = __ddiv_rn(dot3r(g[3 * t], g[3 * t + 1], g[3 * t + 2], g[3 * t], g[3 * t + 1], g[3 * t + 2]),
                                    u2);
        double c;
        if (m_inf > 0.0) {
            const double m2 = rmul(m_inf, m_inf);
            double base = radd(1.0, rmul(rmul(rmul(0.5, rsub(gamma, 1.0)), m2), rsub(1.0, q2)));
            if (base < 1e-10) base = 1e-10;
            const double rho = pow(base, __ddiv_rn(1.0, rsub(gamma, 1.0)));
            c = rmul(__ddiv_rn(2.0, rmul(gamma, m2)), rsub(pow(rho, gamma), 1.0));
        } else {
            c = rsub(1.0, q2);
        }
        if (cp) cp[t] = c;
        const double w = rmul(c, area[t]);
        fx = radd(fx, rmul(w, nout[3 * t]));
        fy = radd(fy, rmul(w, nout[3 * t + 1]));
        fz = radd(fz, rmul(w, nout[3 * t + 2]));
    }
    sh[0][threadIdx.x] = fx;
    sh[1][threadIdx.x] = fy;
    sh[2][threadIdx.x] = fz;
    __syncthreads();
    for (int o = WALL_BLOCK / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o)
            for (int d = 0; d < 3; ++d) sh[d][threadIdx.x] = radd(sh[d][threadIdx.x], sh[d][threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x < 3) part[3 * blockIdx.x + threadIdx.x] = sh[threadIdx.x][0];
}

__global__ void k_wall_total(int n_blocks, const double* __restrict__ part, double s_ref, double* __restrict__ cf) {
    if (threadIdx.x < 3) {
        double s = 0.0;
        for (int b = 0; b < n_blocks; ++b) s = radd(s, part[3 * b + threadIdx.x]);
        cf[threadIdx.x] = __ddiv_rn(-s, s_ref);
    }
}

template <class T>
void upload(DBuf<T>& d, const std::vector<T>& h) {
    d.alloc(h.size());
    if (!h.empty()) UP3D_CUDA(cudaMemcpy(d.get(), h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
}

}  // namespace
}  // namespace up3d

using namespace up3d;

extern "C" {

int up3d_wall_create(const up3d_mesh* m, const int32_t* elements, const int64_t* wall_faces, int64_t n_w,
                     up3d_wall** out) {
    return guarded([&] {
        UP3D_REQUIRE(m && elements && out && (n_w == 0 || wall_faces), UP3D_ERR_ARGUMENT,
                     "up3d_wall_create: null argument");
        UP3D_REQUIRE(n_w >= 0 && n_w < (1ll << 31), UP3D_ERR_VALUE, "up3d_wall_create: bad size");
        const int64_t N = m->N, E = m->E;
        std::vector<char> on_wall(N, 0);
        for (int64_t i = 0; i < 3 * n_w; ++i) {
            UP3D_REQUIRE(wall_faces[i] >= 0 && wall_faces[i] < N, UP3D_ERR_VALUE,
                         "up3d_wall_create: wall node out of range");
            on_wall[wall_faces[i]] = 1;
        }
        // owners: the tet faces whose three nodes are all wall nodes, keyed by
        // their sorted node triple (face f opposite local node f)
        using Key = std::array<int32_t, 3>;
        std::vector<std::pair<Key, int32_t>> tf;
        static const int FD[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};
        for (int64_t e = 0; e < E; ++e)
            for (int f = 0; f < 4; ++f) {
                Key k = {elements[4 * e + FD[f][0]], elements[4 * e + FD[f][1]], elements[4 * e + FD[f][2]]};
                if (!on_wall[k[0]] || !on_wall[k[1]] || !on_wall[k[2]]) continue;
                std::sort(k.begin(), k.end());
                tf.push_back({k, (int32_t)e});
            }
        std::sort(tf.begin(), tf.end());
        std::vector<int4> tri(n_w);
        for (int64_t t = 0; t < n_w; ++t) {
            Key k = {(int32_t)wall_faces[3 * t], (int32_t)wall_faces[3 * t + 1], (int32_t)wall_faces[3 * t + 2]};
            Key s = k;
            std::sort(s.begin(), s.end());
            auto lo = std::lower_bound(tf.begin(), tf.end(), std::make_pair(s, (int32_t)-1));
            auto hi = lo;
            while (hi != tf.end() && hi->first == s) ++hi;
            UP3D_REQUIRE(hi - lo == 1, UP3D_ERR_VALUE, "up3d_wall_create: wall face not owned by exactly one tet");
            tri[t] = make_int4(k[0], k[1], k[2], lo->second);
        }
        // edge adjacency: edges shared by exactly two triangles
        struct Edge {
            int32_t a, b;
            int32_t t, k;
        };
        std::vector<Edge> edges;
        edges.reserve(3 * n_w);
        for (int64_t t = 0; t < n_w; ++t) {
            const int32_t v[3] = {tri[t].x, tri[t].y, tri[t].z};
            for (int k = 0; k < 3; ++k) {
                const int32_t a = v[k], b = v[(k + 1) % 3];
                edges.push_back({std::min(a, b), std::max(a, b), (int32_t)t, k});
            }
        }
        std::sort(edges.begin(), edges.end(), [](const Edge& x, const Edge& y) {
            return x.a != y.a ? x.a < y.a : (x.b != y.b ? x.b < y.b : (x.t != y.t ? x.t < y.t : x.k < y.k));
        });
        std::vector<int32_t> adj(3 * n_w, -1);
        for (size_t i = 0; i < edges.size();) {
            size_t j = i;
            while (j < edges.size() && edges[j].a == edges[i].a && edges[j].b == edges[i].b) ++j;
            if (j - i == 2) {
                adj[3 * edges[i].t + edges[i].k] = edges[i + 1].t;
                adj[3 * edges[i + 1].t + edges[i + 1].k] = edges[i].t;
            }
            i = j;
        }
        int cur = 0;
        UP3D_CUDA(cudaGetDevice(&cur));
        UP3D_CUDA(cudaSetDevice(m->device));
        auto* w = new up3d_wall();
        try {
            w->device = m->device;
            w->n_w = n_w;
            w->n_nodes = N;
            upload(w->tri, tri);
            upload(w->adj, adj);
            const size_t n = n_w > 0 ? (size_t)n_w : 1;
            w->g0.alloc(3 * n);
            w->g1.alloc(3 * n);
            w->area.alloc(n);
            w->nout.alloc(3 * n);
            w->part.alloc(3 * WALL_GRID);
            w->cf.alloc(3);
        } catch (...) {
            delete w;
            cudaSetDevice(cur);
            throw;
        }
        UP3D_CUDA(cudaSetDevice(cur));
        *out = w;
    });
}

int up3d_wall_destroy(up3d_wall* w) {
    return guarded([&] { delete w; });
}

int up3d_wall_forces(up3d_wall* w, const up3d_mesh* m, const double* phi, double u_inf, double m_inf,
                     double gamma, double s_ref, int smooth_passes, double* grad_out, double* area_out,
                     double* normal_out, double* outward_out, double* cp_out, double* cf, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(w && m && phi && cf, UP3D_ERR_ARGUMENT, "up3d_wall_forces: null argument");
        UP3D_REQUIRE(m->N == w->n_nodes, UP3D_ERR_VALUE, "up3d_wall_forces: the wall belongs to another mesh");
        UP3D_REQUIRE(smooth_passes >= 0 && u_inf > 0.0 && s_ref != 0.0, UP3D_ERR_VALUE,
                     "up3d_wall_forces: bad parameter");
        cudaStream_t s = S(stream);
        if (w->n_w == 0) {
            cf[0] = cf[1] = cf[2] = 0.0;
            return;
        }
        const unsigned grid = grid_for(w->n_w, WALL_BLOCK, WALL_GRID);
        k_wall_tri<<<grid, WALL_BLOCK, 0, s>>>(w->n_w, w->tri.get(), m->nodes4.get(), m->conn.get(), phi,
                                               w->g0.get(), w->area.get(), w->nout.get(), normal_out);
        UP3D_CHECK_LAUNCH();
        double* g = w->g0.get();
        double* h = w->g1.get();
        for (int p = 0; p < smooth_passes; ++p) {
            k_wall_smooth<<<grid, WALL_BLOCK, 0, s>>>(w->n_w, w->adj.get(), w->area.get(), w->nout.get(), 0.2, g,
                                                      h);
            UP3D_CHECK_LAUNCH();
            std::swap(g, h);
        }
        k_wall_cp<<<WALL_GRID, WALL_BLOCK, 0, s>>>(w->n_w, g, w->area.get(), w->nout.get(), u_inf * u_inf,
                                                   m_inf, gamma, cp_out, w->part.get());
        UP3D_CHECK_LAUNCH();
        k_wall_total<<<1, 32, 0, s>>>(WALL_GRID, w->part.get(), s_ref, w->cf.get());
        UP3D_CHECK_LAUNCH();
        if (grad_out)
            UP3D_CUDA(cudaMemcpyAsync(grad_out, g, sizeof(double) * 3 * w->n_w, cudaMemcpyDeviceToDevice, s));
        if (area_out)
            UP3D_CUDA(cudaMemcpyAsync(area_out, w->area.get(), sizeof(double) * w->n_w, cudaMemcpyDeviceToDevice, s));
        if (outward_out)
            UP3D_CUDA(cudaMemcpyAsync(outward_out, w->nout.get(), sizeof(double) * 3 * w->n_w,
                                      cudaMemcpyDeviceToDevice, s));
        UP3D_CUDA(cudaMemcpyAsync(cf, w->cf.get(), sizeof(double) * 3, cudaMemcpyDeviceToHost, s));
        UP3D_CUDA(cudaStreamSynchronize(s));
    });
}

}  // extern "C"
