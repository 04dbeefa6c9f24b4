// Per-side Newton Terms 2 and 3 of the level-set (cut-element) assembly
// (kernels/cut_assembly.py:401-488), as COO triplets on extended DOFs.
//
// Term 2, element e kept with s_e lim_e != 0:
//   (dof[e][a], read[e][b], w2 (gBr_e,a gB_e,b)),  w2 = 2/u^2 s_e lim_e V_e
// Term 3, element e kept with s_u lim_u(e) != 0, u = upstream[e]:
//   (dof[e][a], read[u][k], w3 (gBr_e,a gB_u,k)),  w3 = 2/u^2 s_u lim_u V_e
// gBr = grad_row . B (the row factor: the field the residual scatters),
// gB = grad . B (the column factor: the field the density reads).  The
// output order is the reference's: every Term-2 block of the qualifying
// elements in ascending order, then every Term-3 block, each block a-major;
// positions come from scans of the per-element flags, so the triplets are
// deterministic.

#include <cub/cub.cuh>

#include "internal.cuh"

namespace up3d {
namespace {

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

__device__ __forceinline__ bool emits2(const uint8_t* keep, const double* s_e, const double* lim, int64_t e) {
    return keep[e] && rmul(s_e[e], lim[e]) != 0.0;
}
// (an upstream index outside [0, E) never reads lim: the call reports it
// as an error before any triplet is written)
__device__ __forceinline__ bool emits3(const uint8_t* keep, const double* s_u, const double* lim,
                                       const int64_t* up, int64_t e, int64_t E) {
    const int64_t u = up[e];
    return keep[e] && u >= 0 && u < E && rmul(s_u[e], lim[u]) != 0.0;
}

__global__ void k_side_flags(int64_t E, const uint8_t* __restrict__ keep, const double* __restrict__ s_e,
                             const double* __restrict__ s_u, const double* __restrict__ lim,
                             const int64_t* __restrict__ up, int64_t* __restrict__ f2, int64_t* __restrict__ f3) {
    GRID_STRIDE(e, E) {
        f2[e] = emits2(keep, s_e, lim, e) ? 1 : 0;
        f3[e] = emits3(keep, s_u, lim, up, e, E) ? 1 : 0;
    }
}

__device__ __forceinline__ void gB_row_of(const double* __restrict__ B, int64_t e, const double* __restrict__ g,
                                          double out[4]) {
    const double gx = g[3 * e], gy = g[3 * e + 1], gz = g[3 * e + 2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
        out[a] = dot3r(gx, gy, gz, B[12 * e + 3 * a], B[12 * e + 3 * a + 1], B[12 * e + 3 * a + 2]);
}

__global__ void k_side_fill(int64_t E, const double* __restrict__ B, const double* __restrict__ V,
                            const uint8_t* __restrict__ keep, const int64_t* __restrict__ dof,
                            const int64_t* __restrict__ read, const double* __restrict__ grad,
                            const double* __restrict__ grad_row, const double* __restrict__ lim,
                            const double* __restrict__ s_e, const double* __restrict__ s_u,
                            const int64_t* __restrict__ up, double two_inv_u2, const int64_t* __restrict__ o2,
                            const int64_t* __restrict__ o3, int64_t n2, int64_t* __restrict__ rows,
                            int64_t* __restrict__ cols, double* __restrict__ data) {
    GRID_STRIDE(e, E) {
        const bool t2 = emits2(keep, s_e, lim, e);
        const bool t3 = emits3(keep, s_u, lim, up, e, E);
        if (!t2 && !t3) continue;
        double gbr[4], gb[4];
        gB_row_of(B, e, grad_row, gbr);
        if (t2) {
            gB_row_of(B, e, grad, gb);
            const double w2 = rmul(rmul(two_inv_u2, rmul(s_e[e], lim[e])), V[e]);
            const int64_t base = 16 * o2[e];
            for (int a = 0; a < 4; ++a)
                for (int b = 0; b < 4; ++b) {
                    rows[base + 4 * a + b] = dof[4 * e + a];
                    cols[base + 4 * a + b] = read[4 * e + b];
                    data[base + 4 * a + b] = rmul(w2, rmul(gbr[a], gb[b]));
                }
        }
        if (t3) {
            const int64_t u = up[e];
            gB_row_of(B, u, grad, gb);
            const double w3 = rmul(rmul(two_inv_u2, rmul(s_u[e], lim[u])), V[e]);
            const int64_t base = 16 * (n2 + o3[e]);
            for (int a = 0; a < 4; ++a)
                for (int k = 0; k < 4; ++k) {
                    rows[base + 4 * a + k] = dof[4 * e + a];
                    cols[base + 4 * a + k] = read[4 * u + k];
                    data[base + 4 * a + k] = rmul(w3, rmul(gbr[a], gb[k]));
                }
        }
    }
}

__global__ void k_check_up(int64_t E, const int64_t* __restrict__ up, int* __restrict__ bad) {
    GRID_STRIDE(e, E) if (up[e] < 0 || up[e] >= E) *bad = 1;
}

}  // namespace
}  // namespace up3d

using namespace up3d;

extern "C" {

int up3d_terms23_side_coo(const up3d_mesh* m, const uint8_t* keep, const int64_t* dofvec, const int64_t* readvec,
                          const double* grad, const double* grad_row, const double* lim_mask, const double* s_e,
                          const double* s_u, const int64_t* upstream, double u_inf, int64_t* rows, int64_t* cols,
                          double* data, int64_t capacity, int64_t* count, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(m && keep && dofvec && grad && lim_mask && s_e && s_u && upstream && count, UP3D_ERR_ARGUMENT,
                     "up3d_terms23_side_coo: null argument");
        UP3D_REQUIRE(u_inf > 0.0, UP3D_ERR_VALUE, "up3d_terms23_side_coo: u_inf must be positive");
        cudaStream_t s = S(stream);
        const int64_t E = m->E;
        const int64_t* read = readvec ? readvec : dofvec;
        const double* grow = grad_row ? grad_row : grad;
        DBuf<int64_t> f2, f3, o2, o3;
        DBuf<int> bad;
        f2.alloc(E + 1);
        f3.alloc(E + 1);
        o2.alloc(E + 1);
        o3.alloc(E + 1);
        bad.alloc(1);
        UP3D_CUDA(cudaMemsetAsync(bad.get(), 0, sizeof(int), s));
        k_check_up<<<grid_for(E, 256), 256, 0, s>>>(E, upstream, bad.get());
        UP3D_CHECK_LAUNCH();
        k_side_flags<<<grid_for(E, 256), 256, 0, s>>>(E, keep, s_e, s_u, lim_mask, upstream, f2.get(), f3.get());
        UP3D_CHECK_LAUNCH();
        UP3D_CUDA(cudaMemsetAsync(f2.get() + E, 0, sizeof(int64_t), s));
        UP3D_CUDA(cudaMemsetAsync(f3.get() + E, 0, sizeof(int64_t), s));
        DBuf<unsigned char> tmp;
        size_t bytes = 0;
        UP3D_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, f2.get(), o2.get(), E + 1, s));
        tmp.alloc(bytes);
        UP3D_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), bytes, f2.get(), o2.get(), E + 1, s));
        UP3D_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), bytes, f3.get(), o3.get(), E + 1, s));
        int64_t n23[2] = {0, 0};
        int hbad = 0;
        UP3D_CUDA(cudaMemcpyAsync(&n23[0], o2.get() + E, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        UP3D_CUDA(cudaMemcpyAsync(&n23[1], o3.get() + E, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        UP3D_CUDA(cudaMemcpyAsync(&hbad, bad.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
        UP3D_CUDA(cudaStreamSynchronize(s));
        UP3D_REQUIRE(!hbad, UP3D_ERR_VALUE, "up3d_terms23_side_coo: upstream element out of range");
        const int64_t total = 16 * (n23[0] + n23[1]);
        *count = total;
        if (!rows) return;  // count only
        UP3D_REQUIRE(cols && data && capacity >= total, UP3D_ERR_VALUE,
                     "up3d_terms23_side_coo: output capacity below the triplet count");
        if (total == 0) return;
        k_side_fill<<<grid_for(E, 256), 256, 0, s>>>(E, m->B.get(), m->V.get(), keep, dofvec, read, grad, grow,
                                                     lim_mask, s_e, s_u, upstream, 2.0 * (1.0 / (u_inf * u_inf)), o2.get(),
                                                     o3.get(), n23[0], rows, cols, data);
        UP3D_CHECK_LAUNCH();
        UP3D_CUDA(cudaStreamSynchronize(s));
    });
}

}  // extern "C"
