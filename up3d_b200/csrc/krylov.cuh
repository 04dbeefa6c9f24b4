// Device BLAS-1 helpers and the Krylov operator abstraction (krylov.cu).
#pragma once

#include "internal.cuh"

namespace up3d {

// Reproducible reductions and vector updates on one stream.
struct Blas {
    cudaStream_t s;
    DBuf<double> partial, scal;
    double* host = nullptr;  // pinned scalar readback
    explicit Blas(cudaStream_t s);
    ~Blas();
    void multidot(const double* V, int64_t ldv, int K, const double* y, int64_t n, double* out_dev);
    double dot(const double* x, const double* y, int64_t n);
    double nrm2(const double* x, int64_t n);
    void axpby(double a, const double* x, double b, double* y, int64_t n);
    void scale(double* x, double a, int64_t n);
    void multiaxpy(const double* V, int64_t ldv, int K, const double* h_dev, double* y, int64_t n);
};

// y = A x (+ extra x): the P1-pattern matrix plus, for the Newton Jacobian,
// the Term-3 entries outside the pattern.
struct Operator {
    up3d_csr A{};
    up3d_csr extra{};
    mutable DBuf<double> tmp;
    void apply(const double* x, double* y, cudaStream_t s) const;
};

void amg_apply(void* amg, const double* r, double* z, cudaStream_t s);
void amg_destroy(void* amg);
void* amg_setup(const up3d_csr& A, const up3d_amg_options& opt, cudaStream_t s);
void amg_refresh(void* amg, const up3d_csr& A, cudaStream_t s);
const up3d_amg_info* amg_info(void* amg);

}  // namespace up3d

// Preconditioner handle: identity, point Jacobi or an AMG hierarchy.
struct up3d_precond {
    int kind = 0;  // 0 identity, 1 Jacobi, 2 AMG
    int64_t n = 0;
    up3d::DBuf<double> dinv;
    void* amg = nullptr;
    up3d_precond() = default;
    ~up3d_precond() {
        if (amg) up3d::amg_destroy(amg);
    }
    void apply(const double* r, double* z, cudaStream_t s);
};
