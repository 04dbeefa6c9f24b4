// Device BLAS-1 helpers and the Krylov operator abstraction (krylov.cu).
#pragma once

#include "internal.cuh"

struct up3d_coupled;

namespace up3d {

// y = A x (+ xA x) on the device (linear.cu); dir = identity rows or NULL
template <class T>
void launch_spmv(int64_t n, const int32_t* indptr, const int32_t* indices, const T* data, const T* x, T* y,
                 const uint8_t* dir, cudaStream_t s);
template <class T>
void launch_spmv2(int64_t n, const int32_t* indptr, const int32_t* indices, const T* data, const int32_t* xptr,
                  const int32_t* xidx, const T* xdata, const T* x, T* y, const uint8_t* dir, cudaStream_t s);

// The coupled (phi, Gamma) operator of a wake-cut mesh (wake.cu): y =
// J_ff x + B (K x + g) in full reduced size, t = K x + g when t != NULL.
int64_t coupled_rows(const up3d_coupled* c);
void coupled_apply(const up3d_coupled* c, const up3d_csr& J, const up3d_csr& extra, const double* x,
                   const double* g, double* y, double* t, cudaStream_t s);

// Reproducible reductions and vector updates on one stream.
// Vector arguments are double or float; dot products accumulate in FP64.
struct Blas {
    cudaStream_t s;
    DBuf<double> partial, scal;
    DBuf<unsigned int> counter;   // blocks arrived, for the last-block reductions (re-armed by it)
    double* host = nullptr;  // pinned scalar readback
    explicit Blas(cudaStream_t s);
    ~Blas();
    // out[k] = V_k . y for k < K, then y . y at out[K] when self_dot
    template <class T>
    void multidot(const T* V, int64_t ldv, int K, const T* y, int64_t n, double* out_dev, bool self_dot = false);
    template <class T>
    double dot(const T* x, const T* y, int64_t n);
    template <class T>
    double nrm2(const T* x, int64_t n);
    void axpby(double a, const double* x, double b, double* y, int64_t n);
    template <class T>
    void scale(T* x, double a, int64_t n);
    template <class T>
    void multiaxpy(const T* V, int64_t ldv, int K, const double* h_dev, T* y, int64_t n);
    // y -= V h (K <= 64) in one sweep that also forms V^T y (dots) or y.y
    // (!dots) of the new y into out_dev
    template <class T>
    void axpy_dots(const T* V, int64_t ldv, int K, const double* h_dev, T* y, int64_t n, bool dots,
                   double* out_dev);
};

// y = A x (+ extra x): the P1-pattern matrix plus, for the Newton Jacobian,
// the Term-3 entries outside the pattern.  With `coupled` set, A (+ extra)
// is a wake-cut mesh's Jacobian and the operator is the coupled system's
// J_ff + B K on the reduced unknowns (FP64 only).
struct Operator {
    up3d_csr A{};
    up3d_csr extra{};
    const float* data32 = nullptr;   // FP32 copies of the values (mixed precision)
    const float* extra32 = nullptr;
    const up3d_coupled* coupled = nullptr;
    int64_t rows() const { return coupled ? coupled_rows(coupled) : A.n; }
    void apply(const double* x, double* y, cudaStream_t s) const;
    void apply(const float* x, float* y, cudaStream_t s) const;
};

void amg_apply(void* amg, const double* r, double* z, cudaStream_t s);
void amg_apply_f32(void* amg, const float* r, float* z, cudaStream_t s);
void amg_destroy(void* amg);
void* amg_setup(const up3d_csr& A, const up3d_amg_options& opt, cudaStream_t s);
void amg_refresh(void* amg, const up3d_csr& A, cudaStream_t s);
const up3d_amg_info* amg_info(void* amg);
void* ilu0_create(const up3d_csr* A, int sweeps, int tri_sweeps, cudaStream_t s);
void ilu0_apply(void* ilu, const double* r, double* z, cudaStream_t s);
void ilu0_destroy(void* ilu);
void ilu0_factors(const void* ilu, double* out, double* shift, cudaStream_t s);

}  // namespace up3d

// Preconditioner handle: identity, point Jacobi or an AMG hierarchy.
struct up3d_precond {
    int kind = 0;  // 0 identity, 1 Jacobi, 2 AMG, 3 ILU(0)
    int64_t n = 0;
    up3d::DBuf<double> dinv;
    void* amg = nullptr;
    void* ilu = nullptr;
    up3d_precond() = default;
    ~up3d_precond() {
        if (amg) up3d::amg_destroy(amg);
        if (ilu) up3d::ilu0_destroy(ilu);
    }
    void apply(const double* r, double* z, cudaStream_t s);
    void apply(const float* r, float* z, cudaStream_t s);
};
