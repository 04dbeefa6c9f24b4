/*
 * up3d_oracle.c -- CPU ORACLE of the pyfp3d element-loop hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates, in plain C with OpenMP, the
 * algorithms of the reference (swayli94/UP3D, package pyfp3d) for the hot
 * path: element geometry, face adjacency, greedy colouring, CSR pattern,
 * element velocities, isentropic physics, the multi-hop upstream walk, the
 * upwinded density and its sensitivities, residual / Picard matrix / Newton
 * Jacobian assembly and CSR SpMV.  It is the checker that the CUDA library is
 * compared against in tests/, the CPU leg of bench.py and the body of
 * smoke()'s check; the product never links or calls it.
 *
 * Parity of this restatement is pinned by the .npz fixtures under tests/golden, which were
 * produced by running the reference itself (tests/golden/make_golden.py).
 *
 * Each function cites the reference file:line it restates.  Summation orders
 * follow the reference (colour-ordered scatter, ascending elements within a
 * colour) so that the CPU timing is the reference's parallel structure.
 * Compiled without -ffast-math and without FMA contraction.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_API __attribute__((visibility("default")))

/* ------------------------------------------------------------------ */
/* physics/isentropic.py                                               */
/* ------------------------------------------------------------------ */

/* density_isentropic, physics/isentropic.py:30-58 (vacuum guard :56-57) */
static inline double orc_rho(double q2, double m_inf, double gamma) {
    double exponent = 1.0 / (gamma - 1.0);
    double base = 1.0 + 0.5 * (gamma - 1.0) * (m_inf * m_inf) * (1.0 - q2);
    if (base < 1e-10) base = 1e-10;
    return pow(base, exponent);
}

/* mach_number_squared, physics/isentropic.py:80-97 */
static inline double orc_mach2(double q2, double m_inf, double gamma) {
    double num = q2 * (m_inf * m_inf);
    double den = 1.0 + 0.5 * (gamma - 1.0) * (m_inf * m_inf) * (1.0 - q2);
    return num / den;
}

/* density_derivative_wrt_q_sq, physics/isentropic.py:164-180 */
static inline double orc_drho(double q2, double m_inf, double gamma) {
    double rho = orc_rho(q2, m_inf, gamma);
    return -0.5 * (m_inf * m_inf) * pow(rho, 2.0 - gamma);
}

/* mach_squared_derivative_wrt_q_sq, physics/isentropic.py:184-206 */
static inline double orc_dmach2(double q2, double m_inf, double gamma) {
    double D = 1.0 + 0.5 * (gamma - 1.0) * (m_inf * m_inf) * (1.0 - q2);
    return (m_inf * m_inf) * (1.0 + 0.5 * (gamma - 1.0) * (m_inf * m_inf)) / (D * D);
}

/* q2_at_mach, physics/isentropic.py:262-289 */
ORC_API double orc_q2_at_mach(double mach, double m_inf, double gamma) {
    if (m_inf == 0.0) return INFINITY;
    double m2 = mach * mach;
    return m2 * (1.0 + 0.5 * (gamma - 1.0) * (m_inf * m_inf)) /
           ((m_inf * m_inf) * (1.0 + 0.5 * (gamma - 1.0) * m2));
}

/* density_field, physics/isentropic.py:236-258 */
ORC_API void orc_density_field(const double* q2, int64_t n, double m_inf, double gamma,
                               double* out) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) out[i] = orc_rho(q2[i], m_inf, gamma);
}

/* mach_squared_field, physics/isentropic.py:318-334 */
ORC_API void orc_mach2_field(const double* q2, int64_t n, double m_inf, double gamma,
                             double* out) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) out[i] = orc_mach2(q2[i], m_inf, gamma);
}

/* limit_q2_field, physics/isentropic.py:293-314 */
ORC_API void orc_limit_q2_field(const double* q2, int64_t n, double m_inf, double m_cap,
                                double gamma, double* out) {
    double cap = orc_q2_at_mach(m_cap, m_inf, gamma);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) out[i] = q2[i] < cap ? q2[i] : cap;
}

/* density_derivative_wrt_q_sq_field, physics/isentropic.py:338-354 */
ORC_API void orc_drho_field(const double* q2, int64_t n, double m_inf, double gamma,
                            double* out) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) out[i] = orc_drho(q2[i], m_inf, gamma);
}

/* ------------------------------------------------------------------ */
/* mesh/metrics.py                                                     */
/* ------------------------------------------------------------------ */

/* precompute_element_geometry, mesh/metrics.py:177-204 (volume from the
 * triple product, :27-70; degeneracy test relative to edge lengths,
 * :155-164; B_e rows = J^{-T} grad_ref N_i, :96-126, :166-173).
 * The inverse is the adjugate form: rows of J^{-1} are the cross products
 * of J's columns divided by det J.  Returns the index of the first
 * degenerate tet, or -1. */
ORC_API int64_t orc_element_geometry(const double* nodes, const int32_t* el, int64_t E,
                                     double* B, double* V) {
    int64_t bad = -1;
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < E; ++e) {
        const double* x0 = nodes + 3 * (int64_t)el[4 * e + 0];
        const double* x1 = nodes + 3 * (int64_t)el[4 * e + 1];
        const double* x2 = nodes + 3 * (int64_t)el[4 * e + 2];
        const double* x3 = nodes + 3 * (int64_t)el[4 * e + 3];
        double v1[3], v2[3], v3[3];
        for (int d = 0; d < 3; ++d) {
            v1[d] = x1[d] - x0[d];
            v2[d] = x2[d] - x0[d];
            v3[d] = x3[d] - x0[d];
        }
        double c23[3] = {v2[1] * v3[2] - v2[2] * v3[1], v2[2] * v3[0] - v2[0] * v3[2],
                         v2[0] * v3[1] - v2[1] * v3[0]};
        double c31[3] = {v3[1] * v1[2] - v3[2] * v1[1], v3[2] * v1[0] - v3[0] * v1[2],
                         v3[0] * v1[1] - v3[1] * v1[0]};
        double c12[3] = {v1[1] * v2[2] - v1[2] * v2[1], v1[2] * v2[0] - v1[0] * v2[2],
                         v1[0] * v2[1] - v1[1] * v2[0]};
        double det = v1[0] * c23[0] + v1[1] * c23[1] + v1[2] * c23[2];
        V[e] = fabs(det) / 6.0;
        double s1 = sqrt(v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2]);
        double s2 = sqrt(v2[0] * v2[0] + v2[1] * v2[1] + v2[2] * v2[2]);
        double s3 = sqrt(v3[0] * v3[0] + v3[1] * v3[1] + v3[2] * v3[2]);
        double scale = s1 * s2 * s3;
        if (scale == 0.0 || fabs(det) < 1e-12 * scale) {
#pragma omp critical
            { if (bad < 0 || e < bad) bad = e; }
            for (int k = 0; k < 12; ++k) B[12 * e + k] = 0.0;
            continue;
        }
        double inv = 1.0 / det;
        double* b = B + 12 * e;
        for (int d = 0; d < 3; ++d) {
            b[3 + d] = c23[d] * inv;
            b[6 + d] = c31[d] * inv;
            b[9 + d] = c12[d] * inv;
            b[d] = -(b[3 + d] + b[6 + d] + b[9 + d]);
        }
    }
    return bad;
}

static int cmp_i64(const void* a, const void* b) {
    int64_t x = *(const int64_t*)a, y = *(const int64_t*)b;
    return (x > y) - (x < y);
}

/* Face ordering of a tet: face f is opposite local node f,
 * mesh/metrics.py:224-232. */
static const int orc_face_nodes[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};

/* build_face_adjacency, mesh/metrics.py:208-278: neighbour across face f of
 * e, or -1.  Matching faces by a sort of (sorted-node-triple, e*4+f) keys
 * instead of the reference's hash map gives the same pairing on a manifold
 * mesh (each interior face is shared by exactly two tets). */
typedef struct { int32_t a, b, c; int64_t owner; } orc_face_key;
static int cmp_face(const void* p, const void* q) {
    const orc_face_key* x = (const orc_face_key*)p;
    const orc_face_key* y = (const orc_face_key*)q;
    if (x->a != y->a) return x->a < y->a ? -1 : 1;
    if (x->b != y->b) return x->b < y->b ? -1 : 1;
    if (x->c != y->c) return x->c < y->c ? -1 : 1;
    return (x->owner > y->owner) - (x->owner < y->owner);
}
ORC_API void orc_face_adjacency(const int32_t* el, int64_t E, int32_t* fn) {
    orc_face_key* keys = (orc_face_key*)malloc(sizeof(orc_face_key) * 4 * (size_t)E);
    for (int64_t e = 0; e < E; ++e)
        for (int f = 0; f < 4; ++f) {
            int32_t a = el[4 * e + orc_face_nodes[f][0]];
            int32_t b = el[4 * e + orc_face_nodes[f][1]];
            int32_t c = el[4 * e + orc_face_nodes[f][2]];
            int32_t t;
            if (a > b) { t = a; a = b; b = t; }
            if (b > c) { t = b; b = c; c = t; }
            if (a > b) { t = a; a = b; b = t; }
            orc_face_key k = {a, b, c, 4 * e + f};
            keys[4 * e + f] = k;
            fn[4 * e + f] = -1;
        }
    qsort(keys, 4 * (size_t)E, sizeof(orc_face_key), cmp_face);
    for (int64_t i = 0; i + 1 < 4 * E; ++i) {
        if (keys[i].a == keys[i + 1].a && keys[i].b == keys[i + 1].b &&
            keys[i].c == keys[i + 1].c) {
            int64_t p = keys[i].owner, q = keys[i + 1].owner;
            fn[p] = (int32_t)(q / 4);
            fn[q] = (int32_t)(p / 4);
            ++i;
        }
    }
    free(keys);
}

/* centroids = nodes[elements].mean(axis=1), kernels/upwind.py:750
 * (numpy reduces the size-4 axis sequentially, then divides by 4). */
ORC_API void orc_centroids(const double* nodes, const int32_t* el, int64_t E, double* cen) {
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < E; ++e)
        for (int d = 0; d < 3; ++d) {
            double s = nodes[3 * (int64_t)el[4 * e] + d];
            s += nodes[3 * (int64_t)el[4 * e + 1] + d];
            s += nodes[3 * (int64_t)el[4 * e + 2] + d];
            s += nodes[3 * (int64_t)el[4 * e + 3] + d];
            cen[3 * e + d] = s / 4.0;
        }
}

/* ------------------------------------------------------------------ */
/* mesh/coloring.py                                                    */
/* ------------------------------------------------------------------ */

/* node_to_element_csr, mesh/coloring.py:46-62: incident elements of every
 * node in ascending element order. */
ORC_API void orc_node_to_element(const int32_t* el, int64_t E, int64_t N, int64_t* off,
                                 int64_t* elems) {
    memset(off, 0, sizeof(int64_t) * (size_t)(N + 1));
    for (int64_t k = 0; k < 4 * E; ++k) off[el[k] + 1]++;
    for (int64_t n = 0; n < N; ++n) off[n + 1] += off[n];
    int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (size_t)N);
    memcpy(fill, off, sizeof(int64_t) * (size_t)N);
    for (int64_t k = 0; k < 4 * E; ++k) elems[fill[el[k]]++] = k / 4;
    free(fill);
}

/* _greedy_coloring_kernel + greedy_coloring, mesh/coloring.py:66-126:
 * visit elements in order, take the smallest colour not used by any element
 * sharing a node.  Returns n_colors, or -1 past 256 colours (:89-93). */
ORC_API int32_t orc_greedy_coloring(const int32_t* el, int64_t E, int64_t N,
                                    int32_t* colors) {
    int64_t* off = (int64_t*)malloc(sizeof(int64_t) * (size_t)(N + 1));
    int64_t* inc = (int64_t*)malloc(sizeof(int64_t) * 4 * (size_t)E);
    orc_node_to_element(el, E, N, off, inc);
    int64_t mark[256];
    for (int c = 0; c < 256; ++c) mark[c] = -1;
    for (int64_t e = 0; e < E; ++e) colors[e] = -1;
    int32_t n_colors = 0;
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
        if (c >= 256) { n_colors = -1; break; }
        colors[e] = c;
        if (c + 1 > n_colors) n_colors = c + 1;
    }
    free(off);
    free(inc);
    return n_colors;
}

/* color_partition_csr, mesh/coloring.py:129-145 (stable sort by colour). */
ORC_API void orc_color_partition(const int32_t* colors, int64_t E, int32_t n_colors,
                                 int64_t* offsets, int64_t* elems) {
    memset(offsets, 0, sizeof(int64_t) * (size_t)(n_colors + 1));
    for (int64_t e = 0; e < E; ++e) offsets[colors[e] + 1]++;
    for (int c = 0; c < n_colors; ++c) offsets[c + 1] += offsets[c];
    int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n_colors + 1));
    memcpy(fill, offsets, sizeof(int64_t) * (size_t)(n_colors + 1));
    for (int64_t e = 0; e < E; ++e) elems[fill[colors[e]]++] = e;
    free(fill);
}

/* ------------------------------------------------------------------ */
/* kernels/jacobian.py: pattern and scatter map                        */
/* ------------------------------------------------------------------ */

/* build_csr_pattern, kernels/jacobian.py:60-75: sorted, de-duplicated
 * node-to-node pattern.  Pass 1 (indices == NULL) fills indptr and returns
 * nnz; pass 2 fills indices. */
ORC_API int64_t orc_csr_pattern(const int32_t* el, int64_t E, int64_t N, int64_t* indptr,
                                int32_t* indices) {
    int64_t* off = (int64_t*)malloc(sizeof(int64_t) * (size_t)(N + 1));
    int64_t* inc = (int64_t*)malloc(sizeof(int64_t) * 4 * (size_t)E);
    orc_node_to_element(el, E, N, off, inc);
    if (indices == NULL) indptr[0] = 0;
#pragma omp parallel
    {
        int64_t cap = 64;
        int64_t* buf = (int64_t*)malloc(sizeof(int64_t) * (size_t)cap);
#pragma omp for schedule(static)
        for (int64_t n = 0; n < N; ++n) {
            int64_t need = 4 * (off[n + 1] - off[n]);
            if (need > cap) {
                cap = need;
                buf = (int64_t*)realloc(buf, sizeof(int64_t) * (size_t)cap);
            }
            int64_t m = 0;
            for (int64_t k = off[n]; k < off[n + 1]; ++k)
                for (int j = 0; j < 4; ++j) buf[m++] = el[4 * inc[k] + j];
            qsort(buf, (size_t)m, sizeof(int64_t), cmp_i64);
            int64_t u = 0;
            for (int64_t t = 0; t < m; ++t)
                if (t == 0 || buf[t] != buf[t - 1]) {
                    if (indices) indices[indptr[n] + u] = (int32_t)buf[t];
                    ++u;
                }
            if (!indices) indptr[n + 1] = u;
        }
        free(buf);
    }
    if (!indices)
        for (int64_t n = 0; n < N; ++n) indptr[n + 1] += indptr[n];
    free(off);
    free(inc);
    return indptr[N];
}

/* build_elem_to_csr, kernels/jacobian.py:78-103 (lower-bound search). */
ORC_API void orc_elem_to_csr(const int32_t* el, int64_t E, const int64_t* indptr,
                             const int32_t* indices, int64_t* e2c) {
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < E; ++e)
        for (int i = 0; i < 4; ++i) {
            int32_t row = el[4 * e + i];
            for (int j = 0; j < 4; ++j) {
                int32_t col = el[4 * e + j];
                int64_t a = indptr[row], b = indptr[row + 1];
                while (a < b) {
                    int64_t mid = (a + b) / 2;
                    if (indices[mid] < col) a = mid + 1; else b = mid;
                }
                e2c[16 * e + 4 * i + j] = a;
            }
        }
}

/* ------------------------------------------------------------------ */
/* kernels/gradient.py                                                 */
/* ------------------------------------------------------------------ */

/* element_velocity_q2, kernels/gradient.py:33-64 */
ORC_API void orc_velocities(const int32_t* el, const double* B, const double* phi, int64_t E,
                            double* grad, double* q2) {
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < E; ++e) {
        double gx = 0.0, gy = 0.0, gz = 0.0;
        for (int i = 0; i < 4; ++i) {
            double p = phi[el[4 * e + i]];
            gx += p * B[12 * e + 3 * i + 0];
            gy += p * B[12 * e + 3 * i + 1];
            gz += p * B[12 * e + 3 * i + 2];
        }
        grad[3 * e] = gx;
        grad[3 * e + 1] = gy;
        grad[3 * e + 2] = gz;
        q2[e] = gx * gx + gy * gy + gz * gz;
    }
}

/* ------------------------------------------------------------------ */
/* kernels/upwind.py                                                   */
/* ------------------------------------------------------------------ */

/* upstream_elements, kernels/upwind.py:69-125 */
ORC_API void orc_upstream(const int32_t* fn, const double* cen, const double* nodes,
                          const int32_t* el, const double* grad, int64_t E, int max_hops,
                          int64_t* out) {
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < E; ++e) {
        double gx = grad[3 * e], gy = grad[3 * e + 1], gz = grad[3 * e + 2];
        double pmin = 1e300, pmax = -1e300;
        for (int k = 0; k < 4; ++k) {
            const double* x = nodes + 3 * (int64_t)el[4 * e + k];
            double p = x[0] * gx + x[1] * gy + x[2] * gz;
            if (p < pmin) pmin = p;
            if (p > pmax) pmax = p;
        }
        double target = 0.8 * (pmax - pmin);
        int64_t cur = e;
        double reach = 0.0;
        int hops = 0;
        while (hops < max_hops && reach < target) {
            int64_t best = -1;
            double best_disp = 0.0;
            for (int f = 0; f < 4; ++f) {
                int64_t nb = fn[4 * cur + f];
                if (nb >= 0) {
                    double d = (cen[3 * nb] - cen[3 * cur]) * gx +
                               (cen[3 * nb + 1] - cen[3 * cur + 1]) * gy +
                               (cen[3 * nb + 2] - cen[3 * cur + 2]) * gz;
                    if (d < best_disp) { best_disp = d; best = nb; }
                }
            }
            if (best < 0) break;
            cur = best;
            reach += -best_disp;
            hops += 1;
        }
        out[e] = cur;
    }
}

static inline double orc_switch(double m2, double mc2, double C) {
    double m = m2 > mc2 ? m2 : mc2;
    double v = 1.0 - mc2 / m;
    return C * (v > 0.0 ? v : 0.0);
}

/* rho_tilde_sweep, kernels/upwind.py:457-500 */
ORC_API void orc_rho_tilde(const double* q2, const double* rho, const int64_t* up, int64_t n,
                           double m_inf, double m_crit, double C, double gamma,
                           double rho_floor, double* nu_out, double* rt_out) {
    double mc2 = m_crit * m_crit;
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < n; ++e) {
        int64_t u = up[e];
        double nu_e = orc_switch(orc_mach2(q2[e], m_inf, gamma), mc2, C);
        double nu_u = orc_switch(orc_mach2(q2[u], m_inf, gamma), mc2, C);
        double nu = nu_e > nu_u ? nu_e : nu_u;
        nu_out[e] = nu;
        double rt = rho[e] - nu * (rho[e] - rho[u]);
        rt_out[e] = rt > rho_floor ? rt : rho_floor;
    }
}

/* classify_upwind_branches, kernels/upwind.py:504-541 */
ORC_API void orc_classify(const double* q2, const double* rho, const int64_t* up, int64_t n,
                          double m_inf, double m_crit, double C, double gamma,
                          double rho_floor, int8_t* br) {
    double mc2 = m_crit * m_crit;
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < n; ++e) {
        int64_t u = up[e];
        if (u == e) { br[e] = rho[e] <= rho_floor ? 3 : 0; continue; }
        double nu_e = orc_switch(orc_mach2(q2[e], m_inf, gamma), mc2, C);
        double nu_u = orc_switch(orc_mach2(q2[u], m_inf, gamma), mc2, C);
        double nu = nu_e > nu_u ? nu_e : nu_u;
        double rt = rho[e] - nu * (rho[e] - rho[u]);
        if (rt <= rho_floor) br[e] = 3;
        else if (nu == 0.0) br[e] = 0;
        else if (nu_e >= nu_u) br[e] = 1;
        else br[e] = 2;
    }
}

/* rho_tilde_frozen_sweep, kernels/upwind.py:545-593 */
ORC_API void orc_rho_tilde_frozen(const double* q2, const double* rho, const int64_t* up,
                                  const int8_t* br, int64_t n, double m_inf, double m_crit,
                                  double C, double gamma, double rho_floor, double* nu_out,
                                  double* rt_out) {
    double mc2 = m_crit * m_crit;
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < n; ++e) {
        int b = br[e];
        if (b == 3) { nu_out[e] = 0.0; rt_out[e] = rho_floor; continue; }
        if (b == 0) { nu_out[e] = 0.0; rt_out[e] = rho[e]; continue; }
        int64_t u = up[e];
        double nu = b == 1 ? orc_switch(orc_mach2(q2[e], m_inf, gamma), mc2, C)
                           : orc_switch(orc_mach2(q2[u], m_inf, gamma), mc2, C);
        nu_out[e] = nu;
        rt_out[e] = rho[e] - nu * (rho[e] - rho[u]);
    }
}

/* nu' on the active switch branch: C (M_c^2 / M^4) dM^2/dq^2,
 * kernels/upwind.py:633-634, :720-721 */
static inline double orc_dnu(double q2, double m2, double mc2, double C, double m_inf,
                             double gamma) {
    return C * (mc2 / (m2 * m2)) * orc_dmach2(q2, m_inf, gamma);
}

/* rho_tilde_frozen_sensitivities_sweep, kernels/upwind.py:597-643 */
ORC_API void orc_sens_frozen(const double* q2, const double* rho, const int64_t* up,
                             const int8_t* br, int64_t n, double m_inf, double m_crit,
                             double C, double gamma, double rho_floor, double* se,
                             double* su) {
    double mc2 = m_crit * m_crit;
    (void)rho_floor;
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < n; ++e) {
        int b = br[e];
        if (b == 3) { se[e] = 0.0; su[e] = 0.0; continue; }
        double drho_e = orc_drho(q2[e], m_inf, gamma);
        if (b == 0) { se[e] = drho_e; su[e] = 0.0; continue; }
        int64_t u = up[e];
        double drho_u = orc_drho(q2[u], m_inf, gamma);
        double djump = rho[e] - rho[u];
        if (b == 1) {
            double m2 = orc_mach2(q2[e], m_inf, gamma);
            double nu = orc_switch(m2, mc2, C);
            double dnu_e = m2 > mc2 ? orc_dnu(q2[e], m2, mc2, C, m_inf, gamma) : 0.0;
            se[e] = drho_e * (1.0 - nu) - djump * dnu_e;
            su[e] = nu * drho_u;
        } else {
            double m2u = orc_mach2(q2[u], m_inf, gamma);
            double nu = orc_switch(m2u, mc2, C);
            double dnu_u = m2u > mc2 ? orc_dnu(q2[u], m2u, mc2, C, m_inf, gamma) : 0.0;
            se[e] = drho_e * (1.0 - nu);
            su[e] = nu * drho_u - djump * dnu_u;
        }
    }
}

/* rho_tilde_sensitivities_sweep, kernels/upwind.py:647-730 */
ORC_API void orc_sens(const double* q2, const double* rho, const int64_t* up, int64_t n,
                      double m_inf, double m_crit, double C, double gamma, double rho_floor,
                      double* se, double* su) {
    double mc2 = m_crit * m_crit;
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < n; ++e) {
        int64_t u = up[e];
        double rho_e = rho[e];
        double drho_e = orc_drho(q2[e], m_inf, gamma);
        if (u == e) {
            if (rho_e <= rho_floor) { se[e] = 0.0; su[e] = 0.0; }
            else { se[e] = drho_e; su[e] = 0.0; }
            continue;
        }
        double m2 = orc_mach2(q2[e], m_inf, gamma);
        double m2u = orc_mach2(q2[u], m_inf, gamma);
        double nu_e = orc_switch(m2, mc2, C);
        double nu_u = orc_switch(m2u, mc2, C);
        double nu = nu_e > nu_u ? nu_e : nu_u;
        double rho_u = rho[u];
        double rt = rho_e - nu * (rho_e - rho_u);
        if (rt <= rho_floor) { se[e] = 0.0; su[e] = 0.0; continue; }
        if (nu == 0.0) { se[e] = drho_e; su[e] = 0.0; continue; }
        double drho_u = orc_drho(q2[u], m_inf, gamma);
        double djump = rho_e - rho_u;
        if (nu_e >= nu_u) {
            double dnu_e = m2 > mc2 ? orc_dnu(q2[e], m2, mc2, C, m_inf, gamma) : 0.0;
            se[e] = drho_e * (1.0 - nu) - djump * dnu_e;
            su[e] = nu * drho_u;
        } else {
            double dnu_u = orc_dnu(q2[u], m2u, mc2, C, m_inf, gamma);
            se[e] = drho_e * (1.0 - nu);
            su[e] = nu * drho_u - djump * dnu_u;
        }
    }
}

/* ------------------------------------------------------------------ */
/* kernels/residual.py, kernels/jacobian.py: colour-ordered assembly   */
/* ------------------------------------------------------------------ */

/* assemble_residual_colored, kernels/residual.py:44-76 */
ORC_API void orc_residual(const int64_t* coff, const int64_t* celems, int32_t n_colors,
                          const int32_t* el, const double* B, const double* V,
                          const double* rt, const double* grad, int64_t N, double* R) {
    memset(R, 0, sizeof(double) * (size_t)N);
    for (int c = 0; c < n_colors; ++c) {
#pragma omp parallel for schedule(static)
        for (int64_t k = coff[c]; k < coff[c + 1]; ++k) {
            int64_t e = celems[k];
            double w = rt[e] * V[e];
            double gx = grad[3 * e], gy = grad[3 * e + 1], gz = grad[3 * e + 2];
            for (int i = 0; i < 4; ++i) {
                const double* b = B + 12 * e + 3 * i;
                R[el[4 * e + i]] += w * (gx * b[0] + gy * b[1] + gz * b[2]);
            }
        }
    }
}

/* assemble_matrix_data_colored, kernels/jacobian.py:106-130 */
ORC_API void orc_matrix_data(const int64_t* coff, const int64_t* celems, int32_t n_colors,
                             const int64_t* e2c, const double* B, const double* V,
                             const double* rt, int64_t nnz, double* data) {
    memset(data, 0, sizeof(double) * (size_t)nnz);
    for (int c = 0; c < n_colors; ++c) {
#pragma omp parallel for schedule(static)
        for (int64_t k = coff[c]; k < coff[c + 1]; ++k) {
            int64_t e = celems[k];
            double w = rt[e] * V[e];
            for (int i = 0; i < 4; ++i) {
                const double* bi = B + 12 * e + 3 * i;
                for (int j = 0; j < 4; ++j) {
                    const double* bj = B + 12 * e + 3 * j;
                    data[e2c[16 * e + 4 * i + j]] +=
                        w * (bi[0] * bj[0] + bi[1] * bj[1] + bi[2] * bj[2]);
                }
            }
        }
    }
}

/* assemble_jacobian_data_colored, kernels/jacobian.py:133-181 (Term 2 only
 * when w2 != 0, :171-180) */
ORC_API void orc_jacobian_data(const int64_t* coff, const int64_t* celems, int32_t n_colors,
                               const int64_t* e2c, const double* B, const double* V,
                               const double* rt, const double* grad, const double* se,
                               double inv_u2, int64_t nnz, double* data) {
    memset(data, 0, sizeof(double) * (size_t)nnz);
    for (int c = 0; c < n_colors; ++c) {
#pragma omp parallel for schedule(static)
        for (int64_t k = coff[c]; k < coff[c + 1]; ++k) {
            int64_t e = celems[k];
            double w1 = rt[e] * V[e];
            double g0 = grad[3 * e], g1 = grad[3 * e + 1], g2 = grad[3 * e + 2];
            double w2 = 2.0 * inv_u2 * se[e] * V[e];
            for (int i = 0; i < 4; ++i) {
                const double* bi = B + 12 * e + 3 * i;
                double gi = g0 * bi[0] + g1 * bi[1] + g2 * bi[2];
                for (int j = 0; j < 4; ++j) {
                    const double* bj = B + 12 * e + 3 * j;
                    double val = w1 * (bi[0] * bj[0] + bi[1] * bj[1] + bi[2] * bj[2]);
                    if (w2 != 0.0) val += w2 * gi * (g0 * bj[0] + g1 * bj[1] + g2 * bj[2]);
                    data[e2c[16 * e + 4 * i + j]] += val;
                }
            }
        }
    }
}

/* fill_term3_coo, kernels/jacobian.py:184-229 */
ORC_API void orc_term3_coo(const int64_t* active, int64_t n_active, const int32_t* el,
                           const double* B, const double* V, const double* grad,
                           const int64_t* up, const double* su, double inv_u2, int64_t* rows,
                           int64_t* cols, double* vals) {
#pragma omp parallel for schedule(static)
    for (int64_t a = 0; a < n_active; ++a) {
        int64_t e = active[a], u = up[e];
        double ge0 = grad[3 * e], ge1 = grad[3 * e + 1], ge2 = grad[3 * e + 2];
        double gu0 = grad[3 * u], gu1 = grad[3 * u + 1], gu2 = grad[3 * u + 2];
        double w = 2.0 * inv_u2 * su[e] * V[e];
        for (int i = 0; i < 4; ++i) {
            const double* be = B + 12 * e + 3 * i;
            double gi = ge0 * be[0] + ge1 * be[1] + ge2 * be[2];
            double wi = w * gi;
            for (int k = 0; k < 4; ++k) {
                const double* bu = B + 12 * u + 3 * k;
                int64_t idx = 16 * a + 4 * i + k;
                rows[idx] = el[4 * e + i];
                cols[idx] = el[4 * u + k];
                vals[idx] = wi * (gu0 * bu[0] + gu1 * bu[1] + gu2 * bu[2]);
            }
        }
    }
}

/* CSR SpMV y = A x (the scipy sparsetools product inside spla.cg/gmres,
 * solve/picard.py:375-380, solve/linear.py:182) */
ORC_API void orc_spmv(const int64_t* indptr, const int32_t* indices, const double* data,
                      const double* x, int64_t n, double* y) {
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n; ++r) {
        double s = 0.0;
        for (int64_t k = indptr[r]; k < indptr[r + 1]; ++k) s += data[k] * x[indices[k]];
        y[r] = s;
    }
}

/* Number of OpenMP threads the oracle runs with (for reporting). */
ORC_API int orc_num_threads(void) {
    int n = 1;
#pragma omp parallel
    {
#pragma omp single
        {
#ifdef _OPENMP
            extern int omp_get_num_threads(void);
            n = omp_get_num_threads();
#endif
        }
    }
    return n;
}

/* ------------------------------------------------------------------ */
/* Weighted upwind modes, kernels/upwind.py:128-454                     */
/* ------------------------------------------------------------------ */

/* compute_face_normals, kernels/upwind.py:128-172: outward unit normal of
 * face f (opposite local node f), out (n, 4, 3). */
ORC_API void orc_face_normals(const double* X, const int32_t* el, int64_t n, double* out) {
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < n; ++e)
        for (int f = 0; f < 4; ++f) {
            const double* a = X + 3 * (int64_t)el[4 * e + orc_face_nodes[f][0]];
            const double* b = X + 3 * (int64_t)el[4 * e + orc_face_nodes[f][1]];
            const double* c = X + 3 * (int64_t)el[4 * e + orc_face_nodes[f][2]];
            const double* p = X + 3 * (int64_t)el[4 * e + f];
            double e1x = b[0] - a[0], e1y = b[1] - a[1], e1z = b[2] - a[2];
            double e2x = c[0] - a[0], e2y = c[1] - a[1], e2z = c[2] - a[2];
            double nx = e1y * e2z - e1z * e2y;
            double ny = e1z * e2x - e1x * e2z;
            double nz = e1x * e2y - e1y * e2x;
            double nn = sqrt(nx * nx + ny * ny + nz * nz);
            if (nn > 0.0) { nx /= nn; ny /= nn; nz /= nn; }
            double ox = (a[0] + b[0] + c[0]) / 3.0 - p[0];
            double oy = (a[1] + b[1] + c[1]) / 3.0 - p[1];
            double oz = (a[2] + b[2] + c[2]) / 3.0 - p[2];
            if (nx * ox + ny * oy + nz * oz < 0.0) { nx = -nx; ny = -ny; nz = -nz; }
            out[12 * e + 3 * f] = nx;
            out[12 * e + 3 * f + 1] = ny;
            out[12 * e + 3 * f + 2] = nz;
        }
}

/* build_upstream_neighborhoods, kernels/upwind.py:313-341: the elements
 * within `depth` face hops of e, e excluded, ascending.  With idx == NULL
 * fills off (n + 1) and returns the total; else fills idx from off. */
ORC_API int64_t orc_neighborhoods(const int32_t* fn, int64_t n, int depth, int64_t* off, int32_t* idx) {
    int64_t total = 0;
    if (!idx) off[0] = 0;
    int64_t cap = 16;
    int64_t* seen = (int64_t*)malloc(sizeof(int64_t) * cap);
    int64_t* frontier = (int64_t*)malloc(sizeof(int64_t) * cap);
    int64_t* next = (int64_t*)malloc(sizeof(int64_t) * cap);
    for (int64_t e = 0; e < n; ++e) {
        int64_t ns = 0, nf = 0;
        seen[ns++] = e;
        frontier[nf++] = e;
        for (int d = 0; d < depth; ++d) {
            int64_t nn = 0;
            for (int64_t i = 0; i < nf; ++i)
                for (int f = 0; f < 4; ++f) {
                    int64_t nb = fn[4 * frontier[i] + f];
                    if (nb < 0) continue;
                    int found = 0;
                    for (int64_t j = 0; j < ns && !found; ++j) found = seen[j] == nb;
                    if (found) continue;
                    if (ns + 1 > cap || nn + 1 > cap) {
                        cap *= 2;
                        seen = (int64_t*)realloc(seen, sizeof(int64_t) * cap);
                        frontier = (int64_t*)realloc(frontier, sizeof(int64_t) * cap);
                        next = (int64_t*)realloc(next, sizeof(int64_t) * cap);
                    }
                    seen[ns++] = nb;
                    next[nn++] = nb;
                }
            int64_t* t = frontier;
            frontier = next;
            next = t;
            nf = nn;
        }
        qsort(seen, (size_t)ns, sizeof(int64_t), cmp_i64);
        if (idx) {
            int64_t w = off[e];
            for (int64_t j = 0; j < ns; ++j)
                if (seen[j] != e) idx[w++] = (int32_t)seen[j];
        } else {
            total += ns - 1;
            off[e + 1] = total;
        }
    }
    free(seen);
    free(frontier);
    free(next);
    return idx ? off[n] : total;
}

/* rho_tilde_kernel_sweep, kernels/upwind.py:345-454 */
ORC_API void orc_rho_tilde_kernel(const double* q2, const double* rho, const double* grad, const double* X,
                                  const int32_t* el, const double* cen, const int64_t* nb_off,
                                  const int32_t* nb_idx, int64_t n, double m_inf, double m_crit, double C,
                                  double gamma, double rho_floor, double reach_frac, double sig_s,
                                  double sig_p, double* nu_out, double* rt_out) {
    double mc2 = m_crit * m_crit;
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < n; ++e) {
        double gx = grad[3 * e], gy = grad[3 * e + 1], gz = grad[3 * e + 2];
        double gmag = sqrt(gx * gx + gy * gy + gz * gz);
        double nu_e = orc_switch(orc_mach2(q2[e], m_inf, gamma), mc2, C);
        if (gmag <= 0.0) { nu_out[e] = nu_e; rt_out[e] = rho[e]; continue; }
        double vx = gx / gmag, vy = gy / gmag, vz = gz / gmag;
        double pmin = 1e300, pmax = -1e300;
        for (int k = 0; k < 4; ++k) {
            const double* x = X + 3 * (int64_t)el[4 * e + k];
            double pr = x[0] * vx + x[1] * vy + x[2] * vz;
            if (pr < pmin) pmin = pr;
            if (pr > pmax) pmax = pr;
        }
        double extent = pmax - pmin;
        double target = reach_frac * extent;
        double ss = sig_s * extent, sp = sig_p * extent;
        double inv2ss = 1.0 / (2.0 * (ss * ss) + 1e-300);
        double inv2sp = 1.0 / (2.0 * (sp * sp) + 1e-300);
        double w_sum = 0.0, rho_acc = 0.0, m2_acc = 0.0;
        for (int64_t j = nb_off[e]; j < nb_off[e + 1]; ++j) {
            int64_t c = nb_idx[j];
            double dx = cen[3 * c] - cen[3 * e], dy = cen[3 * c + 1] - cen[3 * e + 1],
                   dz = cen[3 * c + 2] - cen[3 * e + 2];
            double up = -(vx * dx + vy * dy + vz * dz);
            if (up <= 0.0) continue;
            double d2 = dx * dx + dy * dy + dz * dz;
            double perp2 = d2 - up * up;
            if (perp2 < 0.0) perp2 = 0.0;
            double w = exp(-((up - target) * (up - target) * inv2ss + perp2 * inv2sp));
            w_sum += w;
            rho_acc += w * rho[c];
            m2_acc += w * orc_mach2(q2[c], m_inf, gamma);
        }
        if (w_sum <= 0.0) { nu_out[e] = nu_e; rt_out[e] = rho[e]; continue; }
        double rho_up = rho_acc / w_sum, m2_up = m2_acc / w_sum;
        double nu_u = orc_switch(m2_up, mc2, C);
        double nu = nu_e > nu_u ? nu_e : nu_u;
        nu_out[e] = nu;
        if (nu <= 0.0) { rt_out[e] = rho[e]; continue; }
        double rt = rho[e] - nu * (rho[e] - rho_up);
        rt_out[e] = rt > rho_floor ? rt : rho_floor;
    }
}

/* rho_tilde_weighted_sweep ("blend"), kernels/upwind.py:176-309 */
ORC_API void orc_rho_tilde_blend(const double* q2, const double* rho, const double* grad, const double* X,
                                 const int32_t* el, const double* cen, const int32_t* fn, int64_t n,
                                 double m_inf, double m_crit, double C, double gamma, double rho_floor,
                                 double p_weight, double reach_frac, double gain_max, double* nu_out,
                                 double* rt_out) {
    double mc2 = m_crit * m_crit;
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < n; ++e) {
        double gx = grad[3 * e], gy = grad[3 * e + 1], gz = grad[3 * e + 2];
        double gmag = sqrt(gx * gx + gy * gy + gz * gz);
        double nu_e = orc_switch(orc_mach2(q2[e], m_inf, gamma), mc2, C);
        if (gmag <= 0.0) { nu_out[e] = nu_e; rt_out[e] = rho[e]; continue; }
        double vx = gx / gmag, vy = gy / gmag, vz = gz / gmag;
        double w_sum = 0.0, rho_acc = 0.0, m2_acc = 0.0, reach_acc = 0.0;
        for (int f = 0; f < 4; ++f) {
            int64_t nb = fn[4 * e + f];
            if (nb < 0) continue;
            double dx = cen[3 * nb] - cen[3 * e], dy = cen[3 * nb + 1] - cen[3 * e + 1],
                   dz = cen[3 * nb + 2] - cen[3 * e + 2];
            double dlen = sqrt(dx * dx + dy * dy + dz * dz);
            if (dlen <= 0.0) continue;
            double up = -(vx * dx + vy * dy + vz * dz);
            double a = up / dlen;
            if (a <= 0.0) continue;
            double w = pow(a, p_weight);
            w_sum += w;
            rho_acc += w * rho[nb];
            m2_acc += w * orc_mach2(q2[nb], m_inf, gamma);
            reach_acc += w * up;
        }
        if (w_sum <= 0.0) { nu_out[e] = nu_e; rt_out[e] = rho[e]; continue; }
        double rho_up = rho_acc / w_sum, m2_up = m2_acc / w_sum, reach = reach_acc / w_sum;
        double nu_u = orc_switch(m2_up, mc2, C);
        double nu = nu_e > nu_u ? nu_e : nu_u;
        nu_out[e] = nu;
        if (nu <= 0.0) { rt_out[e] = rho[e]; continue; }
        double pmin = 1e300, pmax = -1e300;
        for (int k = 0; k < 4; ++k) {
            const double* x = X + 3 * (int64_t)el[4 * e + k];
            double pr = x[0] * vx + x[1] * vy + x[2] * vz;
            if (pr < pmin) pmin = pr;
            if (pr > pmax) pmax = pr;
        }
        double reach_target = reach_frac * (pmax - pmin);
        double g = reach_target / (reach > 1e-30 ? reach : 1e-30);
        if (g < 1.0) g = 1.0;
        else if (g > gain_max) g = gain_max;
        double rt = rho[e] - nu * g * (rho[e] - rho_up);
        rt_out[e] = rt > rho_floor ? rt : rho_floor;
    }
}
