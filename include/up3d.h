/*
 * up3d.h -- C ABI of the B200 (sm_100a) element-loop hot path of the pyfp3d
 * full-potential solver.
 *
 * Conventions
 *   - Every array argument of a per-step call is a DEVICE pointer on the
 *     mesh's device; `stream` is a cudaStream_t (NULL = legacy default).
 *   - Calls are asynchronous on `stream` unless they return a host value
 *     (documented per call), in which case they synchronise that stream.
 *   - Every call returns an up3d status; up3d_last_error() gives the message
 *     of the last failure on the calling thread.
 *   - A mesh handle is not thread-safe: one host thread (and one stream at a
 *     time) per handle, like the reference's per-mesh workspaces.
 *   - Element connectivity is int32 (n_tets, 4); node coordinates are f64
 *     (n_nodes, 3); CSR indices are int32.
 *
 * Each declaration names the reference interface it replaces
 * (file:line in swayli94/UP3D).
 */
#ifndef UP3D_H
#define UP3D_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct up3d_mesh up3d_mesh; /* opaque per-mesh device state */
typedef void* up3d_stream;          /* cudaStream_t */

/* Status codes; the Python layer maps them to the reference's exceptions. */
enum up3d_status {
    UP3D_OK = 0,
    UP3D_ERR_VALUE = -1,           /* ValueError: degenerate tet, > 256 colours, bad shapes */
    UP3D_ERR_RUNTIME = -2,         /* RuntimeError: CUDA failure, Krylov non-convergence */
    UP3D_ERR_NOT_IMPLEMENTED = -3, /* NotImplementedError */
    UP3D_ERR_ARGUMENT = -4         /* null pointer, wrong size, misuse */
};

/* Flow / upwind parameters shared by the per-step calls.  Defaults of the
 * reference drivers: gamma 1.4, u_inf 1, m_cap 3, m_crit 0.95, C 1.5,
 * rho_floor 0.05 (pyfp3d/solve/newton.py:525-528, physics/isentropic.py:21-26). */
typedef struct {
    double m_inf;
    double gamma;
    double u_inf;
    double m_cap;
    double m_crit;
    double upwind_c;
    double rho_floor;
} up3d_flow;

/* Monitors of one residual evaluation (device-resident struct written by the
 * calls that take it; the reference keeps them as UpwindOperator attributes,
 * pyfp3d/kernels/upwind.py:816-818, and eval_residual locals,
 * pyfp3d/solve/newton.py:349-371). */
typedef struct {
    double nu_max;
    int64_t n_supersonic;
    int64_t n_floored;
    int64_t n_limited;
    int64_t n_term3_active;
    int64_t n_term3_extra; /* Term-3 entries outside the P1 pattern */
} up3d_monitors;

typedef struct {
    int64_t n_nodes;
    int64_t n_tets;
    int64_t nnz;             /* P1 pattern */
    int32_t max_row_len;
    int32_t max_node_degree; /* incident elements per node */
    int32_t n_colors;        /* -1 until up3d_mesh_coloring ran */
    int32_t device;
} up3d_mesh_info;

const char* up3d_last_error(void);
int up3d_version(void);

/* ---------------------------------------------------------------- setup */

/* PicardOperator.__init__ (pyfp3d/kernels/jacobian.py:246-262) and
 * UpwindOperator.__init__ (pyfp3d/kernels/upwind.py:744-781): element
 * geometry B_e, V_e (mesh/metrics.py:177-204), face adjacency
 * (mesh/metrics.py:208-278), centroids (kernels/upwind.py:750), the P1 CSR
 * pattern (kernels/jacobian.py:60-75) and the row-gather maps.  `nodes` and
 * `elements` are HOST arrays.  UP3D_ERR_VALUE on a degenerate tet
 * (mesh/metrics.py:155-164) or an out-of-range node index. */
int up3d_mesh_create(const double* nodes, const int32_t* elements, int64_t n_nodes,
                     int64_t n_tets, int device, up3d_stream stream, up3d_mesh** out);
int up3d_mesh_destroy(up3d_mesh* mesh);
int up3d_mesh_get_info(const up3d_mesh* mesh, up3d_mesh_info* info);

/* PicardOperator._pattern.indptr / .indices (device views, valid for the
 * mesh's lifetime). */
int up3d_mesh_pattern(const up3d_mesh* mesh, const int32_t** indptr, const int32_t** indices);

/* PicardOperator.B (n_tets,4,3), .V (n_tets) into caller device buffers. */
int up3d_mesh_geometry(const up3d_mesh* mesh, double* B, double* V, up3d_stream stream);

/* UpwindOperator.centroids (n_tets,3) into a caller device buffer. */
int up3d_mesh_centroids(const up3d_mesh* mesh, double* centroids, up3d_stream stream);

/* UpwindOperator.face_neighbors (n_tets,4) int32: read, and overwrite (the
 * per-side masking of pyfp3d/wake/multivalued.py:463-467). */
int up3d_mesh_face_neighbors(const up3d_mesh* mesh, int32_t* out, up3d_stream stream);
int up3d_mesh_set_face_neighbors(up3d_mesh* mesh, const int32_t* in, up3d_stream stream);

/* color_partition_csr (pyfp3d/mesh/coloring.py:129-145): greedy colouring
 * identical to the reference's (same visit order, smallest free colour).
 * HOST outputs: color_offsets (n_colors+1), color_elems (n_tets); pass NULL
 * for both to only compute and cache n_colors.  UP3D_ERR_VALUE past 256
 * colours.  Synchronous. */
int up3d_mesh_coloring(up3d_mesh* mesh, int64_t* color_offsets, int64_t* color_elems,
                       int32_t* n_colors);

/* PicardOperator.elem_to_csr (kernels/jacobian.py:78-103), int64
 * (n_tets,4,4) device buffer. */
int up3d_mesh_elem_to_csr(const up3d_mesh* mesh, int64_t* out, up3d_stream stream);

/* ------------------------------------------------------ element sweeps */

/* PicardOperator.velocities -> element_velocity_q2
 * (kernels/jacobian.py:264-270, kernels/gradient.py:33-64). */
int up3d_velocities(const up3d_mesh* mesh, const double* phi, double* grad, double* q2,
                    up3d_stream stream);

/* element_velocity_q2 on raw arrays (kernels/gradient.py:33-64): elements
 * int32 (n_tets,4), B (n_tets,4,3), all device pointers. */
int up3d_element_velocity_q2(const int32_t* elements, const double* B, const double* phi, int64_t n_tets,
                             double* grad, double* q2, up3d_stream stream);

/* limit_q2_field (physics/isentropic.py:293-314); if n_limited is non-NULL
 * it receives (device int64) the count of elements with out != q2. */
int up3d_limit_q2(const double* q2, int64_t n, double m_inf, double m_cap, double gamma,
                  double* out, int64_t* n_limited, up3d_stream stream);
/* density_field (physics/isentropic.py:236-258). */
int up3d_density(const double* q2, int64_t n, double m_inf, double gamma, double* out,
                 up3d_stream stream);
/* mach_squared_field (physics/isentropic.py:318-334). */
int up3d_mach_squared(const double* q2, int64_t n, double m_inf, double gamma, double* out,
                      up3d_stream stream);
/* density_derivative_wrt_q_sq_field (physics/isentropic.py:338-354). */
int up3d_density_derivative(const double* q2, int64_t n, double m_inf, double gamma,
                            double* out, up3d_stream stream);
/* mach_squared_derivative_wrt_q_sq_field (physics/isentropic.py:358-374). */
int up3d_mach_squared_derivative(const double* q2, int64_t n, double m_inf, double gamma,
                                 double* out, up3d_stream stream);
/* pressure_coefficient, elementwise (physics/isentropic.py:122-143). */
int up3d_pressure_coefficient(const double* q2, int64_t n, double m_inf, double gamma,
                              double* out, up3d_stream stream);

/* upstream_elements (kernels/upwind.py:69-125), max_hops 4.  `grad` is
 * (n_tets,3); `upstream` is int64 (n_tets). */
int up3d_upwind_walk(const up3d_mesh* mesh, const double* grad, int64_t* upstream,
                     up3d_stream stream);

/* rho_tilde_sweep + monitors (kernels/upwind.py:457-500, :816-818).
 * `monitors` (device) may be NULL. */
int up3d_rho_tilde(const double* q2, const double* rho, const int64_t* upstream, int64_t n,
                   const up3d_flow* flow, double* nu, double* rho_tilde,
                   up3d_monitors* monitors, up3d_stream stream);
/* classify_upwind_branches (kernels/upwind.py:504-541); branch int8. */
int up3d_classify_branches(const double* q2, const double* rho, const int64_t* upstream,
                           int64_t n, const up3d_flow* flow, int8_t* branch,
                           up3d_stream stream);
/* rho_tilde_frozen_sweep + monitors (kernels/upwind.py:545-593, :861-863). */
int up3d_rho_tilde_frozen(const double* q2, const double* rho, const int64_t* upstream,
                          const int8_t* branch, int64_t n, const up3d_flow* flow, double* nu,
                          double* rho_tilde, up3d_monitors* monitors, up3d_stream stream);
/* rho_tilde_sensitivities_sweep (kernels/upwind.py:647-730). */
int up3d_rho_tilde_sens(const double* q2, const double* rho, const int64_t* upstream,
                        int64_t n, const up3d_flow* flow, double* s_e, double* s_u,
                        up3d_stream stream);
/* rho_tilde_frozen_sensitivities_sweep (kernels/upwind.py:597-643). */
int up3d_rho_tilde_frozen_sens(const double* q2, const double* rho, const int64_t* upstream,
                               const int8_t* branch, int64_t n, const up3d_flow* flow,
                               double* s_e, double* s_u, up3d_stream stream);

/* ------------------------------------------------------------ assembly */

/* PicardOperator.assemble_residual (kernels/jacobian.py:361-375 ->
 * kernels/residual.py:44-76).  rho_tilde NULL means rho == 1.  Like the
 * reference, the call also leaves grad(phi) (n_tets,3) and q^2 in the
 * velocity workspace: `grad_out` / `q2_out` when given, else a
 * library-internal buffer. */
int up3d_residual(up3d_mesh* mesh, const double* phi, const double* rho_tilde, double* R,
                  double* grad_out, double* q2_out, up3d_stream stream);

/* PicardOperator.assemble_matrix (kernels/jacobian.py:272-286 ->
 * :106-130): CSR data on the P1 pattern.  rho_tilde NULL means rho == 1. */
int up3d_picard_matrix(up3d_mesh* mesh, const double* rho_tilde, double* data,
                       up3d_stream stream);

/* PicardOperator.assemble_newton_jacobian (kernels/jacobian.py:288-359):
 * Terms 1+2 (+ the in-pattern part of Term 3) into `data` on the P1
 * pattern; Term-3 entries outside the pattern are kept in the mesh
 * workspace for up3d_jacobian_export.  lim_mask (uint8, NULL = none) gates
 * s_e by lim[e] and s_u by lim[upstream[e]].  Inputs are not modified.
 * Host outputs (synchronous): n_term3_active, n_extra, newton_nnz (nnz of
 * the merged matrix, exact zeros dropped when Term 3 is active, as scipy's
 * CSR addition does). */
int up3d_jacobian(up3d_mesh* mesh, const double* phi, const double* rho_tilde,
                  const double* s_e, const double* s_u, const int64_t* upstream, double u_inf,
                  const uint8_t* lim_mask, double* data, int64_t* n_term3_active,
                  int64_t* n_extra, int64_t* newton_nnz, up3d_stream stream);

/* The same two calls under data-only names: up3d_picard_matrix_data is
 * up3d_picard_matrix, up3d_jacobian_data is up3d_jacobian (the data array
 * on the P1 pattern, the new nnz / pattern through up3d_jacobian_export). */
int up3d_picard_matrix_data(up3d_mesh* mesh, const double* rho_tilde, double* data,
                            up3d_stream stream);
int up3d_jacobian_data(up3d_mesh* mesh, const double* phi, const double* rho_tilde,
                       const double* s_e, const double* s_u, const int64_t* upstream, double u_inf,
                       const uint8_t* lim_mask, double* data, int64_t* n_term3_active,
                       int64_t* n_extra, int64_t* newton_nnz, up3d_stream stream);

/* The merged CSR (P1 pattern data + Term-3 extras) of the last up3d_jacobian
 * or up3d_residual_jacobian call into caller device buffers of sizes
 * n_nodes+1 and newton_nnz. */
int up3d_jacobian_export(up3d_mesh* mesh, const double* data, int32_t* indptr,
                         int32_t* indices, double* merged, up3d_stream stream);

/* newton_nnz of the last Jacobian (kernels/jacobian.py:358): the P1 nnz, or,
 * when Term 3 is active, the non-zeros of the merged matrix.  Synchronous. */
int up3d_jacobian_nnz(up3d_mesh* mesh, const double* data, int64_t* newton_nnz,
                      up3d_stream stream);

/* Fused eval_residual + assemble_coupled without a wake
 * (pyfp3d/solve/newton.py:345-372 and :435-452 with T = I): velocities,
 * limiter, density, walk, live flux (or the frozen flux when `upstream_frozen`
 * and `branch_frozen` are non-NULL), sensitivities, residual R (n_nodes) and
 * the Newton Jacobian data on the P1 pattern (NULL skips the Jacobian).
 * Monitors (device, may be NULL).  rho_tilde_out / upstream_out (device,
 * may be NULL) receive the flux and the walk.  Term 3 (kernels/jacobian.py:
 * 184-229, :344-358): the merge is built symbolically (one warp per row)
 * while the set of active elements or their upstream elements change; once
 * the same pattern comes twice in a row its per-destination contributor
 * lists are recorded, and while it repeats (the frozen finish, late Newton
 * steps) Term 3 is a values-only sum per destination in the same order --
 * the same bits. */
int up3d_residual_jacobian(up3d_mesh* mesh, const double* phi, const up3d_flow* flow,
                           const int64_t* upstream_frozen, const int8_t* branch_frozen,
                           double* R, double* data, double* rho_tilde_out,
                           int32_t* upstream_out, up3d_monitors* monitors,
                           up3d_stream stream);
/* Term-3 builds served by the values-only path on this mesh so far (no
 * reference counterpart). */
int up3d_mesh_term3_cache_hits(const up3d_mesh* mesh, int64_t* hits);

/* ------------------------------------------------------ adjoint */

/* Vector-Jacobian product of the residual (the discrete adjoint's
 * right-hand sides; no reference counterpart -- the reference has no
 * adjoint): for L = lam^T R(phi, X, M_inf) + sum_e w_q2[e] q2_e(phi, X),
 * with the upstream elements and, when branch != NULL, the frozen branches
 * held fixed (the Newton Jacobian's linearisation), writes dL/dX (device,
 * N x 3, may be NULL), dL/dM_inf (device scalar, may be NULL) and
 * sum_e w_q2[e] dq2_e/dphi (device, N, may be NULL; needs w_q2).  q2_e =
 * |grad phi_e|^2 / u_inf^2.  lam (N) and w_q2 (E) are device arrays and
 * either may be NULL (zero).  The lam^T dR/dphi part is J^T lam: see
 * up3d_jacobian_transpose.  Deterministic. */
int up3d_residual_vjp(up3d_mesh* mesh, const double* phi, const up3d_flow* flow,
                      const int64_t* upstream, const int8_t* branch, const double* lam,
                      const double* w_q2, double* dphi, double* dX, double* dM,
                      up3d_stream stream);

/* Values of J^T on the (symmetric) P1 pattern: data_t[z] = data[slot of
 * the transposed entry of z] (device arrays of nnz). */
int up3d_jacobian_transpose(up3d_mesh* mesh, const double* data, double* data_t,
                            up3d_stream stream);

/* ------------------------------------------------------ weighted upwind */

/* compute_face_normals (kernels/upwind.py:128-172): outward unit normal of
 * face f (opposite local node f) into out (n_tets, 4, 3), device. */
int up3d_face_normals(const up3d_mesh* mesh, double* out, up3d_stream stream);

/* build_upstream_neighborhoods (kernels/upwind.py:313-341): the elements
 * within `depth` face hops of each element, itself excluded, ascending;
 * built once per depth and kept on the mesh (rebuilt after
 * up3d_mesh_set_face_neighbors).  Device views of the CSR (offsets int64
 * n_tets + 1, indices int32) and the total; any output may be NULL.
 * Depths up to 4 (at most 160 elements) are built on the device, deeper
 * ones on the host (OpenMP breadth-first search) and uploaded.
 * UP3D_ERR_VALUE for depth < 1.  Synchronises the stream when it builds. */
int up3d_mesh_neighborhoods(up3d_mesh* mesh, int depth, const int64_t** offsets,
                            const int32_t** indices, int64_t* total, up3d_stream stream);

/* The same from a face-neighbour table alone (device int32 (n, 4), -1 =
 * boundary), into caller buffers: with indices == NULL fills offsets
 * (n + 1, device int64) and *total (host; synchronises the stream); then,
 * with indices (device int32, *total), fills them. */
int up3d_face_neighborhoods(const int32_t* face_neighbors, int64_t n, int depth, int64_t* offsets,
                            int32_t* indices, int64_t* total, up3d_stream stream);

/* rho_tilde_kernel_sweep (kernels/upwind.py:345-454), the "kernel" mode of
 * UpwindOperator(weighted=True) (:744-819): rho_up and M^2_up as Gaussian
 * averages over the depth-hop neighbourhood centred one streamwise reach
 * upstream.  grad (n_tets, 3), q2, rho, nu, rho_tilde (n_tets) device;
 * monitors (device, may be NULL) get nu_max / n_supersonic / n_floored. */
int up3d_rho_tilde_kernel(up3d_mesh* mesh, const double* grad, const double* q2, const double* rho,
                          const up3d_flow* flow, int depth, double reach_frac,
                          double sigma_s_frac, double sigma_p_frac, double* nu,
                          double* rho_tilde, up3d_monitors* monitors, up3d_stream stream);

/* rho_tilde_weighted_sweep (kernels/upwind.py:176-309), the "blend" mode:
 * an upstream-weighted blend over the face neighbours with reach
 * compensation.  Arrays as up3d_rho_tilde_kernel. */
int up3d_rho_tilde_blend(const up3d_mesh* mesh, const double* grad, const double* q2,
                         const double* rho, const up3d_flow* flow, double p_weight,
                         double reach_frac, double reach_gain_max, double* nu,
                         double* rho_tilde, up3d_monitors* monitors, up3d_stream stream);

/* ------------------------------------------------------ wake constraint */

typedef struct up3d_wake up3d_wake; /* opaque: fold map, reduction plans */

/* WakeConstraint.__init__ / reduce_operator (constraints/wake.py:32-97):
 * the "+"-side copies of the wake-sheet nodes (slaves, ids in [n_red,
 * n_cut)) fold onto their originals (masters, ids in [0, n_red)); for a
 * cut-mesh operator A with the CSR pattern (a_indptr int64 n_cut + 1,
 * a_indices int32) the plans of A_red = T^T A T and of the Gamma columns
 * H = T^T A G (G[slave_k, station_k] = 1, n_red x n_stations) are built on
 * the host and kept on `device`.  All inputs are HOST arrays.
 * UP3D_ERR_VALUE when n_cut != n_red + n_dup (the reference's ValueError)
 * or an index is out of range.  One handle serves every A of this pattern. */
int up3d_wake_create(int64_t n_cut, int64_t n_red, int64_t n_dup, const int64_t* masters,
                     const int64_t* slaves, const int64_t* node_station, int32_t n_stations,
                     const int64_t* a_indptr, const int32_t* a_indices, int device,
                     up3d_wake** out);
int up3d_wake_destroy(up3d_wake* wake);
int up3d_wake_info(const up3d_wake* wake, int64_t* n_red, int64_t* nnz_red, int64_t* nnz_h,
                   int32_t* n_stations);
/* Device views of the A_red pattern (n_red + 1, nnz_red; columns ascending)
 * and of H's (n_red + 1, nnz_h; columns = stations ascending). */
int up3d_wake_patterns(const up3d_wake* wake, const int32_t** red_indptr,
                       const int32_t** red_indices, const int32_t** h_indptr,
                       const int32_t** h_indices);
/* Values of A_red and H (h_data may be NULL) from A's values (device, the
 * pattern given at creation).  Each reduced entry sums, for every cut row
 * folding onto its row (the row itself, then its slaves ascending), that
 * row's entries folding onto its column, in stored order: the grouping of
 * the reference's T^T (A T). */
int up3d_wake_reduce(const up3d_wake* wake, const double* a_data, double* red_data,
                     double* h_data, up3d_stream stream);
/* reduced_rhs (constraints/wake.py:99-102): out = T^T b - sum_j gamma_j h_j
 * with h_j H's station-j column (h_data from up3d_wake_reduce); b (n_cut),
 * gamma (n_stations), out (n_red), all device. */
int up3d_wake_reduced_rhs(const up3d_wake* wake, const double* b, const double* gamma,
                          const double* h_data, double* out, up3d_stream stream);
/* expand (constraints/wake.py:104-112): phi_cut (n_cut) = phi_red on the
 * original nodes, phi_red[master] + gamma[station] on each slave. */
int up3d_wake_expand(const up3d_wake* wake, const double* phi_red, const double* gamma,
                     double* phi_cut, up3d_stream stream);

/* ------------------------------------------------------ wall post-processing */

typedef struct up3d_wall up3d_wall; /* opaque: wall triangles, owners, adjacency */

/* The wall triangles of `mesh` (wall_faces HOST int64 (n_w, 3), stored
 * winding; elements HOST int32 (n_tets, 4), the mesh's connectivity): each
 * triangle's owning tet (wall_outward_normals, post/surface.py:192-231;
 * UP3D_ERR_VALUE unless exactly one tet owns it) and its edge neighbours
 * (wall_triangle_adjacency, :121-144) are found here, on the host. */
int up3d_wall_create(const up3d_mesh* mesh, const int32_t* elements, const int64_t* wall_faces,
                     int64_t n_w, up3d_wall** out);
int up3d_wall_destroy(up3d_wall* wall);

/* wall_force_coefficients (post/surface.py:309-363): per triangle the
 * in-plane P1 gradient of phi (triangle_tangential_gradients, :80-118),
 * smooth_passes of the normal-gated edge-neighbour smoothing (:147-189,
 * cos threshold 0.2), Cp by the exact isentropic law at m_inf > 0 or
 * Bernoulli at m_inf = 0 (physics/isentropic.py:122-160), and
 * cf = -sum Cp A n_out / s_ref into the HOST array cf (3).  phi is the
 * device potential of the mesh; grad_out (n_w, 3, after smoothing),
 * area_out (n_w), normal_out (n_w, 3, the stored winding's unit normal),
 * outward_out (n_w, 3) and cp_out (n_w) are device arrays, each may be
 * NULL.  Synchronises the stream. */
int up3d_wall_forces(up3d_wall* wall, const up3d_mesh* mesh, const double* phi, double u_inf,
                     double m_inf, double gamma, double s_ref, int smooth_passes, double* grad_out,
                     double* area_out, double* normal_out, double* outward_out, double* cp_out,
                     double* cf, up3d_stream stream);

/* ------------------------------------------------------ level-set sides */

/* newton_terms23_side_coo (kernels/cut_assembly.py:401-488): one side's
 * Newton Terms 2 and 3 as COO triplets on extended DOFs.  keep (uint8 E),
 * dofvec / readvec (int64 E x 4: where the element's residual lands / which
 * DOFs its side field reads; readvec NULL = dofvec), grad / grad_row
 * (E x 3: the read and the scatter field's gradients; grad_row NULL =
 * grad), lim_mask (f64 E, 1 or 0), s_e, s_u (f64 E), upstream (int64 E),
 * all device.  Term-2 blocks of the kept elements with s_e lim != 0, in
 * ascending element order, then Term-3 blocks of those with
 * s_u lim[upstream] != 0, 16 triplets per block (a-major).  With rows ==
 * NULL only *count (host) is set; then rows, cols (int64) and data (f64)
 * of `capacity` >= *count entries are filled.  UP3D_ERR_VALUE for an
 * upstream index outside [0, E).  Synchronises the stream. */
int up3d_terms23_side_coo(const up3d_mesh* mesh, const uint8_t* keep, const int64_t* dofvec,
                          const int64_t* readvec, const double* grad, const double* grad_row,
                          const double* lim_mask, const double* s_e, const double* s_u,
                          const int64_t* upstream, double u_inf, int64_t* rows, int64_t* cols,
                          double* data, int64_t capacity, int64_t* count, up3d_stream stream);

/* ------------------------------------------------------ batched cases */

/* up3d_residual_jacobian for several cases in one mesh (their meshes
 * concatenated as disconnected components, no reference counterpart: the
 * reference solves one case at a time): element e takes the flow of its
 * case, flows[case_of[e]] (host array of n_cases; one u_inf for all),
 * case_of a device int32 array of n_tets.  One launch of each pass covers
 * every case.  With frozen arrays, an element whose branch is negative
 * stays live (cases freeze one by one).  branch_out (device int8, may be
 * NULL) receives each element's branch: the frozen one, or the one a live
 * element took (classify_upwind_branches, kernels/upwind.py:504-541).
 * UP3D_ERR_VALUE for a case index outside [0, n_cases).
 * flows == NULL reuses the flow table of the last call with flows on this
 * mesh (same n_cases, else UP3D_ERR_VALUE) without validating case_of
 * again: no host synchronisation, so a residual-only call (data == NULL)
 * can be captured in a CUDA graph.  An index outside [0, n_cases) then
 * reads case 0. */
int up3d_residual_jacobian_batched(up3d_mesh* mesh, const double* phi, int n_cases,
                                   const up3d_flow* flows, const int32_t* case_of,
                                   const int64_t* upstream_frozen, const int8_t* branch_frozen,
                                   double* R, double* data, double* rho_tilde_out,
                                   int32_t* upstream_out, int8_t* branch_out,
                                   up3d_monitors* monitors, up3d_stream stream);

/* ------------------------------------------------------ launch shapes */

/* Launch shapes of the fused evaluation's two passes (no reference
 * counterpart: numba picks its own).  Every shape computes the same bits:
 * the element sweep's per-element arithmetic does not depend on the grid,
 * and the row gather sums every row in a fixed order whatever its lanes
 * per row.
 *   elem_persistent  0: one thread per element (grid capped at 64 blocks
 *                    per SM); 1: one resident wave of blocks looping over
 *                    256-element tiles
 *   elem_threads_per_sm  register budget of the Newton-Jacobian sweep as
 *                    the resident threads per SM it allows: 512 (256-thread
 *                    blocks, up to 128 registers, no spills), 640 (128-thread
 *                    blocks, up to 102) or 768 (256-thread blocks, up to 80,
 *                    spilling to L1)
 *   row_lanes        lanes per row of the row gather: 4, 8, 16 or 32
 *   row_plan8        1: the row gather reads each upper slot's
 *                    contributors from a fixed-width record (built at mesh
 *                    set-up when no slot has more than 8); 0: from the
 *                    offset list.  Ignored when the mesh has no records.
 *   assembly         1: single-pass tiled assembly -- one CTA per tile of
 *                    spatially compact elements evaluates the tile's
 *                    elements with their state in shared memory and sums
 *                    the residual and Jacobian outputs there (outputs that
 *                    straddle tiles through a partial-sum buffer and a
 *                    short combine pass); 0: the two-pass form above (an
 *                    element sweep writing per-element local matrices to
 *                    HBM and a row gather reading them back).  The two
 *                    forms sum each output in a different fixed order, so
 *                    they agree to rounding, not bit for bit; each is
 *                    bit-reproducible.
 *   tile_elems       elements per tile of the tiled form: 128 or 256 (the
 *                    plan is rebuilt when it changes; the summation order
 *                    depends on it)
 *   tile_stretch     1, 2 or 4: the tiles' bisection counts extents along
 *                    x divided by this factor, so tiles come out that many
 *                    times longer along x -- the freestream direction of
 *                    the channel cases, along which the upwind walk runs
 *                    (fewer walks leave their tile); the summation order
 *                    depends on it
 *   elem_us, row_us  autotune output: median time per launch of the
 *                    chosen shapes (0 when set by hand) */
typedef struct {
    int32_t elem_persistent;
    int32_t elem_threads_per_sm;
    int32_t row_lanes;
    int32_t row_plan8;
    int32_t assembly;
    int32_t tile_elems;
    int32_t tile_stretch;
    int32_t reserved;
    double elem_us;
    double row_us;
} up3d_tuning;

/* Default: {0, 512, 8, 0, 0, 256, 1} (the two-pass form, measured faster on
 * the benchmark meshes; the autotuner times both).  UP3D_ERR_VALUE for a
 * shape outside the lists. */
int up3d_mesh_set_tuning(up3d_mesh* mesh, const up3d_tuning* tuning);
int up3d_mesh_get_tuning(const up3d_mesh* mesh, up3d_tuning* tuning);

/* The tile plan of the tiled assembly (built on first use, or here, for
 * `tile_elems` elements per tile; no reference counterpart -- the
 * reference scatters element contributions colour by colour,
 * kernels/jacobian.py:106-181).  Builds the plan when it is missing or of
 * another tile size; synchronises the stream. */
typedef struct {
    int32_t tile_elems;
    int32_t tile_stretch;       /* tiles this many times longer along x than across */
    int32_t max_nodes;          /* most distinct nodes of one tile */
    int32_t max_edges;          /* most distinct element edges of one tile */
    int64_t n_tiles;
    int64_t n_tile_nodes;       /* sum over tiles of their distinct nodes */
    int64_t n_tile_edges;       /* sum over tiles of their distinct element edges */
    int64_t n_partials;         /* partial sums per evaluation */
    int64_t n_combined_nodes;   /* residual/diagonal outputs summed from partials */
    int64_t n_combined_slots;   /* upper Jacobian slots summed from partials */
    double build_s;             /* host time of the plan build */
} up3d_tile_info;
int up3d_mesh_tile_info(up3d_mesh* mesh, int32_t tile_elems, up3d_tile_info* info, up3d_stream stream);

/* The same plan built on the host from host arrays, for tests and
 * inspection (no device is touched): elements and face_neighbors (n_tets,
 * 4) int32, centroids (n_tets, 3), the P1 pattern (indptr, indices).
 * up3d_tile_plan_host_array copies one named array of the plan ("perm",
 * "iperm", "eoff", "noff", "uoff", "tnode", "lconn", "nent_off", "nent",
 * "ndst", "uent_off", "uent", "udst", "cn_off", "cn_idx", "cn_dst",
 * "ce_off", "ce_idx", "ce_dst", "fnbr") into dst (NULL: size only) and
 * returns its byte size. */
typedef struct up3d_tile_plan up3d_tile_plan; /* opaque host-side plan */
int up3d_tile_plan_host_create(const int32_t* elements, const int32_t* face_neighbors, const double* centroids,
                               int64_t n_nodes, int64_t n_tets, const int32_t* indptr, const int32_t* indices,
                               int32_t tile_elems, int32_t tile_stretch, up3d_tile_plan** out);
int up3d_tile_plan_host_info(const up3d_tile_plan* plan, up3d_tile_info* info);
int up3d_tile_plan_host_array(const up3d_tile_plan* plan, const char* name, void* dst, int64_t* nbytes);
int up3d_tile_plan_host_destroy(up3d_tile_plan* plan);

/* Times every candidate shape of the two passes on this mesh (the Newton
 * Jacobian sweep at phi and the flow, live upwind selection; `reps` timed
 * launches each after one warm-up, median kept), then the tiled form at
 * each tile size (the whole evaluation), installs the fastest form and
 * shapes and returns them in `tuning` (may be NULL); for the tiled form
 * elem_us is the whole evaluation and row_us 0.  Builds the tile plans
 * (host work) and overwrites the mesh's internal workspaces only;
 * synchronises the stream. */
int up3d_autotune(up3d_mesh* mesh, const double* phi, const up3d_flow* flow, int reps,
                  up3d_tuning* tuning, up3d_stream stream);

/* ------------------------------------------------------ accounting */

/* Number of library kernel launches since the library was loaded (the
 * reference has no counterpart; used to report device launches per step). */
int up3d_launch_count(int64_t* out);

/* The library's device memory (no reference counterpart: numpy / scipy
 * allocate on the host).  Every device buffer of the library comes from a
 * per-device cache of cudaMalloc'd blocks: a freed block is kept, once the
 * device has finished the work in flight (the synchronisation cudaFree
 * implies), and handed to a later request of the same size or at most a
 * quarter smaller, so repeated set-ups of a problem (a fresh workspace per
 * solve) make no driver allocation.  The cache holds at most
 * UP3D_POOL_CACHE_MB MiB (read at the first allocation; default 4096, 0
 * turns caching off; past it the least recently freed blocks are released
 * down to three quarters of it); when cudaMalloc runs out of memory the device's
 * cached blocks are released and the allocation retried once.
 * up3d_pool_stats: bytes cached and handed out, and the requests served
 * from the cache (hits) or by cudaMalloc (misses) since the library was
 * loaded.  up3d_pool_release: cudaFree of every cached block (for a caller
 * that needs the memory elsewhere); released_bytes may be NULL. */
int up3d_pool_stats(int64_t* cached_bytes, int64_t* live_bytes, int64_t* hits, int64_t* misses);
int up3d_pool_release(int64_t* released_bytes);
/* Enable (1) / disable (0) per-phase CUDA-event timing and reset it. */
int up3d_profile(int enable);
/* Per phase slot (0 element sweep, 1 row gather, 2 Term-3 build, 3 SpMV,
 * 4 Krylov vector work): summed milliseconds, timed calls and kernel
 * launches since up3d_profile(1).  Synchronises the recorded events. */
int up3d_profile_read(double* ms, int64_t* calls, int64_t* launches, int n_slots);

/* ------------------------------------------------------ linear algebra */

/* CSR SpMV y = A x (the scipy product inside spla.cg / spla.gmres,
 * solve/picard.py:375-380, solve/linear.py:182).  `dirichlet` (uint8 per
 * row, NULL = none) makes constrained rows act as identity and drops
 * constrained columns: the free-DOF operator A[free][:, free] embedded in
 * full size (solve/linear.py:20-58). */
int up3d_spmv(int64_t n_rows, const int32_t* indptr, const int32_t* indices,
              const double* data, const double* x, double* y, const uint8_t* dirichlet,
              up3d_stream stream);
/* FP32 variant (mixed precision). */
int up3d_spmv_f32(int64_t n_rows, const int32_t* indptr, const int32_t* indices,
                  const float* data, const float* x, float* y, const uint8_t* dirichlet,
                  up3d_stream stream);

/* A device CSR operand of the solvers.  `dirichlet` (NULL = none) embeds the
 * free-DOF system A[free][:, free] in full size (identity rows, dropped
 * columns); right-hand sides must then be zero on constrained rows. */
typedef struct {
    int64_t n;
    const int32_t* indptr;
    const int32_t* indices;
    const double* data;
    const uint8_t* dirichlet;
} up3d_csr;

typedef struct up3d_precond up3d_precond; /* opaque preconditioner */

/* Smoothed-aggregation AMG (build_amg_preconditioner, solve/linear.py:61-81,
 * pyamg.smoothed_aggregation_solver defaults: theta 0, standard aggregation,
 * Jacobi-smoothed prolongator with omega 4/3 / rho(D^-1 A), Galerkin
 * coarsening).  The V-cycle smooths with damped Jacobi on the device; fp32
 * selects FP32 level operators and cycle with an FP64 coarsest solve. */
typedef struct {
    int max_levels;     /* default 10 */
    int64_t max_coarse; /* dense FP64 solve at or below this size (default 500) */
    int presmooth;      /* Jacobi sweeps (default 2) */
    int postsmooth;     /* Jacobi sweeps (default 2) */
    int fp32;           /* 0 FP64 cycle, 1 FP32 cycle, 2 both (FP64 vectors take the
                           FP64 cycle, FP32 vectors the FP32 one) */
} up3d_amg_options;

typedef struct {
    int32_t n_levels;
    int64_t n_coarse;
    double operator_complexity;
    int64_t level_rows[16];
} up3d_amg_info;

/* Builds the hierarchy of A (solve/linear.py:61-81): aggregation and the
 * level patterns on the host, every value (D^-1, omega, P, R A P, the
 * coarsest inverse) on the device; the cycle runs on the device. */
int up3d_amg_setup(const up3d_csr* A, const up3d_amg_options* options, up3d_precond** out,
                   up3d_stream stream);
int up3d_amg_get_info(const up3d_precond* M, up3d_amg_info* info);
/* Recomputes the values of a hierarchy for a new matrix with the same
 * pattern and Dirichlet mask as its setup matrix: the reference rebuilds
 * pyamg's hierarchy from scratch every amg_rebuild_every Newton steps
 * (solve/newton.py:1016-1022); with every connection strong the aggregates
 * depend on the pattern alone, so the result equals a fresh up3d_amg_setup
 * bit for bit.  UP3D_ERR_VALUE when the pattern or mask differ.
 * Synchronises the stream. */
int up3d_amg_refresh(up3d_precond* M, const up3d_csr* A, up3d_stream stream);

/* Point-Jacobi preconditioner z = D^{-1} r (constrained rows: identity). */
/* ILU(0) preconditioner on A's own pattern (replaces solve/linear.py:84-131
 * build_ilu_preconditioner; the reference's threshold ILU is scipy's serial
 * spilu): the fixed-point form of ILU(0) (Chow and Patel, SIAM J. Sci.
 * Comput. 37, 2015), `sweeps` sweeps from L = strict lower part of A over
 * its diagonal and U = upper part; applied as U^-1 L^-1 r with
 * `tri_sweeps` Jacobi sweeps per triangle.  Honours A->dirichlet (identity
 * rows, dropped columns).  Every row needs its diagonal in the pattern
 * (UP3D_ERR_VALUE otherwise); a non-finite factorisation is redone on
 * A + 1e-3 mean|a_ii| I, and UP3D_ERR_RUNTIME if that fails too.  FP64
 * vectors only (up3d_gmres_ir refuses it).  sweeps, tri_sweeps in [1, 100]
 * (UP3D_ERR_VALUE otherwise). */
int up3d_precond_ilu0(const up3d_csr* A, int sweeps, int tri_sweeps, up3d_precond** out, up3d_stream stream);
/* The ILU(0) factors (nnz values on A's pattern: L strictly below the
 * diagonal, unit diagonal implied; U on and above) into `lu` (device), and
 * the diagonal shift the factorisation used into *shift (host). */
int up3d_precond_ilu0_factors(const up3d_precond* M, double* lu, double* shift, up3d_stream stream);
int up3d_precond_jacobi(const up3d_csr* A, up3d_precond** out, up3d_stream stream);
/* z = M r */
int up3d_precond_apply(up3d_precond* M, const double* r, double* z, up3d_stream stream);
/* One V-cycle of an AMG hierarchy from up3d_amg_setup (pyamg's
 * ml.aspreconditioner() applied once): z = M r.  UP3D_ERR_VALUE when M is
 * not an AMG hierarchy. */
int up3d_amg_vcycle(up3d_precond* M, const double* r, double* z, up3d_stream stream);
/* The same cycle on FP32 vectors, as the mixed-precision GMRES applies it
 * (the FP32 cycle of a hierarchy built with fp32 = 1 or 2, else the FP64
 * cycle between conversions). */
int up3d_amg_vcycle_f32(up3d_precond* M, const float* r, float* z, up3d_stream stream);
int up3d_precond_destroy(up3d_precond* M);

/* Preconditioned CG (scipy.sparse.linalg.cg as called by solve_cg_amg,
 * solve/linear.py:204-239, and solve_subsonic, solve/picard.py:375-380):
 * x holds x0 on entry and the iterate on exit; converged when
 * ||b - A x|| <= max(rtol ||b||, atol).  info = 0 converged, else maxiter.
 * Synchronous. */
int up3d_cg(const up3d_csr* A, const double* b, double* x, double rtol, double atol,
            int maxiter, up3d_precond* M, int64_t* iters, double* resid, int* info,
            up3d_stream stream);

/* Restarted left-preconditioned GMRES (scipy.sparse.linalg.gmres as called
 * by solve_gmres, solve/linear.py:134-201): operator A (+ `extra`, the
 * Term-3 entries outside the P1 pattern, may be NULL); `maxiter` counts
 * restart cycles; inner = total Arnoldi steps.  Synchronous. */
int up3d_gmres(const up3d_csr* A, const up3d_csr* extra, const double* b, double* x,
               double rtol, double atol, int restart, int maxiter, up3d_precond* M,
               int64_t* inner, double* resid, int* info, up3d_stream stream);
/* ------------------------------------------- coupled (phi, Gamma) Newton system */

typedef struct up3d_coupled up3d_coupled; /* opaque: far-field rows, Kutta rows, basis */

/* NewtonWorkspace's coupled system (solve/newton.py:97-502, the "probe"
 * Kutta estimator) on the unknowns of a wake handle: dir_nodes (HOST, n_dir
 * distinct reduced ids) are the far-field rows (`dir_red`, :243-256); K
 * (HOST CSR, n_stations rows, int64 k_indptr / k_cols = reduced ids of free
 * rows, k_vals) is dF/dphi_free (:276-292, the tip taper already applied);
 * the Kutta targets average phi[kutta_upper] - phi[kutta_lower] over each
 * station's TE entries (te_station, n_te entries, TE order: kutta_targets,
 * constraints/wake.py:196-212) and are scaled by taper (n_stations, HOST).
 * The handle refers to `wake`, which must outlive it.  UP3D_ERR_VALUE for
 * ids out of range, a K column on a far-field row or a station without
 * TE entries.  Calls on one handle must not overlap. */
int up3d_coupled_create(const up3d_wake* wake, int64_t n_dir, const int64_t* dir_nodes,
                        const int64_t* k_indptr, const int64_t* k_cols, const double* k_vals,
                        int64_t n_te, const int64_t* te_station, const int64_t* kutta_upper,
                        const int64_t* kutta_lower, const double* taper, up3d_coupled** out);
int up3d_coupled_destroy(up3d_coupled* coupled);
/* Replaces K (HOST CSR as at creation): the pressure Kutta estimator's
 * eliminated row -D^-1 K_p, rebuilt every Newton step (kutta_blocks,
 * solve/newton.py:459-502).  Synchronous. */
int up3d_coupled_set_kutta_row(up3d_coupled* coupled, const int64_t* k_indptr, const int64_t* k_cols,
                               const double* k_vals);
/* set_mach's affine far-field basis (solve/newton.py:295-324): far-field
 * values vals0 + V Gamma (HOST vals0 n_dir, V n_dir x n_stations row-major,
 * rows in dir_nodes order). */
int up3d_coupled_set_farfield(up3d_coupled* coupled, const double* vals0, const double* V);
/* Device view of the far-field row mask (n_red, 1 on far-field rows): the
 * `dirichlet` of the reduced Picard block's up3d_csr. */
int up3d_coupled_dirichlet(const up3d_coupled* coupled, const uint8_t** mask);
/* eval_residual's state (solve/newton.py:340-344): phi_red = phi_f on free
 * rows and vals0 + V gamma on far-field rows (phi_red may alias phi_f),
 * phi_cut = T phi_red + G gamma.  Device vectors (n_red, n_stations,
 * n_red, n_cut). */
int up3d_coupled_state(const up3d_coupled* coupled, const double* phi_f, const double* gamma,
                       double* phi_red, double* phi_cut, up3d_stream stream);
/* eval_residual's outputs (:399-419): R_red = T^T R_cut on free rows, 0 on
 * far-field rows; F = taper * kutta_targets(phi_cut) - gamma (F NULL: the
 * fold alone, phi_cut and gamma unused). */
int up3d_coupled_residual(const up3d_coupled* coupled, const double* R_cut, const double* phi_cut,
                          const double* gamma, double* R_red, double* F, up3d_stream stream);
/* The eliminated coupled step's operator (:1029-1032, :1079):
 * t = K x + g (g may be NULL), y = J_ff x + B t on free rows with
 * B = J_red[free, dir] V + H_J[free] (assemble_coupled, :430-457), y = x on
 * far-field rows.  J (+ extra, may be NULL) is the Jacobian of the CUT mesh
 * (n_cut rows, no Dirichlet mask); J_red, H_J and B are never formed: the
 * operator is T^T J (T u + G t) with u = x on free rows and V t on
 * far-field rows.  x = 0, g = F gives B F; t (n_stations, may be NULL)
 * returns K x + g, the step's dGamma. */
int up3d_coupled_apply(const up3d_coupled* coupled, const up3d_csr* J, const up3d_csr* extra,
                       const double* x, const double* g, double* y, double* t, up3d_stream stream);


/* up3d_gmres on the coupled operator (up3d_coupled_apply with g = NULL):
 * the inexact Newton solve of solve_newton_lifting (solve/newton.py:
 * 1029-1046).  b and x are reduced-size vectors, b zero on far-field rows;
 * M (may be NULL) must be of reduced size -- the AMG of the reduced Picard
 * block with the far-field mask (:1013-1022).  Synchronous. */
int up3d_gmres_coupled(const up3d_coupled* coupled, const up3d_csr* J, const up3d_csr* extra,
                       const double* b, double* x, double rtol, double atol, int restart,
                       int maxiter, up3d_precond* M, int64_t* inner, double* resid, int* info,
                       up3d_stream stream);
/* Mixed-precision GMRES with FP64 iterative refinement (the mixed form of
 * the Newton linear solve the reference does with spla.gmres,
 * solve/newton.py:1029-1040).  The outer loop forms r = b - A x with A's
 * FP64 values and tests up3d_gmres's criterion: with M, the preconditioned
 * residual ||M r|| <= ||M b|| min(1, max(rtol, atol / ||b||)) (M applied in
 * FP32); without, ||r|| <= max(rtol ||b||, atol).  It stops there, after
 * refine_max corrections, or once the corrections have used restart x
 * maxiter Arnoldi steps (the cap of one up3d_gmres call).  Each correction
 * solves A d = r by restarted GMRES in FP32 -- A's FP32 values `data32`
 * (and `extra32` for `extra`), FP32 vectors, M applied in FP32 (an FP32 AMG
 * hierarchy keeps its coarsest solve in FP64) -- to max(inner_rtol,
 * tol / ||M r||) relative, and is added to x in FP64; once a correction
 * fails to halve the tested residual, FP64 GMRES finishes the solve from
 * the current iterate within the remaining steps.  inner = total Arnoldi
 * steps, outer = corrections, resid = ||b - A x||.  Synchronous. */
int up3d_gmres_ir(const up3d_csr* A, const up3d_csr* extra, const float* data32,
                  const float* extra32, const double* b, double* x, double rtol, double atol,
                  int restart, int maxiter, int refine_max, double inner_rtol, up3d_precond* M,
                  int64_t* inner, int64_t* outer, double* resid, int* info, up3d_stream stream);

/* ------------------------------------------------ allocation-free solve */

/* CG with point-Jacobi preconditioning that allocates no device or pinned
 * memory: for callers that cannot let this library call cudaMalloc /
 * cudaFree (a process whose device memory belongs to another allocator or a
 * fixed pre-reserved pool, or a time-critical loop that cannot take the
 * implicit synchronisation of those calls).  Working vectors live in one
 * static device array of UP3D_NOALLOC_MAX_ROWS rows (about 10.5 MB).  Same
 * arguments and result as up3d_cg with an up3d_precond_jacobi
 * preconditioner.  UP3D_ERR_VALUE for more rows than the limit.  With
 * CUDA's default lazy module loading the driver commits the array on a
 * device at the first call there (one driver-side allocation, which fails
 * with out-of-memory if another allocator has already reserved the whole
 * device): make the first call on each device -- or run with
 * CUDA_MODULE_LOADING=EAGER -- before a pool reserves the device, and
 * before capturing any stream; later calls allocate nothing and the array
 * stays resident until the process exits.  Every call looks the array's
 * device address up (cudaGetSymbolAddress) with the caller's device
 * current.  All calls share the array: calls that overlap on the GPU race
 * and must be serialised by the caller.  Synchronous (x is complete on
 * return, b = 0 included).  This entry point has no counterpart in the
 * reference. */
#define UP3D_NOALLOC_MAX_ROWS (1 << 18)
int up3d_cg_jacobi_noalloc(const up3d_csr* A, const double* b, double* x, double rtol,
                           double atol, int maxiter, int64_t* iters, double* resid,
                           int* info, up3d_stream stream);

#ifdef __cplusplus
}
#endif

#endif /* UP3D_H */
