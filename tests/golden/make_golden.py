"""Generate the golden fixtures of the element-loop hot path by running the
reference (pyfp3d, pure Python + Numba) on synthetic Kuhn bump meshes.

Usage (needs the reference source tree; it cannot run where that tree is
absent, which is why its outputs are committed):

    python tests/golden/make_golden.py /path/to/UP3D [--weighted-only | --wake-only | --wall-only |
                                                      --sides-only | --lifting-only |
                                                      --naca-only]

Every array is produced by the reference's own public entry points, composed
exactly as ``NewtonWorkspace.eval_residual`` / ``assemble_coupled`` compose
them (``pyfp3d/solve/newton.py:345-372``, ``:430-452``) with no wake
(T = I):

  PicardOperator(nodes, elements)                     kernels/jacobian.py:246
  UpwindOperator(nodes, elements, weighted=False)     kernels/upwind.py:744
  op.velocities(phi)                                  kernels/jacobian.py:264
  limit_q2_field / density_field / mach_squared_field physics/isentropic.py:293,236,318
  upw.rho_tilde / freeze_upwind_state / rho_tilde_frozen /
  rho_tilde_sensitivities / rho_tilde_frozen_sensitivities
                                                      kernels/upwind.py:783-920
  op.assemble_residual / assemble_matrix / assemble_newton_jacobian
                                                      kernels/jacobian.py:272-375
  solve_subsonic (pyamg swapped for scipy spilu)      solve/picard.py:271-417
  UpwindOperator(weighted=True, mode="kernel"|"blend"), compute_face_normals
                                                      kernels/upwind.py:128-454, :744-819
  WakeConstraint, kutta_targets                       constraints/wake.py:32-127, :196-212
  wall_force_coefficients and its pieces              post/surface.py:80-363
  per-side walks, newton_terms23_side_coo             wake/multivalued.py:456-466,
                                                      kernels/cut_assembly.py:401-488
  NewtonWorkspace, solve_newton_lifting (direct)      solve/newton.py:97-1141
  solve_newton_transonic (the committed NACA recipe)  solve/newton.py:1144-1307
  solve_subsonic_lifting (pyamg swapped for spilu)    solve/picard.py:420-883
  cut_wake on the NACA0012 2.5D coarse mesh and on a
  swept part-span sheet; farfield_dirichlet           mesh/wake_cut.py:225-594,
                                                      constraints/dirichlet.py:98-182
  TEControlVolumes (pressure Kutta estimator)         constraints/te_pressure.py:73-323

The optional reference dependencies that are absent here (meshio, pyamg) are
replaced by empty modules before import; neither is on the hot path.
"""

from __future__ import annotations

import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO))

from up3d_b200.mesh.kuhn import bump_channel, pocket_state, seeded_state  # noqa: E402

M_CRIT = 0.95
UPWIND_C = 1.5
RHO_FLOOR = 0.05
M_CAP = 3.0
GAMMA = 1.4


def import_reference(ref_root: str):
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/up3d_numba_cache")
    for name in ("meshio", "pyamg"):
        if name not in sys.modules:
            sys.modules[name] = types.ModuleType(name)
    sys.path.insert(0, ref_root)
    import pyfp3d.kernels.jacobian as jac
    import pyfp3d.kernels.upwind as upw
    import pyfp3d.physics.isentropic as isen
    return jac, upw, isen


def chain(jac, upw_mod, isen, op, upw, phi, m_inf, u_inf=1.0):
    """Residual + Jacobian chain of eval_residual/assemble_coupled."""
    out = {"phi": phi, "m_inf": np.float64(m_inf), "u_inf": np.float64(u_inf)}
    grad, q2 = op.velocities(phi)
    grad, q2 = grad.copy(), q2.copy()
    q2n = q2 / u_inf ** 2
    q2l = isen.limit_q2_field(q2n, m_inf, M_CAP, GAMMA)
    lim = q2l == q2n
    rho = isen.density_field(q2l, m_inf, GAMMA)
    out.update(grad=grad, q2=q2, q2l=q2l, lim=lim, rho=rho,
               mach2=isen.mach_squared_field(q2l, m_inf, GAMMA))
    rho_t = upw.rho_tilde(grad, q2l, rho, m_inf, UPWIND_C, M_CRIT, GAMMA,
                          RHO_FLOOR).copy()
    out.update(rho_tilde=rho_t, nu=upw.nu.copy(),
               upstream=upw._upstream.copy(),
               nu_max=np.float64(upw.nu_max),
               n_supersonic=np.int64(upw.n_supersonic),
               n_floored=np.int64(upw.n_floored))
    up, br = upw.freeze_upwind_state(grad, q2l, rho, m_inf, UPWIND_C,
                                     M_CRIT, GAMMA, RHO_FLOOR)
    rt_f = upw.rho_tilde_frozen(q2l, rho, up, br, m_inf, UPWIND_C, M_CRIT,
                                GAMMA, RHO_FLOOR).copy()
    se_f, su_f = upw.rho_tilde_frozen_sensitivities(
        q2l, rho, up, br, m_inf, UPWIND_C, M_CRIT, GAMMA, RHO_FLOOR)
    out.update(branch=br, rho_tilde_frozen=rt_f, nu_frozen=upw.nu.copy(),
               s_e_frozen=se_f.copy(), s_u_frozen=su_f.copy())
    s_e, s_u, upstream = upw.rho_tilde_sensitivities(
        grad, q2l, rho, m_inf, UPWIND_C, M_CRIT, GAMMA, RHO_FLOOR)
    s_e, s_u, upstream = s_e.copy(), s_u.copy(), upstream.copy()
    out.update(s_e=s_e, s_u=s_u)
    R = op.assemble_residual(phi, rho_t).copy()
    A = op.assemble_matrix(rho_t)
    J = op.assemble_newton_jacobian(phi, rho_t, s_e, s_u, upstream,
                                    u_inf=u_inf,
                                    lim_mask=None if lim.all() else lim)
    out.update(R=R, A_data=A.data.copy(), J_data=J.data.copy(),
               J_indices=J.indices.astype(np.int32),
               J_indptr=J.indptr.astype(np.int64),
               n_term3_active=np.int64(op.n_term3_active),
               newton_nnz=np.int64(op.newton_nnz))
    return out


def mesh_arrays(op, upw, mesh, full=True):
    out = {"nodes": mesh.nodes, "elements": mesh.elements,
           "dirichlet_nodes": mesh.dirichlet_nodes,
           "shape": np.array(mesh.shape, dtype=np.int64),
           "B": op.B, "V": op.V,
           "face_neighbors": upw.face_neighbors,
           "centroids": upw.centroids,
           "color_offsets": op.color_offsets, "color_elems": op.color_elems,
           "indptr": op._pattern.indptr.astype(np.int64),
           "indices": op._pattern.indices.astype(np.int32),
           "laplace_data": op.assemble_matrix().data.copy()}
    if full:
        out["elem_to_csr"] = op.elem_to_csr
    return out


# Arrays dropped from the large-mesh fixture: each is either recomputed from
# the kept ones in the tests or pinned on the small mesh.
_LARGE_DROP = {"mesh/B", "mesh/centroids", "mesh/color_elems", "grad", "q2",
               "mach2", "nu", "nu_frozen", "rho_tilde_frozen", "s_e_frozen",
               "s_u_frozen", "lim", "q2l", "rho"}


def _compact(v):
    v = np.asarray(v)
    if v.dtype == np.int64 and v.size > 1 and np.abs(v).max() < 2**31:
        return v.astype(np.int32)
    return v


def make_case(jac, upw_mod, isen, name, mesh, states, full=True):
    op = jac.PicardOperator(mesh.nodes, mesh.elements)
    upw = upw_mod.UpwindOperator(mesh.nodes, mesh.elements, weighted=False)
    arrays = {f"mesh/{k}": v for k, v in mesh_arrays(op, upw, mesh, full).items()}
    if not full:
        arrays["mesh/B_checksum"] = np.array([op.B.sum(), np.abs(op.B).sum()])
    for label, (phi, m_inf) in states.items():
        res = chain(jac, upw_mod, isen, op, upw, phi, m_inf)
        for k, v in res.items():
            if not full and (k in _LARGE_DROP):
                continue
            arrays[f"{label}/{k}"] = v
    arrays = {k: _compact(v) for k, v in arrays.items()
              if full or k not in _LARGE_DROP}
    path = HERE / f"{name}.npz"
    np.savez_compressed(path, **arrays)
    print(f"wrote {path} ({path.stat().st_size / 1e6:.2f} MB)")


def make_picard(name, mesh, m_inf):
    """Converged subsonic Picard solution of the reference driver."""
    import scipy.sparse.linalg as spla
    import pyfp3d.solve.linear as lin
    from pyfp3d.solve.picard import solve_subsonic
    import pyfp3d.physics.isentropic as isen

    def _ilu_preconditioner(A):
        ilu = spla.spilu(A.tocsc(), drop_tol=1e-5, fill_factor=20.0)
        return None, spla.LinearOperator(A.shape, matvec=ilu.solve)

    saved = lin.build_amg_preconditioner
    lin.build_amg_preconditioner = _ilu_preconditioner
    try:
        vals = mesh.nodes[mesh.dirichlet_nodes, 0].copy()
        res = solve_subsonic(mesh.nodes, mesh.elements, mesh.dirichlet_nodes,
                             vals, m_inf)
    finally:
        lin.build_amg_preconditioner = saved
    jac_mod = sys.modules["pyfp3d.kernels.jacobian"]
    op = jac_mod.PicardOperator(mesh.nodes, mesh.elements)
    _, q2 = op.velocities(res["phi"])
    cp = np.array([isen.pressure_coefficient(q, m_inf, GAMMA) for q in q2])
    np.savez_compressed(
        HERE / f"{name}.npz", phi=res["phi"], rho=res["rho"], cp=cp,
        m_inf=np.float64(m_inf),
        residual_history=np.array(res["residual_history"]),
        drho_history=np.array(res["drho_history"]),
        n_picard=np.int64(res["n_picard"]), converged=res["converged"],
        nodes=mesh.nodes, elements=mesh.elements,
        dirichlet_nodes=mesh.dirichlet_nodes)
    print(f"wrote {name}: n_picard={res['n_picard']} "
          f"|R|={res['residual_history'][-1]:.2e}")


# The weighted upwind modes (kernels/upwind.py:128-454): outward face
# normals, the BFS neighbourhoods, and rho_tilde / nu / monitors of the
# "kernel" (streamline-Gaussian) and "blend" (face-ring) operators, with the
# default parameters and one other set.
WEIGHTED_PARAMS = {
    "default": dict(p_weight=3.0, reach_frac=1.0, reach_gain_max=4.0, nbr_depth=3,
                    sigma_s_frac=0.35, sigma_p_frac=0.35),
    "alt": dict(p_weight=2.0, reach_frac=0.8, reach_gain_max=3.0, nbr_depth=2,
                sigma_s_frac=0.5, sigma_p_frac=0.25),
}


def make_weighted(jac, upw_mod, isen, name, mesh, states):
    op = jac.PicardOperator(mesh.nodes, mesh.elements)
    arrays = {"mesh/nodes": mesh.nodes, "mesh/elements": mesh.elements}
    fnorm = np.empty((len(mesh.elements), 4, 3), dtype=np.float64)
    upw_mod.compute_face_normals(np.ascontiguousarray(mesh.nodes, dtype=np.float64),
                                 np.ascontiguousarray(mesh.elements), fnorm)
    arrays["mesh/face_normals"] = fnorm
    for pname, prm in WEIGHTED_PARAMS.items():
        for mode in ("kernel", "blend"):
            upw = upw_mod.UpwindOperator(mesh.nodes, mesh.elements, weighted=True, mode=mode,
                                         **prm)
            if mode == "kernel":
                arrays[f"{pname}/nb_off"] = upw._nb_off.astype(np.int64)
                arrays[f"{pname}/nb_idx"] = upw._nb_idx.astype(np.int32)
            for label, (phi, m_inf) in states.items():
                grad, q2 = op.velocities(phi)
                grad, q2 = grad.copy(), q2.copy()
                q2l = isen.limit_q2_field(q2, m_inf, M_CAP, GAMMA)
                rho = isen.density_field(q2l, m_inf, GAMMA)
                rt = upw.rho_tilde(grad, q2l, rho, m_inf, UPWIND_C, M_CRIT, GAMMA, RHO_FLOOR).copy()
                key = f"{pname}/{mode}/{label}"
                arrays[f"{key}/rho_tilde"] = rt
                arrays[f"{key}/nu"] = upw.nu.copy()
                arrays[f"{key}/nu_max"] = np.float64(upw.nu_max)
                arrays[f"{key}/n_supersonic"] = np.int64(upw.n_supersonic)
                arrays[f"{key}/n_floored"] = np.int64(upw.n_floored)
                if pname == "default" and mode == "kernel":
                    arrays[f"state/{label}/phi"] = phi
                    arrays[f"state/{label}/m_inf"] = np.float64(m_inf)
    path = HERE / f"{name}.npz"
    np.savez_compressed(path, **arrays)
    print(f"wrote {path} ({path.stat().st_size / 1e6:.2f} MB)")


def make_wake(jac, upw_mod, isen, name):
    """WakeConstraint (constraints/wake.py:32-127) and kutta_targets
    (:196-212) of the reference on synthetic plane-sheet cuts of the
    channel (up3d_b200.mesh.wake_cut.cut_channel_sheet): a Picard matrix
    (symmetric) and a Newton Jacobian at a pocket state (Term-3 entries
    off the P1 pattern), with one station per spanwise line and with a
    single station."""
    import scipy.sparse as sp
    from pyfp3d.constraints.wake import WakeConstraint, kutta_targets
    from up3d_b200.mesh.wake_cut import cut_channel_sheet
    rng = np.random.default_rng(7)
    mesh = bump_channel(10, 4, 4, amplitude=0.08, seed=1)
    arrays = {}
    for tag, single in (("multi", False), ("single", True)):
        cut = cut_channel_sheet(mesh, single_station=single)
        wc = cut.wc
        pre = f"{tag}/"
        arrays.update({pre + "nodes": cut.nodes, pre + "elements": cut.elements,
                       pre + "dirichlet_nodes": cut.dirichlet_nodes})
        op = jac.PicardOperator(cut.nodes, cut.elements)
        rho = rng.uniform(0.5, 1.5, len(cut.elements))
        mats = {"picard": op.assemble_matrix(rho)}
        upw = upw_mod.UpwindOperator(cut.nodes, cut.elements, weighted=False)
        phi0 = pocket_state(mesh, "mixed")
        phi_cut = np.concatenate([phi0, phi0[wc.master_nodes] + 0.01 * (1 + wc.node_station)])
        res = chain(jac, upw_mod, isen, op, upw, phi_cut, 0.8)
        mats["newton"] = sp.csr_matrix((res["J_data"], res["J_indices"], res["J_indptr"]),
                                       shape=(len(cut.nodes),) * 2)
        for mname, A in mats.items():
            A = A.tocsr()
            con = WakeConstraint(A, wc)
            A_red, H = con.reduce_operator(A)
            A_red = A_red.tocsr().copy()
            A_red.sum_duplicates()
            A_red.sort_indices()
            H = H.tocsr().copy()
            H.sum_duplicates()
            H.sort_indices()
            b = rng.standard_normal(A.shape[0])
            gamma = rng.standard_normal(wc.n_stations)
            phi_red = rng.standard_normal(con.n_reduced)
            q = f"{pre}{mname}/"
            arrays.update({q + "A_indptr": A.indptr.astype(np.int64), q + "A_indices": A.indices.astype(np.int32),
                           q + "A_data": A.data.copy(),
                           q + "red_indptr": A_red.indptr.astype(np.int64),
                           q + "red_indices": A_red.indices.astype(np.int32), q + "red_data": A_red.data,
                           q + "H_indptr": H.indptr.astype(np.int64), q + "H_indices": H.indices.astype(np.int32),
                           q + "H_data": H.data, q + "h_dense": con._h.copy(),
                           q + "b": b, q + "gamma": gamma, q + "rhs": con.reduced_rhs(b, gamma),
                           q + "phi_red": phi_red, q + "expand": con.expand(phi_red, gamma)})
        vals = cut.nodes[cut.dirichlet_nodes, 0] * 1.1
        dn, dv = WakeConstraint(mats["picard"].tocsr(), wc).to_reduced_dirichlet(cut.dirichlet_nodes, vals)
        arrays.update({pre + "dir_values": vals, pre + "red_dir_nodes": dn, pre + "red_dir_values": dv,
                       pre + "phi_cut": phi_cut, pre + "kutta": kutta_targets(phi_cut, wc)})
    path = HERE / f"{name}.npz"
    np.savez_compressed(path, **arrays)
    print(f"wrote {path} ({path.stat().st_size / 1e6:.2f} MB)")


def make_wall(name):
    """wall_force_coefficients and its pieces (post/surface.py:80-363) of the
    reference on the channel's lower wall: per-triangle tangential gradient,
    area and outward normal, edge adjacency, per-triangle Cp and the force
    coefficients, at incompressible and compressible Mach numbers, two
    incidences and with / without gradient smoothing."""
    import pyfp3d.post.surface as surf
    from up3d_b200.adjoint import lower_wall_faces
    mesh = bump_channel(12, 5, 4, amplitude=0.08, seed=2)
    wf = lower_wall_faces(mesh.elements, mesh.shape)[:, 1:]
    arrays = {"nodes": mesh.nodes, "elements": mesh.elements, "wall_faces": wf}
    g, area, tn = surf.triangle_tangential_gradients(mesh.nodes, wf, mesh.freestream())
    arrays.update(tri_normal=tn, area=area,
                  out_normal=surf.wall_outward_normals(mesh.nodes, mesh.elements, wf),
                  adjacency=surf.wall_triangle_adjacency(wf))
    cases = {"seed_m05": (seeded_state(mesh, 1), 0.5), "mixed_m08": (pocket_state(mesh, "mixed"), 0.8),
             "seed_m0": (seeded_state(mesh, 2), 0.0)}
    for label, (phi, m) in cases.items():
        g, _, _ = surf.triangle_tangential_gradients(mesh.nodes, wf, phi)
        arrays[f"{label}/phi"] = phi
        arrays[f"{label}/m_inf"] = np.float64(m)
        arrays[f"{label}/grad"] = g
        for alpha in (0.0, 4.0):
            for sp_ in (0, 2):
                r = surf.wall_force_coefficients(mesh.nodes, mesh.elements, wf, phi, alpha_deg=alpha,
                                                 u_inf=1.0, s_ref=2.5, m_inf=m, smooth_passes=sp_)
                q = f"{label}/a{int(alpha)}_s{sp_}/"
                arrays[q + "cl"] = np.float64(r["cl"])
                arrays[q + "cd"] = np.float64(r["cd_pressure"])
                arrays[q + "cf"] = np.asarray(r["cf"])
                arrays[q + "cp_tri"] = np.asarray(r["cp_tri"])
    path = HERE / f"{name}.npz"
    np.savez_compressed(path, **arrays)
    print(f"wrote {path} ({path.stat().st_size / 1e6:.2f} MB)")


def make_sides(jac, upw_mod, isen, name):
    """The level-set path's per-side pieces: the upwind walk and rho~ on a
    face graph restricted to one side's elements (the masking of
    wake/multivalued.py:456-466) and newton_terms23_side_coo
    (kernels/cut_assembly.py:401-488) on a synthetic side record
    (keep mask, residual and read DOF maps with auxiliary DOFs past the
    nodes, row and column gradients, limiter mask, sensitivities, upstream
    elements)."""
    from pyfp3d.kernels.cut_assembly import newton_terms23_side_coo
    rng = np.random.default_rng(11)
    mesh = bump_channel(10, 4, 3, amplitude=0.08, seed=1)
    op = jac.PicardOperator(mesh.nodes, mesh.elements)
    phi = pocket_state(mesh, "mixed")
    grad, q2 = op.velocities(phi)
    grad, q2 = grad.copy(), q2.copy()
    q2l = isen.limit_q2_field(q2, 0.8, M_CAP, GAMMA)
    rho = isen.density_field(q2l, 0.8, GAMMA)
    cz = mesh.nodes[mesh.elements].mean(axis=1)[:, 2]
    arrays = {"nodes": mesh.nodes, "elements": mesh.elements, "phi": phi}
    for label, keep in (("upper", cz > 0.5), ("lower", cz <= 0.5)):
        upw = upw_mod.UpwindOperator(mesh.nodes, mesh.elements)
        fn = upw.face_neighbors.copy()
        nb_ok = np.where(fn >= 0, keep[np.clip(fn, 0, None)], False)
        fn[~(nb_ok & keep[:, None])] = -1
        upw.face_neighbors = np.ascontiguousarray(fn)
        rt = upw.rho_tilde(grad, q2l, rho, 0.8, UPWIND_C, M_CRIT, GAMMA, RHO_FLOOR).copy()
        arrays.update({f"{label}/keep": keep, f"{label}/fn": fn, f"{label}/upstream": upw._upstream.copy(),
                       f"{label}/rho_tilde": rt, f"{label}/nu": upw.nu.copy()})
        if label == "upper":
            up_walk = upw._upstream.copy()
    E, N = len(mesh.elements), len(mesh.nodes)
    el = mesh.elements.astype(np.int64)
    aux = rng.random(E) < 0.3
    dofvec = np.where(aux[:, None] & (rng.random((E, 4)) < 0.5), N + (el % 37), el)
    readvec = np.where(rng.random((E, 4)) < 0.15, N + (el % 23), dofvec)
    grad_row = grad + np.where(rng.random(E)[:, None] < 0.2, 1e-3 * rng.standard_normal((E, 3)), 0.0)
    s_e = np.where(rng.random(E) < 0.6, rng.standard_normal(E), 0.0)
    s_u = np.where(rng.random(E) < 0.5, rng.standard_normal(E), 0.0)
    side = {"keep": rng.random(E) < 0.7, "dofvec": dofvec, "readvec": readvec, "grad": grad,
            "grad_row": grad_row, "lim_mask": (rng.random(E) < 0.9).astype(np.float64), "s_e": s_e,
            "s_u": s_u, "upstream": up_walk}
    rows, cols, data = newton_terms23_side_coo(op, side, u_inf=1.3)
    arrays.update({f"t23/{k}": np.asarray(v) for k, v in side.items()})
    arrays.update({"t23/rows": rows, "t23/cols": cols, "t23/data": data})
    path = HERE / f"{name}.npz"
    np.savez_compressed(path, **arrays)
    print(f"wrote {path} ({path.stat().st_size / 1e6:.2f} MB), {len(data)} triplets")



LIFTING_CASES = {
    # name: (channel shape, M_inf, alpha_deg, farfield_spanwise_gamma)
    "sub": ((12, 6, 4), 0.5, 3.0, False),
    "trans": ((16, 6, 4), 0.8, 2.0, True),
}


def make_lifting(name):
    """The coupled (phi, Gamma) Newton system of the reference
    (NewtonWorkspace, solve_newton_lifting: solve/newton.py:97-1141, the
    probe Kutta estimator) on a bump channel cut by a plane sheet normal to
    y (up3d_b200.mesh.wake_cut.cut_channel_sheet(normal="y")) with the
    far-field vortex centred on the trailing-edge line: the workspace's
    far-field split, basis and Kutta row; eval_residual and the
    assemble_coupled blocks at a seeded state with the coupled product
    J_ff x + B (K x) and B F; and the converged solve from the freestream
    (precond="direct": exact Newton steps, no pyamg)."""
    from types import SimpleNamespace
    from pyfp3d.mesh.wake_cut import WakeCut as RefWakeCut
    from pyfp3d.solve.newton import NewtonWorkspace, solve_newton_lifting
    from pyfp3d.constraints.dirichlet import freestream_phi
    from up3d_b200.mesh.wake_cut import channel_vortex_center, cut_channel_sheet
    rng = np.random.default_rng(11)
    arrays = {}
    for case, (shape, m_inf, alpha, spanwise) in LIFTING_CASES.items():
        mesh = bump_channel(*shape, amplitude=0.08, seed=3)
        cut = cut_channel_sheet(mesh, normal="y")
        wc = RefWakeCut()
        for k in ("n_nodes_orig", "master_nodes", "slave_nodes", "te_nodes", "station_z",
                  "node_station", "te_station", "kutta_upper", "kutta_lower"):
            setattr(wc, k, getattr(cut.wc, k))
        mc = SimpleNamespace(nodes=cut.nodes, elements=cut.elements, boundary_faces=cut.boundary_faces)
        vc = channel_vortex_center(cut)
        ws = NewtonWorkspace(mc, wc, alpha, vortex_center=vc, farfield_spanwise_gamma=spanwise)
        ws.set_mach(m_inf)
        pre = f"{case}/"
        # the converged solve first (the transonic seed perturbs it)
        res = solve_newton_lifting(mc, wc, m_inf, alpha_deg=alpha, vortex_center=vc,
                                   farfield_spanwise_gamma=spanwise, n_picard_seed=0, precond="direct")
        assert res["converged"], case
        arrays.update({pre + "sol_phi": res["phi"], pre + "sol_gamma": res["gamma"],
                       pre + "sol_residual_history": np.array(res["residual_history"]),
                       pre + "sol_F_history": np.array(res["F_history"]),
                       pre + "sol_n_newton": np.int64(res["n_newton"]),
                       pre + "sol_n_nu_active": np.int64(res["n_nu_active"]),
                       pre + "sol_n_term3_active": np.int64(res["n_term3_active"] or 0)})
        K = ws.K.tocsr()
        arrays.update({pre + "shape": np.array(shape), pre + "m_inf": np.float64(m_inf),
                       pre + "alpha_deg": np.float64(alpha), pre + "spanwise": np.bool_(spanwise),
                       pre + "vortex_center": np.array(vc, dtype=np.float64),
                       pre + "nodes": cut.nodes, pre + "elements": cut.elements,
                       pre + "farfield_faces": cut.boundary_faces["farfield"],
                       pre + "dir_red": ws.dir_red.astype(np.int64), pre + "free": ws.free.astype(np.int64),
                       pre + "vals0_red": ws.vals0_red, pre + "V_red": ws.V_red,
                       pre + "K_indptr": K.indptr.astype(np.int64), pre + "K_indices": K.indices.astype(np.int64),
                       pre + "K_data": K.data})
        # a seeded state: a smooth perturbation of the freestream (subsonic
        # case) or of the converged solution (transonic case: supersonic
        # elements and Term 3 active), small Gamma perturbations
        x = cut.nodes[:ws.n_red, 0]
        wiggle = np.sin(1.3 * x) * (1.0 + 0.1 * rng.standard_normal(ws.n_red))
        if m_inf < 0.7:
            phi_red = freestream_phi(cut.nodes[:ws.n_red], alpha, 1.0) + 0.01 * wiggle
            gamma = 0.01 * rng.standard_normal(ws.n_st)
        else:
            phi_red = res["phi"][:ws.n_red] + 0.002 * wiggle
            gamma = res["gamma"] + 0.001 * rng.standard_normal(ws.n_st)
        phi_free = phi_red[ws.free].copy()
        R_free, F, state = ws.eval_residual(phi_free, gamma, UPWIND_C, M_CRIT, M_CAP, RHO_FLOOR)
        J_ff, B = ws.assemble_coupled(state, UPWIND_C, M_CRIT, RHO_FLOOR)
        J_ff = J_ff.tocsr()
        Bd = B.toarray()
        xv = rng.standard_normal(ws.n_free)
        if case == "sub":
            # a tapered Kutta row (tip_taper) and a lagged external
            # right-hand side (external_rhs) on the same case
            taper = np.linspace(1.0, 0.4, ws.n_st)
            b_ext = 1e-4 * np.sin(3.0 * cut.nodes[:, 0]) * np.cos(2.0 * cut.nodes[:, 2])
            rt = solve_newton_lifting(mc, wc, m_inf, alpha_deg=alpha, vortex_center=vc,
                                      farfield_spanwise_gamma=spanwise, n_picard_seed=0, precond="direct",
                                      tip_taper=taper, external_rhs=b_ext)
            assert rt["converged"]
            arrays.update({pre + "taper": taper, pre + "external_rhs": b_ext, pre + "taper_phi": rt["phi"],
                           pre + "taper_gamma": rt["gamma"], pre + "taper_n_newton": np.int64(rt["n_newton"])})
        arrays.update({pre + "seed_phi_free": phi_free, pre + "seed_gamma": gamma,
                       pre + "seed_R_free": R_free, pre + "seed_F": F,
                       pre + "seed_phi_cut": state["phi_cut"],
                       pre + "seed_n_supersonic": np.int64(state["n_nu_active"]),
                       pre + "Jff_indptr": J_ff.indptr.astype(np.int64),
                       pre + "Jff_indices": J_ff.indices.astype(np.int64), pre + "Jff_data": J_ff.data,
                       pre + "B": Bd, pre + "x": xv, pre + "y": J_ff @ xv + B @ (ws.K @ xv),
                       pre + "BF": B @ F, pre + "n_term3_active": np.int64(ws.op.n_term3_active or 0)})
    path = HERE / f"{name}.npz"
    np.savez_compressed(path, **arrays)
    print(f"wrote {path} ({path.stat().st_size / 1e6:.2f} MB)")



NACA_CASES = {
    # name: (M_inf, alpha_deg)
    "m05": (0.5, 2.0),
    "m07": (0.7, 1.0),
}


def make_naca(ref_root, name):
    """The reference's NACA0012 2.5D coarse mesh (cases/meshes/
    naca0012_2.5d/coarse.msh, MSH 2.2 binary) read with
    up3d_b200.mesh.reader.read_mesh -- its mesh_stats checked against the
    reference's committed coarse_stats.csv -- then cut by the reference's
    own cut_wake (mesh/wake_cut.py:225-441) and solved by its
    solve_newton_lifting (precond="direct", from the freestream) at two
    flow conditions; the wall Cp and force coefficients of each solution
    (post/surface.py:309-363).  The mesh arrays, the cut, the stats and the
    solutions are stored: the mesh file itself is not needed afterwards."""
    import csv
    from types import SimpleNamespace
    import pyfp3d.post.surface as surf
    from pyfp3d.mesh.reader import Mesh as RefMesh
    from pyfp3d.mesh.wake_cut import cut_wake
    from pyfp3d.solve.newton import solve_newton_lifting
    from up3d_b200.mesh.reader import mesh_stats, read_mesh
    from up3d_b200.mesh.wake_cut import cut_arrays
    base = Path(ref_root) / "cases" / "meshes" / "naca0012_2.5d"
    mesh = read_mesh(base / "coarse.msh")
    ref_stats = {r["metric"]: float(r["value"]) for r in csv.DictReader(open(base / "coarse_stats.csv"))}
    st = mesh_stats(mesh)
    for k, v in st.items():
        assert abs(v - ref_stats[k]) <= 1e-12 * abs(ref_stats[k]), (k, v, ref_stats[k])
    assert len(mesh.boundary_faces["wake"]) == ref_stats["n_wake_faces"]
    rm = RefMesh()
    rm.nodes, rm.elements = mesh.nodes, mesh.elements
    rm.boundary_faces = dict(mesh.boundary_faces)
    rm.element_tags, rm.tag_names, rm.name = mesh.element_tags, list(mesh.tag_names), mesh.name
    mc, wc = cut_wake(rm)
    arrays = {"nodes": mesh.nodes, "elements": mesh.elements,
              "stats_keys": np.array(list(ref_stats.keys())), "stats_values": np.array(list(ref_stats.values()))}
    for tag, faces in mesh.boundary_faces.items():
        arrays["faces/" + tag] = np.asarray(faces, dtype=np.int64)
    arrays.update(cut_arrays(mc, wc))
    for case, (m_inf, alpha) in NACA_CASES.items():
        res = solve_newton_lifting(mc, wc, m_inf, alpha_deg=alpha, n_picard_seed=0, precond="direct")
        assert res["converged"], case
        wall = np.asarray(mc.boundary_faces["wall"])
        f = surf.wall_force_coefficients(mc.nodes, mc.elements, wall, res["phi"], alpha_deg=alpha, m_inf=m_inf)
        pre = f"{case}/"
        arrays.update({pre + "m_inf": np.float64(m_inf), pre + "alpha_deg": np.float64(alpha),
                       pre + "phi": res["phi"], pre + "gamma": res["gamma"],
                       pre + "residual_history": np.array(res["residual_history"]),
                       pre + "n_newton": np.int64(res["n_newton"]),
                       pre + "n_nu_active": np.int64(res["n_nu_active"]),
                       pre + "cp_tri": np.asarray(f["cp_tri"]), pre + "cl": np.float64(f["cl"]),
                       pre + "cd_pressure": np.float64(f["cd_pressure"])})
        print(case, res["n_newton"], res["gamma"].mean(), f["cl"], res["n_nu_active"])
    # the reference's own transonic case (cases/analysis/a1_solver_bottleneck:
    # M0.80, alpha 1.25 deg, Mach ramp from 0.70 with its committed recipe)
    # (its level-0 Picard warm start with scipy spilu standing in for pyamg)
    import scipy.sparse.linalg as spla
    import pyfp3d.solve.linear as lin
    from pyfp3d.solve.newton import solve_newton_transonic

    def _ilu_preconditioner(A):
        ilu = spla.spilu(A.tocsc(), drop_tol=1e-5, fill_factor=20.0)
        return None, spla.LinearOperator(A.shape, matvec=ilu.solve)

    saved = lin.build_amg_preconditioner
    lin.build_amg_preconditioner = _ilu_preconditioner
    try:
        rt = solve_newton_transonic(mc, wc, m_inf=0.8, alpha_deg=1.25, m_start=0.70, dm=0.025, dm_min=0.003,
                                    freeze_tol=1e-6,
                                    newton_kw=dict(freeze_refresh_max=8, precond="direct", n_newton_max=60))
    finally:
        lin.build_amg_preconditioner = saved
    assert rt["converged"]
    arrays.update({"m08/phi": rt["phi"], "m08/gamma": rt["gamma"], "m08/n_nu_active": np.int64(rt["n_nu_active"]),
                   "m08/levels": np.array([[m, n, r] for m, n, r in rt["level_history"]])})
    print("m08", rt["gamma"], len(rt["level_history"]), sum(n for _, n, _ in rt["level_history"]))
    path = HERE / f"{name}.npz"
    np.savez_compressed(path, **arrays)
    print(f"wrote {path} ({path.stat().st_size / 1e6:.2f} MB)")
    # the medium mesh (61,788 tets): the mesh of the reference's one
    # published hot-path timing (Picard matrix assembly, 2.1 ms)
    med = read_mesh(base / "medium.msh")
    ref_stats = {r["metric"]: float(r["value"]) for r in csv.DictReader(open(base / "medium_stats.csv"))}
    for k, v in mesh_stats(med).items():
        assert abs(v - ref_stats[k]) <= 1e-12 * abs(ref_stats[k]), (k, v, ref_stats[k])
    path = HERE / "naca_medium_mesh.npz"
    np.savez_compressed(path, nodes=med.nodes, elements=med.elements,
                        stats_keys=np.array(list(ref_stats.keys())), stats_values=np.array(list(ref_stats.values())),
                        **{"faces/" + k: np.asarray(v, dtype=np.int32) for k, v in med.boundary_faces.items()})
    print(f"wrote {path} ({path.stat().st_size / 1e6:.2f} MB)")



def swept_sheet_mesh():
    """A tagged mesh with a swept, part-span wake sheet, built from the
    bump channel 12x6x5 (seed 4): x sheared by 0.3 z, the inflow plane is
    the "wall" (the sheet's trailing edge lies on it, one station per TE
    node because the shear sweeps it), the outflow plane "farfield", the
    other sides "symmetry" / "top" / "side"; the sheet is the interior
    plane j = 3 for k <= 3 (its edge at k = 3 is an interior free edge)."""
    from up3d_b200.mesh.reader import Mesh
    mesh = bump_channel(12, 6, 5, amplitude=0.08, seed=4)
    nx, ny, nz = mesh.shape
    nodes = mesh.nodes.copy()
    nodes[:, 0] += 0.3 * nodes[:, 2]
    el = mesh.elements.astype(np.int64)
    ijk = np.stack(np.unravel_index(np.arange(len(nodes)), (nx + 1, ny + 1, nz + 1)), axis=1)
    faces = el[:, [[1, 2, 3], [0, 2, 3], [0, 1, 3], [0, 1, 2]]].reshape(-1, 3)
    key = np.sort(faces, axis=1)
    _, inv, cnt = np.unique(key, axis=0, return_inverse=True, return_counts=True)
    bnd = faces[cnt[inv.ravel()] == 1]
    fi = ijk[bnd]
    groups = {}
    for name, (axis, val) in (("wall", (0, 0)), ("farfield", (0, nx)), ("symmetry", (2, 0)), ("top", (2, nz)),
                              ("side", (1, 0)), ("side2", (1, ny))):
        sel = np.all(fi[:, :, axis] == val, axis=1)
        groups[name] = bnd[sel]
        bnd, fi = bnd[~sel], fi[~sel]
    assert len(bnd) == 0
    interior = faces[cnt[inv.ravel()] == 2]
    _, first = np.unique(np.sort(interior, axis=1), axis=0, return_index=True)
    interior = interior[np.sort(first)]
    ii = ijk[interior]
    groups["wake"] = interior[np.all(ii[:, :, 1] == 3, axis=1) & np.all(ii[:, :, 2] <= 3, axis=1)]
    m = Mesh()
    m.nodes, m.elements = nodes, mesh.elements
    m.boundary_faces = {k: v.astype(np.int32) for k, v in groups.items()}
    m.element_tags = np.zeros(len(m.elements), dtype=np.int32)
    m.tag_names = ["fluid"]
    m.name = "swept_sheet"
    return m


def make_swept_cut(name):
    """The reference's cut_wake (mesh/wake_cut.py:225-594) on
    swept_sheet_mesh(): several stations, interior free-edge nodes."""
    from pyfp3d.mesh.reader import Mesh as RefMesh
    from pyfp3d.mesh.wake_cut import cut_wake
    from up3d_b200.mesh.wake_cut import cut_arrays
    m = swept_sheet_mesh()
    rm = RefMesh()
    rm.nodes, rm.elements, rm.boundary_faces = m.nodes, m.elements, dict(m.boundary_faces)
    rm.element_tags, rm.tag_names, rm.name = m.element_tags, list(m.tag_names), m.name
    mc, wc = cut_wake(rm)
    print("swept cut:", wc.n_stations, "stations,", len(wc.free_nodes), "free nodes,", len(wc.slave_nodes), "copies")
    arrays = {"nodes": m.nodes, "elements": m.elements}
    for tag, faces in m.boundary_faces.items():
        arrays["faces/" + tag] = np.asarray(faces, dtype=np.int64)
    arrays.update(cut_arrays(mc, wc))
    # the spanwise far field on this cut (several stations, the sheet's tip
    # inside the span: the Gamma(z) interpolation anchored to 0 at the tip)
    from pyfp3d.constraints.dirichlet import farfield_dirichlet
    g_st = np.array([0.10, 0.20, 0.15])
    vc = (0.0, float(m.nodes[wc.master_nodes[0], 1]))
    for beta in (1.0, 0.8):
        dn, dv = farfield_dirichlet(mc, wc, 2.0, g_st, 1.0, vc, beta=beta, spanwise_gamma=True)
        arrays.update({f"ff_beta{beta}/nodes": dn, f"ff_beta{beta}/values": dv})
    arrays.update({"ff_gamma": g_st, "ff_vortex_center": np.array(vc)})
    # the coupled Newton on this cut (three stations, tip nodes single-valued)
    from pyfp3d.solve.newton import solve_newton_lifting
    res = solve_newton_lifting(mc, wc, 0.3, alpha_deg=2.0, vortex_center=vc, farfield_spanwise_gamma=True,
                               n_picard_seed=0, precond="direct")
    assert res["converged"]
    arrays.update({"newton/phi": res["phi"], "newton/gamma": res["gamma"],
                   "newton/n_newton": np.int64(res["n_newton"])})
    print("swept newton", res["n_newton"], res["gamma"])
    path = HERE / f"{name}.npz"
    np.savez_compressed(path, **arrays)
    print(f"wrote {path} ({path.stat().st_size / 1e6:.2f} MB)")



def make_lifting_picard(name):
    """The reference's nested lifting Picard (solve_subsonic_lifting,
    solve/picard.py:420-883; pyamg swapped for scipy spilu, as in
    make_picard) to convergence on the lifting channel's subsonic case and
    on the NACA0012 coarse mesh at the reference's own subsonic case (M0.5,
    alpha 1.25 deg), and its solve_newton_lifting with the default 5-step
    Picard warm start (precond="direct") on the lifting channel."""
    from types import SimpleNamespace
    import scipy.sparse.linalg as spla
    import pyfp3d.solve.linear as lin
    from pyfp3d.mesh.wake_cut import WakeCut as RefWakeCut
    from pyfp3d.solve.newton import solve_newton_lifting
    from pyfp3d.solve.picard import solve_subsonic_lifting
    from up3d_b200.mesh.wake_cut import channel_vortex_center, cut_channel_sheet, load_cut

    def _ilu_preconditioner(A):
        ilu = spla.spilu(A.tocsc(), drop_tol=1e-5, fill_factor=20.0)
        return None, spla.LinearOperator(A.shape, matvec=ilu.solve)

    def ref_wc(wc):
        r = RefWakeCut()
        for k in ("n_nodes_orig", "master_nodes", "slave_nodes", "free_nodes", "te_nodes", "station_z",
                  "node_station", "te_station", "kutta_upper", "kutta_lower"):
            setattr(r, k, getattr(wc, k))
        return r

    saved = lin.build_amg_preconditioner
    lin.build_amg_preconditioner = _ilu_preconditioner
    arrays = {}
    try:
        shape, m_inf, alpha, spanwise = LIFTING_CASES["sub"]
        cut = cut_channel_sheet(bump_channel(*shape, amplitude=0.08, seed=3), normal="y")
        mc = SimpleNamespace(nodes=cut.nodes, elements=cut.elements, boundary_faces=cut.boundary_faces)
        vc = channel_vortex_center(cut)
        runs = {"channel": (mc, ref_wc(cut.wc), m_inf, alpha, vc)}
        g = np.load(HERE / "naca_coarse.npz")
        nmc, nwc = load_cut(g)
        runs["naca"] = (nmc, ref_wc(nwc), 0.5, 1.25, (0.25, 0.0))
        for tag, (m, wc, mi, al, vcen) in runs.items():
            res = solve_subsonic_lifting(m, wc, mi, alpha_deg=al, vortex_center=vcen)
            assert res["converged"], tag
            pre = f"{tag}/"
            arrays.update({pre + "m_inf": np.float64(mi), pre + "alpha_deg": np.float64(al),
                           pre + "vortex_center": np.array(vcen, dtype=np.float64),
                           pre + "phi": res["phi"], pre + "gamma": res["gamma"],
                           pre + "n_picard": np.int64(res["n_picard"]),
                           pre + "n_solves_total": np.int64(res["n_solves_total"]),
                           pre + "residual_history": np.array(res["residual_history"]),
                           pre + "drho_history": np.array(res["drho_history"])})
            print(tag, "picard", res["n_picard"], res["n_solves_total"], res["gamma"][:3])
        # the pseudo-transient forms on the channel case
        # (warm-started near the solution: the damped iterations converge
        # slowly from the freestream)
        gl = np.load(HERE / "lifting_newton.npz")
        warm = dict(phi_init=gl["sub/sol_phi"], gamma_init=0.98 * gl["sub/sol_gamma"], n_picard_max=400)
        for tag, kw in (("channel_theta", dict(damping_theta=0.05, **warm)),
                        ("channel_dt", dict(pseudo_dt=1.0, **warm))):
            res = solve_subsonic_lifting(mc, ref_wc(cut.wc), m_inf, alpha_deg=alpha, vortex_center=vc, **kw)
            assert res["converged"], tag
            arrays.update({tag + "/phi": res["phi"], tag + "/gamma": res["gamma"],
                           tag + "/n_picard": np.int64(res["n_picard"])})
            print(tag, res["n_picard"], res["n_solves_total"])
        res = solve_newton_lifting(mc, ref_wc(cut.wc), m_inf, alpha_deg=alpha, vortex_center=vc,
                                   precond="direct")
        assert res["converged"]
        arrays.update({"channel_newton_seeded/phi": res["phi"], "channel_newton_seeded/gamma": res["gamma"],
                       "channel_newton_seeded/n_newton": np.int64(res["n_newton"]),
                       "channel_newton_seeded/residual_history": np.array(res["residual_history"])})
        print("seeded newton", res["n_newton"], res["residual_history"])
    finally:
        lin.build_amg_preconditioner = saved
    path = HERE / f"{name}.npz"
    np.savez_compressed(path, **arrays)
    print(f"wrote {path} ({path.stat().st_size / 1e6:.2f} MB)")



MV_SHEET = {"shape": (16, 6, 5), "amplitude": 0.08, "seed": 3, "te_x": 2.5, "sheet_z": 0.55,
            "m_inf": 0.8, "jump": 0.05}


def mv_case():
    """The level-set case: the bump channel cut by the horizontal half-plane
    z = sheet_z downstream of x = te_x (TE line across the span, y from 1
    to 0 so that "+" is +z), a transonic pocket state on the main DOFs and a
    jump on the aux DOFs."""
    c = MV_SHEET
    mesh = bump_channel(*c["shape"], amplitude=c["amplitude"], seed=c["seed"])
    te = np.array([[c["te_x"], 1.0, c["sheet_z"]], [c["te_x"], 0.0, c["sheet_z"]]])
    return mesh, te, np.array([1.0, 0.0, 0.0])


def mv_state(mesh, node_side, ext_dof_of_node):
    phi_main = pocket_state(mesh, "mixed")
    cut_nodes = np.flatnonzero(ext_dof_of_node >= 0)
    gam = MV_SHEET["jump"] * (1.0 + 0.3 * mesh.nodes[cut_nodes, 0])
    aux = phi_main[cut_nodes] - node_side[cut_nodes] * gam
    return np.concatenate([phi_main, aux])


def make_multivalued(name):
    """The reference's level-set path -- WakeLevelSet (wake/levelset.py),
    CutElementMap (wake/cut_elements.py), MultivaluedOperator
    (wake/multivalued.py) with the cut-element assembly of
    kernels/cut_assembly.py -- on the bump channel cut by a half-plane sheet
    (mv_case): the level set at the nodes, the cut census and extended DOF
    numbering, the extended matrix with the continuity closure and with the
    wake least-squares closure (mass-conservation TE rows, no TE nodes on
    this sheet), the per-side upwinded densities and monitors, the per-side
    Newton records, live and frozen, at M0.8 with a jump on the aux DOFs."""
    from pyfp3d.physics.isentropic import density_field
    from pyfp3d.wake.cut_elements import CutElementMap
    from pyfp3d.wake.levelset import WakeLevelSet
    from pyfp3d.wake.multivalued import MultivaluedOperator
    mesh, te, direction = mv_case()
    ls = WakeLevelSet(te, direction)
    s_, d_, q_ = ls.evaluate(mesh.nodes)
    cm = CutElementMap(mesh.nodes, mesh.elements, ls)
    mv = MultivaluedOperator(mesh.nodes, mesh.elements, cm, levelset=ls)
    m_inf = MV_SHEET["m_inf"]
    phi_ext = mv_state(mesh, cm.node_side, cm.ext_dof_of_node)
    arrays = {"te_points": te, "direction": direction, "s": s_, "d": d_, "q": q_,
              "normals_cut": ls.surface_normals(mesh.nodes[mesh.elements[cm.cut_elems]].mean(axis=1)),
              "phi_ext": phi_ext, "node_side": cm.node_side, "te_nodes": cm.te_nodes,
              "cut_elems": cm.cut_elems, "te_lower_elems": cm.te_lower_elems,
              "beyond_tip_elems": cm.beyond_tip_elems, "shifted_nodes": cm.shifted_nodes,
              "ext_dof_of_node": cm.ext_dof_of_node, "dofs_upper": cm.dofs_upper, "dofs_lower": cm.dofs_lower,
              "n_total": np.int64(cm.n_total_dofs)}
    _, q2 = mv.op.velocities(phi_ext[:mv.n_main])
    rho = density_field(q2, m_inf).copy()
    arrays["rho_main"] = rho

    def put(tag, A):
        A = A.tocsr()
        A.sort_indices()
        arrays.update({tag + "/indptr": A.indptr.astype(np.int64), tag + "/indices": A.indices.astype(np.int64),
                       tag + "/data": A.data})

    put("A_laplace", mv.assemble_matrix(None))
    put("A_continuity", mv.assemble_matrix(rho))
    rho_up, rho_lo = mv.element_densities(phi_ext, m_inf)
    arrays.update({"rho_up": rho_up, "rho_lo": rho_lo})
    put("A_wake_ls", mv.assemble_matrix((rho_up, rho_lo), closure="wake_ls", te_kutta="mass"))
    rt_u, rt_l = mv.element_rho_tilde(phi_ext, m_inf, UPWIND_C, M_CRIT)
    arrays.update({"rt_up": rt_u.copy(), "rt_lo": rt_l.copy(), "mon": np.array(
        [mv.nu_max, mv.n_nu_active, mv.n_floored, mv.n_limited], dtype=np.float64),
        "nu_active_elements": mv.nu_active_elements()})
    up, lo = mv.side_potentials(phi_ext)
    arrays.update({"phi_up": up, "phi_lo": lo,
                   "node_jump": mv.node_jump(phi_ext, np.flatnonzero(cm.ext_dof_of_node >= 0)),
                   "mach2": mv.element_mach2(phi_ext, m_inf)})
    for tag, fz in (("live", None), ("frozen", mv.freeze_side_state(phi_ext, m_inf, UPWIND_C, M_CRIT))):
        if fz is not None:
            for k, side in enumerate(("upper", "lower")):
                arrays[f"freeze/{side}/upstream"] = fz[k][0].copy()
                arrays[f"freeze/{side}/branch"] = fz[k][1].copy()
        sides = mv.newton_side_data(phi_ext, m_inf, UPWIND_C, M_CRIT, frozen=fz)
        for side, rec in zip(("upper", "lower"), sides):
            for key in ("rho_tilde", "s_e", "s_u", "upstream", "grad", "lim_mask", "keep", "dofvec", "readvec",
                        "grad_row"):
                arrays[f"{tag}/{side}/{key}"] = np.asarray(rec[key]).copy()
        arrays[f"{tag}/mon"] = np.array([mv.nu_max, mv.n_nu_active, mv.n_floored, mv.n_limited], dtype=np.float64)
    print("multivalued: cut", len(cm.cut_elems), "aux", cm.n_ext_dofs, "nu_active", mv.n_nu_active,
          "mixed plain", int(mv._mixed_plain_mask().sum()))
    path = HERE / f"{name}.npz"
    np.savez_compressed(path, **arrays)
    print(f"wrote {path} ({path.stat().st_size / 1e6:.2f} MB)")


def make_lagged_lu(name):
    """The reference's lagged-LU Newton (solve_newton_lifting(precond=
    "direct", direct_refactor_every=1000), solve/newton.py:978-1008: one
    sparse LU, the later steps GMRES on the fresh coupled operator with the
    stale LU as preconditioner to direct_reuse_rtol) on both lifting
    channels from the freestream: the converged state and the step, refactor
    and GMRES counts."""
    from types import SimpleNamespace
    from pyfp3d.mesh.wake_cut import WakeCut as RefWakeCut
    from pyfp3d.solve.newton import solve_newton_lifting
    from up3d_b200.mesh.wake_cut import channel_vortex_center, cut_channel_sheet
    arrays = {}
    for case, (shape, m_inf, alpha, spanwise) in LIFTING_CASES.items():
        cut = cut_channel_sheet(bump_channel(*shape, amplitude=0.08, seed=3), normal="y")
        wc = RefWakeCut()
        for k in ("n_nodes_orig", "master_nodes", "slave_nodes", "te_nodes", "station_z",
                  "node_station", "te_station", "kutta_upper", "kutta_lower"):
            setattr(wc, k, getattr(cut.wc, k))
        mc = SimpleNamespace(nodes=cut.nodes, elements=cut.elements, boundary_faces=cut.boundary_faces)
        vc = channel_vortex_center(cut)
        res = solve_newton_lifting(mc, wc, m_inf, alpha_deg=alpha, vortex_center=vc,
                                   farfield_spanwise_gamma=spanwise, n_picard_seed=0, precond="direct",
                                   direct_refactor_every=1000)
        assert res["converged"], case
        pre = f"{case}/"
        arrays.update({pre + "phi": res["phi"], pre + "gamma": res["gamma"],
                       pre + "n_newton": np.int64(res["n_newton"]),
                       pre + "n_refactor": np.int64(res["n_refactor"]),
                       pre + "n_gmres_total": np.int64(res["n_gmres_total"]),
                       pre + "residual_history": np.array(res["residual_history"])})
        print("lagged LU", case, res["n_newton"], res["n_refactor"], res["n_gmres_total"])
    path = HERE / f"{name}.npz"
    np.savez_compressed(path, **arrays)
    print(f"wrote {path} ({path.stat().st_size / 1e6:.2f} MB)")


def make_weighted_picard(name):
    """The reference's nested lifting Picard with the weighted upwind modes
    (solve_subsonic_lifting(upwind_weighted=True), solve/picard.py:440-447,
    :592-603; pyamg swapped for scipy spilu, as in make_picard) on the
    transonic lifting channel (16 x 6 x 4, M0.8, alpha 2 deg, spanwise far
    field), modes "kernel" and "blend", from the freestream."""
    from types import SimpleNamespace
    import scipy.sparse.linalg as spla
    import pyfp3d.solve.linear as lin
    from pyfp3d.mesh.wake_cut import WakeCut as RefWakeCut
    from pyfp3d.solve.picard import solve_subsonic_lifting
    from up3d_b200.mesh.wake_cut import channel_vortex_center, cut_channel_sheet

    def _ilu_preconditioner(A):
        ilu = spla.spilu(A.tocsc(), drop_tol=1e-5, fill_factor=20.0)
        return None, spla.LinearOperator(A.shape, matvec=ilu.solve)

    def ref_wc(wc):
        r = RefWakeCut()
        for k in ("n_nodes_orig", "master_nodes", "slave_nodes", "free_nodes", "te_nodes", "station_z",
                  "node_station", "te_station", "kutta_upper", "kutta_lower"):
            setattr(r, k, getattr(wc, k))
        return r

    saved = lin.build_amg_preconditioner
    lin.build_amg_preconditioner = _ilu_preconditioner
    arrays = {}
    try:
        shape, m_inf, alpha, spanwise = LIFTING_CASES["trans"]
        cut = cut_channel_sheet(bump_channel(*shape, amplitude=0.08, seed=3), normal="y")
        mc = SimpleNamespace(nodes=cut.nodes, elements=cut.elements, boundary_faces=cut.boundary_faces)
        vc = channel_vortex_center(cut)
        for mode in ("kernel", "blend"):
            res = solve_subsonic_lifting(mc, ref_wc(cut.wc), m_inf, alpha_deg=alpha, vortex_center=vc,
                                         upwind_weighted=True, upwind_mode=mode,
                                         farfield_spanwise_gamma=spanwise, n_picard_max=200)
            assert res["converged"], mode
            pre = f"{mode}/"
            arrays.update({pre + "phi": res["phi"], pre + "gamma": res["gamma"],
                           pre + "n_picard": np.int64(res["n_picard"]),
                           pre + "n_nu_active": np.int64(res["n_nu_active"]),
                           pre + "drho_history": np.array(res["drho_history"])})
            print("weighted picard", mode, res["n_picard"], res["n_nu_active"], res["gamma"][:2])
        arrays.update({"m_inf": np.float64(m_inf), "alpha_deg": np.float64(alpha),
                       "vortex_center": np.array(vc, dtype=np.float64)})
    finally:
        lin.build_amg_preconditioner = saved
    path = HERE / f"{name}.npz"
    np.savez_compressed(path, **arrays)
    print(f"wrote {path} ({path.stat().st_size / 1e6:.2f} MB)")


def make_te_pressure(name):
    """The pressure-equality Kutta estimator (constraints/te_pressure.py,
    TEControlVolumes) on the NACA0012 coarse cut: its control-volume
    velocities, station residual and exact rows (Kp_cut, D) at the probe
    solution of case m05, and solve_newton_lifting with
    kutta_estimator="pressure" (precond="direct", from the freestream) at
    M0.5, alpha 1.25 deg, untapered and with a tip taper."""
    from types import SimpleNamespace
    from pyfp3d.constraints.dirichlet import farfield_dirichlet
    from pyfp3d.constraints.te_pressure import TEControlVolumes
    from pyfp3d.mesh.wake_cut import WakeCut as RefWakeCut
    from pyfp3d.solve.newton import solve_newton_lifting
    from up3d_b200.mesh.wake_cut import load_cut
    g = np.load(HERE / "naca_coarse.npz")
    mc, wc0 = load_cut(g)
    wc = RefWakeCut()
    for k in ("n_nodes_orig", "master_nodes", "slave_nodes", "free_nodes", "te_nodes", "station_z",
              "node_station", "te_station", "kutta_upper", "kutta_lower", "wake_faces_minus", "wake_faces_plus"):
        setattr(wc, k, getattr(wc0, k))
    dn, _ = farfield_dirichlet(mc, wc, 1.25, np.zeros(wc.n_stations))
    cvs = TEControlVolumes(mc, wc, dirichlet_nodes=dn)
    phi = g["m05/phi"]
    qu, ql = cvs.te_velocities(phi)
    Kp, D = cvs.newton_rows(phi)
    Kp = Kp.tocsr()
    arrays = {"phi": phi, "qu": qu, "ql": ql, "F_raw": cvs.residual_stations(phi),
              "Kp_indptr": Kp.indptr.astype(np.int64), "Kp_indices": Kp.indices.astype(np.int64),
              "Kp_data": Kp.data, "D": D, "D_frozen": cvs.gamma_jacobian(phi, mode="frozen"),
              "implied": cvs.implied_targets(phi, g["m05/gamma"] * 0.9)}
    for tag, taper in (("plain", None), ("taper", np.array([0.7]))):
        res = solve_newton_lifting(mc, wc, 0.5, alpha_deg=1.25, n_picard_seed=0, precond="direct",
                                   kutta_estimator="pressure", tip_taper=taper)
        assert res["converged"], tag
        arrays.update({tag + "/phi": res["phi"], tag + "/gamma": res["gamma"],
                       tag + "/kutta_sigma": np.asarray(res["kutta_sigma"]),
                       tag + "/n_newton": np.int64(res["n_newton"])})
        if res["kutta_weld_sign"] is not None:
            arrays[tag + "/kutta_weld_sign"] = np.asarray(res["kutta_weld_sign"])
        print(tag, res["n_newton"], res["gamma"], res["kutta_sigma"])
    path = HERE / f"{name}.npz"
    np.savez_compressed(path, **arrays)
    print(f"wrote {path} ({path.stat().st_size / 1e6:.2f} MB)")


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    jac, upw_mod, isen = import_reference(ref_root)
    if "--weighted-only" in sys.argv:
        _weighted(jac, upw_mod, isen)
        return
    if "--wake-only" in sys.argv:
        make_wake(jac, upw_mod, isen, "wake_constraint")
        return
    if "--wall-only" in sys.argv:
        make_wall("wall_forces")
        return
    if "--sides-only" in sys.argv:
        make_sides(jac, upw_mod, isen, "side_terms")
        return
    if "--lifting-only" in sys.argv:
        make_lifting("lifting_newton")
        make_lifting_picard("lifting_picard")
        make_weighted_picard("weighted_picard")
        make_lagged_lu("lagged_lu")
        return
    if "--multivalued-only" in sys.argv:
        make_multivalued("multivalued")
        return
    if "--lagged-lu-only" in sys.argv:
        make_lagged_lu("lagged_lu")
        return
    if "--weighted-picard-only" in sys.argv:
        make_weighted_picard("weighted_picard")
        return
    if "--naca-only" in sys.argv:
        make_naca(ref_root, "naca_coarse")
        make_swept_cut("swept_cut")
        make_te_pressure("te_pressure")
        return

    small = bump_channel(10, 4, 3, amplitude=0.08, seed=1)
    s_states = {
        "freestream_m05": (small.freestream(), 0.5),
        "seed0_m085": (seeded_state(small, 0), 0.85),
        "accelerating_m08": (pocket_state(small, "accelerating"), 0.8),
        "shockpoint_m08": (pocket_state(small, "shockpoint"), 0.8),
        "mixed_m08": (pocket_state(small, "mixed"), 0.8),
        "limited_m08": (2.5 * pocket_state(small, "mixed"), 0.8),
    }
    make_case(jac, upw_mod, isen, "small_bump", small, s_states, full=True)

    c1 = bump_channel(40, 10, 10, amplitude=0.05, seed=0)
    c1_states = {
        "seed0_m05": (seeded_state(c1, 0), 0.5),
        "mixed_m08": (pocket_state(c1, "mixed"), 0.8),
    }
    make_case(jac, upw_mod, isen, "c1_bump", c1, c1_states, full=False)
    make_picard("c1_picard", c1, 0.5)
    _weighted(jac, upw_mod, isen)
    make_wake(jac, upw_mod, isen, "wake_constraint")
    make_wall("wall_forces")
    make_sides(jac, upw_mod, isen, "side_terms")
    make_lifting("lifting_newton")
    make_naca(ref_root, "naca_coarse")
    make_swept_cut("swept_cut")
    make_lifting_picard("lifting_picard")
    make_weighted_picard("weighted_picard")
    make_lagged_lu("lagged_lu")
    make_multivalued("multivalued")
    make_te_pressure("te_pressure")


def _weighted(jac, upw_mod, isen):
    small = bump_channel(10, 4, 3, amplitude=0.08, seed=1)
    w_states = {
        "freestream_m05": (small.freestream(), 0.5),
        "seed0_m085": (seeded_state(small, 0), 0.85),
        "accelerating_m08": (pocket_state(small, "accelerating"), 0.8),
        "shockpoint_m08": (pocket_state(small, "shockpoint"), 0.8),
        "mixed_m08": (pocket_state(small, "mixed"), 0.8),
        "supersonic_m08": (1.3 * small.freestream(), 0.8),
    }
    make_weighted(jac, upw_mod, isen, "weighted_upwind", small, w_states)


if __name__ == "__main__":
    main()
