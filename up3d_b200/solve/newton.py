"""Non-lifting transonic Newton solve on the B200.

The reference's coupled Newton driver (pyfp3d/solve/newton.py:516-1141,
``solve_newton_lifting``) and its Mach continuation (:1144-1307,
``solve_newton_transonic``) restricted to the wake-free channel: T = I, no
circulation unknowns, Dirichlet inflow/outflow.  The per-iteration chain is
the same -- exact Jacobian with Eisenstat-Walker forcing, GMRES(60) with a
smoothed-aggregation AMG preconditioner built on the Picard block every
``amg_rebuild_every`` steps, a merit line search with at most five
halvings, the level fail-fast, and the frozen (upstream, branch) finish once
the residual drops below ``freeze_tol`` -- with every vector on the device:
the residual and Jacobian come from one fused evaluation, and only scalars
(norms, monitors) return to the host.

``precision="mixed"`` runs the linear solve as FP64 iterative refinement
around an FP32 preconditioner (FP32 AMG); the residual, the Newton update
and the convergence test stay FP64.
"""

from __future__ import annotations

import time
from typing import Dict, Optional

import numpy as np

from .. import _lib as L
from ..mesh.device import DeviceMesh, get_mesh
from .fused import FlowParams, ResidualJacobian
from .linear import amg_for, solve_cg, solve_gmres, solve_gmres_mixed, with_dirichlet


def _ew_forcing(r_norm, r_norm_prev, eta_prev, eta0=1e-2, gamma_ew=0.9, eta_max=1e-2,
                eta_floor=1e-10):
    """Eisenstat-Walker choice 2 with safeguard (pyfp3d/solve/newton.py:504-513)."""
    if r_norm_prev is None:
        return eta0
    eta = gamma_ew * (r_norm / r_norm_prev) ** 2
    safeguard = gamma_ew * eta_prev ** 2
    if safeguard > 0.1:
        eta = max(eta, safeguard)
    return float(min(eta_max, max(eta, eta_floor)))


def mach_schedule(m_target: float, m_start: float = 0.70, dm: float = 0.05):
    """Ascending Mach ramp ending exactly at m_target
    (pyfp3d/solve/continuation.py:72-78)."""
    if m_target <= m_start:
        return [float(m_target)]
    ms = list(np.arange(m_start, m_target - 1e-12, dm))
    ms.append(m_target)
    return [float(m) for m in ms]


class ChannelWorkspace:
    """Per-mesh device state of the channel solves: the mesh, the fused
    evaluator, the Dirichlet split and the Picard operator."""

    # meshes from this size on get their launch shapes autotuned once
    TUNE_MIN_TETS = 100_000

    def __init__(self, nodes, elements, dirichlet_nodes, u_inf: float = 1.0,
                 mesh: Optional[DeviceMesh] = None, tune: bool = True):
        t = L.require_cuda()
        self.mesh = mesh if mesh is not None else get_mesh(nodes, elements)
        from ..kernels.jacobian import PicardOperator
        self.op = PicardOperator(t.as_tensor(np.asarray(self.mesh.nodes)),
                                 t.as_tensor(np.asarray(self.mesh.elements)), mesh=self.mesh)
        self.ev = ResidualJacobian(self.mesh)
        n = self.mesh.n_nodes
        self.u_inf = float(u_inf)
        self.dn = L.to_device(np.asarray(dirichlet_nodes), t.int64)
        self.mask = t.zeros(n, dtype=t.uint8, device="cuda")
        self.mask[self.dn] = 1
        self.free = self.mask == 0
        x = t.from_numpy(np.ascontiguousarray(self.mesh.nodes[:, 0])).cuda()
        self.phi_dir = t.zeros(n, dtype=t.float64, device="cuda")
        self.phi_dir[self.dn] = self.u_inf * x[self.dn]
        self.freestream = self.u_inf * x
        if tune and self.mesh.n_tets >= self.TUNE_MIN_TETS and self.mesh.tuning()["elem_us"] == 0.0:
            # launch shapes timed at the freestream (every element walks);
            # every shape computes the same bits
            self.mesh.autotune(self.freestream, FlowParams(m_inf=0.7, u_inf=self.u_inf))

    def residual(self, phi, flow: FlowParams, frozen=None, jacobian=False):
        """R (device view), monitors; R on constrained rows is ignored."""
        self.ev.evaluate(phi, flow, jacobian=jacobian, frozen=frozen, keep_state=True)
        return self.ev.R, self.ev.read_monitors()

    def r_free(self, R):
        return R.masked_fill(self.mask.bool(), 0.0)

    def picard_matrix(self):
        return with_dirichlet(self.op.assemble_matrix(self.ev.rho_tilde), self.mask)

    def freeze(self, phi, flow: FlowParams):
        """(upstream, branch) at phi, kernels/upwind.py:821-843."""
        from ..kernels.upwind import UpwindOperator
        from ..physics.isentropic import density_field, limit_q2_field
        t = L.torch()
        grad, q2 = self.op.velocities(phi)
        q2l = limit_q2_field(q2 / flow.u_inf ** 2, flow.m_inf, flow.m_cap, flow.gamma)
        rho = density_field(q2l, flow.m_inf, flow.gamma)
        if not hasattr(self, "_upw"):
            self._upw = UpwindOperator(t.as_tensor(np.asarray(self.mesh.nodes)),
                                       t.as_tensor(np.asarray(self.mesh.elements)), mesh=self.mesh)
        up, br = self._upw.freeze_upwind_state(grad, q2l, rho, flow.m_inf, flow.upwind_c,
                                               flow.m_crit, flow.gamma, flow.rho_floor)
        return up.clone(), br.clone()


def picard_seed(ws: ChannelWorkspace, flow: FlowParams, phi, n_iter: int = 5, rtol: float = 1e-7,
                amg_fp32=False):
    """Upwinded density Picard warm start (the seed of
    pyfp3d/solve/newton.py:708-720): A(rho_tilde(phi)) phi_new = b."""
    t = L.torch()
    for _ in range(n_iter):
        ws.residual(phi, flow)
        A = ws.op.assemble_matrix(ws.ev.rho_tilde)
        rhs = -A.matvec(ws.phi_dir)
        rhs[ws.dn] = 0.0
        Af = with_dirichlet(A, ws.mask)
        ws.amg = M = amg_for(Af, getattr(ws, "amg", None), fp32=amg_fp32)
        x, _, info = solve_cg(Af, rhs, M=M, rtol=rtol, maxiter=2000,
                              x0=t.where(ws.free, phi, t.zeros_like(phi)))
        phi = t.where(ws.free, x, ws.phi_dir)
    return phi


def solve_newton(ws: ChannelWorkspace, flow: FlowParams, phi_init=None, n_picard_seed: int = 5,
                 n_newton_max: int = 30, tol_residual: float = 1e-10, amg_rebuild_every: int = 2,
                 gmres_restart: int = 60, gmres_maxiter: int = 10, line_search: bool = True,
                 freeze_tol: Optional[float] = None, freeze_refresh_max: int = 2,
                 freeze_max_reverts: int = 3, precision: str = "fp64",
                 verbose: bool = False) -> Dict[str, object]:
    """Newton at one Mach level (pyfp3d/solve/newton.py:516-1141 without
    the wake / Kutta blocks)."""
    t = L.require_cuda()
    if precision not in ("fp64", "mixed"):
        raise ValueError(f"precision must be 'fp64' or 'mixed', not {precision!r}")
    # mixed: one hierarchy with both cycles -- FP64 for the Picard seed's CG
    # (FP64 vectors), FP32 inside the refined GMRES (FP32 vectors)
    amg_fp32 = "both" if precision == "mixed" else False
    timings = {"seed": 0.0, "assembly": 0.0, "precond": 0.0, "linsolve": 0.0, "residual": 0.0}

    def clock():
        t.cuda.synchronize()
        return time.perf_counter()

    t_wall0 = clock()
    if phi_init is not None:
        phi = L.to_device(phi_init, t.float64).clone()
        phi = t.where(ws.free, phi, ws.phi_dir)
    elif n_picard_seed > 0:
        phi = picard_seed(ws, flow, ws.freestream.clone(), n_picard_seed, amg_fp32=amg_fp32)
    else:
        phi = ws.freestream.clone()
    timings["seed"] = clock() - t_wall0

    residual_history, eta_history, newton_orders = [], [], []
    n_gmres_total = n_gmres_stalled = n_refine_total = 0
    converged = False
    M_pre = None
    eta_prev = None
    frozen = None
    freeze_point = None
    freeze_cooldown = 0
    n_freeze_reverts = n_freeze_refresh = 0
    freeze_armed = freeze_tol is not None
    prev_live_residual = None
    residual_unfrozen = None
    r_level_best = np.inf

    a = clock()
    R, mon = ws.residual(phi, flow, frozen=frozen)
    Rf = ws.r_free(R)
    merit = float(Rf @ Rf)
    timings["residual"] += clock() - a

    for it in range(n_newton_max):
        r_norm = float(Rf.abs().max())
        residual_history.append(r_norm)
        if len(residual_history) >= 3:
            r2, r1, r0 = residual_history[-1], residual_history[-2], residual_history[-3]
            if r2 > 0 and r1 > 0 and r0 > 0 and r1 != r0:
                newton_orders.append(float(np.log(r2 / r1) / np.log(r1 / r0)))
        if verbose:
            print(f"  newton {it:2d}: |R|={r_norm:.3e} lim={mon['n_limited']} "
                  f"flr={mon['n_floored']} sup={mon['n_supersonic']}"
                  + (" [frozen]" if frozen is not None else ""))
        r_level_best = min(r_level_best, r_norm)
        clean = mon["n_limited"] == 0 and mon["n_floored"] == 0

        if frozen is not None and freeze_point is not None:
            if r_norm > 10.0 * freeze_point[1] or not clean:
                phi = freeze_point[0].clone()
                frozen = freeze_point = None
                freeze_cooldown = 5
                n_freeze_reverts += 1
                r_level_best = np.inf
                if n_freeze_reverts >= freeze_max_reverts:
                    freeze_armed = False
                R, mon = ws.residual(phi, flow)
                Rf = ws.r_free(R)
                merit = float(Rf @ Rf)
                continue
        if freeze_cooldown > 0:
            freeze_cooldown -= 1
        if r_norm > 100.0 * r_level_best and r_norm > 1e-3:
            break
        live_stalled = (len(residual_history) >= 7 and r_norm < 1e-3
                        and r_norm > 0.25 * min(residual_history[-7:-1])
                        and r_norm < 2.0 * min(residual_history[-7:-1]))
        if (frozen is None and freeze_armed and freeze_cooldown == 0 and flow.m_inf > 0.0
                and (r_norm < freeze_tol or live_stalled) and clean):
            frozen = ws.freeze(phi, flow)
            freeze_point = (phi.clone(), r_norm)
            r_level_best = np.inf
        if clean and r_norm < tol_residual:
            if frozen is None:
                converged = True
                break
            R_live, mon_live = ws.residual(phi, flow)
            residual_unfrozen = float(ws.r_free(R_live).abs().max())
            if residual_unfrozen < tol_residual:
                converged = True
                R, mon = R_live, mon_live
                break
            if prev_live_residual is not None and residual_unfrozen > 0.5 * prev_live_residual:
                converged = True
                break
            if n_freeze_refresh >= freeze_refresh_max:
                converged = True
                break
            prev_live_residual = residual_unfrozen
            n_freeze_refresh += 1
            frozen = ws.freeze(phi, flow)
            freeze_point = (phi.clone(), residual_unfrozen)
            r_level_best = np.inf
            R, mon = ws.residual(phi, flow, frozen=frozen)
            Rf = ws.r_free(R)
            merit = float(Rf @ Rf)
            continue

        # exact Jacobian at the current state (and the Picard block)
        a = clock()
        ws.residual(phi, flow, frozen=frozen, jacobian=True)
        J = ws.ev.jacobian()
        Jf = with_dirichlet(J, ws.mask)
        timings["assembly"] += clock() - a
        a = clock()
        if M_pre is None or it % amg_rebuild_every == 0:
            # a rebuild on the fixed P1 pattern is a refresh of the values
            ws.amg = M_pre = amg_for(ws.picard_matrix(), getattr(ws, "amg", None), fp32=amg_fp32)
        timings["precond"] += clock() - a
        eta = _ew_forcing(r_norm, residual_history[-2] if it > 0 else None, eta_prev)
        eta_prev = eta
        eta_history.append(eta)
        a = clock()
        rhs = -Rf
        if precision == "mixed":
            # FP32 Jacobian values and FP32 AMG inside FP64-refined GMRES,
            # the FP64 solve's restart, criterion and step cap
            dphi, n_it, n_ref, info = solve_gmres_mixed(Jf, rhs, M=M_pre, rtol=eta, restart=gmres_restart,
                                                        maxiter=gmres_maxiter, refine_max=10,
                                                        inner_rtol=1e-5)
            n_refine_total += n_ref
        else:
            dphi, n_it, info = solve_gmres(Jf, rhs, M=M_pre, rtol=eta, restart=gmres_restart,
                                           maxiter=gmres_maxiter, on_fail="return")
        timings["linsolve"] += clock() - a
        n_gmres_total += n_it
        n_gmres_stalled += info != 0
        dphi = dphi.masked_fill(ws.mask.bool(), 0.0)

        lam, best, accepted = 1.0, None, False
        a = clock()
        for _ in range(5):
            phi_try = phi + lam * dphi
            R_try, mon_try = ws.residual(phi_try, flow, frozen=frozen)
            Rf_try = ws.r_free(R_try)
            merit_try = float(Rf_try @ Rf_try)
            if np.isfinite(merit_try) and (not line_search or merit_try <= merit):
                accepted = True
                break
            if np.isfinite(merit_try) and (best is None or merit_try < best[0]):
                best = (merit_try, lam, phi_try.clone(), mon_try)
            lam *= 0.5
        if not accepted:
            if best is None:
                raise RuntimeError(f"Newton line search failed at iteration {it}")
            merit_try, lam, phi_try, mon_try = best
            R_try, mon_try = ws.residual(phi_try, flow, frozen=frozen)
            Rf_try = ws.r_free(R_try)
        timings["residual"] += clock() - a
        phi = phi_try
        R, mon, Rf, merit = R_try, mon_try, Rf_try, merit_try

    timings["wall"] = clock() - t_wall0
    return {"phi": phi, "converged": converged,
            "n_newton": len(residual_history) - (1 if converged else 0),
            "residual_history": residual_history, "eta_history": eta_history,
            "newton_orders": newton_orders, "n_gmres_total": n_gmres_total,
            "n_gmres_stalled": n_gmres_stalled, "n_refinements": n_refine_total,
            "froze": frozen is not None,
            "frozen_state": frozen,
            "n_freeze_refresh": n_freeze_refresh, "residual_unfrozen": residual_unfrozen,
            "n_freeze_reverts": n_freeze_reverts, "nu_max": mon["nu_max"],
            "n_supersonic": mon["n_supersonic"], "n_limited": mon["n_limited"],
            "n_floored": mon["n_floored"], "n_term3_active": mon["n_term3_active"],
            "timings": timings}


def solve_newton_transonic(first, *args, **kw) -> Dict[str, object]:
    """Upward Mach continuation (pyfp3d/solve/newton.py:1144-1307).  With a
    cut mesh and its WakeCut first -- the reference's signature
    (mesh_cut, wc, m_inf, alpha_deg, ...) -- the coupled lifting solve
    (solve.lifting.solve_newton_transonic); with a ChannelWorkspace first,
    the wake-free channel solve (solve_channel_transonic)."""
    if isinstance(first, ChannelWorkspace):
        return solve_channel_transonic(first, *args, **kw)
    from .lifting import solve_newton_transonic as lifting
    return lifting(first, *args, **kw)


def __getattr__(name):
    # the reference's module also holds the coupled lifting workspace and
    # driver (solve/newton.py:97-1141); they live in solve.lifting
    if name in ("NewtonWorkspace", "solve_newton_lifting"):
        from . import lifting
        return getattr(lifting, name)
    raise AttributeError(name)


def solve_channel_transonic(ws: ChannelWorkspace, m_inf: float, m_start: float = 0.70,
                            dm: float = 0.05, dm_min: float = 0.01, freeze_tol: Optional[float] = 1e-6,
                            precision: str = "fp64", verbose: bool = False,
                            **newton_kw) -> Dict[str, object]:
    """Upward Mach continuation of the channel solve (the ramp of
    pyfp3d/solve/newton.py:1144-1307 without the wake): each level
    warm-starts from the previous converged level; a failed level is
    retried with the Mach step halved down to dm_min."""
    t = L.require_cuda()
    t0 = time.perf_counter()
    levels = mach_schedule(m_inf, m_start, dm)
    level_history = []
    last_good = None
    result = None
    i = 0
    while i < len(levels):
        m = levels[i]
        flow = FlowParams(m_inf=m, u_inf=ws.u_inf)
        kw = dict(newton_kw)
        kw.setdefault("freeze_tol", freeze_tol)
        if last_good is not None:
            kw.update(phi_init=last_good["phi"], n_picard_seed=0)
        if verbose:
            print(f"newton continuation level M = {m:.4f}")
        result = solve_newton(ws, flow, precision=precision, verbose=verbose, **kw)
        level_history.append((m, result["n_newton"], result["residual_history"][-1],
                              result["n_gmres_total"]))
        if not result["converged"]:
            m_prev = m_start if i == 0 else levels[i - 1]
            dm_new = 0.5 * (m - m_prev)
            if i == 0 or dm_new < dm_min:
                break
            levels.insert(i, m_prev + dm_new)
            continue
        last_good = result
        i += 1
    t.cuda.synchronize()
    result = dict(result)
    result["level_history"] = level_history
    result["wall_total"] = time.perf_counter() - t0
    return result
