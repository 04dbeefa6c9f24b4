"""Non-lifting subsonic Picard solve on the B200 (pyfp3d/solve/picard.py:
271-417, ``solve_subsonic``): relaxed density Picard, each outer iteration
assembling A(rho) on the device, building the AMG hierarchy and solving the
free-DOF system with CG+AMG, all vectors device-resident.  Only the
convergence scalars return to the host.
"""

from __future__ import annotations

import time
from typing import Dict, Optional

import numpy as np

from .. import _lib as L
from ..kernels.jacobian import PicardOperator
from ..physics.isentropic import density_field, mach_squared_field
from .linear import amg_for, solve_cg, with_dirichlet


def solve_subsonic(nodes, elements, dirichlet_nodes, dirichlet_values, m_inf: float,
                   gamma_air: float = 1.4, u_inf: float = 1.0, body_source_rhs=None,
                   phi_init=None, omega: float = 1.0, n_picard_max: int = 40,
                   tol_rho: float = 1e-10, rtol: float = 1e-12, maxiter: int = 3000,
                   amg_fp32: bool = False) -> Dict[str, object]:
    """Same arguments and result keys as the reference; the result also
    carries ``timings`` (assembly / precond / linsolve / residual seconds)."""
    t = L.require_cuda()
    t0 = time.perf_counter()
    op = PicardOperator(t.as_tensor(np.asarray(nodes)), t.as_tensor(np.asarray(elements)))
    n = op.n_nodes
    dn = L.to_device(np.asarray(dirichlet_nodes), t.int64)
    vals = L.to_device(np.asarray(dirichlet_values, dtype=np.float64), t.float64)
    mask = t.zeros(n, dtype=t.uint8, device="cuda")
    mask[dn] = 1
    free = mask == 0
    b_wall = None
    if body_source_rhs is not None:
        b_wall = L.to_device(body_source_rhs, t.float64)
        if b_wall.shape != (n,):
            raise ValueError(f"body_source_rhs must be ({n},), got {tuple(b_wall.shape)}")
    if phi_init is not None:
        phi = L.to_device(phi_init, t.float64).clone()
        phi[dn] = vals
        _, q2 = op.velocities(phi)
        rho = density_field(q2 / u_inf ** 2, m_inf, gamma_air).clone()
    else:
        phi = t.zeros(n, dtype=t.float64, device="cuda")
        phi[dn] = vals
        rho = t.ones(op.n_tets, dtype=t.float64, device="cuda")
    phi_dir = t.zeros(n, dtype=t.float64, device="cuda")
    phi_dir[dn] = vals

    timings = {"assembly": 0.0, "precond": 0.0, "linsolve": 0.0, "residual": 0.0}
    residual_history, drho_history = [], []
    n_cg_total = 0
    converged = False

    def tick():
        t.cuda.synchronize()
        return time.perf_counter()

    M = None
    for _ in range(n_picard_max):
        a = tick()
        A = op.assemble_matrix(rho)
        # b_free = -A[free][:, dir] vals (+ b_wall[free]), embedded in full size
        rhs = -A.matvec(phi_dir)
        if b_wall is not None:
            rhs = rhs + b_wall
        rhs[dn] = 0.0
        Af = with_dirichlet(A, mask)
        b2 = tick()
        timings["assembly"] += b2 - a
        M = amg_for(Af, M, fp32=amg_fp32)
        c = tick()
        timings["precond"] += c - b2
        x, n_it, info = solve_cg(Af, rhs, M=M, rtol=rtol, maxiter=maxiter)
        if info != 0:
            raise RuntimeError(f"CG did not converge (info={info})")
        n_cg_total += n_it
        d = tick()
        timings["linsolve"] += d - c
        phi_new = t.where(free, x, phi_dir)
        phi = phi_new if omega == 1.0 else phi + omega * (phi_new - phi)
        _, q2 = op.velocities(phi)
        rho_new = density_field(q2 / u_inf ** 2, m_inf, gamma_air).clone()
        R = op.assemble_residual(phi, rho_new)
        if b_wall is not None:
            R = R - b_wall
        res = float(R[free].abs().max())
        drho = float((rho_new - rho).abs().max())
        residual_history.append(res)
        drho_history.append(drho)
        rho = rho_new
        timings["residual"] += tick() - d
        if drho < tol_rho:
            converged = True
            break

    _, q2 = op.velocities(phi)
    mach2_max = float(mach_squared_field(q2 / u_inf ** 2, m_inf, gamma_air).max())
    timings["wall"] = time.perf_counter() - t0
    return {"phi": phi.cpu().numpy(), "n_picard": len(residual_history), "converged": converged,
            "residual_history": residual_history, "drho_history": drho_history,
            "rho": rho.cpu().numpy(), "mach2_max": mach2_max, "n_cg_total": n_cg_total,
            "timings": timings}


def __getattr__(name):
    # the reference's module also holds the nested lifting Picard
    # (solve/picard.py:420-883); it lives in solve.lifting
    if name == "solve_subsonic_lifting":
        from .lifting import solve_subsonic_lifting
        return solve_subsonic_lifting
    raise AttributeError(name)
