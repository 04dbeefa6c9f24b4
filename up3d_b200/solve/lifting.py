"""Wake-coupled (lifting) Newton solve on the B200.

``NewtonWorkspace`` and ``solve_newton_lifting`` keep the signatures of
pyfp3d/solve/newton.py:97-1141 for the "probe" Kutta estimator: the
unknowns are the free reduced potentials phi_f and the station
circulations Gamma; far-field values are affine in Gamma (set_mach's basis
vals0 + V Gamma); the wake sheet's "+"-side copies follow
phi_cut = T phi_red + G Gamma.  Each Newton step eliminates the Kutta rows
(F = taper * kutta_targets(phi_cut) - Gamma, dF/dphi_f = K,
dF/dGamma = -I) and solves

    (J_ff + B K) dphi = -R_f - B F,   dGamma = K dphi + F,

with B = J_red[free, dir] V + H_J[free], by GMRES(60) preconditioned with
smoothed-aggregation AMG on the reduced Picard block.  On the device none of
J_red, J_ff or B is formed: the coupled operator is one expand, one SpMV of
the cut-mesh Jacobian (Term 3 included) and one fold (up3d_coupled_apply),
so the same cut-mesh Jacobian the fused evaluation writes serves the
solve.  Vectors are reduced-size CUDA tensors with the far-field rows
carried as identity rows; only norms and monitors return to the host.

``solve_subsonic_lifting`` is the nested lifting Picard
(pyfp3d/solve/picard.py:420-883), also the Newton driver's warm start.

kutta_estimator="pressure" replaces the probe row by the pressure
equality on wall-adjacent TE control volumes (constraints/te_pressure.py):
its state-dependent eliminated row -D^-1 K_p is rebuilt on the host per
Newton step (n_stations rows over the TE fans' nodes) and uploaded to the
coupled handle.  precond="direct" takes exact steps (dense LU of the
reduced J_ff on the device with the Woodbury update for the Kutta
coupling), with direct_refactor_every > 1 GMRES steps on a stale LU in
between; precond="ilu" preconditions GMRES with a device ILU(0) of the
reduced J_ff, rebuilt every step (the reference's host threshold ILU has no
device form; see solve.linear.build_ilu_preconditioner).
"""

from __future__ import annotations

import ctypes
import time
from typing import Dict, Optional

import numpy as np

from .. import _lib as L
from ..constraints.dirichlet import FarfieldBasis, freestream_phi, kutta_row
from ..constraints.wake import WakeConstraint
from ..mesh.device import DeviceCSR, device_view, get_mesh
from .fused import FlowParams, ResidualJacobian
from .linear import _csr_struct, amg_for, build_ilu_preconditioner
from .newton import _ew_forcing


class CoupledOperator:
    """J_ff + B K of one Newton step (the cut-mesh Jacobian J bound to a
    workspace's coupled handle)."""

    def __init__(self, ws: "NewtonWorkspace", J: DeviceCSR):
        self.ws = ws
        self.J = J
        self.shape = (ws.n_red, ws.n_red)
        self._c = _csr_struct(J, None)

    def apply(self, x, g=None):
        """(J_ff x + B (K x + g), K x + g), reduced-size x (far-field rows
        pass through)."""
        t = L.torch()
        y = t.empty(self.ws.n_red, dtype=t.float64, device="cuda")
        tv = t.empty(max(self.ws.n_st, 1), dtype=t.float64, device="cuda")
        L.call("up3d_coupled_apply", self.ws._coupled, ctypes.byref(self._c), None, x.data_ptr(),
               L.ptr(g), y.data_ptr(), tv.data_ptr(), L.stream_ptr())
        return y, tv[:self.ws.n_st]

    def matvec(self, x):
        return self.apply(x)[0]

    __matmul__ = matvec

    def solve(self, b, M=None, rtol=1e-5, atol=0.0, restart=60, maxiter=10, x0=None):
        """GMRES on this operator (up3d_gmres_coupled): (x, inner steps,
        info) with info 0 when converged."""
        t = L.torch()
        x = t.zeros_like(b) if x0 is None else x0.clone()
        inner, resid, info = ctypes.c_int64(), ctypes.c_double(), ctypes.c_int()
        L.call("up3d_gmres_coupled", self.ws._coupled, ctypes.byref(self._c), None, b.data_ptr(),
               x.data_ptr(), float(rtol), float(atol), int(restart), int(maxiter),
               None if M is None else M.handle, ctypes.byref(inner), ctypes.byref(resid),
               ctypes.byref(info), L.stream_ptr())
        return x, int(inner.value), int(info.value)


class NewtonWorkspace:
    """Per-case device state of the coupled Newton solve
    (pyfp3d/solve/newton.py:97-324): the cut mesh and its fused evaluator,
    the wake fold, the far-field split, the Kutta row K and, per Mach level,
    the far-field basis."""

    TUNE_MIN_TETS = 100_000

    def __init__(self, mesh_cut, wc, alpha_deg: float = 0.0, u_inf: float = 1.0,
                 gamma_air: float = 1.4, vortex_center=(0.25, 0.0),
                 farfield_spanwise_gamma: bool = False, tip_taper=None,
                 kutta_estimator: str = "probe", external_rhs=None, tune: bool = True):
        t = L.require_cuda()
        if kutta_estimator not in ("probe", "pressure"):
            raise ValueError(f"unknown kutta_estimator {kutta_estimator!r}")
        self.mesh_cut, self.wc = mesh_cut, wc
        self.alpha_deg, self.u_inf, self.gamma_air = float(alpha_deg), float(u_inf), float(gamma_air)
        self.vortex_center = tuple(vortex_center)
        self.spanwise = bool(farfield_spanwise_gamma)
        self.kutta_estimator = kutta_estimator
        n_st = wc.n_stations
        self.tip_taper = (np.ones(n_st) if tip_taper is None
                          else np.asarray(tip_taper, dtype=np.float64).copy())
        if self.tip_taper.shape != (n_st,):
            raise ValueError(f"tip_taper must be ({n_st},), got {self.tip_taper.shape}")
        nodes = np.asarray(mesh_cut.nodes, dtype=np.float64)
        self.mesh = get_mesh(nodes, mesh_cut.elements)
        self.ev = ResidualJacobian(self.mesh)
        from ..kernels.jacobian import PicardOperator
        self.op = PicardOperator(t.as_tensor(nodes), t.as_tensor(np.asarray(self.mesh.elements)), mesh=self.mesh)
        self.external_rhs = None
        if external_rhs is not None:
            b = np.asarray(external_rhs, dtype=np.float64)
            if b.shape != (len(nodes),):
                raise ValueError(f"external_rhs must be ({len(nodes)},) on the cut mesh, got {b.shape}")
            self.external_rhs = L.to_device(b, t.float64)
        # the wake fold on the cut mesh's P1 pattern (the Picard block's)
        A0 = self.op.assemble_matrix(t.ones(self.mesh.n_tets, dtype=t.float64, device="cuda"))
        self.con = WakeConstraint(A0, wc)
        self._plan = self.con._plan            # keeps the wake handle alive
        self.n_red, self.n_st = self.con.n_reduced, n_st
        # far-field split (Gamma-, rho- and beta-independent) and the Kutta row
        self.basis = FarfieldBasis(mesh_cut, wc, self.alpha_deg, self.u_inf, self.vortex_center,
                                   self.spanwise)
        self.dir_red, self.free = self.basis.dir_red, self.basis.free
        self.n_free = len(self.free)
        K = self.K = kutta_row(wc, self.basis.is_dir, self.tip_taper)
        self._taper_active = not np.all(self.tip_taper == 1.0)
        # pressure estimator: TE control volumes and the frozen scaling
        self.cvs = None
        self.kutta_sigma = self.kutta_weld_sign = None
        self.kutta_sigma_sign_flips = 0
        if kutta_estimator == "pressure":
            from ..constraints.te_pressure import TEControlVolumes
            self.cvs = TEControlVolumes(mesh_cut, wc, dirichlet_nodes=self.basis.dir_cut,
                                        geometry=self.mesh.geometry())
            red_of = np.arange(len(nodes), dtype=np.int64)
            red_of[np.asarray(wc.slave_nodes, dtype=np.int64)] = np.asarray(wc.master_nodes, dtype=np.int64)
            import scipy.sparse as sp
            self._T = sp.csr_matrix((np.ones(len(nodes)), (np.arange(len(nodes)), red_of)),
                                    shape=(len(nodes), self.n_red))
        h = ctypes.c_void_p()
        dr = np.ascontiguousarray(self.dir_red, dtype=np.int64)
        kp = np.ascontiguousarray(K.indptr, dtype=np.int64)
        kc = np.ascontiguousarray(K.indices, dtype=np.int64)
        kv = np.ascontiguousarray(K.data, dtype=np.float64)
        ts = np.ascontiguousarray(wc.te_station, dtype=np.int64)
        ku = np.ascontiguousarray(wc.kutta_upper, dtype=np.int64)
        kl = np.ascontiguousarray(wc.kutta_lower, dtype=np.int64)
        tp = np.ascontiguousarray(self.tip_taper, dtype=np.float64)
        L.call("up3d_coupled_create", self._plan.handle, len(dr), dr.ctypes.data, kp.ctypes.data,
               kc.ctypes.data, kv.ctypes.data, len(ts), ts.ctypes.data, ku.ctypes.data, kl.ctypes.data,
               tp.ctypes.data, ctypes.byref(h))
        self._coupled = h.value
        mp = ctypes.c_void_p()
        L.call("up3d_coupled_dirichlet", self._coupled, ctypes.byref(mp))
        self.mask = device_view(mp.value, (self.n_red,), np.uint8)
        self.m_inf = self.beta = self.vals0_red = self.V_red = None
        self.amg = None
        if tune and self.mesh.n_tets >= self.TUNE_MIN_TETS and self.mesh.tuning()["elem_us"] == 0.0:
            fs = L.to_device(freestream_phi(nodes, self.alpha_deg, self.u_inf), t.float64)
            self.mesh.autotune(fs, FlowParams(m_inf=0.7, u_inf=self.u_inf))

    def __del__(self):
        h = getattr(self, "_coupled", None)
        if h:
            try:
                L.lib().up3d_coupled_destroy(h)
            except Exception:
                pass
            self._coupled = None

    def set_mach(self, m_inf: float) -> None:
        """Prandtl-Glauert beta and the far-field basis vals0 + V Gamma
        (newton.py:295-324)."""
        if not 0.0 <= m_inf < 1.0:
            raise ValueError(f"Newton driver needs 0 <= M_inf < 1, got {m_inf}")
        self.m_inf = float(m_inf)
        self.beta = float(np.sqrt(1.0 - m_inf ** 2))
        self.vals0_red, self.V_red = self.basis.at_mach(self.beta)
        v0c = np.ascontiguousarray(self.vals0_red)
        Vc = np.ascontiguousarray(self.V_red)
        L.call("up3d_coupled_set_farfield", self._coupled, v0c.ctypes.data, Vc.ctypes.data)

    def flow(self, upwind_c=1.5, m_crit=0.95, m_cap=3.0, rho_floor=0.05) -> FlowParams:
        return FlowParams(m_inf=self.m_inf, gamma=self.gamma_air, u_inf=self.u_inf, m_cap=m_cap,
                          m_crit=m_crit, upwind_c=upwind_c, rho_floor=rho_floor)

    def eval_residual(self, phi_f, gamma, upwind_c: float, m_crit: float, m_cap: float,
                      rho_floor: float, frozen=None, jacobian: bool = False):
        """(R_f, F, state) at (phi_f, Gamma) (newton.py:326-428): phi_f a
        reduced-size CUDA tensor (far-field rows ignored), R_f reduced-size
        with zeros on the far-field rows.  jacobian=True also leaves the
        cut-mesh Jacobian in the evaluator (assemble_coupled reads it)."""
        t = L.torch()
        phi_f = L.to_device(phi_f, t.float64)
        g = L.to_device(np.atleast_1d(gamma) if not L.is_torch(gamma) else gamma, t.float64)
        phi_red = t.empty(self.n_red, dtype=t.float64, device="cuda")
        phi_cut = t.empty(self.mesh.n_nodes, dtype=t.float64, device="cuda")
        L.call("up3d_coupled_state", self._coupled, phi_f.data_ptr(), g.data_ptr(), phi_red.data_ptr(),
               phi_cut.data_ptr(), L.stream_ptr())
        flow = self.flow(upwind_c, m_crit, m_cap, rho_floor)
        self.ev.evaluate(phi_cut, flow, jacobian=jacobian, frozen=frozen, keep_state=True)
        R_cut = self.ev.R if self.external_rhs is None else self.ev.R - self.external_rhs
        R_red = t.empty(self.n_red, dtype=t.float64, device="cuda")
        F = t.empty(max(self.n_st, 1), dtype=t.float64, device="cuda")
        L.call("up3d_coupled_residual", self._coupled, R_cut.data_ptr(), phi_cut.data_ptr(), g.data_ptr(),
               R_red.data_ptr(), F.data_ptr(), L.stream_ptr())
        if self.cvs is not None:
            F = L.to_device(self._pressure_F(phi_cut, g.cpu().numpy()), t.float64)
        mon = self.ev.read_monitors()
        state = {"phi_red": phi_red, "phi_cut": phi_cut, "gamma": g, "flow": flow, "frozen": frozen,
                 "n_limited": mon["n_limited"], "n_floored": mon["n_floored"], "nu_max": mon["nu_max"],
                 "n_nu_active": mon["n_supersonic"], "n_term3_active": mon["n_term3_active"],
                 "jacobian": jacobian}
        return R_red, F[:self.n_st], state

    def assemble_coupled(self, state, upwind_c: float = 1.5, m_crit: float = 0.95,
                         rho_floor: float = 0.05, frozen=None) -> CoupledOperator:
        """The coupled operator J_ff + B K at the state of eval_residual
        (newton.py:430-457): the evaluation is redone with the Jacobian
        unless it already produced it."""
        if not state.get("jacobian"):
            self.ev.evaluate(state["phi_cut"], state["flow"], jacobian=True, frozen=frozen, keep_state=True)
            state["jacobian"] = True
            state["n_term3_active"] = self.ev.read_monitors()["n_term3_active"]
        return CoupledOperator(self, self.ev.jacobian())

    def _pressure_F(self, phi_cut, gamma):
        """sigma F_raw, or with a tip taper the blend taper sigma F_raw +
        (1 - taper) s Gamma; sigma and s frozen at the first evaluation
        (newton.py:376-416)."""
        F_raw = self.cvs.residual_stations(phi_cut)
        if self.kutta_sigma is None:
            dj = np.diag(self.cvs.gamma_jacobian(phi_cut, mode="exact"))
            ref = np.sign(np.median(dj))
            self.kutta_sigma_sign_flips = int(np.count_nonzero(np.sign(dj) != ref))
            a = np.abs(dj)
            self.kutta_sigma = 1.0 / np.maximum(a, 0.1 * np.median(a))
            sg = np.sign(dj)
            self.kutta_weld_sign = np.where(sg == 0.0, ref, sg)
        if not self._taper_active:
            return self.kutta_sigma * F_raw
        return (self.kutta_sigma * (self.tip_taper * F_raw)
                + (1.0 - self.tip_taper) * (self.kutta_weld_sign * gamma))

    def kutta_blocks(self, state, F):
        """(K, F_elim) of the eliminated step (newton.py:459-502): the probe
        estimator's constant K and F; the pressure estimator's
        K = -D^-1 K_p and F_elim = -D^-1 F / sigma from the exact rows at
        this state (tip taper: D = taper D + (1 - taper) s / sigma, K_p
        scaled by taper), uploaded to the coupled handle."""
        if self.cvs is None:
            return self.K, F
        import scipy.linalg as sla
        import scipy.sparse as sp
        t = L.torch()
        Kp_cut, D = self.cvs.newton_rows(state["phi_cut"])
        Kp = (Kp_cut @ self._T).tocsr()
        Kp.sum_duplicates()
        Fh = F.cpu().numpy() / self.kutta_sigma
        if self._taper_active:
            tp = self.tip_taper
            Kp = (sp.diags(tp) @ Kp).tocsr()
            D = tp[:, None] * D
            D[np.diag_indices_from(D)] += (1.0 - tp) * self.kutta_weld_sign / self.kutta_sigma
        lu = sla.lu_factor(D)
        F_elim = -sla.lu_solve(lu, Fh)
        cols = np.unique(Kp.indices)
        Kd = -sla.lu_solve(lu, Kp[:, cols].toarray())
        n_st = self.n_st
        kp = np.ascontiguousarray(np.arange(n_st + 1, dtype=np.int64) * len(cols))
        kc = np.ascontiguousarray(np.tile(cols.astype(np.int64), n_st))
        kv = np.ascontiguousarray(Kd.ravel())
        L.call("up3d_coupled_set_kutta_row", self._coupled, kp.ctypes.data, kc.ctypes.data, kv.ctypes.data)
        K = sp.csr_matrix((kv, kc, kp), shape=(n_st, self.n_red))
        return K, L.to_device(F_elim, t.float64)

    # dense direct steps are for small cases (the reference's sparse LU
    # path: "seconds at 6e4 dofs"); 20,000 free unknowns are 3.2 GB dense
    DIRECT_MAX_FREE = 20_000

    def dense_lu(self, Aop: CoupledOperator):
        """(LU, pivots) of the dense J_ff = (T^T J T)[free, free] of this
        step (J the cut-mesh Jacobian, reduced by the wake plan of its
        pattern: the fixed grouping of the reference's T^T (J T)), and the
        dense B (n_free, n_stations) from the coupled operator at x = 0,
        g = e_j.  The factorisation is cuSOLVER's dense LU (torch.linalg)."""
        t = L.torch()
        if self.n_free > self.DIRECT_MAX_FREE:
            raise ValueError(f"precond='direct' is for small cases: {self.n_free} free unknowns "
                             f"(limit {self.DIRECT_MAX_FREE}); use precond='amg'")
        J_red = self.jacobian_block(Aop)
        if not hasattr(self, "_free_pos"):
            self._free_pos = t.full((self.n_red,), -1, dtype=t.int64, device="cuda")
            self._free_pos[L.to_device(self.free, t.int64)] = t.arange(self.n_free, device="cuda")
            self._free_d = L.to_device(self.free, t.int64)
        ip = J_red.indptr.to(t.int64)
        rows = t.repeat_interleave(t.arange(self.n_red, device="cuda"), ip[1:] - ip[:-1])
        cols = J_red.indices.to(t.int64)
        fr, fc = self._free_pos[rows], self._free_pos[cols]
        keep = (fr >= 0) & (fc >= 0)
        D = t.zeros((self.n_free, self.n_free), dtype=t.float64, device="cuda")
        D[fr[keep], fc[keep]] = J_red.data[keep]
        zero = t.zeros(self.n_red, dtype=t.float64, device="cuda")
        cols_b = []
        for j in range(self.n_st):
            e = t.zeros(self.n_st, dtype=t.float64, device="cuda")
            e[j] = 1.0
            cols_b.append(Aop.apply(zero, e)[0][self._free_d])
        B = t.stack(cols_b, dim=1) if cols_b else t.zeros((self.n_free, 0), dtype=t.float64, device="cuda")
        LU, piv = t.linalg.lu_factor(D)
        return LU, piv, B

    def jacobian_block(self, Aop: CoupledOperator) -> DeviceCSR:
        """T^T J T of this step's cut-mesh Jacobian (Term-3 entries merged),
        with the far-field mask: J_ff embedded in the reduced numbering, the
        matrix the direct and ILU preconditioners factor."""
        if not hasattr(self, "_con_direct"):
            self._con_direct = WakeConstraint(Aop.J, self.wc)   # plans of the merged Jacobian patterns
        J_red, _ = self._con_direct.reduce_operator(Aop.J)
        J_red.dirichlet = self.mask
        J_red.extra = None
        return J_red

    def direct_step(self, lu, K, rhs):
        """dphi = z - JB S^-1 K z with z = J_ff^-1 rhs, JB = J_ff^-1 B,
        S = I + K JB (newton.py:1003-1008); reduced-size, far-field rows 0."""
        t = L.torch()
        LU, piv, B = lu
        Kd = L.to_device(np.ascontiguousarray(K[:, self.free].toarray()), t.float64)
        z = t.linalg.lu_solve(LU, piv, rhs[self._free_d].unsqueeze(1)).squeeze(1)
        if self.n_st:
            JB = t.linalg.lu_solve(LU, piv, B)
            S = t.eye(self.n_st, dtype=t.float64, device="cuda") + Kd @ JB
            z = z - JB @ t.linalg.solve(S, Kd @ z)
        out = t.zeros(self.n_red, dtype=t.float64, device="cuda")
        out[self._free_d] = z
        return out

    def lagged_step(self, lu, Aop: CoupledOperator, rhs, rtol: float, restart: int, maxiter: int):
        """The lagged-LU reuse step (newton.py:978-996): GMRES on the fresh
        coupled operator J_ff + B K over the free unknowns, preconditioned
        by a stale dense LU of J_ff, to rtol.  Right-preconditioned
        restarted GMRES (classical Gram-Schmidt Arnoldi with one
        re-orthogonalisation pass, Givens rotations), converged when the
        true residual |rhs - A x| <= rtol |rhs|; at most maxiter cycles of
        restart steps.  Returns (dphi reduced-size or
        None when it did not converge, inner steps)."""
        t = L.torch()
        LU, piv, _ = lu
        fr = self._free_d
        b = rhs[fr]
        n = b.numel()
        full = t.zeros(self.n_red, dtype=t.float64, device="cuda")

        def A(v):
            full.zero_()
            full[fr] = v
            return Aop.matvec(full)[fr]

        def Minv(v):
            return t.linalg.lu_solve(LU, piv, v.unsqueeze(1)).squeeze(1)

        b_norm = float(t.linalg.vector_norm(b))
        x = t.zeros(n, dtype=t.float64, device="cuda")
        if b_norm == 0.0:
            out = t.zeros(self.n_red, dtype=t.float64, device="cuda")
            return out, 0
        tol = rtol * b_norm
        m = max(1, min(int(restart), n))
        n_it = 0
        converged = False
        for _ in range(int(maxiter)):
            r = b - A(x)
            beta = float(t.linalg.vector_norm(r))
            if beta <= tol:
                converged = True
                break
            V = t.empty((m + 1, n), dtype=t.float64, device="cuda")
            V[0] = r / beta
            H = np.zeros((m + 1, m))
            cs, sn = np.zeros(m), np.zeros(m)
            g = np.zeros(m + 1)
            g[0] = beta
            k_used = 0
            for k in range(m):
                w = A(Minv(V[k]))
                h = V[:k + 1] @ w                     # classical projection, then one
                w = w - V[:k + 1].T @ h               # re-orthogonalisation pass
                h2 = V[:k + 1] @ w
                w = w - V[:k + 1].T @ h2
                hk = (h + h2).cpu().numpy()
                hn = float(t.linalg.vector_norm(w))
                H[:k + 1, k] = hk
                H[k + 1, k] = hn
                for i in range(k):
                    a_, b_ = H[i, k], H[i + 1, k]
                    H[i, k] = cs[i] * a_ + sn[i] * b_
                    H[i + 1, k] = -sn[i] * a_ + cs[i] * b_
                den = float(np.hypot(H[k, k], H[k + 1, k]))
                cs[k], sn[k] = (1.0, 0.0) if den == 0.0 else (H[k, k] / den, H[k + 1, k] / den)
                H[k, k] = den
                H[k + 1, k] = 0.0
                g[k + 1] = -sn[k] * g[k]
                g[k] = cs[k] * g[k]
                n_it += 1
                k_used = k + 1
                if hn != 0.0:
                    V[k + 1] = w / hn
                if abs(g[k + 1]) <= tol or hn == 0.0:
                    break
            y = np.linalg.solve(np.triu(H[:k_used, :k_used]), g[:k_used])
            yd = t.from_numpy(y).cuda()
            x = x + Minv(V[:k_used].T @ yd)
        else:
            converged = float(t.linalg.vector_norm(b - A(x))) <= tol
        if not converged:
            return None, n_it
        out = t.zeros(self.n_red, dtype=t.float64, device="cuda")
        out[fr] = x
        return out, n_it

    def picard_block(self) -> DeviceCSR:
        """T^T A(rho_tilde) T with the far-field mask: the AMG source
        (newton.py:1013-1022), rho_tilde of the last evaluation."""
        A = self.op.assemble_matrix(self.ev.rho_tilde)
        A_red, _ = self.con.reduce_operator(A)
        A_red.dirichlet = self.mask
        A_red.extra = None
        return A_red

    def freeze(self, state):
        """(upstream, branch) at the state (kernels/upwind.py:821-843)."""
        from ..kernels.upwind import UpwindOperator
        from ..physics.isentropic import density_field, limit_q2_field
        t = L.torch()
        fl = state["flow"]
        grad, q2 = self.op.velocities(state["phi_cut"])
        q2l = limit_q2_field(q2 / fl.u_inf ** 2, fl.m_inf, fl.m_cap, fl.gamma)
        rho = density_field(q2l, fl.m_inf, fl.gamma)
        if not hasattr(self, "_upw"):
            self._upw = UpwindOperator(t.as_tensor(np.asarray(self.mesh.nodes)),
                                       t.as_tensor(np.asarray(self.mesh.elements)), mesh=self.mesh)
        up, br = self._upw.freeze_upwind_state(grad, q2l, rho, fl.m_inf, fl.upwind_c, fl.m_crit,
                                               fl.gamma, fl.rho_floor)
        return up.clone(), br.clone()


def solve_newton_lifting(mesh_cut, wc, m_inf: float, alpha_deg: float = 0.0, u_inf: float = 1.0,
                         gamma_air: float = 1.4, vortex_center=(0.25, 0.0),
                         farfield_spanwise_gamma: bool = False, upwind_c: float = 1.5,
                         m_crit: float = 0.95, m_cap: float = 3.0, rho_floor: float = 0.05,
                         phi_init=None, gamma_init=None, n_picard_seed: int = 5,
                         n_newton_max: int = 30, tol_residual: float = 1e-10,
                         tol_gamma: float = 1e-8, ew_eta0: float = 1e-2, ew_gamma: float = 0.9,
                         ew_eta_max: float = 1e-2, amg_rebuild_every: int = 2,
                         precond: str = "amg", direct_refactor_every: int = 1,
                         direct_reuse_rtol: float = 1e-8, gmres_restart: int = 60, gmres_maxiter: int = 10,
                         line_search: bool = True, rtol_seed: float = 1e-7,
                         tol_residual_loose: Optional[float] = None,
                         tol_residual_rel: Optional[float] = None, accept_on_stall: bool = False,
                         freeze_tol: Optional[float] = None,
                         freeze_refresh_max: int = 2, freeze_max_reverts: int = 3,
                         workspace: Optional[NewtonWorkspace] = None, tip_taper=None,
                         kutta_estimator: str = "probe", external_rhs=None,
                         verbose: bool = False) -> Dict[str, object]:
    """Fully coupled (phi_red, Gamma) Newton at one Mach level
    (pyfp3d/solve/newton.py:516-1141): Eisenstat-Walker forcing, GMRES(60)
    with AMG on the reduced Picard block (rebuilt every amg_rebuild_every
    steps), merit |R|^2 + |F|^2 line search with at most five halvings,
    the level fail-fast and the optional frozen-selection finish.
    Converged when |R_f|_inf < tol_residual and |F|_inf < tol_gamma with no
    limited or floored element; tol_residual_loose / tol_residual_rel /
    accept_on_stall accept an intermediate continuation level earlier
    (after at least one step, never while frozen) as the reference does.
    Start: phi_init / gamma_init, else n_picard_seed outer iterations of
    solve_subsonic_lifting (tol_rho 1e-3, rtol_seed), else the freestream."""
    t = L.require_cuda()
    if m_inf > 0.0 and upwind_c <= 0.0:
        raise ValueError("the Newton driver runs with the walk upwind machinery active for m_inf > 0; "
                         "pass upwind_c > 0")
    if precond not in ("amg", "direct", "ilu"):
        raise ValueError(f"unknown precond {precond!r}")
    if direct_refactor_every < 1:
        raise ValueError(f"direct_refactor_every must be >= 1, got {direct_refactor_every}")
    ws = workspace
    if ws is None:
        ws = NewtonWorkspace(mesh_cut, wc, alpha_deg, u_inf, gamma_air, vortex_center,
                             farfield_spanwise_gamma, tip_taper=tip_taper,
                             kutta_estimator=kutta_estimator, external_rhs=external_rhs)
    elif ws.kutta_estimator != kutta_estimator:
        raise ValueError(f"workspace was built with kutta_estimator={ws.kutta_estimator!r} but "
                         f"{kutta_estimator!r} was requested")
    ws.set_mach(m_inf)
    timings = {"seed": 0.0, "assembly": 0.0, "precond": 0.0, "linsolve": 0.0, "residual": 0.0}

    def clock():
        t.cuda.synchronize()
        return time.perf_counter()

    t_wall0 = clock()
    if phi_init is not None:
        phi_f = (phi_init[:ws.n_red].to(device="cuda", dtype=t.float64).clone() if L.is_torch(phi_init)
                 else L.to_device(np.asarray(phi_init, dtype=np.float64)[:ws.n_red], t.float64).clone())
        gamma = (t.zeros(ws.n_st, dtype=t.float64, device="cuda") if gamma_init is None
                 else L.to_device(np.atleast_1d(np.asarray(gamma_init, dtype=np.float64)), t.float64).clone())
    elif n_picard_seed > 0:
        seed = solve_subsonic_lifting(mesh_cut, wc, m_inf=m_inf, alpha_deg=alpha_deg, u_inf=u_inf,
                                      gamma_air=gamma_air, vortex_center=vortex_center, upwind_c=upwind_c,
                                      m_crit=m_crit, m_cap=m_cap, n_picard_max=n_picard_seed, tol_rho=1e-3,
                                      rtol=rtol_seed, farfield_spanwise_gamma=farfield_spanwise_gamma,
                                      workspace=ws)
        phi_f = seed["phi"][:ws.n_red].clone()
        gamma = L.to_device(np.atleast_1d(seed["gamma"]), t.float64).clone()
    else:
        phi_f = L.to_device(freestream_phi(np.asarray(mesh_cut.nodes)[:ws.n_red], alpha_deg, u_inf),
                            t.float64)
        gamma = (t.zeros(ws.n_st, dtype=t.float64, device="cuda") if gamma_init is None
                 else L.to_device(np.atleast_1d(np.asarray(gamma_init, dtype=np.float64)), t.float64).clone())
    timings["seed"] = clock() - t_wall0

    def merit_of(R, F):
        return float(R @ R) + (float(F @ F) if ws.n_st else 0.0)

    res_kw = dict(upwind_c=upwind_c, m_crit=m_crit, m_cap=m_cap, rho_floor=rho_floor)
    residual_history, F_history, gamma_history, eta_history, newton_orders = [], [], [], [], []
    n_gmres_total = n_gmres_stalled = 0
    converged = False
    accept_reason = None
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
    n_term3_last = 0
    n_refactor = 0
    lu, lu_age = None, 0

    a = clock()
    R, F, state = ws.eval_residual(phi_f, gamma, **res_kw)
    merit = merit_of(R, F)
    timings["residual"] += clock() - a

    for it in range(n_newton_max):
        r_norm = float(R.abs().max())
        f_norm = float(F.abs().max()) if ws.n_st else 0.0
        residual_history.append(r_norm)
        F_history.append(f_norm)
        gamma_history.append(gamma.cpu().numpy().copy())
        if len(residual_history) >= 3:
            r2, r1, r0 = residual_history[-1], residual_history[-2], residual_history[-3]
            if r2 > 0 and r1 > 0 and r0 > 0 and r1 != r0:
                newton_orders.append(float(np.log(r2 / r1) / np.log(r1 / r0)))
        if verbose:
            print(f"  newton {it:2d}: |R|={r_norm:.3e} |F|={f_norm:.3e} lim={state['n_limited']} "
                  f"flr={state['n_floored']}" + (" [frozen]" if frozen is not None else ""))
        r_level_best = min(r_level_best, r_norm)
        clean = state["n_limited"] == 0 and state["n_floored"] == 0

        if frozen is not None and freeze_point is not None:
            if r_norm > 10.0 * freeze_point[2] or not clean:
                phi_f, gamma = freeze_point[0].clone(), freeze_point[1].clone()
                frozen = freeze_point = None
                freeze_cooldown = 5
                n_freeze_reverts += 1
                r_level_best = np.inf
                if n_freeze_reverts >= freeze_max_reverts:
                    freeze_armed = False
                R, F, state = ws.eval_residual(phi_f, gamma, **res_kw)
                merit = merit_of(R, F)
                continue
        if freeze_cooldown > 0:
            freeze_cooldown -= 1
        if r_norm > 100.0 * r_level_best and r_norm > 1e-3:
            break
        live_stalled = (len(residual_history) >= 7 and r_norm < 1e-3
                        and r_norm > 0.25 * min(residual_history[-7:-1])
                        and r_norm < 2.0 * min(residual_history[-7:-1]))
        if (frozen is None and freeze_armed and freeze_cooldown == 0 and m_inf > 0.0
                and (r_norm < freeze_tol or live_stalled) and clean):
            frozen = ws.freeze(state)
            freeze_point = (phi_f.clone(), gamma.clone(), r_norm)
            r_level_best = np.inf
        accept = None
        if f_norm < tol_gamma and clean:
            if r_norm < tol_residual:
                accept = "tol"
            elif frozen is None and it > 0:
                if tol_residual_loose is not None and r_norm < tol_residual_loose:
                    accept = "loose_tol"
                elif tol_residual_rel is not None and r_norm <= tol_residual_rel * residual_history[0]:
                    accept = "rel_drop"
                elif accept_on_stall and live_stalled:
                    accept = "stall"
        if accept is not None:
            if frozen is None:
                converged = True
                accept_reason = accept
                break
            R_live, F_live, st_live = ws.eval_residual(phi_f, gamma, **res_kw)
            residual_unfrozen = float(R_live.abs().max())
            if residual_unfrozen < tol_residual:
                converged = True
                R, F, state = R_live, F_live, st_live
                break
            if prev_live_residual is not None and residual_unfrozen > 0.5 * prev_live_residual:
                converged = True
                break
            if n_freeze_refresh >= freeze_refresh_max:
                converged = True
                break
            prev_live_residual = residual_unfrozen
            n_freeze_refresh += 1
            frozen = ws.freeze(st_live)
            freeze_point = (phi_f.clone(), gamma.clone(), residual_unfrozen)
            r_level_best = np.inf
            R, F, state = ws.eval_residual(phi_f, gamma, frozen=frozen, **res_kw)
            merit = merit_of(R, F)
            continue

        a = clock()
        Aop = ws.assemble_coupled(state, frozen=frozen)
        n_term3_last = state["n_term3_active"]
        timings["assembly"] += clock() - a
        a = clock()
        if precond == "amg" and (M_pre is None or it % amg_rebuild_every == 0):
            ws.amg = M_pre = amg_for(ws.picard_block(), ws.amg)
        elif precond == "ilu":
            # ILU of J_ff itself, every step (newton.py:1023-1024)
            M_pre = build_ilu_preconditioner(ws.jacobian_block(Aop))
        timings["precond"] += clock() - a
        # rhs = -R_f - B F_elim  (B F_elim = the coupled operator at x = 0)
        a = clock()
        K_elim, F_elim = ws.kutta_blocks(state, F)
        zero = t.zeros(ws.n_red, dtype=t.float64, device="cuda")
        BF, _ = Aop.apply(zero, F_elim)
        rhs = -R - BF
        if precond == "direct":
            # exact step: dense LU of J_ff and the Woodbury update for the
            # rank-n_stations coupling B K (newton.py:966-1011); with
            # direct_refactor_every > 1 the steps in between run GMRES on
            # the fresh operator with the stale LU as preconditioner and
            # refactor when that GMRES does not converge
            dphi = None
            if lu is not None and lu_age < direct_refactor_every:
                dphi, n_it = ws.lagged_step(lu, Aop, rhs, direct_reuse_rtol, gmres_restart, 2)
                n_gmres_total += n_it
            if dphi is None:
                b2 = clock()
                lu = ws.dense_lu(Aop)
                lu_age = 0
                timings["precond"] += clock() - b2
                n_refactor += 1
                dphi = ws.direct_step(lu, K_elim, rhs)
            lu_age += 1
            eta_history.append(0.0)
        else:
            eta = _ew_forcing(r_norm, residual_history[-2] if it > 0 else None, eta_prev, ew_eta0, ew_gamma,
                              ew_eta_max)
            eta_prev = eta
            eta_history.append(eta)
            dphi, n_it, info = Aop.solve(rhs, M=M_pre, rtol=eta, restart=gmres_restart, maxiter=gmres_maxiter)
            n_gmres_total += n_it
            n_gmres_stalled += info != 0
        dphi = dphi.masked_fill(ws.mask.bool(), 0.0)
        _, dgamma = Aop.apply(dphi, F_elim)        # dGamma = K dphi + F_elim
        timings["linsolve"] += clock() - a

        lam, best, accepted = 1.0, None, False
        a = clock()
        for _ in range(5):
            phi_try = phi_f + lam * dphi
            g_try = gamma + lam * dgamma
            R_try, F_try, st_try = ws.eval_residual(phi_try, g_try, frozen=frozen, **res_kw)
            merit_try = merit_of(R_try, F_try)
            if np.isfinite(merit_try) and (not line_search or merit_try <= merit):
                accepted = True
                break
            if np.isfinite(merit_try) and (best is None or merit_try < best[0]):
                best = (merit_try, lam)
            lam *= 0.5
        if not accepted:
            if best is None:
                raise RuntimeError(f"Newton line search failed at iteration {it} "
                                   f"(merit {merit:.3e} -> {merit_try:.3e})")
            merit_try, lam = best
            phi_try = phi_f + lam * dphi
            g_try = gamma + lam * dgamma
            R_try, F_try, st_try = ws.eval_residual(phi_try, g_try, frozen=frozen, **res_kw)
        timings["residual"] += clock() - a
        phi_f, gamma = phi_try, g_try
        R, F, state, merit = R_try, F_try, st_try, merit_try

    timings["wall"] = clock() - t_wall0
    if converged and accept_reason is None:
        accept_reason = "tol"
    return {"phi": state["phi_cut"], "gamma": gamma, "converged": converged, "accept_reason": accept_reason,
            "n_newton": len(residual_history) - (1 if converged else 0),
            "residual_history": residual_history, "F_history": F_history,
            "gamma_history": gamma_history, "newton_orders": newton_orders, "eta_history": eta_history,
            "n_gmres_total": n_gmres_total, "n_gmres_stalled": n_gmres_stalled,
            "froze": frozen is not None, "n_freeze_refresh": n_freeze_refresh,
            "residual_unfrozen": residual_unfrozen, "n_freeze_reverts": n_freeze_reverts,
            "nu_max": state["nu_max"], "n_nu_active": state["n_nu_active"],
            "n_limited": state["n_limited"], "n_floored": state["n_floored"],
            "n_term3_active": n_term3_last, "timings": timings, "workspace": ws,
            "n_refactor": n_refactor,
            "kutta_estimator": ws.kutta_estimator, "kutta_sigma": ws.kutta_sigma,
            "kutta_sigma_sign_flips": ws.kutta_sigma_sign_flips, "kutta_weld_sign": ws.kutta_weld_sign}


def solve_newton_transonic(mesh_cut, wc, m_inf: float, alpha_deg: float, m_start: float = 0.70,
                           dm: float = 0.05, dm_min: float = 0.01, upwind_c: float = 1.5,
                           m_crit: float = 0.95, upwind_c_post=None, freeze_tol: Optional[float] = 1e-6,
                           intermediate_tol: Optional[float] = None, newton_kw: Optional[dict] = None,
                           verbose: bool = False) -> Dict[str, object]:
    """Upward Mach continuation of the coupled solve
    (pyfp3d/solve/newton.py:1144-1307): every level warm-starts (phi, Gamma)
    from the last converged one and reuses its workspace; a level that
    fails is retried with the Mach step halved down to dm_min; with
    intermediate_tol the original-schedule levels before the last accept
    loosely; upwind_c_post re-solves the final level at each listed
    upwind_c.  Level 0 starts from the Picard warm start (or newton_kw's
    phi_init)."""
    from .newton import mach_schedule
    if m_inf < m_start:
        raise ValueError(f"upward ramp only: m_inf {m_inf} < m_start {m_start}")
    kw = dict(newton_kw or {})
    kw.setdefault("upwind_c", upwind_c)
    kw.setdefault("m_crit", m_crit)
    kw.setdefault("freeze_tol", freeze_tol)
    ws = kw.pop("workspace", None)
    t0 = time.perf_counter()
    result, last_good = None, None
    level_history, level_results = [], []
    levels = mach_schedule(m_inf, m_start, dm)
    loose = [True] * (len(levels) - 1) + [False]

    def run(m, lvl_kw):
        nonlocal ws
        a = time.perf_counter()
        res = solve_newton_lifting(mesh_cut, wc, m_inf=m, alpha_deg=alpha_deg, workspace=ws,
                                   verbose=verbose, **lvl_kw)
        ws = res["workspace"]
        level_history.append((m, res["n_newton"], res["residual_history"][-1]))
        level_results.append({"m": m, "upwind_c": lvl_kw["upwind_c"], "converged": res["converged"],
                              "accept_reason": res["accept_reason"], "n_newton": res["n_newton"],
                              "residual_history": res["residual_history"], "F_history": res["F_history"],
                              "gamma_history": res["gamma_history"], "n_lin_iters": res["n_gmres_total"],
                              "wall_s": time.perf_counter() - a, "timings": res["timings"]})
        return res

    i = 0
    while i < len(levels):
        m = levels[i]
        lvl_kw = dict(kw)
        if intermediate_tol is not None and loose[i]:
            lvl_kw.update(tol_residual_loose=intermediate_tol, tol_residual_rel=1e-3, accept_on_stall=True,
                          freeze_tol=None)
        if last_good is not None:
            lvl_kw.update(phi_init=last_good["phi"], gamma_init=last_good["gamma"].cpu().numpy(),
                          n_picard_seed=0)
        if verbose:
            print(f"newton continuation level M = {m:.4f}")
        result = run(m, lvl_kw)
        if not result["converged"]:
            m_prev = m_start if i == 0 else levels[i - 1]
            dm_new = 0.5 * (m - m_prev)
            if i == 0 or dm_new < dm_min:
                break
            levels.insert(i, m_prev + dm_new)
            loose.insert(i, False)
            continue
        last_good = result
        i += 1
    if result["converged"] and upwind_c_post:
        for c_post in upwind_c_post:
            lvl_kw = dict(kw)
            lvl_kw.update(upwind_c=c_post, phi_init=result["phi"], gamma_init=result["gamma"].cpu().numpy(),
                          n_picard_seed=0)
            result = run(m_inf, lvl_kw)
            if not result["converged"]:
                break
    result = dict(result)
    result["level_history"] = level_history
    result["level_results"] = level_results
    result["wall_total"] = time.perf_counter() - t0
    return result


def solve_subsonic_lifting(mesh_cut, wc, m_inf: float, alpha_deg: float = 0.0, u_inf: float = 1.0,
                           gamma_air: float = 1.4, vortex_center=(0.25, 0.0), gamma_fixed=None,
                           omega: float = 1.0, omega_gamma: float = 0.9, tol_gamma: float = 1e-8,
                           tol_rho: float = 1e-10, n_picard_max: int = 40, rtol: float = 1e-10,
                           maxiter: int = 3000, amg_rebuild_every: int = 4, forcing: float = 0.0,
                           upwind_c: float = 1.5, m_crit: float = 0.95, upwind_weighted: bool = False,
                           upwind_mode: str = "kernel", upwind_p_weight: float = 3.0,
                           upwind_reach_frac: float = 1.0, upwind_reach_gain_max: float = 4.0,
                           upwind_nbr_depth: int = 3, upwind_sigma_s_frac: float = 0.35,
                           upwind_sigma_p_frac: float = 0.35,
                           phi_init=None, gamma_init=None, kutta_per_outer: Optional[int] = None,
                           m_cap: float = 3.0, omega_rho: float = 1.0, pseudo_dt: Optional[float] = None,
                           pseudo_dt_growth: float = 1.1, pseudo_dt_max_ratio: float = 100.0,
                           damping_theta: Optional[float] = None, tol_residual: Optional[float] = None,
                           farfield_spanwise_gamma: bool = False, body_source_rhs=None,
                           workspace: Optional[NewtonWorkspace] = None,
                           rho_floor: float = 0.05) -> Dict[str, object]:
    """Nested lifting Picard (pyfp3d/solve/picard.py:420-883): per outer
    iteration the upwinded density of the current potential weights the
    stiffness matrix, reduced by the wake fold, with an AMG hierarchy
    rebuilt every amg_rebuild_every outers; the inner loop solves the
    free-node system by CG (warm-started when m_inf > 0, forcing gives the
    inexact atol) for the current Gamma and updates Gamma from the Kutta
    targets -- secant steps until |target - Gamma| < tol_gamma (at most 30),
    or kutta_per_outer plain under-relaxed steps.  Converged when the Kutta
    loop met tol_gamma, the density lag max|rho_new - rho| < tol_rho and
    (with tol_residual) |T^T R|inf < tol_residual.  Matrix, right-hand
    side, CG, density and residual run on the device; Gamma (n_stations
    numbers) and the convergence scalars on the host.  damping_theta adds
    theta diag(A_free) of each outer, pseudo_dt the lumped volumes over an
    adaptive dtau, to the matrix and D phi_k to the right-hand side (the
    reference's pseudo-transient forms).  upwind_weighted takes rho~ from
    the weighted upwind modes (UpwindOperator(weighted=True, mode=...),
    kernels/upwind.py:176-454, with the reference's parameters) instead of
    the walk, and the residual from PicardOperator.assemble_residual at
    that rho~, as the reference's loop does (picard.py:592-603, :703-710,
    :803-813)."""
    t = L.require_cuda()
    from ..physics.isentropic import mach_squared_field
    from .linear import solve_cg
    if not 0.0 <= m_inf < 1.0:
        raise ValueError(f"solve_subsonic_lifting needs 0 <= M_inf < 1, got {m_inf}")
    if pseudo_dt is not None and damping_theta is not None:
        raise ValueError("pseudo_dt and damping_theta are mutually exclusive stabilizers -- pick one")
    t_wall0 = time.perf_counter()
    ws = workspace
    if ws is None:
        ws = NewtonWorkspace(mesh_cut, wc, alpha_deg, u_inf, gamma_air, vortex_center, farfield_spanwise_gamma)
    ws.set_mach(m_inf)
    n_red, n_st = ws.n_red, ws.n_st
    flow = ws.flow(upwind_c if m_inf > 0.0 else 0.0, m_crit, m_cap, rho_floor)
    mask_b = ws.mask.bool()
    timings = {"assembly": 0.0, "precond": 0.0, "linsolve": 0.0, "residual": 0.0, "kutta": 0.0}

    def clock():
        t.cuda.synchronize()
        return time.perf_counter()

    b_fold = None
    if body_source_rhs is not None:
        b = np.asarray(body_source_rhs, dtype=np.float64)
        if b.shape != (ws.mesh.n_nodes,):
            raise ValueError(f"body_source_rhs must be ({ws.mesh.n_nodes},) on the cut mesh, got {b.shape}")
        b_cut = L.to_device(b, t.float64)
        b_fold = t.empty(n_red, dtype=t.float64, device="cuda")
        L.call("up3d_coupled_residual", ws._coupled, b_cut.data_ptr(), None, None, b_fold.data_ptr(), None,
               L.stream_ptr())

    def state_of(phi_f, g):
        """(phi_red, phi_cut): far-field rows vals(Gamma), copies expanded."""
        g_d = L.to_device(np.ascontiguousarray(g, dtype=np.float64), t.float64)
        phi_red = t.empty(n_red, dtype=t.float64, device="cuda")
        phi_cut = t.empty(ws.mesh.n_nodes, dtype=t.float64, device="cuda")
        L.call("up3d_coupled_state", ws._coupled, phi_f.data_ptr(), g_d.data_ptr(), phi_red.data_ptr(),
               phi_cut.data_ptr(), L.stream_ptr())
        return phi_red, phi_cut

    def fold(v_cut):
        out = t.empty(n_red, dtype=t.float64, device="cuda")
        L.call("up3d_coupled_residual", ws._coupled, v_cut.data_ptr(), None, None, out.data_ptr(), None,
               L.stream_ptr())
        return out

    probes = L.to_device(np.concatenate([wc.kutta_upper, wc.kutta_lower]).astype(np.int64), t.int64)
    n_te = len(wc.kutta_upper)
    counts = np.bincount(wc.te_station, minlength=n_st)

    def kutta_host(phi_cut):
        """kutta_targets (constraints/wake.py:196-212) in the reference's
        bincount order, on the host (2 n_TE values cross)."""
        v = phi_cut[probes].cpu().numpy()
        return np.bincount(wc.te_station, weights=v[:n_te] - v[n_te:], minlength=n_st) / counts

    weighted = upwind_weighted and upwind_c > 0.0 and m_inf > 0.0
    if weighted:
        from ..kernels.upwind import UpwindOperator
        from ..physics.isentropic import density_field, limit_q2_field
        upw_w = UpwindOperator(t.as_tensor(np.asarray(ws.mesh.nodes)), t.as_tensor(np.asarray(ws.mesh.elements)),
                               weighted=True, mode=upwind_mode, p_weight=upwind_p_weight,
                               reach_frac=upwind_reach_frac, reach_gain_max=upwind_reach_gain_max,
                               nbr_depth=upwind_nbr_depth, sigma_s_frac=upwind_sigma_s_frac,
                               sigma_p_frac=upwind_sigma_p_frac, mesh=ws.mesh)

    def evaluate(phi_cut):
        """(rho~, monitors, R) at phi_cut: the fused evaluation (walk
        flux), or the weighted modes' rho~ and the residual at it."""
        if not weighted:
            ws.ev.evaluate(phi_cut, flow, jacobian=False, keep_state=True)
            return ws.ev.rho_tilde.clone(), ws.ev.read_monitors(), ws.ev.R
        grad, q2 = ws.op.velocities(phi_cut)
        q2l = limit_q2_field(q2 / u_inf ** 2, m_inf, m_cap, gamma_air)
        rho = density_field(q2l, m_inf, gamma_air)
        rt = upw_w.rho_tilde(grad, q2l, rho, m_inf, upwind_c, m_crit, gamma_air, rho_floor).clone()
        R = ws.op.assemble_residual(phi_cut, rt).clone()
        mon = {"nu_max": float(upw_w.nu_max), "n_supersonic": int(upw_w.n_supersonic),
               "n_floored": int(upw_w.n_floored), "n_limited": int((q2l != q2 / u_inf ** 2).sum())}
        return rt, mon, R

    if gamma_fixed is not None:
        gamma = np.broadcast_to(np.atleast_1d(np.asarray(gamma_fixed, dtype=np.float64)), (n_st,)).copy()
    elif gamma_init is not None:
        gamma = np.atleast_1d(np.asarray(gamma_init, dtype=np.float64)).copy()
    else:
        gamma = np.zeros(n_st, dtype=np.float64)
    if phi_init is not None:
        phi_cut = (phi_init.to(device="cuda", dtype=t.float64).clone() if L.is_torch(phi_init)
                   else L.to_device(np.asarray(phi_init, dtype=np.float64), t.float64).clone())
        phi_red = phi_cut[:n_red].clone()
    else:
        phi_cut = L.to_device(freestream_phi(np.asarray(mesh_cut.nodes), alpha_deg, u_inf), t.float64)
        phi_red = None
    rho_t, mon, _ = evaluate(phi_cut)
    # pseudo-transient term D (picard.py:586-596, :736-745): the local
    # theta diag(A_free) of each outer, or the lumped volumes over dtau
    diag_pos = None
    d_tau = None
    dt_cur = pseudo_dt
    if pseudo_dt is not None:
        _, V = ws.mesh.geometry()
        m_h = np.zeros(ws.mesh.n_nodes)
        np.add.at(m_h, np.asarray(ws.mesh.elements).reshape(-1), np.repeat(V.cpu().numpy() / 4.0, 4))
        m_cut = L.to_device(m_h, t.float64)
        m_red = fold(m_cut)                         # T^T m, zero on far-field rows
        d_tau = m_red / dt_cur

    residual_history, drho_history, gamma_history = [], [], [gamma.copy()]
    n_cg_total = n_solves_total = 0
    M = None
    converged = False
    kutta_converged = gamma_fixed is not None
    zeros = t.zeros(n_red, dtype=t.float64, device="cuda")
    for outer in range(n_picard_max):
        a = clock()
        A_cut = ws.op.assemble_matrix(rho_t)
        A_red = ws.con.reduce_operator(A_cut)[0]
        if damping_theta is not None or d_tau is not None:
            if diag_pos is None:
                ip = A_red.indptr.to(t.int64)
                rows = t.repeat_interleave(t.arange(n_red, device="cuda"), ip[1:] - ip[:-1])
                diag_pos = t.nonzero(A_red.indices.to(t.int64) == rows).flatten()
            if damping_theta is not None:
                d_tau = (damping_theta * A_red.data[diag_pos]).masked_fill(mask_b, 0.0)
            data = A_red.data.clone()
            data[diag_pos] += d_tau
            A_red = DeviceCSR(A_red.indptr, A_red.indices, data, A_red.shape)
        A_red.dirichlet = ws.mask
        A_red.extra = None
        timings["assembly"] += clock() - a
        if M is None or outer % amg_rebuild_every == 0:
            a = clock()
            ws.amg = M = amg_for(A_red, ws.amg)
            timings["precond"] += clock() - a
        x0 = phi_red.masked_fill(mask_b, 0.0) if (m_inf > 0.0 and phi_red is not None) else None

        def solve_for(g, x0):
            a = clock()
            _, u_cut = state_of(zeros, g)
            rhs = -fold(A_cut.matvec(u_cut))
            if b_fold is not None:
                rhs = rhs + b_fold
            if d_tau is not None and x0 is not None:
                rhs = rhs + d_tau * x0
            if m_inf > 0.0 and forcing > 0.0:
                r0 = rhs - A_red.matvec(x0, dirichlet=ws.mask) if x0 is not None else rhs
                atol_k = forcing * float(t.linalg.vector_norm(r0))
            else:
                atol_k = 0.0
            b2 = clock()
            timings["assembly"] += b2 - a
            x, n_it, info = solve_cg(A_red, rhs, M=M, rtol=rtol, atol=atol_k, maxiter=maxiter, x0=x0)
            timings["linsolve"] += clock() - b2
            if info != 0:
                raise RuntimeError(f"CG did not converge (info={info})")
            return state_of(x, g), n_it

        n_inner = 30 if kutta_per_outer is None else kutta_per_outer
        prev_gamma = prev_target = None
        if gamma_fixed is not None:
            (phi_red_new, cut_new), n_it = solve_for(gamma, x0)
            n_cg_total += n_it
            n_solves_total += 1
        else:
            for _ in range(n_inner):
                (phi_red_new, cut_new), n_it = solve_for(gamma, x0)
                n_cg_total += n_it
                n_solves_total += 1
                a = clock()
                if m_inf > 0.0:
                    x0 = phi_red_new.masked_fill(mask_b, 0.0)
                target = kutta_host(cut_new)
                kutta_converged = float(np.max(np.abs(target - gamma))) < tol_gamma
                if not kutta_converged:
                    if prev_gamma is None or kutta_per_outer is not None:
                        new_gamma = gamma + omega_gamma * (target - gamma)
                    else:
                        dg = gamma - prev_gamma
                        slope = np.where(np.abs(dg) > 1e-14, (target - prev_target) / np.where(dg == 0, 1, dg), 0.0)
                        denom = 1.0 - slope
                        relaxed = gamma + omega_gamma * (target - gamma)
                        new_gamma = np.where(np.abs(denom) > 1e-3,
                                             (target - slope * gamma) / np.where(denom == 0, 1, denom), relaxed)
                    prev_gamma, prev_target = gamma, target
                    gamma = new_gamma
                    gamma_history.append(gamma.copy())
                timings["kutta"] += clock() - a
                if kutta_converged:
                    break
        phi_red = phi_red_new if (omega == 1.0 or phi_red is None) else phi_red + omega * (phi_red_new - phi_red)
        phi_cut = ws.con.expand(phi_red, gamma)
        a = clock()
        rho_t_new, mon, R_eval = evaluate(phi_cut)
        R = R_eval if b_fold is None else R_eval - b_cut
        residual_history.append(float(fold(R).abs().max()))
        drho = float((rho_t_new - rho_t).abs().max())
        drho_history.append(drho)
        rho_t = rho_t_new if omega_rho == 1.0 else rho_t + omega_rho * (rho_t_new - rho_t)
        if pseudo_dt is not None and len(drho_history) >= 2:
            if drho < drho_history[-2]:
                dt_cur = min(dt_cur * pseudo_dt_growth, pseudo_dt * pseudo_dt_max_ratio)
            elif drho > 2.0 * drho_history[-2]:
                dt_cur = max(dt_cur / 2.0, pseudo_dt)
            d_tau = m_red / dt_cur
        timings["residual"] += clock() - a
        if kutta_converged and drho < tol_rho and (tol_residual is None or residual_history[-1] < tol_residual):
            converged = True
            break

    _, q2 = ws.op.velocities(phi_cut)
    mach2_max = float(mach_squared_field(q2 / u_inf ** 2, m_inf, gamma_air).max())
    timings["wall"] = time.perf_counter() - t_wall0
    return {"phi": phi_cut, "gamma": gamma, "n_picard": len(residual_history), "converged": converged,
            "kutta_converged": kutta_converged, "residual_history": residual_history,
            "drho_history": drho_history, "gamma_history": gamma_history, "timings": timings, "rho": rho_t,
            "mach2_max": mach2_max, "nu_max": mon["nu_max"], "n_nu_active": mon["n_supersonic"],
            "n_limited": mon["n_limited"], "n_floored": mon["n_floored"], "n_cg_total": n_cg_total,
            "n_solves_total": n_solves_total, "workspace": ws}
