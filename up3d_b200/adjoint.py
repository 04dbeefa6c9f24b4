"""Discrete adjoint of the full-potential channel solve: shape and Mach
gradients of the lift-like and drag-like wall-pressure integrals.

The reference has no adjoint; this module adds one on top of its discrete
equations (the residual of kernels/jacobian.py and kernels/upwind.py):

* ``BumpShape`` -- the bump channel of mesh.kuhn with the lower wall lifted
  by the base Gaussian plus ``n_side x n_side`` Gaussian shape modes whose
  amplitudes are the design parameters (centres on a grid over the bump,
  jittered from a seed);
* ``wall_force_objective`` -- F = cf . e, e = z (lift-like) or x
  (drag-like), with cf the reference's pressure-force coefficient of the
  lower wall (post/surface.py:309-363 with alpha 0, S_ref 1, no smoothing):
  per wall triangle the in-plane P1 gradient of phi (:80-118), the exact
  isentropic Cp of its speed (physics/isentropic.py:122-143), the
  body-outward normal taken from the owning tet (:192-230), cf = -sum Cp A
  n_out -- written in torch so that autograd gives its explicit partials
  with respect to phi, the node coordinates and M_inf;
* ``lift_objective`` -- the earlier element-Cp integral (Cp of the face's
  element at its limited speed), kept for comparison;
* ``ResidualFunction`` -- R(phi, X, M_inf) as a torch.autograd.Function
  whose backward is the hand-written device product up3d_residual_vjp
  (node coordinates, Mach) plus J^T g (phi);
* ``adjoint_gradient`` -- dF/dp and dF/dM_inf at a converged state:
  J^T lam = dF/dphi solved by GMRES + AMG on the free DOFs, then
  dF/dX = dF/dX|explicit - lam^T dR/dX, chained through dX/dp;
* ``frozen_objective`` -- F after re-converging the discrete equations with
  a given (upstream, branch) selection held fixed: the function whose
  derivative the adjoint at a frozen finish is (for finite differences).
"""

from __future__ import annotations

import ctypes
import time
from typing import Dict, Optional

import numpy as np

from . import _lib as L
from .mesh.kuhn import BumpMesh, bump_channel

GAMMA = 1.4


class BumpShape:
    """Parametric bump channel.  Node z = z_box + H(x, y) (1 - z_box / lz)
    with H = A exp(-(x - x_c)^2 / width) + sum_k p_k exp(-((x - x_k)^2 +
    (y - y_k)^2) / mode_width): p = 0 reproduces bump_channel(amplitude=A)
    bit for bit."""

    def __init__(self, nx: int, ny: int, nz: int, amplitude: float = 0.05, seed: int = 0,
                 n_side: int = 4, mode_width: float = 0.02, centre_seed: int = 7,
                 span_x=(1.7, 2.3), bump_center: float = 2.0, bump_width: float = 0.04):
        box = bump_channel(nx, ny, nz, amplitude=0.0, seed=seed)
        self.box = box.nodes
        self.elements = box.elements
        self.dirichlet_nodes = box.dirichlet_nodes
        self.shape = box.shape
        self.lengths = box.lengths
        self.amplitude = float(amplitude)
        self.bump_center, self.bump_width = bump_center, bump_width
        self.mode_width = float(mode_width)
        ly = self.lengths[1]
        xs = np.linspace(span_x[0], span_x[1], n_side)
        ys = (np.arange(n_side) + 0.5) * ly / n_side
        rng = np.random.default_rng(centre_seed)
        cx, cy = np.meshgrid(xs, ys, indexing="ij")
        jit = rng.uniform(-0.25, 0.25, size=(2, n_side * n_side))
        self.centres = np.stack([cx.ravel() + jit[0] * (xs[1] - xs[0] if n_side > 1 else 0.1),
                                 cy.ravel() + jit[1] * ly / n_side], axis=1)
        x, y, z = self.box[:, 0], self.box[:, 1], self.box[:, 2]
        self._blend = 1.0 - z / self.lengths[2]
        self._base = self.amplitude * np.exp(-((x - bump_center) ** 2) / bump_width)
        self.modes = np.exp(-((x[:, None] - self.centres[None, :, 0]) ** 2
                              + (y[:, None] - self.centres[None, :, 1]) ** 2) / self.mode_width)

    @property
    def n_params(self) -> int:
        return self.modes.shape[1]

    def nodes(self, p=None) -> np.ndarray:
        h = self._base if p is None else self._base + self.modes @ np.asarray(p, dtype=np.float64)
        out = self.box.copy()
        out[:, 2] = out[:, 2] + h * self._blend
        return out

    def dz_dp(self) -> np.ndarray:
        """(N, n_params): d z / d p_k."""
        return self.modes * self._blend[:, None]

    def mesh(self, p=None) -> BumpMesh:
        return BumpMesh(nodes=np.ascontiguousarray(self.nodes(p)), elements=self.elements,
                        dirichlet_nodes=self.dirichlet_nodes, shape=self.shape, lengths=self.lengths)


def lower_wall_faces(elements: np.ndarray, shape) -> np.ndarray:
    """(F, 4) int64: element, then the face's three nodes, for every face
    on the lower wall (all three nodes at k = 0); face f of an element is
    opposite its local node f (mesh/metrics.py:224-232)."""
    nz = shape[2]
    on_wall = (elements % (nz + 1)) == 0
    out = []
    for f in range(4):
        keep = [j for j in range(4) if j != f]
        sel = np.nonzero(on_wall[:, keep].all(axis=1))[0]
        out.append(np.column_stack([sel, elements[sel][:, keep]]))
    faces = np.concatenate(out).astype(np.int64)
    return faces[np.argsort(faces[:, 0], kind="stable")]


def _cp_torch(q2n, mach, gamma=GAMMA, m_cap=3.0):
    """Pressure coefficient of the limited speed (physics/isentropic.py:
    122-143 on the limiter of :262-314)."""
    t = L.torch()
    hgm = 0.5 * (gamma - 1.0)
    m2 = mach * mach
    cap = m_cap ** 2 * (1.0 + hgm * m2) / (m2 * (1.0 + hgm * m_cap ** 2))
    q2l = t.minimum(q2n, cap)
    b = t.clamp(1.0 + hgm * m2 * (1.0 - q2l), min=1e-10)
    rho = b ** (1.0 / (gamma - 1.0))
    return 2.0 / (gamma * m2) * (rho ** gamma - 1.0)


def lift_objective(X, q2n_elem, faces_dev, mach, interior_nodes_dev, gamma=GAMMA, axis: int = 2):
    """F = -sum_f Cp_e(f) (S_f . e_axis), S_f the outward area vector of the
    face (away from the element's fourth node): the lift-like force on the
    lower wall for axis 2 (z), the drag-like one for axis 0 (x).  All
    arguments are torch tensors; X (N, 3), q2n_elem (E) and mach may require
    grad."""
    t = L.torch()
    e = faces_dev[:, 0]
    a, b, c = X[faces_dev[:, 1]], X[faces_dev[:, 2]], X[faces_dev[:, 3]]
    S = 0.5 * t.linalg.cross(b - a, c - a)
    # orientation: outward, away from the element's off-face node
    d = X[interior_nodes_dev] - a
    sign = t.where((S * d).sum(dim=1) > 0, -1.0, 1.0).to(X.dtype)
    Sa = sign.detach() * S[:, axis]
    cp = _cp_torch(q2n_elem[e], mach, gamma)
    return -(cp * Sa).sum()


def wall_force_objective(X, phi, faces_dev, mach, axis: int = 2, u_inf: float = 1.0, gamma=GAMMA):
    """F = cf[axis] of post/surface.py's wall_force_coefficients (alpha 0,
    S_ref 1, no smoothing) on the wall triangles faces_dev[:, 1:4], whose
    owning tets' nodes are faces_dev[:, 4:8] (rows of
    wall_faces_with_owners); X (N, 3) the node coordinates.  Torch tensors;
    X, phi and mach may require grad.  See the module docstring."""
    t = L.torch()
    tri = faces_dev[:, 1:4]
    p0, p1, p2 = X[tri[:, 0]], X[tri[:, 1]], X[tri[:, 2]]
    edge1 = p1 - p0
    edge2 = p2 - p0
    area_vec = t.linalg.cross(edge1, edge2)
    twice_area = t.linalg.norm(area_vec, dim=1)
    n = area_vec / twice_area[:, None]
    e1 = edge1 / t.linalg.norm(edge1, dim=1)[:, None]
    e2 = t.linalg.cross(n, e1)
    u1, v1 = (edge1 * e1).sum(dim=1), (edge1 * e2).sum(dim=1)
    u2, v2 = (edge2 * e1).sum(dim=1), (edge2 * e2).sum(dim=1)
    df1 = phi[tri[:, 1]] - phi[tri[:, 0]]
    df2 = phi[tri[:, 2]] - phi[tri[:, 0]]
    det = u1 * v2 - v1 * u2
    du = (v2 * df1 - v1 * df2) / det
    dv = (-u2 * df1 + u1 * df2) / det
    grad = du[:, None] * e1 + dv[:, None] * e2
    q2 = (grad * grad).sum(dim=1) / u_inf ** 2
    hgm = 0.5 * (gamma - 1.0)
    m2 = mach * mach
    base = t.clamp(1.0 + hgm * m2 * (1.0 - q2), min=1e-10)
    rho = base ** (1.0 / (gamma - 1.0))
    cp = 2.0 / (gamma * m2) * (rho ** gamma - 1.0)
    # body-outward (toward the owning tet, i.e. into the fluid): the sign is
    # a discrete choice, not differentiated
    owner_c = X[faces_dev[:, 4:8]].mean(dim=1)
    face_c = (p0 + p1 + p2) / 3.0
    flip = ((n * (owner_c - face_c)).sum(dim=1) < 0).detach()
    n_out = t.where(flip[:, None], -n, n)
    area = 0.5 * twice_area
    return -(cp * area * n_out[:, axis]).sum()


def wall_faces_with_owners(mesh) -> np.ndarray:
    """(F, 8) int64 rows: owning element, the face's three nodes, the
    owner's four nodes (lower wall of the channel)."""
    faces = lower_wall_faces(mesh.elements, mesh.shape)
    return np.column_stack([faces, mesh.elements[faces[:, 0]].astype(np.int64)])


def transpose_csr(A):
    """A^T of a device CSR (stable, (row, col)-ordered)."""
    t = L.torch()
    from .mesh.device import DeviceCSR
    n = A.shape[0]
    counts = A.indptr[1:] - A.indptr[:-1]
    rows = t.repeat_interleave(t.arange(n, device=A.data.device, dtype=t.int64), counts.to(t.int64))
    cols = A.indices.to(t.int64)
    order = t.sort(cols * n + rows, stable=True).indices
    indptr = t.zeros(A.shape[1] + 1, dtype=t.int64, device=A.data.device)
    indptr[1:] = t.cumsum(t.bincount(cols, minlength=A.shape[1]), 0)
    return DeviceCSR(indptr.to(t.int32), rows[order].to(t.int32).contiguous(),
                     A.data[order].contiguous(), (A.shape[1], n))


class AdjointContext:
    """A converged state on one mesh: the evaluator, the Jacobian at the
    state and the linearisation's upstream / branch."""

    def __init__(self, ws, phi, flow, frozen=None):
        t = L.torch()
        self.ws, self.flow = ws, flow
        self.phi = phi
        ws.ev.evaluate(phi, flow, jacobian=True, frozen=frozen, keep_state=True)
        if frozen is not None:
            self.upstream = L.to_device(frozen[0], t.int64)
            self.branch = L.to_device(frozen[1], t.int8)
        else:
            self.upstream = ws.ev.upstream.to(t.int64)
            self.branch = None
        self.J = ws.ev.jacobian()
        self._JT = None

    @property
    def JT(self):
        if self._JT is None:
            from .mesh.device import DeviceCSR
            t = L.torch()
            J, m = self.J, self.ws.ev.mesh
            if J.data.numel() == m.nnz:
                data_t = t.empty_like(J.data)
                L.call("up3d_jacobian_transpose", m.handle, J.data.data_ptr(), data_t.data_ptr(),
                       L.stream_ptr())
                self._JT = DeviceCSR(J.indptr, J.indices, data_t, J.shape)
            else:
                self._JT = transpose_csr(J)
        return self._JT

    def vjp(self, lam=None, w_q2=None, want_dphi=False):
        """(dphi, dX (N, 3), dM) of L = lam^T R + sum w q2 (up3d_residual_vjp)."""
        t = L.torch()
        m = self.ws.ev.mesh
        dX = t.empty((m.n_nodes, 3), dtype=t.float64, device="cuda")
        dM = t.zeros(1, dtype=t.float64, device="cuda")
        dphi = t.empty(m.n_nodes, dtype=t.float64, device="cuda") if want_dphi else None
        L.call("up3d_residual_vjp", m.handle, self.phi.data_ptr(), self.flow.c(),
               self.upstream.data_ptr(), L.ptr(self.branch), L.ptr(lam), L.ptr(w_q2),
               L.ptr(dphi), dX.data_ptr(), dM.data_ptr(), L.stream_ptr())
        return dphi, dX, dM


class ResidualFunction:
    """R(phi, X, M_inf) on a fixed mesh state as a torch autograd function
    (``ResidualFunction.apply(ctx, phi, X, mach)``): the forward is the
    device residual, the backward the hand-written products J^T g (phi),
    (dR/dX)^T g and (dR/dM)^T g."""

    _fn = None

    @classmethod
    def apply(cls, actx: AdjointContext, phi, X, mach):
        if cls._fn is None:
            import torch

            class _Fn(torch.autograd.Function):
                @staticmethod
                def forward(ctx, phi_, X_, mach_, actx_):
                    ctx.actx = actx_
                    R = actx_.ws.ev.evaluate(phi_.detach(), actx_.flow, jacobian=False,
                                             frozen=None if actx_.branch is None
                                             else (actx_.upstream, actx_.branch),
                                             keep_state=False).clone()
                    return R

                @staticmethod
                def backward(ctx, gR):
                    a = ctx.actx
                    g = gR.detach().contiguous().to(torch.float64)
                    gphi = a.JT.matvec(g)
                    _, dX, dM = a.vjp(lam=g)
                    return gphi, dX, dM.reshape(()), None

            cls._fn = _Fn
        return cls._fn.apply(phi, X, mach, actx)


def adjoint_gradient(shape: BumpShape, mach: float, p=None, m_start: Optional[float] = None,
                     dm: float = 0.05, tol_lambda: float = 1e-12, ws=None,
                     solve_kw: Optional[dict] = None, axis: int = 2) -> Dict[str, object]:
    """Converges the channel at (p, M_inf) on the device, then returns the
    objective F (lift-like for axis 2, drag-like for axis 0), dF/dp
    (n_params), dF/dM_inf, the adjoint lam and timings."""
    t = L.require_cuda()
    from .solve.fused import FlowParams
    from .solve.linear import amg_for, solve_gmres, with_dirichlet
    from .solve.newton import ChannelWorkspace, solve_newton_transonic
    timings = {}
    c0 = time.perf_counter()
    mesh = shape.mesh(p)
    if ws is None:
        ws = ChannelWorkspace(mesh.nodes, mesh.elements, mesh.dirichlet_nodes)
    res = solve_newton_transonic(ws, mach, m_start=mach if m_start is None else m_start, dm=dm,
                                 **(solve_kw or {}))
    t.cuda.synchronize()
    timings["forward_s"] = time.perf_counter() - c0
    if not res["converged"]:
        raise RuntimeError(f"forward solve did not converge: {res['level_history']}")
    c1 = time.perf_counter()
    phi = res["phi"]
    flow = FlowParams(m_inf=mach, u_inf=ws.u_inf)
    actx = AdjointContext(ws, phi, flow, frozen=res.get("frozen_state"))
    mon = ws.ev.read_monitors()  # of the Jacobian evaluation at the state
    # objective and its explicit partials
    X = t.from_numpy(mesh.nodes).cuda().requires_grad_(True)
    phi_g = phi.detach().clone().requires_grad_(True)
    faces_d = t.from_numpy(wall_faces_with_owners(mesh)).cuda()
    M = t.tensor(float(mach), dtype=t.float64, device="cuda", requires_grad=True)
    F = wall_force_objective(X, phi_g, faces_d, M, axis=axis, u_inf=ws.u_inf)
    gX_exp, gphi, gM_exp = t.autograd.grad(F, (X, phi_g, M))
    # J^T lam = dF/dphi on the free DOFs
    rhs = gphi.detach().masked_fill(ws.mask.bool(), 0.0).contiguous()
    JTf = with_dirichlet(actx.JT, ws.mask)
    ws.amg = M_pre = amg_for(ws.picard_matrix(), getattr(ws, "amg", None))
    lam, n_it, info = solve_gmres(JTf, rhs, M=M_pre, rtol=tol_lambda, restart=100, maxiter=50,
                                  on_fail="return")
    lam = lam.masked_fill(ws.mask.bool(), 0.0)
    # total derivatives: explicit - lam^T dR
    _, dX, dMr = actx.vjp(lam=(-lam).contiguous())
    dX_total = gX_exp.detach() + dX
    dz = t.from_numpy(shape.dz_dp()).cuda()
    dFdp = (dX_total[:, 2:3] * dz).sum(dim=0)  # the modes move z only
    dFdM = float(gM_exp) + float(dMr)
    t.cuda.synchronize()
    timings["adjoint_s"] = time.perf_counter() - c1
    return {"F": float(F.detach()), "dF_dp": dFdp.cpu().numpy(), "dF_dM": dFdM,
            "lambda": lam, "dF_dphi": rhs, "gmres_iterations": n_it, "gmres_info": info,
            "n_term3_active": int(mon["n_term3_active"]), "n_supersonic": int(mon["n_supersonic"]),
            "phi": phi, "newton": res, "timings": timings, "context": actx}


def objective_value(shape: BumpShape, mach: float, p=None, m_start: Optional[float] = None,
                    dm: float = 0.05, solve_kw: Optional[dict] = None, axis: int = 2) -> float:
    """F at (p, M_inf) after a converged solve (for finite differences)."""
    t = L.require_cuda()
    from .solve.newton import ChannelWorkspace, solve_newton_transonic
    mesh = shape.mesh(p)
    ws = ChannelWorkspace(mesh.nodes, mesh.elements, mesh.dirichlet_nodes)
    res = solve_newton_transonic(ws, mach, m_start=mach if m_start is None else m_start, dm=dm,
                                 **(solve_kw or {}))
    if not res["converged"]:
        raise RuntimeError("solve did not converge")
    X = t.from_numpy(mesh.nodes).cuda()
    M = t.tensor(float(mach), dtype=t.float64, device="cuda")
    return float(wall_force_objective(X, res["phi"], t.from_numpy(wall_faces_with_owners(mesh)).cuda(), M,
                                      axis=axis, u_inf=ws.u_inf))


def frozen_objective(shape: BumpShape, mach: float, phi0, frozen, p=None, axis: int = 2,
                     tol_residual: float = 1e-13, n_newton_max: int = 20) -> float:
    """F after Newton on the discrete equations with the (upstream, branch)
    selection `frozen` held fixed, from phi0 (a nearby converged state):
    the function whose derivative a frozen-finish adjoint gives.  Exact
    Jacobian (the frozen one), GMRES + AMG to 1e-12, full steps."""
    t = L.require_cuda()
    from .solve.fused import FlowParams
    from .solve.linear import amg_for, solve_gmres, with_dirichlet
    from .solve.newton import ChannelWorkspace
    mesh = shape.mesh(p)
    ws = ChannelWorkspace(mesh.nodes, mesh.elements, mesh.dirichlet_nodes)
    flow = FlowParams(m_inf=float(mach), u_inf=ws.u_inf)
    phi = t.where(ws.free, L.to_device(phi0, t.float64), ws.phi_dir).clone()
    for _ in range(n_newton_max):
        R, _ = ws.residual(phi, flow, frozen=frozen, jacobian=True)
        Rf = ws.r_free(R).clone()
        if float(Rf.abs().max()) < tol_residual:
            break
        J = with_dirichlet(ws.ev.jacobian(), ws.mask)
        ws.amg = M = amg_for(ws.picard_matrix(), getattr(ws, "amg", None))
        dphi, _, _ = solve_gmres(J, -Rf, M=M, rtol=1e-12, restart=100, maxiter=50, on_fail="return")
        phi = phi + dphi.masked_fill(ws.mask.bool(), 0.0)
    else:
        raise RuntimeError("frozen solve did not converge")
    X = t.from_numpy(mesh.nodes).cuda()
    M = t.tensor(float(mach), dtype=t.float64, device="cuda")
    return float(wall_force_objective(X, phi, t.from_numpy(wall_faces_with_owners(mesh)).cuda(), M, axis=axis,
                                      u_inf=ws.u_inf))
