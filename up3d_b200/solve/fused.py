"""Fused residual + Newton Jacobian evaluation on the device.

One call does what ``NewtonWorkspace.eval_residual`` followed by
``assemble_coupled`` do without a wake (pyfp3d/solve/newton.py:345-372,
:430-457 with T = I): velocities, speed limiter, density, upstream walk (or
the frozen selection), upwinded density, its sensitivities, the residual R
and the Newton Jacobian (Terms 1-3) -- one tiled pass over the mesh and a
short combine of the outputs shared by tiles (or, by tuning, two passes: an
element sweep and a row gather), plus the Term-3 merge when supersonic
elements exist.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

from .. import _lib as L
from ..mesh.device import DeviceCSR, DeviceMesh


@dataclass
class FlowParams:
    m_inf: float
    gamma: float = 1.4
    u_inf: float = 1.0
    m_cap: float = 3.0
    m_crit: float = 0.95
    upwind_c: float = 1.5
    rho_floor: float = 0.05

    def c(self) -> L.Flow:
        return L.flow(self.m_inf, self.gamma, self.u_inf, self.m_cap, self.m_crit, self.upwind_c,
                      self.rho_floor)


class ResidualJacobian:
    """Device workspace of the fused evaluation on one mesh."""

    def __init__(self, mesh: DeviceMesh):
        t = L.require_cuda()
        self.mesh = mesh
        self.R = t.empty(mesh.n_nodes, dtype=t.float64, device="cuda")
        self.data = t.empty(mesh.nnz, dtype=t.float64, device="cuda")
        self.rho_tilde = t.empty(mesh.n_tets, dtype=t.float64, device="cuda")
        self.upstream = t.empty(mesh.n_tets, dtype=t.int32, device="cuda")
        self.monitors = L.monitors_buffer()
        self._n_extra = 0
        if mesh.tuning()["assembly"] == 1:
            mesh.tile_info()  # the tile plan now, not inside a timed solve

    def evaluate(self, phi, flow: FlowParams, jacobian: bool = True, frozen=None,
                 keep_state=True, R_out=None, data_out=None):
        """R(phi) (and the Jacobian data on the P1 pattern) into this
        workspace, or into R_out / data_out when given.  `frozen` =
        (upstream int64, branch int8) selects the frozen flux.  keep_state:
        True writes rho~ and the upstream map to ``rho_tilde`` /
        ``upstream``, "upstream" the upstream map only, False neither."""
        up_fz = br_fz = None
        if frozen is not None:
            t = L.torch()
            up_fz = L.to_device(frozen[0], t.int64)
            br_fz = L.to_device(frozen[1], t.int8)
        R = self.R if R_out is None else R_out
        data = self.data if data_out is None else data_out
        L.call("up3d_residual_jacobian", self.mesh.handle, phi.data_ptr(), flow.c(),
               L.ptr(up_fz), L.ptr(br_fz), R.data_ptr(),
               data.data_ptr() if jacobian else None,
               self.rho_tilde.data_ptr() if keep_state is True else None,
               self.upstream.data_ptr() if keep_state else None,
               self.monitors.data_ptr(), L.stream_ptr())
        return R

    def read_monitors(self) -> dict:
        return L.read_monitors(self.monitors)

    def jacobian(self, newton_nnz: int | None = None) -> DeviceCSR:
        """The merged Newton Jacobian of the last evaluate(jacobian=True)."""
        t = L.torch()
        mon = self.read_monitors()
        if mon["n_term3_active"] == 0:
            return DeviceCSR(self.mesh.indptr, self.mesh.indices, self.data,
                             (self.mesh.n_nodes, self.mesh.n_nodes))
        if newton_nnz is None:
            newton_nnz = self.newton_nnz()
        indptr = t.empty(self.mesh.n_nodes + 1, dtype=t.int32, device="cuda")
        indices = t.empty(newton_nnz, dtype=t.int32, device="cuda")
        data = t.empty(newton_nnz, dtype=t.float64, device="cuda")
        L.call("up3d_jacobian_export", self.mesh.handle, self.data.data_ptr(), indptr.data_ptr(),
               indices.data_ptr(), data.data_ptr(), L.stream_ptr())
        return DeviceCSR(indptr, indices, data, (self.mesh.n_nodes, self.mesh.n_nodes))

    def evaluate_host(self, phi_host, flow: FlowParams, R_host, J_host) -> None:
        """One evaluation on host buffers (pinned CPU tensors): copy phi in,
        evaluate R and the Jacobian data on the P1 pattern, copy both back;
        returns when R_host / J_host hold the result."""
        t = L.torch()
        if not hasattr(self, "_phi_in"):
            self._phi_in = t.empty(self.mesh.n_nodes, dtype=t.float64, device="cuda")
        self._phi_in.copy_(phi_host, non_blocking=True)
        self.evaluate(self._phi_in, flow, jacobian=True, keep_state=False)
        R_host.copy_(self.R, non_blocking=True)
        J_host.copy_(self.data, non_blocking=True)
        t.cuda.current_stream().synchronize()

    def newton_nnz(self) -> int:
        """nnz of the merged Jacobian (exact zeros dropped when Term 3 is
        active, like scipy's CSR addition)."""
        out = ctypes.c_int64()
        L.call("up3d_jacobian_nnz", self.mesh.handle, self.data.data_ptr(), ctypes.byref(out),
               L.stream_ptr())
        return int(out.value)


class HostPipeline:
    """Residual + Jacobian evaluations on host buffers, double-buffered:
    uploads and downloads run on two copy streams (PCIe is full duplex), so
    step k's results come back while step k+1's phi goes up and step k+1 is
    evaluated on the compute stream.  Every
    step still copies its phi host -> device and its R and Jacobian data
    device -> host; ``finish()`` returns when all requested results are in
    their host buffers."""

    def __init__(self, ev: ResidualJacobian):
        t = L.require_cuda()
        self.ev = ev
        m = ev.mesh
        self.compute = t.cuda.current_stream()
        self.up = t.cuda.Stream()
        self.down = t.cuda.Stream()
        self.slots = []
        for _ in range(2):
            self.slots.append({
                "phi": t.empty(m.n_nodes, dtype=t.float64, device="cuda"),
                "R": t.empty(m.n_nodes, dtype=t.float64, device="cuda"),
                "J": t.empty(m.nnz, dtype=t.float64, device="cuda"),
                "free": t.cuda.Event(), "loaded": t.cuda.Event(), "done": t.cuda.Event(),
            })
            self.slots[-1]["free"].record(self.down)
        self.k = 0

    def submit(self, phi_host, flow: FlowParams, R_host, J_host) -> None:
        t = L.torch()
        s = self.slots[self.k % 2]
        self.k += 1
        with t.cuda.stream(self.up):
            self.up.wait_event(s["free"])
            s["phi"].copy_(phi_host, non_blocking=True)
            s["loaded"].record(self.up)
        self.compute.wait_event(s["loaded"])
        with t.cuda.stream(self.compute):
            self.ev.evaluate(s["phi"], flow, jacobian=True, keep_state=False, R_out=s["R"],
                             data_out=s["J"])
            s["done"].record(self.compute)
        with t.cuda.stream(self.down):
            self.down.wait_event(s["done"])
            R_host.copy_(s["R"], non_blocking=True)
            J_host.copy_(s["J"], non_blocking=True)
            s["free"].record(self.down)

    def finish(self) -> None:
        self.up.synchronize()
        self.down.synchronize()
        self.compute.synchronize()
