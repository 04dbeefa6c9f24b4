"""Wall Cp and pressure-force coefficients on the B200, with the reference's
signatures (pyfp3d/post/surface.py:80-363).

``wall_force_coefficients`` evaluates, per wall triangle, the in-plane P1
gradient of phi, the optional normal-gated smoothing, Cp and the force
integral on the device (``up3d_wall_forces``); the triangles' owning tets
and edge neighbours are found once per (mesh, wall) and kept.  Arrays in,
same kind out: numpy in, numpy out; CUDA tensors in, CUDA tensors out.
"""

from __future__ import annotations

import ctypes
import zlib

import numpy as np

from .. import _lib as L
from ..mesh.device import get_mesh
from ..physics.isentropic import GAMMA


class _Wall:
    def __init__(self, mesh, elements, wall_faces):
        h = ctypes.c_void_p()
        el = np.ascontiguousarray(elements, dtype=np.int32)
        wf = np.ascontiguousarray(wall_faces, dtype=np.int64)
        L.call("up3d_wall_create", mesh.handle, el.ctypes.data, wf.ctypes.data, len(wf), ctypes.byref(h))
        self.handle, self.mesh, self.n = h.value, mesh, len(wf)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            try:
                L.lib().up3d_wall_destroy(h)
            except Exception:
                pass
            self.handle = None

    def run(self, phi, u_inf, m_inf, gamma, s_ref, smooth_passes, want=()):
        t = L.torch()
        d_phi = L.to_device(phi, t.float64)
        outs = {k: t.empty((self.n, 3) if k in ("grad", "normal", "outward") else self.n, dtype=t.float64,
                           device="cuda")
                for k in want}
        cf = (ctypes.c_double * 3)()
        L.call("up3d_wall_forces", self.handle, self.mesh.handle, d_phi.data_ptr(), float(u_inf), float(m_inf),
               float(gamma), float(s_ref), int(smooth_passes),
               *[outs[k].data_ptr() if k in outs else None for k in ("grad", "area", "normal", "outward", "cp")],
               ctypes.addressof(cf), L.stream_ptr())
        return np.array(cf[:]), outs


_WALLS: dict = {}


def _wall(nodes, elements, wall_faces):
    mesh = get_mesh(nodes, elements)
    wf = np.ascontiguousarray(np.asarray(wall_faces.cpu() if L.is_torch(wall_faces) else wall_faces),
                              dtype=np.int64)
    key = (id(mesh), len(wf), zlib.crc32(wf.tobytes()))
    w = _WALLS.get(key)
    if w is None:
        el = elements.cpu().numpy() if L.is_torch(elements) else elements
        if len(_WALLS) >= 8:
            _WALLS.pop(next(iter(_WALLS)))
        w = _WALLS[key] = _Wall(mesh, el, wf)
    return w


def _out(x, like):
    return x if L.is_torch(like) else x.cpu().numpy()


def triangle_tangential_gradients(nodes, wall_faces, phi, elements=None):
    """(grad_tri, area, normal) per wall triangle, normal of the stored
    winding (post/surface.py:80-118).  The device path works on a mesh
    handle, so it also takes the mesh's elements (the reference's function
    does not); TypeError without them."""
    if elements is None:
        raise TypeError("triangle_tangential_gradients on the device needs elements= (the mesh's tets)")
    w = _wall(nodes, elements, wall_faces)
    _, o = w.run(phi, 1.0, 0.0, GAMMA, 1.0, 0, want=("grad", "area", "normal"))
    return _out(o["grad"], phi), _out(o["area"], phi), _out(o["normal"], phi)


def wall_outward_normals(nodes, elements, wall_faces):
    """Unit wall-triangle normals pointing into the fluid (post/surface.py:
    192-231)."""
    w = _wall(nodes, elements, wall_faces)
    t = L.torch()
    _, o = w.run(t.zeros(len(nodes), dtype=t.float64, device="cuda"), 1.0, 0.0, GAMMA, 1.0, 0, want=("outward",))
    return _out(o["outward"], nodes)


def wall_force_coefficients(nodes, elements, wall_faces, phi, alpha_deg: float = 0.0, u_inf: float = 1.0,
                            s_ref: float = 1.0, m_inf: float = 0.0, smooth_passes: int = 0) -> dict:
    """cl, cd_pressure, cf (3-vector) and cp_tri (post/surface.py:309-363)."""
    w = _wall(nodes, elements, wall_faces)
    cf, o = w.run(phi, u_inf, m_inf, GAMMA, s_ref, smooth_passes, want=("cp",))
    a = np.deg2rad(alpha_deg)
    lift = np.array([-np.sin(a), np.cos(a), 0.0])
    drag = np.array([np.cos(a), np.sin(a), 0.0])
    return {"cl": float(cf @ lift), "cd_pressure": float(cf @ drag), "cf": cf, "cp_tri": _out(o["cp"], phi)}
