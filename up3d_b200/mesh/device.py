"""Device-resident mesh handle (owner of an ``up3d_mesh``) and a device CSR.

One handle serves every operator built on the same (nodes, elements): the
handles are cached by content digest (skipped for arrays that cannot have
changed since they were last seen), so ``PicardOperator`` and
``UpwindOperator`` on one mesh share a single device copy of the geometry,
adjacency and pattern, and the per-mesh setup runs once.
"""

from __future__ import annotations

import ctypes
import hashlib
from collections import OrderedDict

import numpy as np

from .. import _lib as L


class _DevView:
    """__cuda_array_interface__ over library-owned device memory."""

    def __init__(self, addr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {
            "shape": tuple(shape), "typestr": typestr, "data": (int(addr), False),
            "version": 3, "strides": None,
        }


def device_view(addr: int, shape, dtype):
    """Zero-copy torch view of library-owned device memory."""
    t = L.torch()
    typestr = {np.int32: "<i4", np.int64: "<i8", np.float64: "<f8", np.uint8: "|u1"}[dtype]
    return t.as_tensor(_DevView(addr, shape, typestr), device="cuda")


def _as_numpy(x, dtype):
    if L.is_torch(x):
        x = x.detach().cpu().numpy()
    return np.ascontiguousarray(np.asarray(x), dtype=dtype)


class DeviceMesh:
    """Owner of one up3d_mesh handle on one device."""

    def __init__(self, nodes, elements, device: int | None = None):
        t = L.require_cuda()
        nodes = _as_numpy(nodes, np.float64)
        elements = _as_numpy(elements, np.int32)
        if nodes.ndim != 2 or nodes.shape[1] != 3:
            raise ValueError(f"nodes must be (n_nodes, 3), got {nodes.shape}")
        if elements.ndim != 2 or elements.shape[1] != 4:
            raise ValueError(f"elements must be (n_tets, 4), got {elements.shape}")
        self.device = t.cuda.current_device() if device is None else int(device)
        handle = ctypes.c_void_p()
        with t.cuda.device(self.device):
            L.call("up3d_mesh_create", nodes.ctypes.data, elements.ctypes.data, len(nodes),
                   len(elements), self.device, L.stream_ptr(), ctypes.byref(handle))
        self.handle = handle.value
        info = L.MeshInfo()
        L.call("up3d_mesh_get_info", self.handle, ctypes.byref(info))
        self.n_nodes = int(info.n_nodes)
        self.n_tets = int(info.n_tets)
        self.nnz = int(info.nnz)
        self.max_row_len = int(info.max_row_len)
        self.max_node_degree = int(info.max_node_degree)
        self.nodes = nodes
        self.elements = elements
        ip, ix = ctypes.c_void_p(), ctypes.c_void_p()
        L.call("up3d_mesh_pattern", self.handle, ctypes.byref(ip), ctypes.byref(ix))
        # torch-owned copies of the pattern (valid independent of the handle)
        self.indptr = device_view(ip.value, (self.n_nodes + 1,), np.int32).clone()
        self.indices = device_view(ix.value, (self.nnz,), np.int32).clone()
        self._colors = None

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            try:
                L.lib().up3d_mesh_destroy(h)
            except Exception:
                pass
            self.handle = None

    # ---------------------------------------------------------- exports

    def geometry(self):
        t = L.torch()
        B = t.empty((self.n_tets, 4, 3), dtype=t.float64, device="cuda")
        V = t.empty(self.n_tets, dtype=t.float64, device="cuda")
        L.call("up3d_mesh_geometry", self.handle, B.data_ptr(), V.data_ptr(), L.stream_ptr())
        return B, V

    def centroids(self):
        t = L.torch()
        c = t.empty((self.n_tets, 3), dtype=t.float64, device="cuda")
        L.call("up3d_mesh_centroids", self.handle, c.data_ptr(), L.stream_ptr())
        return c

    def face_neighbors(self):
        t = L.torch()
        f = t.empty((self.n_tets, 4), dtype=t.int32, device="cuda")
        L.call("up3d_mesh_face_neighbors", self.handle, f.data_ptr(), L.stream_ptr())
        return f

    def set_face_neighbors(self, fn):
        t = L.torch()
        d = L.to_device(fn, t.int32)
        if tuple(d.shape) != (self.n_tets, 4):
            raise ValueError(f"face_neighbors must be ({self.n_tets}, 4), got {tuple(d.shape)}")
        if int(d.max()) >= self.n_tets or int(d.min()) < -1:
            raise ValueError("face_neighbors entries must be -1 or element indices")
        L.call("up3d_mesh_set_face_neighbors", self.handle, d.data_ptr(), L.stream_ptr())
        t.cuda.current_stream().synchronize()

    def coloring(self):
        if self._colors is None:
            nc = ctypes.c_int32()
            L.call("up3d_mesh_coloring", self.handle, None, None, ctypes.byref(nc))
            off = np.empty(nc.value + 1, dtype=np.int64)
            el = np.empty(self.n_tets, dtype=np.int64)
            L.call("up3d_mesh_coloring", self.handle, off.ctypes.data, el.ctypes.data,
                   ctypes.byref(nc))
            self._colors = (off, el, int(nc.value))
        return self._colors

    # ---------------------------------------------------------- launch shapes

    def tuning(self) -> dict:
        """The launch shapes of the fused evaluation (up3d_tuning)."""
        t = L.Tuning()
        L.call("up3d_mesh_get_tuning", self.handle, ctypes.byref(t))
        return t.as_dict()

    def set_tuning(self, elem_persistent: int = 0, elem_threads_per_sm: int = 512, row_lanes: int = 8,
                   row_plan8: int = 0, assembly: int = 0, tile_elems: int = 256, tile_stretch: int = 1) -> None:
        """Installs launch shapes by hand.  Within one assembly form (and,
        for the tiled form, one tile size and stretch) every shape computes
        the same bits; the forms agree to rounding."""
        t = L.Tuning(elem_persistent, elem_threads_per_sm, row_lanes, row_plan8, assembly, tile_elems,
                     tile_stretch, 0, 0.0, 0.0)
        L.call("up3d_mesh_set_tuning", self.handle, ctypes.byref(t))

    def term3_cache_hits(self) -> int:
        """Term-3 builds served by the values-only path so far."""
        h = ctypes.c_int64()
        L.call("up3d_mesh_term3_cache_hits", self.handle, ctypes.byref(h))
        return int(h.value)

    def tile_info(self, tile_elems: int | None = None) -> dict:
        """Sizes of the tiled assembly's plan (built here when missing)."""
        if tile_elems is None:
            tile_elems = self.tuning()["tile_elems"]
        t = L.TileInfo()
        L.call("up3d_mesh_tile_info", self.handle, int(tile_elems), ctypes.byref(t), L.stream_ptr())
        return t.as_dict()

    def autotune(self, phi, flow, reps: int = 5) -> dict:
        """Times every candidate shape of the element sweep and the row
        gather on this mesh at (phi, flow) and installs the fastest."""
        t = L.Tuning()
        L.call("up3d_autotune", self.handle, phi.data_ptr(), flow.c(), int(reps), ctypes.byref(t),
               L.stream_ptr())
        return t.as_dict()

    def elem_to_csr(self):
        t = L.torch()
        out = t.empty((self.n_tets, 4, 4), dtype=t.int64, device="cuda")
        L.call("up3d_mesh_elem_to_csr", self.handle, out.data_ptr(), L.stream_ptr())
        return out


_CACHE: "OrderedDict[tuple, DeviceMesh]" = OrderedDict()
_CACHE_SIZE = 4
# (identity key) -> (weak references to the caller's two arrays, content key):
# arrays that cannot have changed since they were digested skip the digest
_SEEN: "OrderedDict[tuple, tuple]" = OrderedDict()


def _digest(nodes: np.ndarray, elements: np.ndarray) -> str:
    h = hashlib.sha256()
    h.update(np.asarray(nodes.shape, dtype=np.int64).tobytes())
    h.update(memoryview(nodes).cast("B"))
    h.update(np.asarray(elements.shape, dtype=np.int64).tobytes())
    h.update(memoryview(elements).cast("B"))
    return h.hexdigest()


def _identity(x):
    """A key under which x cannot have changed while it is alive: a torch
    tensor's storage, shape and in-place version counter, or a read-only
    numpy array's buffer; None for anything else (a writeable array)."""
    if L.is_torch(x):
        return ("t", id(x), x.data_ptr(), tuple(x.shape), tuple(x.stride()), str(x.dtype), str(x.device),
                x._version)
    if isinstance(x, np.ndarray) and not x.flags.writeable and x.base is None:
        return ("n", id(x), x.ctypes.data, x.shape, x.strides, x.dtype.str)
    return None


def get_mesh(nodes, elements, device: int | None = None) -> DeviceMesh:
    """Shared DeviceMesh for (nodes, elements) on `device`, cached by a
    digest of their contents.  Torch tensors (tracked by their in-place
    version counter) and read-only numpy arrays that were seen before skip
    the digest; writeable numpy arrays are digested on every call, since
    they may have been changed in place."""
    import weakref
    t = L.require_cuda()
    dev = t.cuda.current_device() if device is None else int(device)
    ident = None
    a, b = _identity(nodes), _identity(elements)
    if a is not None and b is not None:
        ident = (a, b, dev)
        seen = _SEEN.get(ident)
        if seen is not None and seen[0]() is nodes and seen[1]() is elements and seen[2] in _CACHE:
            _CACHE.move_to_end(seen[2])
            return _CACHE[seen[2]]
    nodes_h = _as_numpy(nodes, np.float64)
    elements_h = _as_numpy(elements, np.int32)
    key = (_digest(nodes_h, elements_h), dev)
    m = _CACHE.get(key)
    if m is None:
        m = DeviceMesh(nodes_h, elements_h, dev)
        _CACHE[key] = m
        while len(_CACHE) > _CACHE_SIZE:
            _CACHE.popitem(last=False)
    else:
        _CACHE.move_to_end(key)
    if ident is not None:
        try:
            _SEEN[ident] = (weakref.ref(nodes), weakref.ref(elements), key)
            while len(_SEEN) > 4 * _CACHE_SIZE:
                _SEEN.popitem(last=False)
        except TypeError:   # an object without weak references: no shortcut
            pass
    return m


def clear_cache():
    _CACHE.clear()
    _SEEN.clear()


class DeviceCSR:
    """CSR matrix whose arrays are CUDA tensors (int32 indices, f64/f32 data).

    ``to_scipy()`` makes the host copy the reference's callers expect
    (``scipy.sparse.csr_matrix``)."""

    def __init__(self, indptr, indices, data, shape):
        self.indptr = indptr
        self.indices = indices
        self.data = data
        self.shape = tuple(shape)

    @property
    def nnz(self) -> int:
        return int(self.indices.numel())

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.data.detach().cpu().numpy(),
                              self.indices.detach().cpu().numpy(),
                              self.indptr.detach().cpu().numpy()), shape=self.shape)

    def matvec(self, x, y=None, dirichlet=None):
        """y = A x on the device (FP64 or FP32 by data dtype)."""
        t = L.torch()
        if y is None:
            y = t.empty_like(x)
        fn = "up3d_spmv" if self.data.dtype == t.float64 else "up3d_spmv_f32"
        L.call(fn, self.shape[0], self.indptr.data_ptr(), self.indices.data_ptr(),
               self.data.data_ptr(), x.data_ptr(), y.data_ptr(),
               None if dirichlet is None else dirichlet.data_ptr(), L.stream_ptr())
        return y

    def __matmul__(self, x):
        return self.matvec(x)
