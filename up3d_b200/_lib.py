"""ctypes binding of the up3d C ABI (include/up3d.h) and device-array helpers.

The library is loaded from ``up3d_b200/lib/libup3d.so`` (built in-tree by
``up3d_b200.build``).  There is no fallback: if the library is missing or no
CUDA device is visible, every device entry point raises.

Status codes map to the reference's exception classes:
UP3D_ERR_VALUE -> ValueError, UP3D_ERR_RUNTIME -> RuntimeError,
UP3D_ERR_NOT_IMPLEMENTED -> NotImplementedError, UP3D_ERR_ARGUMENT ->
TypeError.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "lib" / "libup3d.so"
HEADER = HERE.parent / "include" / "up3d.h"

_d = ctypes.c_double
_i64 = ctypes.c_int64
_i32 = ctypes.c_int32
_p = ctypes.c_void_p
_int = ctypes.c_int


class Flow(ctypes.Structure):
    """up3d_flow"""
    _fields_ = [("m_inf", _d), ("gamma", _d), ("u_inf", _d), ("m_cap", _d),
                ("m_crit", _d), ("upwind_c", _d), ("rho_floor", _d)]


class Monitors(ctypes.Structure):
    """up3d_monitors (device-resident; read back with read_monitors)."""
    _fields_ = [("nu_max", _d), ("n_supersonic", _i64), ("n_floored", _i64),
                ("n_limited", _i64), ("n_term3_active", _i64), ("n_term3_extra", _i64)]


class MeshInfo(ctypes.Structure):
    _fields_ = [("n_nodes", _i64), ("n_tets", _i64), ("nnz", _i64), ("max_row_len", _i32),
                ("max_node_degree", _i32), ("n_colors", _i32), ("device", _i32)]


class Tuning(ctypes.Structure):
    """up3d_tuning: launch shapes of the fused evaluation's two passes."""
    _fields_ = [("elem_persistent", _i32), ("elem_threads_per_sm", _i32), ("row_lanes", _i32),
                ("row_plan8", _i32), ("assembly", _i32), ("tile_elems", _i32), ("tile_stretch", _i32),
                ("reserved", _i32), ("elem_us", _d), ("row_us", _d)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class TileInfo(ctypes.Structure):
    """up3d_tile_info: size of the tiled assembly's plan."""
    _fields_ = [("tile_elems", _i32), ("tile_stretch", _i32), ("max_nodes", _i32), ("max_edges", _i32),
                ("n_tiles", _i64), ("n_tile_nodes", _i64),
                ("n_tile_edges", _i64), ("n_partials", _i64), ("n_combined_nodes", _i64),
                ("n_combined_slots", _i64), ("build_s", _d)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


MONITOR_BYTES = ctypes.sizeof(Monitors)

# name -> (restype, argtypes); every entry returns int status
SIGNATURES = {
    "up3d_last_error": (ctypes.c_char_p, []),
    "up3d_version": (_int, []),
    "up3d_mesh_create": (_int, [_p, _p, _i64, _i64, _int, _p, ctypes.POINTER(_p)]),
    "up3d_mesh_destroy": (_int, [_p]),
    "up3d_mesh_get_info": (_int, [_p, ctypes.POINTER(MeshInfo)]),
    "up3d_mesh_pattern": (_int, [_p, ctypes.POINTER(_p), ctypes.POINTER(_p)]),
    "up3d_mesh_geometry": (_int, [_p, _p, _p, _p]),
    "up3d_mesh_centroids": (_int, [_p, _p, _p]),
    "up3d_mesh_face_neighbors": (_int, [_p, _p, _p]),
    "up3d_mesh_set_face_neighbors": (_int, [_p, _p, _p]),
    "up3d_mesh_coloring": (_int, [_p, _p, _p, ctypes.POINTER(_i32)]),
    "up3d_mesh_elem_to_csr": (_int, [_p, _p, _p]),
    "up3d_velocities": (_int, [_p, _p, _p, _p, _p]),
    "up3d_element_velocity_q2": (_int, [_p, _p, _p, _i64, _p, _p, _p]),
    "up3d_limit_q2": (_int, [_p, _i64, _d, _d, _d, _p, _p, _p]),
    "up3d_density": (_int, [_p, _i64, _d, _d, _p, _p]),
    "up3d_mach_squared": (_int, [_p, _i64, _d, _d, _p, _p]),
    "up3d_density_derivative": (_int, [_p, _i64, _d, _d, _p, _p]),
    "up3d_mach_squared_derivative": (_int, [_p, _i64, _d, _d, _p, _p]),
    "up3d_pressure_coefficient": (_int, [_p, _i64, _d, _d, _p, _p]),
    "up3d_upwind_walk": (_int, [_p, _p, _p, _p]),
    "up3d_rho_tilde": (_int, [_p, _p, _p, _i64, ctypes.POINTER(Flow), _p, _p, _p, _p]),
    "up3d_classify_branches": (_int, [_p, _p, _p, _i64, ctypes.POINTER(Flow), _p, _p]),
    "up3d_rho_tilde_frozen": (_int, [_p, _p, _p, _p, _i64, ctypes.POINTER(Flow), _p, _p, _p, _p]),
    "up3d_rho_tilde_sens": (_int, [_p, _p, _p, _i64, ctypes.POINTER(Flow), _p, _p, _p]),
    "up3d_rho_tilde_frozen_sens": (_int, [_p, _p, _p, _p, _i64, ctypes.POINTER(Flow), _p, _p, _p]),
    "up3d_residual": (_int, [_p, _p, _p, _p, _p, _p, _p]),
    "up3d_picard_matrix": (_int, [_p, _p, _p, _p]),
    "up3d_picard_matrix_data": (_int, [_p, _p, _p, _p]),
    "up3d_jacobian": (_int, [_p, _p, _p, _p, _p, _p, _d, _p, _p, ctypes.POINTER(_i64),
                             ctypes.POINTER(_i64), ctypes.POINTER(_i64), _p]),
    "up3d_jacobian_data": (_int, [_p, _p, _p, _p, _p, _p, _d, _p, _p, ctypes.POINTER(_i64),
                             ctypes.POINTER(_i64), ctypes.POINTER(_i64), _p]),
    "up3d_jacobian_export": (_int, [_p, _p, _p, _p, _p, _p]),
    "up3d_jacobian_nnz": (_int, [_p, _p, ctypes.POINTER(_i64), _p]),
    "up3d_residual_jacobian": (_int, [_p, _p, ctypes.POINTER(Flow), _p, _p, _p, _p, _p, _p, _p, _p]),
    "up3d_residual_vjp": (_int, [_p, _p, ctypes.POINTER(Flow), _p, _p, _p, _p, _p, _p, _p, _p]),
    "up3d_jacobian_transpose": (_int, [_p, _p, _p, _p]),
    "up3d_residual_jacobian_batched": (_int, [_p, _p, _int, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p]),
    "up3d_wake_create": (_int, [_i64, _i64, _i64, _p, _p, _p, _i32, _p, _p, _int, ctypes.POINTER(_p)]),
    "up3d_wake_destroy": (_int, [_p]),
    "up3d_wake_info": (_int, [_p, ctypes.POINTER(_i64), ctypes.POINTER(_i64), ctypes.POINTER(_i64),
                              ctypes.POINTER(_i32)]),
    "up3d_wake_patterns": (_int, [_p, ctypes.POINTER(_p), ctypes.POINTER(_p), ctypes.POINTER(_p),
                                  ctypes.POINTER(_p)]),
    "up3d_wake_reduce": (_int, [_p, _p, _p, _p, _p]),
    "up3d_wake_reduced_rhs": (_int, [_p, _p, _p, _p, _p, _p]),
    "up3d_wake_expand": (_int, [_p, _p, _p, _p, _p]),
    "up3d_coupled_create": (_int, [_p, _i64, _p, _p, _p, _p, _i64, _p, _p, _p, _p, ctypes.POINTER(_p)]),
    "up3d_coupled_destroy": (_int, [_p]),
    "up3d_coupled_set_kutta_row": (_int, [_p, _p, _p, _p]),
    "up3d_coupled_set_farfield": (_int, [_p, _p, _p]),
    "up3d_coupled_dirichlet": (_int, [_p, ctypes.POINTER(_p)]),
    "up3d_coupled_state": (_int, [_p, _p, _p, _p, _p, _p]),
    "up3d_coupled_residual": (_int, [_p, _p, _p, _p, _p, _p, _p]),
    "up3d_coupled_apply": (_int, [_p, _p, _p, _p, _p, _p, _p, _p]),
    "up3d_gmres_coupled": (_int, [_p, _p, _p, _p, _p, _d, _d, _int, _int, _p, ctypes.POINTER(_i64),
                                  ctypes.POINTER(_d), ctypes.POINTER(_int), _p]),
    "up3d_terms23_side_coo": (_int, [_p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _d, _p, _p, _p, _i64,
                                     ctypes.POINTER(_i64), _p]),
    "up3d_wall_create": (_int, [_p, _p, _p, _i64, ctypes.POINTER(_p)]),
    "up3d_wall_destroy": (_int, [_p]),
    "up3d_wall_forces": (_int, [_p, _p, _p, _d, _d, _d, _d, _int, _p, _p, _p, _p, _p, _p, _p]),
    "up3d_face_normals": (_int, [_p, _p, _p]),
    "up3d_mesh_neighborhoods": (_int, [_p, _int, ctypes.POINTER(_p), ctypes.POINTER(_p),
                                       ctypes.POINTER(_i64), _p]),
    "up3d_face_neighborhoods": (_int, [_p, _i64, _int, _p, _p, ctypes.POINTER(_i64), _p]),
    "up3d_rho_tilde_kernel": (_int, [_p, _p, _p, _p, ctypes.POINTER(Flow), _int, _d, _d, _d, _p, _p,
                                     _p, _p]),
    "up3d_rho_tilde_blend": (_int, [_p, _p, _p, _p, ctypes.POINTER(Flow), _d, _d, _d, _p, _p, _p, _p]),
    "up3d_mesh_set_tuning": (_int, [_p, ctypes.POINTER(Tuning)]),
    "up3d_mesh_get_tuning": (_int, [_p, ctypes.POINTER(Tuning)]),
    "up3d_autotune": (_int, [_p, _p, ctypes.POINTER(Flow), _int, ctypes.POINTER(Tuning), _p]),
    "up3d_mesh_tile_info": (_int, [_p, _i32, ctypes.POINTER(TileInfo), _p]),
    "up3d_mesh_term3_cache_hits": (_int, [_p, ctypes.POINTER(_i64)]),
    "up3d_tile_plan_host_create": (_int, [_p, _p, _p, _i64, _i64, _p, _p, _i32, _i32, ctypes.POINTER(_p)]),
    "up3d_tile_plan_host_info": (_int, [_p, ctypes.POINTER(TileInfo)]),
    "up3d_tile_plan_host_array": (_int, [_p, ctypes.c_char_p, _p, ctypes.POINTER(_i64)]),
    "up3d_tile_plan_host_destroy": (_int, [_p]),
    "up3d_launch_count": (_int, [ctypes.POINTER(_i64)]),
    "up3d_pool_stats": (_int, [ctypes.POINTER(_i64), ctypes.POINTER(_i64), ctypes.POINTER(_i64),
                               ctypes.POINTER(_i64)]),
    "up3d_pool_release": (_int, [ctypes.POINTER(_i64)]),
    "up3d_profile": (_int, [_int]),
    "up3d_profile_read": (_int, [_p, _p, _p, _int]),
    "up3d_spmv": (_int, [_i64, _p, _p, _p, _p, _p, _p, _p]),
    "up3d_spmv_f32": (_int, [_i64, _p, _p, _p, _p, _p, _p, _p]),
    "up3d_amg_setup": (_int, [_p, _p, ctypes.POINTER(_p), _p]),
    "up3d_amg_get_info": (_int, [_p, _p]),
    "up3d_amg_refresh": (_int, [_p, _p, _p]),
    "up3d_precond_jacobi": (_int, [_p, ctypes.POINTER(_p), _p]),
    "up3d_precond_ilu0": (_int, [_p, _int, _int, ctypes.POINTER(_p), _p]),
    "up3d_precond_ilu0_factors": (_int, [_p, _p, ctypes.POINTER(_d), _p]),
    "up3d_precond_apply": (_int, [_p, _p, _p, _p]),
    "up3d_amg_vcycle": (_int, [_p, _p, _p, _p]),
    "up3d_amg_vcycle_f32": (_int, [_p, _p, _p, _p]),
    "up3d_precond_destroy": (_int, [_p]),
    "up3d_cg": (_int, [_p, _p, _p, _d, _d, _int, _p, ctypes.POINTER(_i64), ctypes.POINTER(_d),
                       ctypes.POINTER(_int), _p]),
    "up3d_gmres": (_int, [_p, _p, _p, _p, _d, _d, _int, _int, _p, ctypes.POINTER(_i64),
                          ctypes.POINTER(_d), ctypes.POINTER(_int), _p]),
    "up3d_gmres_ir": (_int, [_p, _p, _p, _p, _p, _p, _d, _d, _int, _int, _int, _d, _p,
                             ctypes.POINTER(_i64), ctypes.POINTER(_i64), ctypes.POINTER(_d),
                             ctypes.POINTER(_int), _p]),
    "up3d_cg_jacobi_noalloc": (_int, [_p, _p, _p, _d, _d, _int, ctypes.POINTER(_i64),
                                      ctypes.POINTER(_d), ctypes.POINTER(_int), _p]),
}

NOALLOC_MAX_ROWS = 1 << 18  # UP3D_NOALLOC_MAX_ROWS


class CSR(ctypes.Structure):
    """up3d_csr"""
    _fields_ = [("n", _i64), ("indptr", _p), ("indices", _p), ("data", _p), ("dirichlet", _p)]


class AmgOptions(ctypes.Structure):
    """up3d_amg_options"""
    _fields_ = [("max_levels", _int), ("max_coarse", _i64), ("presmooth", _int),
                ("postsmooth", _int), ("fp32", _int)]


class AmgInfo(ctypes.Structure):
    """up3d_amg_info"""
    _fields_ = [("n_levels", _i32), ("n_coarse", _i64), ("operator_complexity", _d),
                ("level_rows", _i64 * 16)]

STATUS_EXC = {-1: ValueError, -2: RuntimeError, -3: NotImplementedError, -4: TypeError}

_lib = None


def header_symbols() -> list[str]:
    """Every function the public header declares."""
    import re
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*|int64_t)\s+(up3d_\w+)\s*\(",
                                 text, flags=re.M)))


def lib():
    """The loaded library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            if os.environ.get("UP3D_AUTOBUILD") == "1":
                from . import build
                build.build()
            else:
                raise RuntimeError(
                    f"up3d CUDA library not built ({LIB_PATH}); run "
                    "`python -m up3d_b200.build` (there is no CPU fallback)")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int, what: str = "") -> None:
    if status != 0:
        msg = lib().up3d_last_error().decode(errors="replace")
        exc = STATUS_EXC.get(status, RuntimeError)
        raise exc(f"{what}: {msg}" if what else msg)


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args), name)


# ------------------------------------------------------------------ torch glue

def torch():
    import torch as _t
    return _t


def require_cuda():
    t = torch()
    if not t.cuda.is_available():
        raise RuntimeError("up3d_b200 needs a CUDA device; none is visible (no CPU fallback)")
    return t


def stream_ptr():
    return torch().cuda.current_stream().cuda_stream


def ptr(t) -> int | None:
    """Device address of a contiguous CUDA tensor (None passes through)."""
    if t is None:
        return None
    if not t.is_cuda:
        raise TypeError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise TypeError("expected a contiguous tensor")
    return t.data_ptr()


def is_torch(x) -> bool:
    try:
        import torch as _t
        return isinstance(x, _t.Tensor)
    except ImportError:
        return False


def to_device(x, dtype, device=None):
    """numpy / torch -> contiguous CUDA tensor of `dtype` (no copy when it
    already is one)."""
    t = require_cuda()
    dev = device if device is not None else t.device("cuda", t.cuda.current_device())
    if is_torch(x):
        y = x.to(device=dev, dtype=dtype)
        return y.contiguous()
    arr = np.ascontiguousarray(x)
    return t.from_numpy(arr).to(device=dev, dtype=dtype, non_blocking=False).contiguous()


def flow(m_inf, gamma=1.4, u_inf=1.0, m_cap=3.0, m_crit=0.95, upwind_c=1.5, rho_floor=0.05) -> Flow:
    return Flow(float(m_inf), float(gamma), float(u_inf), float(m_cap), float(m_crit),
                float(upwind_c), float(rho_floor))


def read_monitors(dev_tensor) -> dict:
    """Copy a device up3d_monitors struct (uint8 tensor) to a dict."""
    host = dev_tensor.cpu().numpy().tobytes()
    m = Monitors.from_buffer_copy(host)
    return {k: getattr(m, k) for k, _ in Monitors._fields_}


PROF_SLOTS = ("elem_sweep", "row_gather", "term3", "spmv", "krylov")


def launch_count() -> int:
    out = ctypes.c_int64()
    call("up3d_launch_count", ctypes.byref(out))
    return int(out.value)


def pool_stats() -> dict:
    """The device block cache: bytes cached and handed out, cache hits and
    misses (up3d_pool_stats)."""
    v = [ctypes.c_int64() for _ in range(4)]
    call("up3d_pool_stats", *(ctypes.byref(x) for x in v))
    return dict(zip(("cached_bytes", "live_bytes", "hits", "misses"), (int(x.value) for x in v)))


def pool_release() -> int:
    """Frees every cached device block; returns the bytes released."""
    out = ctypes.c_int64()
    call("up3d_pool_release", ctypes.byref(out))
    return int(out.value)


def profile(enable: bool) -> None:
    call("up3d_profile", 1 if enable else 0)


def profile_read() -> dict:
    n = len(PROF_SLOTS)
    ms = (ctypes.c_double * n)()
    calls = (ctypes.c_int64 * n)()
    launches = (ctypes.c_int64 * n)()
    call("up3d_profile_read", ctypes.addressof(ms), ctypes.addressof(calls),
         ctypes.addressof(launches), n)
    return {name: {"ms": ms[i], "calls": calls[i], "launches": launches[i]}
            for i, name in enumerate(PROF_SLOTS)}


def monitors_buffer(device=None):
    t = require_cuda()
    return t.zeros(MONITOR_BYTES, dtype=t.uint8, device=device or "cuda")
