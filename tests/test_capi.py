"""The C-ABI library loads without a GPU and exports every symbol the public
header declares (no compute calls here)."""

import ctypes

import pytest

from up3d_b200 import _lib as L


def test_library_built():
    assert L.LIB_PATH.exists(), "run python -m up3d_b200.build"


def test_header_symbols_exported():
    lib = ctypes.CDLL(str(L.LIB_PATH))
    names = L.header_symbols()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_binding_covers_header():
    names = set(L.header_symbols())
    bound = set(L.SIGNATURES)
    assert names - bound == set(), f"header symbols without a ctypes signature: {names - bound}"
    assert bound - names == set(), f"bound but not declared: {bound - names}"


def test_build_targets_sm100a_only():
    from up3d_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_status_mapping():
    assert L.STATUS_EXC[-1] is ValueError
    assert L.STATUS_EXC[-2] is RuntimeError
    assert L.STATUS_EXC[-3] is NotImplementedError
    assert L.lib().up3d_version() == 1


def test_no_device_raises_cleanly():
    """Without a device the Python layer refuses instead of falling back."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is visible")
    from up3d_b200.kernels.jacobian import PicardOperator
    import numpy as np
    with pytest.raises(RuntimeError, match="CUDA device"):
        PicardOperator(np.zeros((4, 3)), np.array([[0, 1, 2, 3]], dtype=np.int32))


def test_pool_accounting_without_a_device():
    """The device block cache's accounting entry points are host-only: with
    nothing allocated they report an empty cache, a release frees nothing,
    and a null argument is refused."""
    s = L.pool_stats()
    if s["live_bytes"] == 0 and s["misses"] == 0:  # no device buffer made in this process
        assert s == {"cached_bytes": 0, "live_bytes": 0, "hits": 0, "misses": 0}
        assert L.pool_release() == 0
    with pytest.raises(TypeError):
        L.call("up3d_pool_stats", None, None, None, None)
