"""The C-ABI library loads and exports every symbol include/p3m.h declares
(no GPU needed: nothing here launches a kernel)."""

import ctypes
import re
from pathlib import Path

import pytest

from gravity_b200 import _abi
from gravity_b200.config import GravityFieldConfig, P3MConfig

HEADER = Path(__file__).resolve().parent.parent / "include" / "p3m.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(p3m_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported_and_bound():
    lib = _abi.load()
    names = declared_functions()
    assert len(names) >= 30
    for name in names:
        assert hasattr(lib, name), f"{name} declared in p3m.h but not exported"
        assert name in _abi.SIGNATURES, f"{name} has no ctypes signature"
    assert sorted(_abi.SIGNATURES) == names


def test_library_is_built_for_sm100a_only():
    """The shared object carries sm_100a device code (checked from nvcc's
    build flags, not by reading the binary)."""
    from gravity_b200 import build

    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert build.LIB_PATH.exists()


def test_config_struct_layout_and_defaults():
    c = _abi.default_config()
    assert c.struct_size == ctypes.sizeof(_abi.P3MConfig)
    py = P3MConfig().to_abi()
    for field, _ in _abi.P3MConfig._fields_:
        if field == "capacity":
            continue
        assert getattr(c, field) == pytest.approx(getattr(py, field)), field


def test_status_strings():
    assert _abi.status_name(_abi.P3M_OK) == "ok"
    assert "capacity" in _abi.status_name(_abi.P3M_ERR_CAPACITY)


def test_create_rejects_invalid_configs_before_touching_a_device():
    lib = _abi.load()
    ctx = ctypes.c_void_p()
    bad = P3MConfig(gravity=GravityFieldConfig(grid_width=512, grid_height=256)).to_abi()
    bad.grid_width = 500
    assert lib.p3m_create(ctypes.byref(bad), ctypes.byref(ctx)) == _abi.P3M_ERR_UNSUPPORTED
    assert b"power of two" in lib.p3m_last_error(None)
    bad = P3MConfig().to_abi()
    bad.struct_size = 4
    assert lib.p3m_create(ctypes.byref(bad), ctypes.byref(ctx)) == _abi.P3M_ERR_INVALID_ARGUMENT
    bad = P3MConfig().to_abi()
    bad.capacity = 0
    assert lib.p3m_create(ctypes.byref(bad), ctypes.byref(ctx)) == _abi.P3M_ERR_INVALID_ARGUMENT
    assert not ctx.value


def test_calls_on_a_null_context_fail_without_crashing():
    lib = _abi.load()
    assert lib.p3m_step(None, 10, 1) == _abi.P3M_ERR_INVALID_ARGUMENT
    assert lib.p3m_synchronize(None) == _abi.P3M_ERR_INVALID_ARGUMENT
    assert lib.p3m_destroy(None) == _abi.P3M_OK


def test_no_device_means_a_loud_error():
    """Without a usable CUDA device the product refuses to run (there is no
    CPU fallback)."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present; the no-device path is not reachable")
    from gravity_b200.pipeline import GravityPipeline

    with pytest.raises(_abi.P3MError):
        GravityPipeline(P3MConfig(capacity=16))
