"""C-ABI checks that need no GPU: the library loads, exports every symbol include/hp2d.h
declares, and rejects unsupported reference flags before touching a device."""
import ctypes as C
import re
from pathlib import Path

import pytest

from hydropol2d_b200 import _abi

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols(header="hp2d.h"):
    text = (ROOT / "include" / header).read_text()
    return sorted(set(re.findall(r"^\s*(?:hp2d_status|const char\*)\s+(hp2d_\w+)\s*\(", text, re.M)))


def test_header_and_binding_agree():
    assert declared_symbols() == sorted(_abi.EXPORTS)
    assert declared_symbols("hp2d_nn.h") == sorted(_abi.NN_EXPORTS)


def test_library_exports_every_declared_symbol(hp2d_lib):
    for name in declared_symbols() + declared_symbols("hp2d_nn.h"):
        assert hasattr(hp2d_lib, name), name


def _create(**kw):
    L = _abi.lib()
    g = _abi.Grid(8, 8, 1.0, _abi.HP2D_FP32)
    p = _abi.default_params(**kw)
    h = C.c_void_p()
    st = L.hp2d_create(C.byref(g), C.byref(p), 0, C.byref(h))
    return st, L.hp2d_create_error().decode(), h


@pytest.mark.parametrize("flag,value", [("flag_subgrid", 1), ("flag_D8", 1),
                                        ("flag_numerical_scheme", 0), ("flag_numerical_scheme", 4),
                                        ("flag_infiltration", 3)])
def test_unsupported_flags_rejected(hp2d_lib, flag, value):
    st, msg, h = _create(**{flag: value})
    assert _abi.STATUS[st] == "HP2D_UNSUPPORTED_FLAG", msg
    assert not h.value


@pytest.mark.parametrize("kw", [dict(outlet_type=3), dict(min_time_step=0.0), dict(max_time_step=0.001),
                                dict(flag_critical=2), dict(flag_reservoir=2)])
def test_invalid_controls_rejected(hp2d_lib, kw):
    st, msg, _ = _create(**kw)
    assert _abi.STATUS[st] == "HP2D_INVALID_ARG", msg


def test_no_device_is_an_error_not_a_fallback(hp2d_lib):
    from tests.conftest import HAS_GPU
    if HAS_GPU:
        pytest.skip("a GPU is present")
    st, msg, _ = _create()
    assert _abi.STATUS[st] == "HP2D_NO_DEVICE", msg


def test_unknown_param_name_rejected():
    with pytest.raises(TypeError):
        _abi.default_params(flag_bogus=1)
