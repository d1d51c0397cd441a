"""CPU checks of the C-ABI boundary: the library loads and exports every declared symbol, and
the host-side layout validation accepts dense layouts (any stride on a length-1 axis) and
rejects others."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _declared():
    text = (ROOT / "include" / "motionest.h").read_text()
    return sorted(set(re.findall(r"\b(me_[a-z0-9_]+)\s*\(", text)))


def test_header_and_binding_agree():
    from motionest import _lib
    assert sorted(_lib.declared_symbols()) == _declared()


def test_library_exports_every_declared_symbol():
    from motionest import build
    lib_path = build.build()
    lib = ctypes.CDLL(str(lib_path))
    for name in _declared():
        assert hasattr(lib, name), name
    lib.me_abi_version.restype = ctypes.c_int
    assert lib.me_abi_version() == 1


def _validate_layout(dims, strides):
    """me_rigid_apply with NULL data pointers: the grid and layout checks run first, on the
    host, so the answer says whether the layout was accepted ("NULL pointer" next) or not."""
    from motionest import _lib
    lib = _lib.load()
    g = _lib.MeGrid()
    g.nx, g.ny, g.nz = dims
    dummy = (ctypes.c_double * 1)()
    addr = ctypes.addressof(dummy)
    for a in range(3):
        g.k[a] = g.tan_rk[a] = g.sin_rk[a] = addr
    rc = lib.me_rigid_apply(None, 0, None, 0, 1, _lib.MeLayout(*strides), ctypes.byref(g),
                            None, 0, 0, None)
    return rc, lib.me_last_error().decode()


@pytest.mark.parametrize("order", ["xyz", "xzy", "yxz", "yzx", "zxy", "zyx"])
def test_every_dense_axis_order_is_accepted(order):
    dims = {"x": 6, "y": 5, "z": 4}
    stride, s = {}, 1
    for a in reversed(order):  # last axis contiguous
        stride[a] = s
        s *= dims[a]
    rc, msg = _validate_layout((6, 5, 4), (stride["x"], stride["y"], stride["z"]))
    assert rc == 1 and "NULL pointer" in msg, msg


@pytest.mark.parametrize("strides", [(20, 5, 1), (5, 1, 40), (21, 4, 1), (24, 4, 1)])
def test_non_dense_layouts_are_rejected(strides):
    rc, msg = _validate_layout((6, 5, 4), strides)
    assert rc == 1 and "dense permutation" in msg, msg


@pytest.mark.parametrize("dims,strides", [((6, 5, 1), (5, 1, 1)), ((6, 5, 1), (5, 1, 999)),
                                          ((6, 1, 4), (4, 4, 1)), ((1, 5, 4), (0, 4, 1))])
def test_length_one_axes_take_any_stride(dims, strides):
    rc, msg = _validate_layout(dims, strides)
    assert rc == 1 and "NULL pointer" in msg, msg
