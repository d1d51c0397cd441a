"""CPU checks of the C-ABI boundary: the library loads and exports every declared symbol."""
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
