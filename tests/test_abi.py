"""CPU tests: the C-ABI library loads and exports every entry point the public
header declares (no compute without a GPU)."""
import ctypes
import os
import re

from onedal_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            src = open(os.path.join(ROOT, "include", h)).read()
            names |= set(re.findall(r"KMB_API\s+[^;(]*?\b(kmb_\w+)\s*\(", src))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    assert {"kmb_train", "kmb_infer", "kmb_context_create"} <= names
    assert names == set(_native.EXPORTED), names ^ set(_native.EXPORTED)


def test_library_exports_every_declared_symbol():
    lib = _native.load_library()
    for name in declared_symbols():
        assert isinstance(getattr(lib, name), ctypes._CFuncPtr), name


def test_status_strings_and_version_without_gpu():
    lib = _native.load_library()
    assert lib.kmb_version().startswith(b"onedal_b200")
    assert b"empty" in lib.kmb_status_string(_native.KMB_ETOO_MANY_EMPTY)
    # calls that need a device report an error instead of crashing
    assert lib.kmb_train(None, 0, 0, None, 0, 0, None, None, None, None, None, None, None) == _native.KMB_EINVAL


def test_context_creation_fails_loudly_without_gpu():
    import torch
    if torch.cuda.is_available():
        return
    import pytest
    with pytest.raises(_native.NativeError):
        _native.Context(0)
