"""The C-ABI library loads without a GPU and exports every symbol declared in
include/nrgb.h; context creation fails cleanly (nonzero status) without one."""
import ctypes
import os
import re

import pytest

import nrgb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "nrgb.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(nrgb_[a-z_0-9]+)\s*\(", src)))


def test_header_and_wrapper_agree():
    assert set(declared_symbols()) == set(nrgb.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = nrgb.load()
    for name in declared_symbols():
        assert hasattr(lib, name), name
    assert lib.nrgb_version().startswith(b"nrgb")


def test_create_without_device_fails_cleanly():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    lib = nrgb.load()
    h = ctypes.c_void_p()
    assert lib.nrgb_create(0, ctypes.byref(h)) != 0


def test_wait_limit_arguments_are_checked_without_a_device():
    lib = nrgb.load()
    assert lib.nrgb_set_wait_limit(None, 3) == 1      # below the allowed range
    assert lib.nrgb_set_wait_limit(None, 31) == 1     # above it
    assert lib.nrgb_set_wait_limit(None, 16) == 1     # null context
    assert lib.nrgb_inject_barrier_shortfall(None, 1) == 1
