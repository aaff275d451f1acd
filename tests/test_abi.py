"""The C-ABI library loads and exports every entry point include/pyg.h
declares; without a GPU it refuses to create a context (no CPU fallback)."""
import ctypes
import os
import re

import pytest

import pyg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = ""
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if h.endswith(".h"):
            with open(os.path.join(ROOT, "include", h)) as f:
                text += f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pyg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = pyg.lib()
    names = declared_symbols()
    assert len(names) > 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    bound = {n for n, _, _ in pyg.SIGNATURES}
    assert set(declared_symbols()) <= bound


def test_version_and_error_string():
    L = pyg.lib()
    assert b"sm_100a" in L.pyg_version()
    assert isinstance(L.pyg_last_error(), bytes)


def test_null_arguments_are_rejected_without_touching_a_device():
    L = pyg.lib()
    assert L.pyg_ctx_create(0, None) == pyg.PYG_ERR_ARG
    assert L.pyg_hashtable_stats(None, None, None, None, None) == pyg.PYG_ERR_ARG


def test_no_cpu_fallback_without_gpu():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    rc = pyg.lib().pyg_ctx_create(0, ctypes.byref(h))
    assert rc == pyg.PYG_ERR_NO_DEVICE
    assert b"device" in pyg.lib().pyg_last_error()
