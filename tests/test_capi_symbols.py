"""The C-ABI library builds for sm_100a, loads without a GPU and exports
every function declared in include/alpacc_b200.h; the product path refuses
to run without a CUDA device (no CPU fallback)."""

import ctypes
import os
import re

import pytest

from alpacc_b200 import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            with open(os.path.join(ROOT, "include", fn)) as f:
                text = re.sub(r"/\*.*?\*/", "", f.read(), flags=re.S)
            names |= set(re.findall(r"\b(alp_\w+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    path = build.build_cuda()
    lib = ctypes.CDLL(path)
    names = _declared()
    assert len(names) >= 15
    for n in sorted(names):
        assert hasattr(lib, n), n


def test_no_cpu_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from alpacc_b200.api import AlpError, Grammar
    with pytest.raises(AlpError):
        Grammar("arithmetic")


def test_ctx_rejects_bad_blob():
    lib = ctypes.CDLL(build.build_cuda())
    h = ctypes.c_void_p()
    lib.alp_ctx_create.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    rc = lib.alp_ctx_create(b"not a blob at all", 17, 0, ctypes.byref(h))
    assert rc != 0 and not h.value
