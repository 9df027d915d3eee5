"""alp_lex_noalloc: lexing for callers that cannot allocate device memory.

The entry point keeps its look-back scratch in a fixed array compiled into
the library instead of growing context scratch with cudaMalloc.  This test
calls it through the C ABI twice in a row (a second, different input checks
that the shared array is cleared between calls) and compares every token with
the allocating entry point alp_lex_into; integer outputs, so equality is exact.
It lives in its own file, collected after every other test.
"""

import ctypes

import numpy as np
import pytest

from alpacc_b200 import synth, tables

pytestmark = pytest.mark.gpu

MAX_BYTES = 128 << 20


def _lex(L, h, fn, d, cap):
    import torch
    term = torch.empty(cap, dtype=torch.int32, device=d.device)
    start = torch.empty(cap, dtype=torch.int64, device=d.device)
    end = torch.empty(cap, dtype=torch.int64, device=d.device)
    n, valid = ctypes.c_int64(0), ctypes.c_int(0)
    rc = fn(h, ctypes.c_void_p(d.data_ptr()), ctypes.c_int64(d.numel()), ctypes.c_void_p(term.data_ptr()),
            ctypes.c_void_p(start.data_ptr()), ctypes.c_void_p(end.data_ptr()), ctypes.c_int64(cap),
            ctypes.byref(n), ctypes.byref(valid))
    assert rc == 0, L.alp_last_error(h)
    k = n.value
    return valid.value, term[:k].cpu().numpy(), start[:k].cpu().numpy(), end[:k].cpu().numpy()


def test_noalloc_matches_alp_lex_into(has_gpu):
    import torch
    from alpacc_b200.api import Grammar, native
    L = native()
    L.alp_lex_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                  ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int)]
    g = Grammar(tables.load("json", "lexer"))
    docs = [synth.json_doc(3_000_000, 8, 0xA1FACC00 + 51), synth.json_doc(1_234_567, 8, 0xA1FACC00 + 52)]
    for doc in docs:  # two calls in a row
        d = torch.from_numpy(doc).cuda()
        cap = doc.size + 1
        ref = _lex(L, g.h, L.alp_lex_into, d, cap)
        got = _lex(L, g.h, L.alp_lex_noalloc, d, cap)
        assert got[0] == ref[0] == 1
        for a, b in zip(got[1:], ref[1:]):
            np.testing.assert_array_equal(a, b)

    # a rejected input reports valid = 0 like the allocating entry point
    bad = torch.from_numpy(np.frombuffer(b'{"a": 1, "b": "unterminated', dtype=np.uint8).copy()).cuda()
    assert _lex(L, g.h, L.alp_lex_noalloc, bad, 64)[0] == 0

    # inputs over the limit are refused before any device work
    n, valid = ctypes.c_int64(0), ctypes.c_int(0)
    small = torch.zeros(16, dtype=torch.uint8, device="cuda")
    rc = L.alp_lex_noalloc(g.h, ctypes.c_void_p(small.data_ptr()), ctypes.c_int64(MAX_BYTES + 1), None, None,
                           None, ctypes.c_int64(0), ctypes.byref(n), ctypes.byref(valid))
    assert rc == 1 and b"limit" in L.alp_last_error(g.h)
