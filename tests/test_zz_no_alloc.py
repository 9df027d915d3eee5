"""alp_lex_noalloc: lexing for callers that cannot allocate device memory.

A serving process that reserved the whole GPU for its own pool, or a path
where a cudaMalloc would synchronise the device, cannot let the library grow
its scratch.  alp_lex_noalloc keeps its look-back scratch in a fixed array
compiled into the library instead.  These tests call it through the C ABI,
two calls in a row per grammar (the second input differs, so a shared array
left dirty by the first call would show), and compare every token with the
allocating entry point alp_lex_into and with the CPU oracle; the outputs are
integers, so equality is exact.  They also check the defining property: after
a warm-up call, further calls make no device allocation.  The file is
collected after every other test.
"""

import ctypes

import numpy as np
import pytest

from alpacc_b200 import synth, tables

pytestmark = pytest.mark.gpu

MAX_BYTES = 128 << 20


def _bind(L):
    L.alp_lex_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                  ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int)]
    L.alp_ctx_info.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]


def _bufs(cap, device):
    import torch
    return (torch.empty(cap, dtype=torch.int32, device=device), torch.empty(cap, dtype=torch.int64, device=device),
            torch.empty(cap, dtype=torch.int64, device=device))


def _call(L, h, fn, d, bufs):
    term, start, end = bufs
    n, valid = ctypes.c_int64(0), ctypes.c_int(0)
    rc = fn(h, ctypes.c_void_p(d.data_ptr()), ctypes.c_int64(d.numel()), ctypes.c_void_p(term.data_ptr()),
            ctypes.c_void_p(start.data_ptr()), ctypes.c_void_p(end.data_ptr()), ctypes.c_int64(term.numel()),
            ctypes.byref(n), ctypes.byref(valid))
    assert rc == 0, L.alp_last_error(h)
    return valid.value, n.value


def _lex(L, h, fn, d, cap):
    bufs = _bufs(cap, d.device)
    v, k = _call(L, h, fn, d, bufs)
    return (v,) + tuple(b[:k].cpu().numpy() for b in bufs)


def _dev_allocs(L, h):
    info = (ctypes.c_int64 * 13)()
    assert L.alp_ctx_info(h, info, 13) == 0
    return int(info[12])


@pytest.mark.parametrize("grammar,make", [
    ("json", lambda size, seed: synth.json_doc(size, 8, seed)),
    ("sexp", lambda size, seed: synth.sexp_doc(size, 20, seed)),
])
def test_noalloc_matches_alp_lex_into_and_oracle(has_gpu, grammar, make):
    import torch
    import oracle
    from alpacc_b200.api import Grammar, native
    L = native()
    _bind(L)
    tb = tables.load(grammar, "lexer")
    g = Grammar(tb)
    o = oracle.Oracle(tb.blob())
    docs = [make(3_000_000, 0xA1FACC00 + 51), make(1_234_567, 0xA1FACC00 + 52)]
    for doc in docs:  # two calls in a row
        d = torch.from_numpy(doc).cuda()
        cap = doc.size + 1
        ref = _lex(L, g.h, L.alp_lex_into, d, cap)
        got = _lex(L, g.h, L.alp_lex_noalloc, d, cap)
        want = o.tokenize(doc.tobytes())
        assert want is not None
        assert got[0] == ref[0] == 1
        for a, b, w in zip(got[1:], ref[1:], want):
            np.testing.assert_array_equal(a, b)
            np.testing.assert_array_equal(a.astype(np.int64), w.astype(np.int64))


def test_noalloc_makes_no_device_allocation(has_gpu):
    import torch
    from alpacc_b200.api import Grammar, native
    L = native()
    _bind(L)
    g = Grammar(tables.load("json", "lexer"))
    docs = [torch.from_numpy(synth.json_doc(size, 8, 0xA1FACC00 + 53 + i)).cuda()
            for i, size in enumerate((5_000_000, 700_001))]
    bufs = _bufs(6_000_000, docs[0].device)
    assert _call(L, g.h, L.alp_lex_noalloc, docs[0], bufs)[0] == 1  # warm-up: kernels loaded on this device
    torch.cuda.synchronize()
    allocs = _dev_allocs(L, g.h)
    free0 = torch.cuda.mem_get_info()[0]
    counts = []
    for d in docs + docs:
        v, k = _call(L, g.h, L.alp_lex_noalloc, d, bufs)
        assert v == 1
        counts.append(k)
    torch.cuda.synchronize()
    assert _dev_allocs(L, g.h) == allocs, "alp_lex_noalloc grew the context's device buffers"
    assert torch.cuda.mem_get_info()[0] == free0, "device memory changed across alp_lex_noalloc calls"
    assert counts[:2] == counts[2:]


def test_noalloc_rejection_and_limit(has_gpu):
    import torch
    from alpacc_b200.api import Grammar, native
    L = native()
    _bind(L)
    g = Grammar(tables.load("json", "lexer"))
    # a rejected input reports valid = 0 like the allocating entry point
    bad = torch.from_numpy(np.frombuffer(b'{"a": 1, "b": "unterminated', dtype=np.uint8).copy()).cuda()
    assert _lex(L, g.h, L.alp_lex_noalloc, bad, 64)[0] == 0
    # inputs over the limit are refused before any device work
    n, valid = ctypes.c_int64(0), ctypes.c_int(0)
    small = torch.zeros(16, dtype=torch.uint8, device="cuda")
    rc = L.alp_lex_noalloc(g.h, ctypes.c_void_p(small.data_ptr()), ctypes.c_int64(MAX_BYTES + 1), None, None,
                           None, ctypes.c_int64(0), ctypes.byref(n), ctypes.byref(valid))
    assert rc == 1 and b"limit" in L.alp_last_error(g.h)
