"""Failure detection without a GPU fault.

* Bounded waits: ``alp_check_bounded_wait`` runs a wait on a status word that
  nothing sets; the wait must give up by itself, the call must report
  ALP_ERR_TIMEOUT, and the same context must lex correctly afterwards.
* Malformed tables: every truncation of a table blob, and every table entry
  that a kernel would use as an index set out of range, must be refused at
  context creation with ALP_ERR_TABLE, before any kernel sees it.
"""

import ctypes
import struct
import time

import numpy as np
import pytest

import oracle
from alpacc_b200 import synth, tables

pytestmark = pytest.mark.gpu

ALP_ERR_TIMEOUT = 3
ALP_ERR_TABLE = 4


def _lib():
    from alpacc_b200.api import native
    L = native()
    L.alp_check_bounded_wait.argtypes = [ctypes.c_void_p]
    return L


def _create(blob: bytes):
    L = _lib()
    h = ctypes.c_void_p()
    rc = L.alp_ctx_create(blob, len(blob), 0, ctypes.byref(h))
    if rc == 0:
        L.alp_ctx_destroy(h)
    else:
        assert not h.value
    return rc


def test_bounded_wait_gives_up_and_context_survives(has_gpu):
    from alpacc_b200.api import Grammar
    tb = tables.load("json", "both")
    g = Grammar(tb)
    o = oracle.Oracle(tb.blob())
    L = _lib()
    doc = synth.json_doc(200000, 8, 17).tobytes()
    want = o.lex_futhark(doc)
    for _ in range(2):
        t0 = time.time()
        rc = L.alp_check_bounded_wait(g.h)
        took = time.time() - t0
        assert rc == ALP_ERR_TIMEOUT, L.alp_last_error(g.h)
        assert took < 60
        got = g.lex_int(doc)
        assert got is not None
        np.testing.assert_array_equal(got[0].cpu().numpy().astype(np.uint32), want[0])
        np.testing.assert_array_equal(got[1].cpu().numpy(), want[1])
        np.testing.assert_array_equal(got[2].cpu().numpy(), want[2])


def test_truncated_blobs_refused(has_gpu):
    rng = np.random.default_rng(5)
    for name in ("json", "sexp"):
        for mode in ("lexer", "both"):
            blob = tables.load(name, mode).blob()
            assert _create(blob) == 0
            cuts = set(rng.integers(0, len(blob), 60).tolist()) | {0, 3, 4, 15, 16, 17, len(blob) - 1}
            for c in sorted(cuts):
                assert _create(blob[:c]) == ALP_ERR_TABLE, (name, mode, c)


def _pad4(n):
    return (n + 3) & ~3


def _sections(blob: bytes):
    """Byte offsets of the blob's sections (layout of alpacc_b200/tables.py)."""
    u32 = lambda o: struct.unpack_from("<I", blob, o)[0]
    off = {}
    hl, hp = u32(8), u32(12)
    o = 16
    if hl:
        S, C, E = u32(o), u32(o + 4), u32(o + 8)
        off["S"], off["C"], off["E"] = S, C, E
        o += 24
        off["cls"] = o; o += 256
        o += _pad4(S * 256 * 2)
        off["cdelta"] = o; o += _pad4(S * (C + 1) * 2)
        off["token"] = o; o += S * 4
        o += _pad4(S)
        off["step"] = o; o += _pad4(E * (C + 1) * 2)
        off["comp"] = o; o += _pad4(E * E * 2)
        off["apply"] = o; o += _pad4(E * S * 2)
    if hp:
        off["parser"] = o
        q, k = u32(o), u32(o + 4)
        n_prods = u32(o + 24)
        o += 32 + 8 * n_prods
        n_pairs = u32(o); off["n_pairs"] = n_pairs; o += 4 + 16 * n_pairs
        n_stack = u32(o); o += 4 + 4 * n_stack
        n_pseq = u32(o); o += 4 + 4 * n_pseq
        n_keys = u32(o); o += 4 + 4 * n_keys * (q + k)
        off["key_pair"] = o
        assert o + 4 * n_keys == len(blob)
    return off


def _set16(blob, o, v):
    b = bytearray(blob)
    struct.pack_into("<H", b, o, v)
    return bytes(b)


def _set32(blob, o, v):
    b = bytearray(blob)
    struct.pack_into("<I", b, o, v)
    return bytes(b)


@pytest.mark.parametrize("name", ["json", "sexp", "arithmetic"])
def test_out_of_range_entries_refused(has_gpu, name):
    blob = tables.load(name, "both").blob()
    off = _sections(blob)
    S, C, E = off["S"], off["C"], off["E"]
    rng = np.random.default_rng(9)
    bad = []
    for _ in range(4):
        bad.append(_set16(blob, off["cdelta"] + 2 * int(rng.integers(0, S * (C + 1))), S))
        bad.append(_set16(blob, off["step"] + 2 * int(rng.integers(0, E * (C + 1))), E))
        bad.append(_set16(blob, off["comp"] + 2 * int(rng.integers(0, E * E)), E))
        bad.append(_set16(blob, off["apply"] + 2 * int(rng.integers(0, E * S)), S))
        b = bytearray(blob)
        b[off["cls"] + int(rng.integers(0, 256))] = 255
        bad.append(bytes(b))
        bad.append(_set32(blob, off["token"] + 4 * int(rng.integers(0, S)), 0x7fff0000))
        bad.append(_set32(blob, off["key_pair"], off["n_pairs"]))
    for b in bad:
        assert _create(b) == ALP_ERR_TABLE
    # a terminal id inside the lexer's range but outside the parser's
    T = struct.unpack_from("<I", blob, off["parser"] + 8)[0]
    assert _create(_set32(blob, off["token"], T)) == ALP_ERR_TABLE
    assert _create(blob) == 0
