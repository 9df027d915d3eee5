"""Python front end over the C ABI (``include/alpacc_b200.h``).

Mirrors the entry points alpacc's Futhark generator emits
(``src/Alpacc/Generator/Futhark/Generator.hs``): ``lex_int`` / ``lex`` return
the token triples (or ``None`` for ``#none``), ``parse_int`` / ``parse`` the
preorder tree, ``pre_productions_int`` the production sequence.  Every call
runs the CUDA kernels of ``_lib/libalpacc_b200.so``; there is no CPU path, and
constructing a :class:`Grammar` without a CUDA device raises.

Arrays come back as torch tensors on the context's device (``*_int``
variants) or as Python lists of names (named variants).
"""

from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple, Union

import numpy as np

from . import build as _build
from . import tables as _tables

ALP_OK, ALP_ERR_ARG, ALP_ERR_CUDA, ALP_ERR_TIMEOUT, ALP_ERR_TABLE, ALP_ERR_CAPACITY, ALP_ERR_MODE = range(7)


class AlpError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("alpacc_b200 error %d: %s" % (code, msg))
        self.code = code


_lib = None


def native() -> ctypes.CDLL:
    """Load (building first if the sources are newer) the CUDA library."""
    global _lib
    if _lib is None:
        path = _build.LIB
        if _build.needs_build():
            _build.build_cuda()
        if not os.path.exists(path):
            raise AlpError(ALP_ERR_CUDA, "native library missing: %s" % path)
        L = ctypes.CDLL(path)
        vp, i64, i32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int
        P = ctypes.POINTER
        L.alp_ctx_create.argtypes = [ctypes.c_char_p, ctypes.c_size_t, i32, P(vp)]
        L.alp_ctx_destroy.argtypes = [vp]
        L.alp_last_error.restype = ctypes.c_char_p
        L.alp_last_error.argtypes = [vp]
        L.alp_set_stream.argtypes = [vp, vp]
        L.alp_ctx_info.argtypes = [vp, P(i64), i32]
        L.alp_memcpy.argtypes = [vp, vp, vp, ctypes.c_size_t]
        L.alp_ctx_profile.argtypes = [vp, i32]
        L.alp_ctx_timings.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t]
        L.alp_lex.argtypes = [vp, vp, i64, P(vp), P(vp), P(vp), P(i64), P(i32)]
        L.alp_lex_into.argtypes = [vp, vp, i64, vp, vp, vp, i64, P(i64), P(i32)]
        L.alp_lex_host.argtypes = [vp, vp, i64, vp, vp, vp, i64, P(i64), P(i32)]
        for name in ("alp_parse",):
            getattr(L, name).argtypes = [vp, vp, i64, P(vp), P(vp), P(vp), P(vp), P(vp), P(i64), P(i32)]
        L.alp_parse_into.argtypes = [vp, vp, i64, vp, vp, vp, vp, vp, i64, P(i64), P(i32)]
        L.alp_parse_host.argtypes = [vp, vp, i64, vp, vp, vp, vp, vp, i64, P(i64), P(i32)]
        L.alp_parse_tokens.argtypes = [vp, vp, vp, vp, i64, P(vp), P(vp), P(vp), P(vp), P(vp), P(i64), P(i32)]
        L.alp_pre_productions.argtypes = [vp, vp, i64, P(vp), P(i64), P(i32)]
        L.alp_lex_batch.argtypes = [vp, vp, vp, i64, P(vp), P(vp), P(vp), P(vp), P(vp), P(i64)]
        L.alp_parse_batch.argtypes = [vp, vp, vp, i64, P(vp), P(vp), P(vp), P(vp), P(vp), P(vp), P(vp), P(i64)]
        L.alp_parse_batch_host.argtypes = [vp, vp, vp, i64, vp, vp, vp, vp, vp, vp, vp, i64, P(i64)]
        L.alp_lex_stream_begin.argtypes = [vp, vp, vp, vp, i64, P(vp)]
        L.alp_lex_stream_push.argtypes = [vp, vp, i64]
        L.alp_lex_stream_tokens.argtypes = [vp, P(i64)]
        L.alp_lex_stream_end.argtypes = [vp, P(i64), P(i32)]
        L.alp_lex_stream_window.argtypes = [vp, vp, vp, vp, i64, i64]
        L.alp_parse_graph_create.argtypes = [vp, vp, i64, vp, i64, i64, i64] + [vp] * 8 + [P(vp)]
        L.alp_parse_graph_launch.argtypes = [vp, vp]
        L.alp_parse_graph_result.argtypes = [vp, P(i64)]
        L.alp_parse_graph_error.argtypes = [vp]
        L.alp_parse_graph_error.restype = ctypes.c_char_p
        L.alp_parse_graph_destroy.argtypes = [vp]
        L.alp_parse_graph_destroy.restype = None
        L.alp_check_bounded_wait.argtypes = [vp]
        L.alp_tune_parse.argtypes = [vp, vp, i64, i32, ctypes.c_char_p, ctypes.c_size_t]
        L.alp_tune_get.argtypes = [vp, P(i32), i32]
        L.alp_tune_set.argtypes = [vp, P(i32), i32]
        L.alp_tune_shapes.argtypes = [P(i32), i32]
        L.alp_lex_stream_free.argtypes = [vp]
        L.alp_lex_stream_free.restype = None
        L.alp_lex_host_stream.argtypes = [vp, vp, i64, i64, vp, vp, vp, i64, P(i64), P(i32)]
        _lib = L
    return _lib


def _torch():
    import torch
    return torch


def _wrap(h, ptr: int, n: int, dtype, device) -> "torch.Tensor":
    """Copy n elements at a context-owned device pointer into a new tensor."""
    torch = _torch()
    out = torch.empty(n, dtype=dtype, device=device)
    if n:
        rc = native().alp_memcpy(h, ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(ptr),
                                 n * out.element_size())
        if rc != ALP_OK:
            raise AlpError(rc, native().alp_last_error(h).decode(errors="replace"))
    return out


@dataclass
class Tree:
    parent: "torch.Tensor"   # int64
    tag: "torch.Tensor"      # uint32 as int64 view-compatible (production or terminal id)
    kind: "torch.Tensor"     # uint8: 0 production, 1 terminal
    start: "torch.Tensor"    # int64
    end: "torch.Tensor"      # int64

    def __len__(self) -> int:
        return int(self.parent.numel())


class Grammar:
    """One grammar's tables loaded on one CUDA device (a Futhark context)."""

    def __init__(self, grammar: Union[str, _tables.Tables], mode: str = "both", device: int = 0):
        torch = _torch()
        if not torch.cuda.is_available():
            raise AlpError(ALP_ERR_CUDA, "no CUDA device: alpacc_b200 runs on the GPU only")
        self.tables = grammar if isinstance(grammar, _tables.Tables) else _tables.load(grammar, mode)
        self.device = torch.device("cuda", device)
        torch.cuda.init()
        with torch.cuda.device(self.device):
            torch.empty(1, device=self.device)  # make the primary context current
        blob = self.tables.blob()
        self._blob = blob
        h = ctypes.c_void_p()
        L = native()
        rc = L.alp_ctx_create(blob, len(blob), device, ctypes.byref(h))
        if rc != ALP_OK:
            raise AlpError(rc, "alp_ctx_create failed")
        self.h = h
        info = (ctypes.c_int64 * 8)()
        L.alp_ctx_info(self.h, info, 8)
        self.info = list(info)

    def close(self):
        if getattr(self, "h", None):
            native().alp_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------- profiling
    def profile(self, on: bool = True) -> None:
        native().alp_ctx_profile(self.h, 1 if on else 0)

    def timings(self) -> List[Tuple[str, float]]:
        buf = ctypes.create_string_buffer(1 << 16)
        native().alp_ctx_timings(self.h, buf, len(buf))
        out = []
        for line in buf.value.decode().splitlines():
            name, ms = line.rsplit(" ", 1)
            out.append((name, float(ms)))
        return out

    # ------------------------------------------------------------------ utils
    def _err(self, rc: int):
        msg = native().alp_last_error(self.h).decode(errors="replace")
        raise AlpError(rc, msg)

    def _stream(self):
        torch = _torch()
        s = torch.cuda.current_stream(self.device).cuda_stream
        native().alp_set_stream(self.h, ctypes.c_void_p(s))

    def _as_device_bytes(self, data) -> "torch.Tensor":
        torch = _torch()
        if isinstance(data, torch.Tensor):
            t = data
            if t.dtype != torch.uint8:
                raise TypeError("input must be uint8")
            return t.to(self.device).contiguous()
        if isinstance(data, (bytes, bytearray, memoryview)):
            arr = np.frombuffer(bytes(data), dtype=np.uint8)
        else:
            arr = np.ascontiguousarray(data, dtype=np.uint8)
        return torch.from_numpy(arr.copy()).to(self.device)

    # ------------------------------------------------------------------ lexer
    def lex_int(self, data) -> Optional[Tuple["torch.Tensor", "torch.Tensor", "torch.Tensor"]]:
        """Tokens as (terminal uint32->int64 tensor, start int64, end int64),
        or None when the input is rejected."""
        torch = _torch()
        x = self._as_device_bytes(data)
        self._stream()
        pt, ps, pe = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        n, valid = ctypes.c_int64(0), ctypes.c_int(0)
        rc = native().alp_lex(self.h, ctypes.c_void_p(x.data_ptr()), x.numel(), ctypes.byref(pt), ctypes.byref(ps),
                              ctypes.byref(pe), ctypes.byref(n), ctypes.byref(valid))
        if rc != ALP_OK:
            self._err(rc)
        if not valid.value:
            return None
        k = n.value
        term = _wrap(self.h, pt.value or 0, k, torch.int32, self.device)
        start = _wrap(self.h, ps.value or 0, k, torch.int64, self.device)
        end = _wrap(self.h, pe.value or 0, k, torch.int64, self.device)
        return term, start, end

    def lex(self, data) -> Optional[List[Tuple[str, Tuple[int, int]]]]:
        r = self.lex_int(data)
        if r is None:
            return None
        names = self.tables.terminal_names
        t, s, e = (x.cpu().numpy() for x in r)
        return [(names[int(a)], (int(b), int(c))) for a, b, c in zip(t, s, e)]

    def lex_host(self, data: np.ndarray):
        """Host buffers in and out (copies inside the call)."""
        arr = np.ascontiguousarray(data, dtype=np.uint8)
        cap = len(arr) + 1
        term = np.empty(cap, np.uint32)
        start = np.empty(cap, np.int64)
        end = np.empty(cap, np.int64)
        n, valid = ctypes.c_int64(0), ctypes.c_int(0)
        self._stream()
        rc = native().alp_lex_host(self.h, arr.ctypes.data_as(ctypes.c_void_p), len(arr),
                                   term.ctypes.data_as(ctypes.c_void_p), start.ctypes.data_as(ctypes.c_void_p),
                                   end.ctypes.data_as(ctypes.c_void_p), cap, ctypes.byref(n), ctypes.byref(valid))
        if rc != ALP_OK:
            self._err(rc)
        if not valid.value:
            return None
        k = n.value
        return term[:k], start[:k], end[:k]

    def lex_stream(self, cap: int) -> "TokenStream":
        """A token stream over input pushed in pieces (alp_lex_stream_*),
        writing up to `cap` tokens into device tensors it owns."""
        return TokenStream(self, cap)

    def lex_host_stream(self, data: np.ndarray, piece: int = 0, out=None):
        """alp_lex_host through alp_lex_host_stream: the input in pieces with
        the copies in and out overlapped with the lexing.  `out`: optional
        (term uint32, start int64, end int64) host arrays (pinned for overlap)."""
        arr = np.ascontiguousarray(data, dtype=np.uint8)
        if out is None:
            cap = len(arr) + 1
            out = (np.empty(cap, np.uint32), np.empty(cap, np.int64), np.empty(cap, np.int64))
        term, start, end = out
        cap = min(len(term), len(start), len(end))
        n, valid = ctypes.c_int64(0), ctypes.c_int(0)
        self._stream()
        ptr = lambda a: ctypes.c_void_p(a.ctypes.data if isinstance(a, np.ndarray) else a.data_ptr())
        rc = native().alp_lex_host_stream(self.h, ptr(arr), len(arr), piece, ptr(term), ptr(start), ptr(end), cap,
                                          ctypes.byref(n), ctypes.byref(valid))
        if rc != ALP_OK:
            self._err(rc)
        if not valid.value:
            return None
        k = n.value
        return term[:k], start[:k], end[:k]

    # ----------------------------------------------------------------- parser
    def _tree(self, pp, pt, pk, ps, pe, n) -> Tree:
        torch = _torch()
        return Tree(_wrap(self.h, pp.value or 0, n, torch.int64, self.device),
                    _wrap(self.h, pt.value or 0, n, torch.int32, self.device),
                    _wrap(self.h, pk.value or 0, n, torch.uint8, self.device),
                    _wrap(self.h, ps.value or 0, n, torch.int64, self.device),
                    _wrap(self.h, pe.value or 0, n, torch.int64, self.device))

    def parse_int(self, data) -> Optional[Tree]:
        """Bytes -> preorder tree (parent, tag, kind, start, end), or None."""
        x = self._as_device_bytes(data)
        self._stream()
        ptrs = [ctypes.c_void_p() for _ in range(5)]
        n, valid = ctypes.c_int64(0), ctypes.c_int(0)
        rc = native().alp_parse(self.h, ctypes.c_void_p(x.data_ptr()), x.numel(), *[ctypes.byref(p) for p in ptrs],
                                ctypes.byref(n), ctypes.byref(valid))
        if rc != ALP_OK:
            self._err(rc)
        if not valid.value:
            return None
        return self._tree(*ptrs, n.value)

    def parse(self, data):
        """Named tree: a list of (parent, ('terminal', name, (start, end)) |
        ('production', name)), or None."""
        t = self.parse_int(data)
        if t is None:
            return None
        tn, pn = self.tables.terminal_names, self.tables.production_names
        par, tag, kind, s, e = (x.cpu().numpy() for x in (t.parent, t.tag, t.kind, t.start, t.end))
        out = []
        for i in range(len(par)):
            if kind[i]:
                out.append((int(par[i]), ("terminal", tn[int(tag[i])], (int(s[i]), int(e[i])))))
            else:
                out.append((int(par[i]), ("production", pn[int(tag[i])])))
        return out

    def parse_tokens_int(self, term, start, end) -> Optional[Tree]:
        """Parser-only ``parse_int``: token arrays (device or host) -> tree."""
        torch = _torch()
        term = torch.as_tensor(term).to(self.device, torch.int32).contiguous()
        start = torch.as_tensor(start).to(self.device, torch.int64).contiguous()
        end = torch.as_tensor(end).to(self.device, torch.int64).contiguous()
        self._stream()
        ptrs = [ctypes.c_void_p() for _ in range(5)]
        n, valid = ctypes.c_int64(0), ctypes.c_int(0)
        rc = native().alp_parse_tokens(self.h, ctypes.c_void_p(term.data_ptr()), ctypes.c_void_p(start.data_ptr()),
                                       ctypes.c_void_p(end.data_ptr()), term.numel(),
                                       *[ctypes.byref(p) for p in ptrs], ctypes.byref(n), ctypes.byref(valid))
        if rc != ALP_OK:
            self._err(rc)
        if not valid.value:
            return None
        return self._tree(*ptrs, n.value)

    def pre_productions_int(self, term) -> Optional["torch.Tensor"]:
        torch = _torch()
        term = torch.as_tensor(term).to(self.device, torch.int32).contiguous()
        self._stream()
        pp = ctypes.c_void_p()
        n, valid = ctypes.c_int64(0), ctypes.c_int(0)
        rc = native().alp_pre_productions(self.h, ctypes.c_void_p(term.data_ptr()), term.numel(), ctypes.byref(pp),
                                          ctypes.byref(n), ctypes.byref(valid))
        if rc != ALP_OK:
            self._err(rc)
        if not valid.value:
            return None
        return _wrap(self.h, pp.value or 0, n.value, torch.int32, self.device)

    def parse_host(self, data: np.ndarray):
        """Host buffers in and out: (parent, tag, kind, start, end) numpy arrays or None."""
        arr = np.ascontiguousarray(data, dtype=np.uint8)
        cap = (len(arr) + 2) * max(1, self.info[6])
        par = np.empty(cap, np.int64)
        tag = np.empty(cap, np.uint32)
        kind = np.empty(cap, np.uint8)
        st = np.empty(cap, np.int64)
        en = np.empty(cap, np.int64)
        n, valid = ctypes.c_int64(0), ctypes.c_int(0)
        self._stream()
        vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        rc = native().alp_parse_host(self.h, vp(arr), len(arr), vp(par), vp(tag), vp(kind), vp(st), vp(en), cap,
                                     ctypes.byref(n), ctypes.byref(valid))
        if rc != ALP_OK:
            self._err(rc)
        if not valid.value:
            return None
        k = n.value
        return par[:k], tag[:k], kind[:k], st[:k], en[:k]

    # ---------------------------------------------------------------- batches
    def _batch_inputs(self, data, offsets):
        torch = _torch()
        x = self._as_device_bytes(data)
        if isinstance(offsets, torch.Tensor):
            off = offsets.to(device=self.device, dtype=torch.int64).contiguous()
        else:
            off = torch.as_tensor(np.ascontiguousarray(offsets, dtype=np.int64)).to(self.device)
        if off.numel() < 2 or int(off[-1]) != x.numel():
            raise ValueError("offsets must run from 0 to len(data)")
        return x, off

    def lex_batch_int(self, data, offsets):
        """Documents back to back (offsets[0..n]) -> (term, start, end,
        tok_off[n+1], valid[n]); spans are relative to each document and a
        document's tokens are meaningful only when valid[d] is 1."""
        torch = _torch()
        x, off = self._batch_inputs(data, offsets)
        nd = off.numel() - 1
        self._stream()
        ptrs = [ctypes.c_void_p() for _ in range(5)]
        total = ctypes.c_int64(0)
        rc = native().alp_lex_batch(self.h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(off.data_ptr()), nd,
                                    *[ctypes.byref(p) for p in ptrs], ctypes.byref(total))
        if rc != ALP_OK:
            self._err(rc)
        k = total.value
        return (_wrap(self.h, ptrs[0].value or 0, k, torch.int32, self.device),
                _wrap(self.h, ptrs[1].value or 0, k, torch.int64, self.device),
                _wrap(self.h, ptrs[2].value or 0, k, torch.int64, self.device),
                _wrap(self.h, ptrs[3].value or 0, nd + 1, torch.int64, self.device),
                _wrap(self.h, ptrs[4].value or 0, nd, torch.uint8, self.device))

    # ---------------------------------------------------------------- tuning
    @staticmethod
    def tile_shapes() -> List[Tuple[int, int]]:
        """(threads, elements per thread) of each previous-smaller-or-equal tile shape."""
        L = native()
        k = L.alp_tune_shapes(None, 0)
        out = (ctypes.c_int32 * (2 * k))()
        L.alp_tune_shapes(out, 2 * k)
        return [(out[2 * i], out[2 * i + 1]) for i in range(k)]

    def get_tuning(self) -> List[int]:
        """[tile shape, pair CTAs per SM, expand CTAs per SM, MLP kernel (0 tcgen05, 1 mma.sync),
        lexer token pass (0 fused, 1 count pass + tile scan + token pass),
        parser position pass (0 fused, 1 pair pass + tile-sum scan + expansion),
        lexer state-scan chunks per lane (8, 16 or 32)]."""
        cfg = (ctypes.c_int32 * 7)()
        native().alp_tune_get(self.h, cfg, 7)
        return list(cfg)

    def set_tuning(self, cfg: Sequence[int]) -> None:
        """Three values (launch shapes), four (and the MLP inference kernel),
        five (and the lexer's token pass), six (and the parser's position
        pass) or seven (and the lexer state scan's chunks per lane)."""
        if len(cfg) not in (3, 4, 5, 6, 7):
            raise ValueError("tuning takes 3 to 7 values")
        c = (ctypes.c_int32 * len(cfg))(*cfg)
        rc = native().alp_tune_set(self.h, c, len(cfg))
        if rc != ALP_OK:
            self._err(rc)

    def tune(self, sample, reps: int = 3) -> dict:
        """alp_tune_parse on `sample` (bytes, numpy or a uint8 tensor): the
        context keeps the fastest launch shapes; returns them with the timings."""
        x = self._as_device_bytes(sample)
        self._stream()
        buf = ctypes.create_string_buffer(1 << 14)
        rc = native().alp_tune_parse(self.h, ctypes.c_void_p(x.data_ptr()), x.numel(), reps, buf, len(buf))
        if rc != ALP_OK:
            self._err(rc)
        rows = []
        for ln in buf.value.decode().splitlines():
            k, v, ms = ln.split()
            rows.append((k, int(v), float(ms)))
        cfg = self.get_tuning()
        return {"config": cfg, "tile_shape": self.tile_shapes()[cfg[0]], "timings": rows}

    def parse_batch_graph(self, data, offsets, cap_nodes: Optional[int] = None, cap_brackets: Optional[int] = None,
                          slack: float = 0.25) -> "ParseGraph":
        """alp_parse_graph_*: the batched parse of these documents' shape as a
        CUDA graph.  Without capacities, one alp_parse_batch call measures the
        batch and the capacities are its node and bracket counts plus `slack`."""
        if cap_nodes is None or cap_brackets is None:
            tree, _, _ = self.parse_batch_int(data, offsets)
            info = (ctypes.c_int64 * 11)()
            native().alp_ctx_info(self.h, info, 11)
            if cap_nodes is None:
                cap_nodes = int(len(tree) * (1 + slack)) + 64
            if cap_brackets is None:
                cap_brackets = int(info[10] * (1 + slack)) + 64
        return ParseGraph(self, data, offsets, cap_nodes, cap_brackets)

    def parse_batch_int(self, data, offsets):
        """Documents back to back -> (Tree, node_off[n+1], valid[n]); parents
        and spans are relative to each document."""
        torch = _torch()
        x, off = self._batch_inputs(data, offsets)
        nd = off.numel() - 1
        self._stream()
        ptrs = [ctypes.c_void_p() for _ in range(7)]
        total = ctypes.c_int64(0)
        rc = native().alp_parse_batch(self.h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(off.data_ptr()), nd,
                                      *[ctypes.byref(p) for p in ptrs], ctypes.byref(total))
        if rc != ALP_OK:
            self._err(rc)
        k = total.value
        tree = self._tree(*ptrs[:5], k)
        return (tree, _wrap(self.h, ptrs[5].value or 0, nd + 1, torch.int64, self.device),
                _wrap(self.h, ptrs[6].value or 0, nd, torch.uint8, self.device))


    def parse_batch_host(self, data, offsets, cap: Optional[int] = None):
        """alp_parse_batch_host: documents back to back in host memory ->
        (parent, tag, kind, start, end, node_off, valid) numpy arrays; parents and
        spans are relative to each document."""
        arr = np.ascontiguousarray(data, dtype=np.uint8)
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        nd = len(off) - 1
        # without a capacity: a guess of one node per byte, and the exact count on a retry
        caps = [cap] if cap is not None else [len(arr) + 2 * nd + 1024, None]
        node_off = np.empty(nd + 1, np.int64)
        valid = np.empty(nd, np.uint8)
        total = ctypes.c_int64(0)
        self._stream()
        vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        for c in caps:
            c = total.value if c is None else c
            outs = [np.empty(max(c, 1), dt) for dt in (np.int64, np.uint32, np.uint8, np.int64, np.int64)]
            rc = native().alp_parse_batch_host(self.h, vp(arr), vp(off), nd, *[vp(o) for o in outs], vp(node_off),
                                               vp(valid), c, ctypes.byref(total))
            if rc != ALP_ERR_CAPACITY:
                break
        if rc != ALP_OK:
            self._err(rc)
        k = total.value
        return tuple(o[:k] for o in outs) + (node_off, valid)


class TokenStream:
    """Input lexed as it arrives: ``push`` pieces (bytes, numpy or uint8
    tensors), then ``end`` for the tokens of the whole stream, equal to
    ``Grammar.lex_int`` of the concatenation (None when rejected).  ``tokens``
    waits for the pushed pieces and gives the count of tokens final so far."""

    def __init__(self, grammar: Grammar, cap: int):
        torch = _torch()
        self.g = grammar
        self.term = torch.empty(max(cap, 1), dtype=torch.int32, device=grammar.device)
        self.start = torch.empty(max(cap, 1), dtype=torch.int64, device=grammar.device)
        self.end_ = torch.empty(max(cap, 1), dtype=torch.int64, device=grammar.device)
        self._pending = []  # pieces the GPU may still read
        self.first = 0
        grammar._stream()
        h = ctypes.c_void_p()
        rc = native().alp_lex_stream_begin(grammar.h, ctypes.c_void_p(self.term.data_ptr()),
                                           ctypes.c_void_p(self.start.data_ptr()),
                                           ctypes.c_void_p(self.end_.data_ptr()), cap, ctypes.byref(h))
        if rc != ALP_OK:
            grammar._err(rc)
        self.h = h

    def push(self, data) -> None:
        x = self.g._as_device_bytes(data)
        self.g._stream()
        rc = native().alp_lex_stream_push(self.h, ctypes.c_void_p(x.data_ptr()), x.numel())
        if rc != ALP_OK:
            self.g._err(rc)
        self._pending.append(x)

    def tokens(self) -> int:
        n = ctypes.c_int64(0)
        rc = native().alp_lex_stream_tokens(self.h, ctypes.byref(n))
        if rc != ALP_OK:
            self.g._err(rc)
        self._pending.clear()
        return n.value

    def window(self, first: int) -> None:
        """Later tokens go to element ``token index - first`` of this stream's
        buffers; tokens before ``first`` are not stored."""
        rc = native().alp_lex_stream_window(self.h, ctypes.c_void_p(self.term.data_ptr()),
                                            ctypes.c_void_p(self.start.data_ptr()),
                                            ctypes.c_void_p(self.end_.data_ptr()), self.term.numel(), first)
        if rc != ALP_OK:
            self.g._err(rc)
        self.first = first

    def finish(self) -> Tuple[int, bool]:
        """Ends the stream: (tokens written in all, accepted)."""
        n, valid = ctypes.c_int64(0), ctypes.c_int(0)
        rc = native().alp_lex_stream_end(self.h, ctypes.byref(n), ctypes.byref(valid))
        self._pending.clear()
        if rc != ALP_OK:
            self.g._err(rc)
        return n.value, bool(valid.value)

    def end(self):
        k, ok = self.finish()
        if not ok:
            return None
        k -= self.first
        return self.term[:k], self.start[:k], self.end_[:k]

    def close(self) -> None:
        if self.h:
            native().alp_lex_stream_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ParseGraph:
    """A batched parse captured once as a CUDA graph: ``load`` new documents of
    the same total size and count, ``launch`` (no wait), then ``result`` for
    (Tree, node_off, valid) as ``Grammar.parse_batch_int`` gives them."""

    def __init__(self, grammar: Grammar, data, offsets, cap_nodes: int, cap_brackets: int):
        torch = _torch()
        self.g = grammar
        x, off = grammar._batch_inputs(data, offsets)
        self.x, self.off = x.clone(), off.clone()
        nd = self.off.numel() - 1
        dev = grammar.device
        self.parent = torch.empty(max(cap_nodes, 1), dtype=torch.int64, device=dev)
        self.tag = torch.empty(max(cap_nodes, 1), dtype=torch.int32, device=dev)
        self.kind = torch.empty(max(cap_nodes, 1), dtype=torch.uint8, device=dev)
        self.start = torch.empty(max(cap_nodes, 1), dtype=torch.int64, device=dev)
        self.end = torch.empty(max(cap_nodes, 1), dtype=torch.int64, device=dev)
        self.node_off = torch.empty(nd + 1, dtype=torch.int64, device=dev)
        self.valid = torch.empty(nd, dtype=torch.uint8, device=dev)
        self.counts = torch.zeros(4, dtype=torch.int64, device=dev)
        torch.cuda.synchronize(dev)
        vp = lambda t: ctypes.c_void_p(t.data_ptr())
        h = ctypes.c_void_p()
        rc = native().alp_parse_graph_create(grammar.h, vp(self.x), self.x.numel(), vp(self.off), nd, cap_nodes,
                                             cap_brackets, vp(self.parent), vp(self.tag), vp(self.kind),
                                             vp(self.start), vp(self.end), vp(self.node_off), vp(self.valid),
                                             vp(self.counts), ctypes.byref(h))
        if rc != ALP_OK:
            grammar._err(rc)
        self.h = h

    def load(self, data, offsets) -> None:
        """New documents with the same byte total and document count."""
        x, off = self.g._batch_inputs(data, offsets)
        if x.numel() != self.x.numel() or off.numel() != self.off.numel():
            raise ValueError("a graph replays one batch shape: same bytes and documents")
        self.x.copy_(x)
        self.off.copy_(off)

    def launch(self) -> None:
        torch = _torch()
        s = torch.cuda.current_stream(self.g.device).cuda_stream
        rc = native().alp_parse_graph_launch(self.h, ctypes.c_void_p(s))
        if rc != ALP_OK:
            raise AlpError(rc, native().alp_parse_graph_error(self.h).decode(errors="replace"))

    def result(self):
        n = ctypes.c_int64(0)
        rc = native().alp_parse_graph_result(self.h, ctypes.byref(n))
        if rc != ALP_OK:
            raise AlpError(rc, native().alp_parse_graph_error(self.h).decode(errors="replace"))
        k = n.value
        tree = Tree(self.parent[:k], self.tag[:k], self.kind[:k], self.start[:k], self.end[:k])
        return tree, self.node_off, self.valid

    def close(self) -> None:
        if self.h:
            native().alp_parse_graph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
