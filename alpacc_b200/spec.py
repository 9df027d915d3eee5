"""Learned boundary-state speculation (host side).

A small MLP reads the 64 bytes before a chunk boundary and predicts the DFA
state there.  Labels come from the exact lexer (``alp_lex_states``: the
composition scan's own state at every 16-byte boundary), training runs the
project's BF16 tensor-core kernels (``alp_mlp_train_step``: forward, backward,
AdamW), and ``alp_lex_speculative`` uses the predictions as chunk start
states, re-running mispredicted chunks until every start is exact.  The
prediction only changes how much work is redone, never the tokens.

There is no counterpart in the reference; its lexer is the plain composition
scan, which this module's results are always checked against.
"""

from __future__ import annotations

import ctypes
import math
from typing import Dict, Optional, Tuple

import numpy as np

from . import api

WIN = 64
EMB, IN, H, OUT = 16, 1024, 128, 32
P_EMB = 0
P_W1 = P_EMB + 256 * EMB
P_B1 = P_W1 + IN * H
P_W2 = P_B1 + H
P_B2 = P_W2 + H * H
P_W3 = P_B2 + H
P_B3 = P_W3 + H * OUT
P_TOTAL = P_B3 + OUT
BF_TOTAL = 256 * EMB + IN * H + H * H + H * OUT


def _L():
    L = api.native()
    if not getattr(L, "_spec_ready", False):
        vp, i64, i32, f32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_float
        P = ctypes.POINTER
        L.alp_lex_states.argtypes = [vp, vp, i64, vp]
        L.alp_mlp_train_step.argtypes = [vp, vp, vp, vp, vp, vp, i32, vp, vp, i32, f32, f32, i32, i32, P(f32), P(f32)]
        L.alp_mlp_predict.argtypes = [vp, vp, vp, i32, vp, i64, vp, i64, vp]
        L.alp_lex_speculative.argtypes = [vp, vp, vp, i32, vp, i64, i64, P(vp), P(vp), P(vp), P(i64), P(i32), P(i64)]
        L._spec_ready = True
    return L


def exact_states(g: "api.Grammar", data) -> "torch.Tensor":
    """State entering byte 16*i for every 16*i < n (uint8 tensor)."""
    import torch
    x = g._as_device_bytes(data)
    out = torch.zeros((x.numel() + 15) // 16 + 1, dtype=torch.uint8, device=g.device)
    g._stream()
    rc = _L().alp_lex_states(g.h, ctypes.c_void_p(x.data_ptr()), x.numel(), ctypes.c_void_p(out.data_ptr()))
    if rc != 0:
        g._err(rc)
    return out[: (x.numel() + 15) // 16]


def windows_at(x: "torch.Tensor", pos: "torch.Tensor") -> "torch.Tensor":
    """[len(pos), 64] bytes before each position (spaces before the start)."""
    import torch
    idx = pos.view(-1, 1) - WIN + torch.arange(WIN, device=x.device).view(1, -1)
    w = torch.full(idx.shape, 0x20, dtype=torch.uint8, device=x.device)
    ok = idx >= 0
    w[ok] = x[idx[ok]]
    return w


def dataset(g: "api.Grammar", docs, per_doc: int, seed: int) -> Tuple["torch.Tensor", "torch.Tensor"]:
    """(windows [N, 64], labels [N]) from 16-byte boundaries of each document,
    labelled by the exact lexer."""
    import torch
    gen = torch.Generator(device="cpu").manual_seed(seed)
    ws, ys = [], []
    for d in docs:
        x = g._as_device_bytes(d)
        st = exact_states(g, x)
        nb = st.numel()
        if nb < 2:
            continue
        k = min(per_doc, nb - 1)
        b = torch.randint(1, nb, (k,), generator=gen).to(g.device)
        ws.append(windows_at(x, b * 16))
        ys.append(st[b])
    return torch.cat(ws), torch.cat(ys)


class BoundaryModel:
    """The MLP's parameters (FP32 masters, BF16 copies, Adam moments) on the
    grammar's device."""

    def __init__(self, g: "api.Grammar", seed: int = 0):
        import torch
        self.g = g
        self.n_states = g.tables.lexer.dfa.n_states
        if self.n_states > OUT:
            raise ValueError("the MLP predicts at most %d states" % OUT)
        dev = g.device
        rng = np.random.default_rng(seed)
        p = np.zeros(P_TOTAL, np.float32)
        p[P_EMB:P_W1] = rng.standard_normal(256 * EMB) * 0.5
        p[P_W1:P_B1] = rng.standard_normal(IN * H) * math.sqrt(2.0 / IN)
        p[P_W2:P_B2] = rng.standard_normal(H * H) * math.sqrt(2.0 / H)
        p[P_W3:P_B3] = rng.standard_normal(H * OUT) * math.sqrt(1.0 / H)
        self.params = torch.from_numpy(p).to(dev)
        self.grads = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.wbf = torch.zeros(BF_TOTAL, dtype=torch.bfloat16, device=dev)
        self.sync_bf16()
        self.step = 0

    def sync_bf16(self):
        p = self.params
        self.wbf[: 256 * EMB] = p[P_EMB:P_W1].to(self.wbf.dtype)
        o = 256 * EMB
        self.wbf[o:o + IN * H] = p[P_W1:P_B1].to(self.wbf.dtype)
        o += IN * H
        self.wbf[o:o + H * H] = p[P_W2:P_B2].to(self.wbf.dtype)
        o += H * H
        self.wbf[o:o + H * OUT] = p[P_W3:P_B3].to(self.wbf.dtype)

    def _ptr(self, t):
        return ctypes.c_void_p(t.data_ptr())

    def train_step(self, win, lab, lr: float = 2e-3, wd: float = 1e-4, update: bool = True):
        loss, acc = ctypes.c_float(0.0), ctypes.c_float(0.0)
        if update:
            self.step += 1
        self.g._stream()
        rc = _L().alp_mlp_train_step(self.g.h, self._ptr(self.params), self._ptr(self.wbf), self._ptr(self.grads),
                                     self._ptr(self.m), self._ptr(self.v), self.n_states, self._ptr(win),
                                     self._ptr(lab), win.shape[0], lr, wd, max(self.step, 1), 1 if update else 0,
                                     ctypes.byref(loss), ctypes.byref(acc))
        if rc != 0:
            self.g._err(rc)
        return loss.value, acc.value

    def train(self, win, lab, epochs: int = 2, batch: int = 4096, lr: float = 2e-3, seed: int = 0) -> Dict:
        import torch
        n = (win.shape[0] // batch) * batch
        gen = torch.Generator(device="cpu").manual_seed(seed)
        hist = []
        total = epochs * (n // batch)
        k = 0
        for _ in range(epochs):
            perm = torch.randperm(win.shape[0], generator=gen)[:n].to(win.device)
            for b in range(0, n, batch):
                idx = perm[b:b + batch]
                # cosine learning-rate decay
                lr_k = lr * 0.5 * (1 + math.cos(math.pi * k / max(1, total)))
                hist.append(self.train_step(win[idx].contiguous(), lab[idx].contiguous(), lr_k))
                k += 1
        return {"steps": k, "last_loss": hist[-1][0] if hist else None, "last_acc": hist[-1][1] if hist else None}

    def predict(self, data, positions) -> "torch.Tensor":
        import torch
        x = self.g._as_device_bytes(data)
        pos = torch.as_tensor(positions, dtype=torch.int64).to(self.g.device).contiguous()
        out = torch.zeros(pos.numel(), dtype=torch.uint8, device=self.g.device)
        self.g._stream()
        rc = _L().alp_mlp_predict(self.g.h, self._ptr(self.wbf), self._ptr(self.params), self.n_states,
                                  self._ptr(x), x.numel(), self._ptr(pos), pos.numel(), self._ptr(out))
        if rc != 0:
            self.g._err(rc)
        return out

    def lex(self, data, chunk: int):
        """Speculative lex_int: (term, start, end) or None, and the stats
        (chunks, first-round mismatches, chunks re-run, rounds)."""
        import torch
        x = self.g._as_device_bytes(data)
        self.g._stream()
        pt, ps, pe = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        n, valid = ctypes.c_int64(0), ctypes.c_int(0)
        stats = (ctypes.c_int64 * 4)()
        rc = _L().alp_lex_speculative(self.g.h, self._ptr(self.wbf), self._ptr(self.params), self.n_states,
                                      self._ptr(x), x.numel(), chunk, ctypes.byref(pt), ctypes.byref(ps),
                                      ctypes.byref(pe), ctypes.byref(n), ctypes.byref(valid), stats)
        if rc != 0:
            self.g._err(rc)
        st = list(stats)
        if not valid.value:
            return None, st
        k = n.value
        return (api._wrap(self.g.h, pt.value or 0, k, torch.int32, self.g.device),
                api._wrap(self.g.h, ps.value or 0, k, torch.int64, self.g.device),
                api._wrap(self.g.h, pe.value or 0, k, torch.int64, self.g.device)), st

    @classmethod
    def constant(cls, g: "api.Grammar", state: int) -> "BoundaryModel":
        """The method without a network: every boundary guesses `state`."""
        import torch
        m = cls(g)
        m.params.zero_()
        m.params[P_B3 + state] = 1.0
        m.sync_bf16()
        return m


def main(argv=None) -> None:
    """``python -m alpacc_b200.spec --predict N [--kernel 0|1]``: N boundary
    predictions (random-init weights, json lexer) at evenly spaced positions
    of a synthetic 64 MiB json document, three calls, and the inference time
    of the last one (CUDA events).  Kernel 0 is the tcgen05 kernel, 1 the
    mma.sync kernel; a small fixed workload for profiling either.
    ``--train S``: S training steps of 4096 windows from a 4 MiB document
    (labels from the exact lexer), and the time of the last one; a small
    fixed workload for profiling the training kernels."""
    import argparse
    import torch
    from . import synth, tables
    ap = argparse.ArgumentParser(prog="python -m alpacc_b200.spec")
    ap.add_argument("--predict", type=int, default=0)
    ap.add_argument("--train", type=int, default=0)
    ap.add_argument("--kernel", type=int, default=0, choices=[0, 1])
    args = ap.parse_args(argv)
    g = api.Grammar(tables.load("json", "lexer"))
    if args.train:
        m = BoundaryModel(g, seed=5)
        win, lab = dataset(g, [synth.json_doc(4 << 20, 8, 3)], 4096 * args.train, 7)
        b = 4096
        for i in range(args.train - 1):
            m.train_step(win[i * b:(i + 1) * b], lab[i * b:(i + 1) * b])
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        loss, acc = m.train_step(win[-b:], lab[-b:])
        e1.record()
        torch.cuda.synchronize()
        print("train steps %d  batch %d  last step %.4f ms  loss %.4f  acc %.4f" % (
            args.train, b, e0.elapsed_time(e1), loss, acc))
        return
    if not args.predict:
        ap.error("one of --predict or --train")
    g.set_tuning(g.get_tuning()[:3] + [args.kernel])
    m = BoundaryModel(g, seed=5)
    size = 64 << 20
    x = torch.from_numpy(synth.json_doc(size, 8, 3)).to(g.device)
    pos = torch.arange(1, args.predict + 1, dtype=torch.int64, device=g.device) * (size // (args.predict + 1))
    for _ in range(2):
        m.predict(x, pos)
    g.profile(True)
    p = m.predict(x, pos)
    ms = sum(t for k, t in g.timings() if "mlp" in k)
    g.profile(False)
    print("predictions %d  kernel %s  %.4f ms  %.1f TFLOP/s  checksum %d" % (
        args.predict, "tcgen05" if args.kernel == 0 else "mma.sync", ms,
        args.predict * 2 * (1024 * 128 + 128 * 128 + 128 * 32) / (ms * 1e-3) / 1e12, int(p.sum())))


if __name__ == "__main__":
    main()
