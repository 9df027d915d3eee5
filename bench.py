#!/usr/bin/env python3
"""Benchmark: bit-exact lex+parse of synthetic JSON on B200.

Default workload (one step): the full json.alp lex+parse (bytes -> preorder
tree with parents, tags, kinds and spans) of one 256 MiB synthetic JSON
document of nesting depth <= 16, through the C ABI (``alp_parse``).  Inputs
are larger than L2, so no flush is needed between steps.

* ``value``   -- input GB/s with the document resident in HBM (device-timed
                 with CUDA events around the ``alp_parse`` calls).
* ``e2e``     -- the same through ``alp_parse_host``: pinned host bytes in,
                 the whole tree back to pinned host memory, copies inside
                 the timed region (parents and spans cross as 32-bit values
                 and are widened on the host; the bytes moved are the ones the
                 call reports).
* ``roofline``-- algorithmic bytes (input + 29 B per output node: i64 parent,
                 u32 tag, u8 kind, i64 start, i64 end) over the step time,
                 against the measured HBM copy bandwidth; plus a per-kernel
                 breakdown from one instrumented step.
* ``cpu_baseline`` -- the data-parallel CPU restatement of the
                 reference's generated lexer and parser (oracle/par.c, OpenMP,
                 every host thread) on the same document, rank 0 only.
* ``parity``  -- SHA-256 of each output array of the e2e call's tree against
                 the sequential oracle's, at full size (rank 0).

Other workloads (``--workload``), one JSON line each, same keys:

* ``lex``    -- json.alp lexer only (lexer-mode terminal ids) on one 512 MiB
                document of nesting depth <= 8 (``alp_lex``); algorithmic bytes
                input + 20 B per token (u32 id, i64 start, i64 end).
* ``batch``  -- 100,000 JSON documents and 50,000 sexp documents with
                log-normal sizes (median 4 KiB, sigma 1.5, capped at 4 MiB),
                each set in one ``alp_parse_batch`` call per step; algorithmic
                bytes input + 29 B per node + offsets and validity; e2e through
                ``alp_parse_batch_host``.
* ``spec``   -- learned boundary-state speculation for the json.alp and
                sexp.alp lexers: the MLP trained on the GPU on exact boundary
                states of documents from other seeds, then
                ``alp_lex_speculative`` at chunk sizes 256/1024/4096 on 512 MiB
                inputs against the plain lexer, with hit rate and re-run
                fraction; the output is compared token for token.

``--impl reference`` times the data-parallel CPU restatement alone (the
reference's own Futhark/Haskell toolchain is not available) on the same
single document.
Under torchrun each rank runs its own inputs (weak scaling, replicas, no
data-path collective); the step time is the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DOC_BYTES = 256 << 20
DEPTH = 16
NODE_BYTES = 8 + 4 + 1 + 8 + 8
MLP_FLOPS = 2 * (64 * 16 * 128 + 128 * 128 + 128 * 32)  # boundary MLP, per prediction
SEED = 0xA1FACC00 + 2
METRIC = "input GB/s lex+parse (json.alp, plain scan, bit-exact)"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _bf16_peak():
    """Dense BF16 tensor-core peak (burst, cuBLAS) in TFLOP/s and its source."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]), "measured"
    except Exception:
        return 1590.0, "fallback"


class ClockSampler:
    """SM clock and clock-event reasons of the timed GPU, read through NVML
    every 2 ms while the timed region runs (read-only queries)."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.max = None
        self.err = None
        self.t = None

    def __enter__(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = None
            try:
                import torch
                p = torch.cuda.get_device_properties(self.index)
                h = nv.nvmlDeviceGetHandleByPciBusId(
                    "%08x:%02x:%02x.0" % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id))
            except Exception:
                h = nv.nvmlDeviceGetHandleByIndex(self.index)
            self.nv, self.h = nv, h
            self.max = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            self.reasons_fn = (getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None)
                               or nv.nvmlDeviceGetCurrentClocksThrottleReasons)
            self.stop = threading.Event()
            self._sample()
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        except Exception as e:  # no NVML: the line says so
            self.err = "%s: %s" % (type(e).__name__, e)
        return self

    def _sample(self):
        try:
            self.samples.append((self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM),
                                 int(self.reasons_fn(self.h))))
        except Exception:
            pass

    def _run(self):
        while not self.stop.is_set():
            self._sample()
            time.sleep(0.002)

    def __exit__(self, *exc):
        if self.t:
            self.stop.set()
            self.t.join(timeout=2)
            self._sample()
            try:
                self.nv.nvmlShutdown()
            except Exception:
                pass

    def summary(self):
        sm = [c for c, _ in self.samples]
        reasons = set()
        for _, r in self.samples:
            for bit, nm in self.REASONS.items():
                if r & bit:
                    reasons.add(nm)
        out = {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max,
               "reasons": sorted(reasons), "samples": len(sm), "source": "nvml, 2 ms"}
        if self.err:
            out["error"] = self.err
        return out


def make_doc(seed: int, size: int) -> np.ndarray:
    from alpacc_b200 import synth
    return synth.json_doc(size, DEPTH, seed)


def _sha256(a: np.ndarray) -> str:
    """SHA-256 of a generated input (outside the timed region), so that a run's
    synthetic workload can be reproduced and compared byte for byte."""
    import hashlib
    return hashlib.sha256(memoryview(np.ascontiguousarray(a)).cast("B")).hexdigest()


def _host_threads() -> int:
    try:
        n = len(os.sched_getaffinity(0))
    except AttributeError:
        n = os.cpu_count() or 1
    return max(1, min(n, 64))


def _par_rate(P, d: bytes, reps: int):
    """Median seconds of `reps` lex+parse runs of the data-parallel CPU
    restatement over the whole document, after one warm-up run; the node
    count of the last run."""
    ok, nodes = P.lex_parse_count(d)  # warm-up
    if not ok:
        raise RuntimeError("CPU restatement rejected the benchmark document")
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        ok, nodes = P.lex_parse_count(d)
        ts.append(time.perf_counter() - t0)
        if not ok:
            raise RuntimeError("CPU restatement rejected the benchmark document")
    return statistics.median(ts), nodes


def _config(size: int, sha: str):
    """The workload as both arms name it (identical objects)."""
    return {"workload": "json.alp full lex+parse, one %d MiB synthetic JSON document (depth <= %d), bytes -> "
                        "preorder tree (i64 parent, u32 tag, u8 kind, i64 start, i64 end per node)"
                        % (size >> 20, DEPTH),
            "doc_bytes": size, "depth": DEPTH, "seed": SEED, "input_sha256": sha,
            "l2": "inputs larger than L2 (no flush needed)"}


def _par_sample(reps: int, size: int):
    """The data-parallel CPU restatement of the templates (oracle/par.c,
    OpenMP) on the benchmark document, on every host thread."""
    import oracle
    from alpacc_b200 import tables
    P = oracle.Par(tables.load("json", "both").blob(), _host_threads())
    doc = oracle.synth_json(size, DEPTH, SEED)
    sha = _sha256(doc)
    d = doc.tobytes()
    t, nodes = _par_rate(P, d, reps)
    return {"value": size / t / 1e9, "unit": "GB/s", "cores": P.threads, "kind": "port",
            "sample": "the whole %d MiB document (%d nodes), lex+parse by the data-parallel restatement of "
                      "futhark/lexer.fut + futhark/parser.fut (oracle/par.c, OpenMP, %d threads), median of %d "
                      "after a warm-up" % (size >> 20, nodes, P.threads, reps),
            "median_s": t}, sha


def cpu_baseline(size: int, reps: int):
    base, _ = _par_sample(reps, size)
    return base


def run_reference(args, rank: int, world: int):
    """The reference arm: the reference's own CPU path for lex+parse is Futhark
    multicore output of the Haskell generator, which cannot be built here (no
    GHC, no futhark); its data-parallel algorithm restated in C with OpenMP
    (oracle/par.c) runs in its place, on the same single document, every host
    thread, input generated by the oracle library's copy of the generator."""
    if rank != 0:
        return
    size = args.doc_mib << 20
    base, sha = _par_sample(max(5, args.steps), size)
    v = base["value"]
    line = {"metric": METRIC, "value": v, "unit": "GB/s", "n_gpus": world, "steps": max(5, args.steps),
            "warmup": 1, "ms_per_step": base["median_s"] * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8", "data": "synthetic", "impl": "reference",
            "config": _config(size, sha), "cpu_baseline": base,
            "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _pcie(local: int, h2d_bytes: int, d2h_bytes: int):
    """Plain pinned-memory copy bandwidth of this GPU's host link, each
    direction alone (CUDA events, best of 3 copies of 512 MiB), and the time
    the step's own copies would take at those rates: the floor of e2e."""
    import torch
    nb = 512 << 20
    dev = torch.empty(nb, dtype=torch.uint8, device=f"cuda:{local}")
    host = torch.empty(nb, dtype=torch.uint8, pin_memory=True)
    out = {}
    for name, dst, src in (("h2d", dev, host), ("d2h", host, dev)):
        best = None
        for _ in range(4):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            dst.copy_(src, non_blocking=True)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        out[name + "_gbs"] = nb / (best * 1e-3) / 1e9
    out["copy_floor_ms"] = (h2d_bytes / out["h2d_gbs"] + d2h_bytes / out["d2h_gbs"]) / 1e6
    del dev, host
    return out


def _sha_arrays(arrs, names, dtypes):
    import hashlib
    out = {}
    for a, nm, dt in zip(arrs, names, dtypes):
        out[nm] = hashlib.sha256(memoryview(np.ascontiguousarray(a).view(dt)).cast("B")).hexdigest()
    return out


def _parity_tree(doc: np.ndarray, got, N: int):
    """SHA-256 of each output array of the GPU's tree against the oracle's
    (oracle/oracle.c: the generated lex_int + parse_int restated
    sequentially), at the benchmark's full size."""
    import oracle
    from alpacc_b200 import tables
    o = oracle.Oracle(tables.load("json", "both").blob())
    t0 = time.perf_counter()
    want = o.lex_parse(doc.tobytes())
    t = time.perf_counter() - t0
    names = ["parent", "tag", "kind", "start", "end"]
    dts = [np.int64, np.uint32, np.uint8, np.int64, np.int64]
    res = {"config": "the benchmark document, whole tree", "arrays": names, "nodes": N,
           "oracle": "oracle/oracle.c orc_lex_futhark + orc_parse_futhark (sequential restatement)",
           "oracle_s": round(t, 2)}
    if want is None:
        res.update(sha256_equal=False, error="oracle rejected the document")
        return res
    sg = _sha_arrays([g[:N] for g in got], names, dts)
    sw = _sha_arrays([w.astype(d) for w, d in zip(want, dts)], names, dts)
    res["oracle_nodes"] = int(len(want[0]))
    res["sha256_equal"] = bool(len(want[0]) == N and sg == sw)
    res["sha256"] = sw
    if not res["sha256_equal"]:
        res["sha256_gpu"] = sg
    return res


def _traffic_table():
    """Per-unit DRAM bytes per launch of each kernel, from the committed ncu summary."""
    out = {}
    try:
        with open(os.path.join(ROOT, "profiles", "traffic_per_unit.txt")) as f:
            for ln in f:
                if ln.startswith("#") or not ln.strip():
                    continue
                k, unit, v = ln.split()
                out[k] = (unit, float(v))
    except OSError:
        pass
    return out


def _kernel_alg_bytes(name, units, parse_layout=True):
    """Algorithmic bytes of one launch: the inputs a kernel must read once and
    the outputs it must write once for its part of the path.  units: n (input
    bytes), m (tokens), L (parser positions), N (nodes), B (brackets), K
    (brackets left after the pairs closed between adjacent positions)."""
    n, m, L, N, B = (units.get(k, 0) for k in ("n", "m", "L", "N", "B"))
    K = units.get("K", B)
    c = (n + 31) // 32
    tok = 10 if parse_layout else 20
    # one document: the expansion takes its ⊢ / ⊣ from the position, so it reads no terminal ids
    ids_in = 2 * L if units.get("one_doc") else 4 * L
    table = {
        "parse_expand_kernel": ids_in + 8 * m + 25 * N + 8 * K,  # ids in, spans in, node fields + kept brackets out
        "parse_expand_kernel(fused)": 2 * L + 8 * m + 25 * N + 8 * K,  # terminals in (keys), spans in, same out
        "lex3_tok_kernel": n + c + tok * m,                    # bytes and chunk states in, tokens out
        "ple_tile_kernel(nodes)": 12 * N,                      # values in, parents out
        "ple_tile_kernel(brackets)": 8 * K,                    # kept brackets' depth values and symbols in
        "lex3_emit_kernel": n + 3 * c + tok * m,               # bytes, chunk states and counts in, tokens out
        "lex3_fold_kernel": n + 2 * c,                         # bytes in, chunk endomorphisms out
        "lex3_count_kernel": n + 3 * c,                        # bytes, chunk states in, counts out
        "parse_pairs_kernel": 4 * L,                           # terminal ids in, pair ids out
    }
    return table.get(name)


def _unit_count(unit, units):
    return {"node": units.get("N", 0), "bracket": units.get("K", units.get("B", 0)), "byte": units.get("n", 0),
            "position": units.get("L", 0)}.get(unit, 0)


def _roofline(kern, units, ms_path, alg_path, parse_layout=True):
    """roofline of the dominant kernel (achieved = its algorithmic bytes per
    launch over its CUDA-event duration) and the whole call as path_roofline."""
    peak, peak_kind = _peaks()
    kms, share, top, _ = _kernels(kern)
    name, tms = top
    base = name.split(":")[-1]
    alg = _kernel_alg_bytes(base, units, parse_layout)
    tt = _traffic_table().get(base)
    roof = {"bound": "hbm", "kernel": name, "peak": peak, "unit": "GB/s", "peak_kind": peak_kind,
            "achieved": None, "frac": None, "traffic": None, "kernel_ms": tms}
    if alg and tms:
        roof["achieved"] = alg / (tms * 1e-3) / 1e9
        roof["frac"] = roof["achieved"] / peak
        roof["algorithmic_bytes"] = alg
    if tt:
        roof["traffic"] = tt[1] * _unit_count(tt[0], units)
        roof["traffic_source"] = "ncu DRAM read+write per %s (profiles/traffic_per_unit.txt) x units" % tt[0]
    path = {"achieved": alg_path / (ms_path * 1e-3) / 1e9, "unit": "GB/s"}
    path["frac"] = path["achieved"] / peak
    roof["kernels_ms"] = kms
    roof["kernel_share"] = share
    return roof, path


def _profiled(g, step, reps: int):
    """Per-kernel milliseconds averaged over `reps` instrumented calls."""
    acc, order = {}, []
    for _ in range(reps):
        g.profile(True)
        step()
        for k, t in g.timings():
            if k not in acc:
                acc[k] = 0.0
                order.append(k)
            acc[k] += t
        g.profile(False)
    return [(k, acc[k] / reps) for k in order]


def _ctx_counts(g):
    import ctypes
    from alpacc_b200 import api
    L = api.native()
    out = (ctypes.c_int64 * 15)()
    L.alp_ctx_info.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    L.alp_ctx_info(g.h, out, 15)
    return {"m": int(out[8]), "L": int(out[9]), "B": int(out[10]), "K": int(out[11]),
            "h2d": int(out[13]), "d2h": int(out[14])}


SEED_LEX = 0xA1FACC00 + 1
SEED_BATCH = 0xA1FACC00 + 3
SEED_TRAIN = 0xA1FACC10


def _dist_init(world: int, backend: str = "nccl"):
    """Process group for N > 1 ranks (one per GPU; gloo for the CPU tests),
    with a short timeout so that ranks waiting for a dead peer fail."""
    if world <= 1:
        return None
    import datetime
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return dist


def _max_over_ranks(ms: float, dist, device) -> float:
    """The step time of the job: the slowest rank's."""
    if not dist:
        return ms
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device if isinstance(device, str) else f"cuda:{device}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _e2e_two_contexts(L, g, h_in, size, N, outs, k, stream, dist, local, world):
    """alp_parse_host on two contexts from two host threads, k calls each, back to back;
    per-document time = elapsed / (2 k).  ctypes releases the GIL during each call."""
    import ctypes
    import threading
    import torch
    from alpacc_b200 import api, tables
    g2 = api.Grammar(tables.load("json", "both"), device=local)
    g2._stream()
    outs2 = [torch.empty(o.shape, dtype=o.dtype, pin_memory=True) for o in outs]
    errs = []

    def calls(gx, ox, n_calls):
        n_, v_ = ctypes.c_int64(0), ctypes.c_int(0)
        for _ in range(n_calls):
            rc = L.alp_parse_host(gx.h, ctypes.c_void_p(h_in.data_ptr()), size,
                                  *[ctypes.c_void_p(o.data_ptr()) for o in ox], N, ctypes.byref(n_), ctypes.byref(v_))
            if rc != 0 or not v_.value or n_.value != N:
                errs.append(rc)

    calls(g2, outs2, 1)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    th = [threading.Thread(target=calls, args=(gx, ox, k)) for gx, ox in ((g, outs), (g2, outs2))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    e1.record(stream)
    torch.cuda.synchronize()
    if errs:
        raise RuntimeError("alp_parse_host failed on a second context: %r" % errs[:3])
    same = all(torch.equal(a, b) for a, b in zip(outs, outs2))
    ms = _max_over_ranks(e0.elapsed_time(e1) / (2 * k), dist, local)
    del outs2, g2
    if not same:
        raise RuntimeError("the two contexts' trees differ")
    return {"value": _gbs(world, size, ms), "unit": "GB/s", "ms_per_doc": ms,
            "contexts": 2, "calls": 2 * k, "trees_equal": True,
            "note": "throughput of a document stream, not one call's latency (the line's e2e value)"}


def _gbs(world: int, bytes_per_rank: int, ms: float) -> float:
    """Whole-job input GB/s: every rank processes bytes_per_rank (weak scaling)."""
    return world * bytes_per_rank / (ms * 1e-3) / 1e9


def _timed(step, steps: int, local: int, dist):
    """ms per step of `steps` calls (CUDA events on the current stream,
    synchronize and barrier on both sides, max over ranks) and the clocks."""
    import torch
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = _max_over_ranks(ev0.elapsed_time(ev1) / steps, dist, local)
    return ms, clk.summary()


def _kernels(kern):
    total_k = sum(t for _, t in kern) or 1.0
    top = max(kern, key=lambda x: x[1]) if kern else ("", 0.0)
    return ({k: round(t, 4) for k, t in kern}, {k: round(t / total_k, 4) for k, t in kern}, top,
            sum(1 + k.count("+") for k, _ in kern))


def _line(metric, value, world, args, ms, config, alg_bytes, kern, e2e, clocks, extra=None, units=None,
          parse_layout=True):
    _, _, _, launches = _kernels(kern)
    roof, path = _roofline(kern, units or {}, ms, alg_bytes, parse_layout)
    line = {"metric": metric, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8", "data": "synthetic", "config": config,
            "roofline": roof, "path_roofline": path,
            "e2e": e2e, "gpu_launches": launches * args.steps, "clocks": clocks}
    if extra:
        line.update(extra)
    return line


def run_lex(args, rank: int, world: int, local: int):
    """json.alp lexer only, one 512 MiB document (lexer-mode ids), alp_lex."""
    import ctypes
    import torch
    from alpacc_b200 import api, synth, tables
    torch.cuda.set_device(local)
    dist = _dist_init(world)
    size = (args.doc_mib << 20) if args.doc_mib_given else 512 << 20
    doc = synth.json_doc(size, 8, SEED_LEX + 1000 * rank)
    g = api.Grammar(tables.load("json", "lexer"), device=local)
    d_in = torch.from_numpy(doc).to(f"cuda:{local}")
    g._stream()
    L = api.native()
    ptrs = [ctypes.c_void_p() for _ in range(3)]
    n_tok, valid = ctypes.c_int64(0), ctypes.c_int(0)

    def step():
        rc = L.alp_lex(g.h, ctypes.c_void_p(d_in.data_ptr()), size, *[ctypes.byref(p) for p in ptrs],
                       ctypes.byref(n_tok), ctypes.byref(valid))
        if rc != 0 or not valid.value:
            raise RuntimeError("alp_lex failed rc=%d: %s" % (rc, L.alp_last_error(g.h).decode()))

    for _ in range(max(3, args.warmup)):
        step()
    M = n_tok.value
    ms, clocks = _timed(step, args.steps, local, dist)
    kern = _profiled(g, step, 3)
    # end to end: pinned host bytes in, tokens back to pinned host memory
    h_in = torch.from_numpy(doc).pin_memory()
    outs = [torch.empty(M, dtype=dt, pin_memory=True) for dt in (torch.int32, torch.int64, torch.int64)]
    n2, v2 = ctypes.c_int64(0), ctypes.c_int(0)

    def e2e_step():
        rc = L.alp_lex_host(g.h, ctypes.c_void_p(h_in.data_ptr()), size, *[ctypes.c_void_p(o.data_ptr()) for o in outs],
                            M, ctypes.byref(n2), ctypes.byref(v2))
        if rc != 0 or n2.value != M:
            raise RuntimeError("alp_lex_host failed rc=%d" % rc)

    e2e_step()
    ms_whole, _ = _timed(e2e_step, max(1, min(args.steps, 5)), local, dist)
    whole = (n2.value, [o[:M].clone() for o in outs])
    # the same through the token stream: 32 MiB pieces, the copies in and out
    # overlapped with the lexing
    piece = 32 << 20

    def e2e_stream():
        rc = L.alp_lex_host_stream(g.h, ctypes.c_void_p(h_in.data_ptr()), size, piece,
                                   *[ctypes.c_void_p(o.data_ptr()) for o in outs], M, ctypes.byref(n2),
                                   ctypes.byref(v2))
        if rc != 0 or n2.value != M or not v2.value:
            raise RuntimeError("alp_lex_host_stream failed rc=%d" % rc)

    e2e_stream()
    if n2.value != whole[0] or not all(torch.equal(o[:M], w) for o, w in zip(outs, whole[1])):
        raise RuntimeError("alp_lex_host_stream tokens differ from alp_lex_host")
    # both host calls widen 32-bit spans on the host: their tokens against alp_lex's
    # 64-bit device arrays, element for element
    step()
    dev = [api._wrap(g.h, p.value, M, dt, f"cuda:{local}") for p, dt in zip(ptrs, (torch.int32, torch.int64,
                                                                                     torch.int64))]
    if not all(torch.equal(o[:M].to(d.device), d) for o, d in zip(outs, dev)):
        raise RuntimeError("alp_lex_host_stream tokens differ from alp_lex's device arrays")
    del dev
    ms_e2e, _ = _timed(e2e_stream, max(1, min(args.steps, 5)), local, dist)
    moved = _ctx_counts(g)  # the spans cross as 32-bit values
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = _line("input GB/s lex (json.alp lexer-only, plain scan, bit-exact)", _gbs(world, size, ms),
                 world, args, ms,
                 {"workload": "json.alp lexer only, one %d MiB synthetic JSON document per GPU (depth <= 8), "
                              "bytes -> (u32 id, i64 start, i64 end) tokens" % (size >> 20),
                  "doc_bytes": size, "tokens": M, "tokens_per_byte": M / size, "parallelism": "replicas",
                  "l2": "inputs larger than L2 (no flush needed)", "seed": SEED_LEX,
                  "input_sha256": _sha256(doc)},
                 size + 20 * M, kern,
                 {"value": _gbs(world, size, ms_e2e), "unit": "GB/s", "h2d_bytes_per_step": moved["h2d"],
                  "d2h_bytes_per_step": moved["d2h"], "ms_per_step": ms_e2e,
                  "api": "alp_lex_host_stream, 32 MiB pieces, pinned host buffers",
                  "d2h_form": "i32 spans (sign-extended into the caller's i64 arrays on the host while later "
                              "chunks are in flight), u32 ids", "bit_exact_vs_device": True,
                  "whole_input": {"api": "alp_lex_host", "value": _gbs(world, size, ms_whole),
                                  "ms_per_step": ms_whole}}, clocks,
                 units={"n": size, "m": M}, parse_layout=False)
    line["path_roofline"]["scope"] = "whole alp_lex call: input bytes + 20 B per token, over the step time"
    print(json.dumps(line), flush=True)


def run_batch(args, rank: int, world: int, local: int):
    """100,000 JSON + 50,000 sexp documents, log-normal sizes, alp_parse_batch."""
    import ctypes
    import torch
    from alpacc_b200 import api, synth, tables
    torch.cuda.set_device(local)
    dist = _dist_init(world)
    dev = f"cuda:{local}"
    L = api.native()
    sets = []
    nj = args.batch_docs
    for name, n_docs, depth, seed in (("json", nj, 8, SEED_BATCH), ("sexp", nj // 2, 20, SEED_BATCH + 1)):
        seed += 1000 * rank
        sizes = synth.lognormal_sizes(n_docs, median=4096, sigma=1.5, cap=4 << 20, seed=seed)
        data, off = synth.batch(name, sizes, depth, seed)
        g = api.Grammar(tables.load(name, "both"), device=local)
        sets.append({"name": name, "g": g, "data": data, "off": off, "n_docs": n_docs,
                     "x": torch.from_numpy(data).to(dev), "o": torch.from_numpy(off).to(dev),
                     "ptrs": [ctypes.c_void_p() for _ in range(7)], "N": ctypes.c_int64(0)})
    sets[0]["g"]._stream()

    def call(st, x, o):
        rc = L.alp_parse_batch(st["g"].h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(o.data_ptr()), st["n_docs"],
                               *[ctypes.byref(p) for p in st["ptrs"]], ctypes.byref(st["N"]))
        if rc != 0:
            raise RuntimeError("alp_parse_batch failed rc=%d: %s" % (rc, L.alp_last_error(st["g"].h).decode()))

    def step():
        for st in sets:
            call(st, st["x"], st["o"])

    for _ in range(max(3, args.warmup)):
        step()
    ms, clocks = _timed(step, args.steps, local, dist)
    kern = []
    for st in sets:
        st["g"].profile(True)
        call(st, st["x"], st["o"])
        kern += [("%s:%s" % (st["name"], k), t) for k, t in st["g"].timings()]
        st["g"].profile(False)
        st["counts"] = _ctx_counts(st["g"])
        valid = _wrap_valid(st)
        st["accepted"] = int(valid.sum())
    # end to end through alp_parse_batch_host: documents and offsets from pinned host
    # memory, the trees (parents and spans as 32-bit values widened on the host), node
    # offsets and validity back to pinned host memory, all inside the timed region
    for st in sets:
        N, D = st["N"].value, st["n_docs"]
        st["h_x"] = torch.from_numpy(st["data"]).pin_memory()
        st["h_o"] = torch.from_numpy(st["off"]).pin_memory()
        st["h_out"] = [torch.empty(N * w, dtype=torch.uint8, pin_memory=True) for w in (8, 4, 1, 8, 8)]
        st["h_noff"] = torch.empty((D + 1) * 8, dtype=torch.uint8, pin_memory=True)
        st["h_valid"] = torch.empty(D, dtype=torch.uint8, pin_memory=True)
    L.alp_parse_batch_host.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int64] + [ctypes.c_void_p] * 7 + \
        [ctypes.c_int64, ctypes.c_void_p]
    h_total = ctypes.c_int64(0)

    def e2e_step():
        for st in sets:
            ptr = lambda t: ctypes.c_void_p(t.data_ptr())
            rc = L.alp_parse_batch_host(st["g"].h, ptr(st["h_x"]), ptr(st["h_o"]), st["n_docs"],
                                        *[ptr(t) for t in st["h_out"]], ptr(st["h_noff"]), ptr(st["h_valid"]),
                                        st["N"].value, ctypes.byref(h_total))
            if rc != 0 or h_total.value != st["N"].value:
                raise RuntimeError("alp_parse_batch_host failed rc=%d" % rc)

    e2e_step()
    ms_e2e, _ = _timed(e2e_step, max(1, min(args.steps, 3)), local, dist)
    h2d = d2h = 0
    for st in sets:
        moved = _ctx_counts(st["g"])
        h2d += moved["h2d"]
        d2h += moved["d2h"]
    # the host arrays of the last e2e call, byte for byte, against alp_parse_batch's on the device
    for st in sets:
        tree, noff, val = st["g"].parse_batch_int(st["x"], st["o"])
        dev = [tree.parent, tree.tag, tree.kind, tree.start, tree.end, noff, val]
        for h, d in zip(st["h_out"] + [st["h_noff"], st["h_valid"]], dev):
            if not torch.equal(h.to(d.device), d.contiguous().view(torch.uint8)):
                raise RuntimeError("alp_parse_batch_host output differs from alp_parse_batch")
        del tree, noff, val, dev

    # the same batches captured once each as a CUDA graph (alp_parse_graph_*),
    # replayed; outputs compared with alp_parse_batch's on the device
    graph = {}
    if not args.no_graph:
        for st in sets:
            for k2 in ("h_x", "h_o", "d_x", "d_o", "h_out", "h_noff", "h_valid"):
                st.pop(k2, None)
        torch.cuda.empty_cache()
        pgs = []
        exact = True
        for st in sets:
            want = st["g"].parse_batch_int(st["x"], st["o"])
            pg = st["g"].parse_batch_graph(st["x"], st["o"], cap_nodes=st["N"].value + 64,
                                           cap_brackets=st["counts"]["B"] + 64)
            pg.launch()
            got = pg.result()
            exact = exact and len(got[0]) == len(want[0]) and torch.equal(got[1], want[1]) and \
                torch.equal(got[2], want[2]) and all(torch.equal(getattr(got[0], f), getattr(want[0], f))
                                                     for f in ("parent", "tag", "kind", "start", "end"))
            del want, got
            pgs.append(pg)
        if not exact:
            raise RuntimeError("graph replay differs from alp_parse_batch")

        def gstep():
            for pg in pgs:
                pg.launch()

        for _ in range(max(3, args.warmup)):
            gstep()
        ms_graph, _ = _timed(gstep, args.steps, local, dist)
        for pg in pgs:
            pg.result()
            pg.close()
        graph = {"api": "alp_parse_graph_create once per grammar, then alp_parse_graph_launch per step",
                 "ms_per_step": ms_graph, "value": _gbs(world, sum(len(st["data"]) for st in sets), ms_graph),
                 "unit": "GB/s", "vs_alp_parse_batch": ms / ms_graph, "bit_exact": True}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    n_bytes = sum(len(st["data"]) for st in sets)
    alg = sum(len(st["data"]) + 29 * st["N"].value + 17 * (st["n_docs"] + 1) for st in sets)
    cfg = {"workload": "batched segmented lex+parse: %d json.alp documents (depth <= 8) and %d "
                       "sexp.alp documents (depth <= 20), log-normal sizes (median 4 KiB, sigma 1.5, cap 4 MiB), "
                       "one alp_parse_batch call per grammar per step" % (sets[0]["n_docs"], sets[1]["n_docs"]),
           "parallelism": "replicas", "l2": "inputs larger than L2 (no flush needed)"}
    for st in sets:
        cfg[st["name"]] = {"docs": st["n_docs"], "bytes": len(st["data"]), "nodes": st["N"].value,
                           "accepted": st["accepted"]}
    _, _, top, _ = _kernels(kern)
    st_top = [st for st in sets if top[0].startswith(st["name"] + ":")][0]
    units = dict(st_top["counts"], n=len(st_top["data"]), N=st_top["N"].value)
    line = _line("input GB/s batched lex+parse (json.alp + sexp.alp documents, bit-exact)",
                 _gbs(world, n_bytes, ms), world, args, ms, cfg, alg, kern,
                 {"value": _gbs(world, n_bytes, ms_e2e), "unit": "GB/s", "h2d_bytes_per_step": h2d,
                  "d2h_bytes_per_step": d2h, "ms_per_step": ms_e2e, "api": "alp_parse_batch_host, pinned buffers",
                  "bit_exact_vs_device": True}, clocks, units=units)
    line["path_roofline"]["scope"] = ("both alp_parse_batch calls: input bytes + 29 B per node + 17 B per "
                                      "document (offsets in, node offsets and validity out), over the step time")
    if graph:
        line["graph"] = graph
    print(json.dumps(line), flush=True)


def run_graph(args, rank: int, world: int, local: int):
    """Small batches of json.alp documents through the captured CUDA graph
    (alp_parse_graph_*), beside alp_parse_batch on the same documents."""
    import ctypes
    import torch
    from alpacc_b200 import api, synth, tables
    torch.cuda.set_device(local)
    dist = _dist_init(world)
    dev = f"cuda:{local}"
    L = api.native()
    g = api.Grammar(tables.load("json", "both"), device=local)
    g._stream()
    shapes = [(64, 1024), (256, 4096), (2048, 8192)]  # documents, median bytes
    head = 1  # the shape the line's value is quoted on
    res = {}
    for si, (n_docs, med) in enumerate(shapes):
        seed = SEED_BATCH + 100 + si + 1000 * rank
        sizes = synth.lognormal_sizes(n_docs, median=med, sigma=1.0, cap=16 * med, seed=seed)
        data, off = synth.batch("json", sizes, 8, seed)
        x, o = torch.from_numpy(data).to(dev), torch.from_numpy(off).to(dev)
        ptrs = [ctypes.c_void_p() for _ in range(7)]
        N = ctypes.c_int64(0)

        def plain():
            rc = L.alp_parse_batch(g.h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(o.data_ptr()), n_docs,
                                   *[ctypes.byref(p) for p in ptrs], ctypes.byref(N))
            if rc != 0:
                raise RuntimeError("alp_parse_batch failed rc=%d" % rc)

        want = g.parse_batch_int(x, o)
        pg = g.parse_batch_graph(x, o)
        pg.launch()
        got = pg.result()
        exact = (len(got[0]) == len(want[0]) and torch.equal(got[1], want[1]) and torch.equal(got[2], want[2]) and
                 all(torch.equal(getattr(got[0], f), getattr(want[0], f))
                     for f in ("parent", "tag", "kind", "start", "end")))
        if not exact:
            raise RuntimeError("graph replay differs from alp_parse_batch")
        for _ in range(max(3, args.warmup)):
            plain()
            pg.launch()
        steps = max(args.steps, 20)
        ms_plain, _ = _timed(plain, steps, local, dist)
        ms_graph, clocks = _timed(pg.launch, steps, local, dist)
        pg.result()
        r = {"docs": n_docs, "bytes": len(data), "nodes": len(want[0]), "graph_ms": ms_graph, "batch_ms": ms_plain,
             "graph_gbs": _gbs(world, len(data), ms_graph), "batch_gbs": _gbs(world, len(data), ms_plain),
             "speedup": ms_plain / ms_graph, "bit_exact": True}
        if si == head:
            kern = _profiled(g, plain, 3)
            counts = _ctx_counts(g)
            # end to end through the graph: pinned input in, the tree out
            hx = torch.from_numpy(data).pin_memory()
            nb = len(want[0])
            hout = [torch.empty(nb * w, dtype=torch.uint8, pin_memory=True) for w in (8, 4, 1, 8, 8)]
            srcs = [pg.parent, pg.tag, pg.kind, pg.start, pg.end]

            def e2e():
                pg.x.copy_(hx, non_blocking=True)
                pg.launch()
                pg.result()
                for dst, src in zip(hout, srcs):
                    dst.copy_(src.view(torch.uint8)[:dst.numel()], non_blocking=True)

            e2e()
            ms_e2e, _ = _timed(e2e, steps, local, dist)
            hd = {"x": data, "N": nb, "counts": counts, "ms": ms_graph, "kern": kern, "clocks": clocks,
                  "e2e": ms_e2e, "h2d": len(data), "d2h": 29 * nb}
        pg.close()
        res["%d docs, median %d B" % (n_docs, med)] = r
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    n_bytes = len(hd["x"])
    cfg = {"workload": "small batches of json.alp documents (depth <= 8, log-normal sizes, sigma 1.0) through "
                       "one captured CUDA graph per batch shape (alp_parse_graph_launch), beside alp_parse_batch "
                       "on the same documents; the value is the %d-document batch" % shapes[head][0],
           "parallelism": "replicas", "l2": "batches fit in L2; every replay re-reads them (no flush)",
           "shapes": res}
    alg = n_bytes + 29 * hd["N"]
    line = _line("input GB/s batched lex+parse, CUDA graph replay (json.alp documents, bit-exact)",
                 _gbs(world, n_bytes, hd["ms"]), world, args, hd["ms"], cfg, alg, hd["kern"],
                 {"value": _gbs(world, n_bytes, hd["e2e"]), "unit": "GB/s", "h2d_bytes_per_step": hd["h2d"],
                  "d2h_bytes_per_step": hd["d2h"], "ms_per_step": hd["e2e"],
                  "api": "alp_parse_graph_launch + alp_parse_graph_result, pinned host buffers"},
                 hd["clocks"], units=dict(hd["counts"], n=n_bytes, N=hd["N"]))
    line["path_roofline"]["scope"] = "one replay: input bytes + 29 B per node, over the replay time"
    print(json.dumps(line), flush=True)


def run_shard(args, rank: int, world: int, local: int):
    """One 512 MiB json.alp document lexed by all ranks together: rank r holds
    the r-th byte range; two all-gathers of a few bytes per rank (state
    functions, then token counts and last starts) place every range's tokens.
    Strong scaling: the document is the same for every N."""
    import torch
    from alpacc_b200 import api, shard, synth, tables
    torch.cuda.set_device(local)
    dist = _dist_init(world)
    size = (args.doc_mib << 20) if args.doc_mib_given else 512 << 20
    doc = synth.json_doc(size, 8, SEED_LEX)
    a, b = size * rank // world, size * (rank + 1) // world
    g = api.Grammar(tables.load("json", "lexer"), device=local)
    x = torch.from_numpy(doc[a:b]).to(f"cuda:{local}")
    g._stream()

    def gather(obj):
        if not dist:
            return [obj]
        out = [None] * world
        dist.all_gather_object(out, obj)
        return out

    res = {}

    def step():
        res["t"] = shard.lex_shard(g, x, a, rank == world - 1, rank, gather)

    for _ in range(max(3, args.warmup)):
        step()
    ms, clocks = _timed(step, args.steps, local, dist)
    kern = _profiled(g, step, 3)
    toks, base, valid = res["t"]
    n_local = int(toks[0].numel())
    total = gather(n_local)
    if world == 1:
        whole = g.lex_int(x)
        if whole is None or not all(torch.equal(u.to(v.dtype), v) for u, v in zip(toks, whole)):
            raise RuntimeError("sharded lexing differs from alp_lex")
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    M = int(sum(total))
    cfg = {"workload": "json.alp lexer, one %d MiB synthetic document (depth <= 8) split into %d contiguous byte "
                       "ranges, one per GPU; two all-gathers per step (state functions; token counts and last "
                       "starts)" % (size >> 20, world),
           "doc_bytes": size, "tokens": M, "parallelism": "byte ranges of one document",
           "l2": "inputs larger than L2 (no flush needed)"}
    line = _line("input GB/s lex of one document across GPUs (json.alp lexer-only, bit-exact)",
                 size / (ms * 1e-3) / 1e9, world, args, ms, cfg, size + 20 * M, kern,
                 {"value": None, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                  "note": "device-resident ranges; see the lex workload for host buffers"}, clocks,
                 units={"n": b - a, "m": n_local}, parse_layout=False)
    line["scaling"] = "strong"
    line["path_roofline"]["scope"] = "whole job: document bytes + 20 B per token over the step time, all GPUs"
    print(json.dumps(line), flush=True)


def _wrap_valid(st):
    import torch
    from alpacc_b200 import api
    return api._wrap(st["g"].h, st["ptrs"][6].value or 0, st["n_docs"], torch.uint8, st["g"].device)


def _spec_eval(name, depth, eval_seed, size, args, local, dist, chunks):
    """Train the boundary MLP on the GPU (pairs labelled by the exact lexer on
    documents from other seeds), then time alp_lex_speculative at each chunk
    size against alp_lex on one document, tokens compared on the device.
    Returns (summary, grammar, model, device input, best (C, ms, tokens), clocks)."""
    import ctypes
    import torch
    from alpacc_b200 import api, spec, synth, tables
    dev = f"cuda:{local}"
    L = api.native()
    g = api.Grammar(tables.load(name, "lexer"), device=local)
    g._stream()
    t0 = time.perf_counter()
    docs = [synth.json_doc(16 << 20, depth, SEED_TRAIN + k) if name == "json"
            else synth.sexp_doc(16 << 20, depth, SEED_TRAIN + k) for k in range(10)]
    win, lab = spec.dataset(g, docs, 1000000, SEED_TRAIN)
    model = spec.BoundaryModel(g, seed=1)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    hist = model.train(win, lab, epochs=1, batch=4096, lr=2e-3)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t1
    del win, lab, docs
    doc = synth.json_doc(size, depth, eval_seed) if name == "json" else synth.sexp_doc(size, depth, eval_seed)
    x = torch.from_numpy(doc).to(dev)
    ptrs = [ctypes.c_void_p() for _ in range(3)]
    n_tok, valid = ctypes.c_int64(0), ctypes.c_int(0)

    def plain():
        rc = L.alp_lex(g.h, ctypes.c_void_p(x.data_ptr()), size, *[ctypes.byref(p) for p in ptrs],
                       ctypes.byref(n_tok), ctypes.byref(valid))
        if rc != 0 or not valid.value:
            raise RuntimeError("alp_lex failed")

    for _ in range(max(3, args.warmup)):
        plain()
    ms_plain, clk = _timed(plain, args.steps, local, dist)
    M = n_tok.value
    ref = [api._wrap(g.h, p.value or 0, M, dt, g.device).clone()
           for p, dt in zip(ptrs, (torch.int32, torch.int64, torch.int64))]
    res = {"train_pairs": int(hist["steps"]) * 4096, "train_s": t_train, "train_acc": hist["last_acc"],
           "prep_s": t1 - t0, "plain_gbs": size / (ms_plain * 1e-3) / 1e9, "plain_ms": ms_plain, "tokens": M,
           "chunks": {}}
    Ls = spec._L()
    sptr = [ctypes.c_void_p() for _ in range(3)]
    sn, sv = ctypes.c_int64(0), ctypes.c_int(0)
    stats = (ctypes.c_int64 * 4)()
    best = None
    for C in chunks:

        def sp():
            rc = Ls.alp_lex_speculative(g.h, ctypes.c_void_p(model.wbf.data_ptr()),
                                        ctypes.c_void_p(model.params.data_ptr()), model.n_states,
                                        ctypes.c_void_p(x.data_ptr()), size, C, *[ctypes.byref(p) for p in sptr],
                                        ctypes.byref(sn), ctypes.byref(sv), stats)
            if rc != 0:
                raise RuntimeError("alp_lex_speculative failed: %s" % L.alp_last_error(g.h).decode())

        for _ in range(max(3, args.warmup)):
            sp()
        ms_sp, _ = _timed(sp, args.steps, local, dist)
        st = list(stats)
        exact = bool(sv.value) and sn.value == M and all(
            torch.equal(api._wrap(g.h, p.value or 0, M, r.dtype, g.device), r) for p, r in zip(sptr, ref))
        res["chunks"][str(C)] = {"gbs": size / (ms_sp * 1e-3) / 1e9, "ms": ms_sp,
                                 "hit_rate": 1.0 - st[1] / max(1, st[0]), "rerun_fraction": st[2] / max(1, st[0]),
                                 "rounds": st[3], "bit_exact": bool(exact), "vs_plain": ms_plain / ms_sp}
        if not exact:
            raise RuntimeError("speculative tokens differ from the plain lexer (%s, C=%d)" % (name, C))
        if best is None or ms_sp < best[1]:
            best = (C, ms_sp, M)
    return res, g, model, x, best, clk


def spec_summary(args, local):
    """The default line's `spec` object: json.alp lexer, one 512 MiB document,
    learned speculation at its better chunk size against the plain lexer."""
    size = 512 << 20
    res, g, model, x, best, _ = _spec_eval("json", 8, SEED_LEX, size, args, local, None, (1024, 4096))
    C = best[0]
    c = res["chunks"][str(C)]
    out = {"workload": "json.alp lexer, one %d MiB document (depth <= 8), MLP trained on %d boundary pairs from "
                       "other seeds" % (size >> 20, res["train_pairs"]),
           "chunk": C, "gbs": c["gbs"], "plain_gbs": res["plain_gbs"], "vs_plain": c["vs_plain"],
           "hit_rate": c["hit_rate"], "rerun_fraction": c["rerun_fraction"], "bit_exact": c["bit_exact"],
           "train_s": res["train_s"], "chunks": res["chunks"]}
    del x, model, g
    return out


def run_spec(args, rank: int, world: int, local: int):
    """Learned boundary-state speculation against the plain lexer."""
    import torch
    torch.cuda.set_device(local)
    dist = _dist_init(world)
    dev = f"cuda:{local}"
    size = (args.doc_mib << 20) if args.doc_mib_given else 512 << 20
    results = {}
    kern_all = []
    best = None
    mlp_line = None
    clocks = None
    for name, depth, eval_seed in (("json", 8, SEED_LEX), ("sexp", 20, SEED_BATCH + 1)):
        res, g, model, x, b, clk = _spec_eval(name, depth, eval_seed, size, args, local, dist, (256, 1024, 4096))
        clocks = clocks or clk
        if name == "json":
            best = b
        g.profile(True)
        model.lex(x, best[0] if name == "json" else 1024)
        kern_all += [("%s:%s" % (name, k), t) for k, t in g.timings()]
        g.profile(False)
        if name == "json":
            # the boundary MLP alone (tcgen05 kernel): one prediction per 1 KiB chunk start
            P = size // 1024 - 1
            cpos = torch.arange(1, P + 1, dtype=torch.int64, device=dev) * 1024
            ts = []
            for _ in range(5):
                g.profile(True)
                model.predict(x, cpos)
                ts.append(sum(t for k, t in g.timings() if "mlp" in k))
                g.profile(False)
            mlp_ms = sorted(ts)[len(ts) // 2]
            peak, kind = _bf16_peak()
            tflops = P * MLP_FLOPS / (mlp_ms * 1e-3) / 1e12
            mlp_line = {"kernel": "mlp_wimg+mlp_infer3 (tcgen05)", "bound": "tensor", "predictions": P,
                        "flops_per_prediction": MLP_FLOPS, "ms": mlp_ms, "achieved": tflops, "peak": peak,
                        "peak_kind": kind + " bf16 burst", "unit": "TFLOP/s", "frac": tflops / peak}
        results[name] = res
        del x
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    C, ms, M = best
    line = _line("input GB/s lex, learned boundary-state speculation (json.alp lexer, bit-exact)",
                 _gbs(world, size, ms), world, args, ms,
                 {"workload": "json.alp lexer on one %d MiB document (depth <= 8) with MLP-predicted chunk "
                              "start states, best chunk size; sexp.alp in 'results'" % (size >> 20),
                  "chunk": C, "doc_bytes": size, "results": results, "parallelism": "replicas",
                  "l2": "inputs larger than L2 (no flush needed)"},
                 size + 20 * M, kern_all,
                 {"value": None, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                  "note": "speculation is a device-resident variant of alp_lex; see the lex workload for e2e"},
                 clocks, units={"n": size, "m": M}, parse_layout=False)
    line["path_roofline"]["scope"] = "alp_lex_speculative: input bytes + 20 B per token, over the step time"
    line["mlp_roofline"] = mlp_line
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--doc-mib", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="skip the full-size comparison with the oracle")
    ap.add_argument("--no-graph", action="store_true", help="batch workload: skip the CUDA-graph replay")
    ap.add_argument("--no-spec", action="store_true", help="default workload: skip the learned-speculation object")
    ap.add_argument("--no-two", action="store_true", help="default workload: skip the two-context serving figure")
    ap.add_argument("--no-tune", action="store_true", help="default launch shapes (no autotuner run): for "
                    "launch lists whose first launches should be the measured ones")
    ap.add_argument("--tuning", default=None, help="comma-separated tuning values (alp_tune_set) instead of the "
                    "autotuner: to repeat a tuned run's configuration, e.g. under a profiler")
    ap.add_argument("--workload", default="parse", choices=["parse", "lex", "batch", "spec", "graph", "shard"])
    ap.add_argument("--batch-docs", type=int, default=100000, help="JSON documents of the batch workload "
                    "(half as many sexp documents); smaller values are for profiling")
    args = ap.parse_args()
    args.doc_mib_given = args.doc_mib is not None
    if args.doc_mib is None:
        args.doc_mib = DOC_BYTES >> 20
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload != "parse":
        return {"lex": run_lex, "batch": run_batch, "spec": run_spec,
                "graph": run_graph, "shard": run_shard}[args.workload](args, rank, world, local)

    import torch
    from alpacc_b200 import api, tables

    torch.cuda.set_device(local)
    dist = _dist_init(world)
    size = args.doc_mib << 20
    doc = make_doc(SEED + 1000 * rank, size)
    g = api.Grammar(tables.load("json", "both"), device=local)
    d_in = torch.from_numpy(doc).to(f"cuda:{local}")
    stream = torch.cuda.current_stream()
    g._stream()

    import ctypes
    L = api.native()
    ptrs = [ctypes.c_void_p() for _ in range(5)]
    n_node, valid = ctypes.c_int64(0), ctypes.c_int(0)

    def step():
        rc = L.alp_parse(g.h, ctypes.c_void_p(d_in.data_ptr()), size, *[ctypes.byref(p) for p in ptrs],
                         ctypes.byref(n_node), ctypes.byref(valid))
        if rc != 0 or not valid.value:
            raise RuntimeError("alp_parse failed rc=%d valid=%d: %s" % (rc, valid.value,
                                                                       L.alp_last_error(g.h).decode()))

    # launch shapes from the autotuner, timed on this document (outside the timed region)
    if args.tuning:
        g.set_tuning([int(x) for x in args.tuning.split(",")])
        tuning = {"config": g.get_tuning(), "tile_shape": g.tile_shapes()[g.get_tuning()[0]], "timings": []}
    elif args.no_tune:
        tuning = {"config": g.get_tuning(), "tile_shape": g.tile_shapes()[g.get_tuning()[0]], "timings": []}
    else:
        tuning = g.tune(d_in, reps=3)
    g._stream()
    for _ in range(max(3, args.warmup)):
        step()
    N = n_node.value
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = _max_over_ranks(ev0.elapsed_time(ev1) / args.steps, dist, local)
    if dist:
        dist.barrier()

    # per-kernel breakdown: CUDA events between the launches of three instrumented
    # steps right after the timed region, averaged per kernel
    kern = _profiled(g, step, 3)
    counts = _ctx_counts(g)

    # end to end through the host-buffer entry point
    h_in = torch.from_numpy(doc).pin_memory()
    outs = [torch.empty(N, dtype=dt, pin_memory=True) for dt in (torch.int64, torch.int32, torch.uint8,
                                                                  torch.int64, torch.int64)]
    n2, v2 = ctypes.c_int64(0), ctypes.c_int(0)

    def e2e_step():
        rc = L.alp_parse_host(g.h, ctypes.c_void_p(h_in.data_ptr()), size,
                              *[ctypes.c_void_p(o.data_ptr()) for o in outs], N, ctypes.byref(n2), ctypes.byref(v2))
        if rc != 0 or not v2.value or n2.value != N:
            raise RuntimeError("alp_parse_host failed rc=%d" % rc)

    e2e_step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    k_e2e = max(1, min(args.steps, 5))
    for _ in range(k_e2e):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = _max_over_ranks(e0.elapsed_time(e1) / k_e2e, dist, local)
    # the bytes the call moved: parents and spans cross as 32-bit values
    moved = _ctx_counts(g)
    pcie = _pcie(local, moved["h2d"], moved["d2h"])
    # a stream of such documents served by two contexts on two host threads, each making
    # the same synchronous alp_parse_host calls (one call's input copy and device work
    # overlap the other's tree copy out): documents per second as input GB/s; one GPU only
    # (a second set of pinned tree buffers and widening threads per rank)
    two = None
    if not args.no_two and world == 1:
        two = _e2e_two_contexts(L, g, h_in, size, N, outs, k_e2e, stream, dist, local, world)

    # full-size parity: the tree the e2e call brought back against the oracle
    # (sequential restatement of the generated lex_int + parse_int)
    parity = None
    if rank == 0 and not args.no_parity:
        parity = _parity_tree(doc, [o.numpy() for o in outs], N)

    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base = cpu_baseline(size, 5)

    # learned speculation on the json.alp lexer, timed apart from the plain scan above
    spec_res = None
    if rank == 0 and world == 1 and not args.no_spec:
        del h_in, outs
        spec_res = spec_summary(args, local)

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    alg_bytes = size + NODE_BYTES * N
    # one mark per kernel, except "a+b" marks that cover two launches
    launches_per_step = sum(1 + k.count("+") for k, _ in kern)
    roof, path = _roofline(kern, dict(counts, n=size, N=N, one_doc=True), ms, alg_bytes)
    path["scope"] = "whole alp_parse call: %d input bytes + %d B per node, over the step time" % (size, NODE_BYTES)
    line = {
        "metric": METRIC,
        "value": _gbs(world, size, ms),
        "unit": "GB/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": max(3, args.warmup),
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u8",
        "data": "synthetic",
        "config": _config(size, _sha256(doc)),
        "details": {"nodes": N, "nodes_per_byte": N / size, "parallelism": "replicas (one document per GPU)",
                    "tokens": counts["m"], "positions": counts["L"], "brackets": counts["B"],
                    "brackets_searched": counts["K"],
                    "tuning": {"config": tuning["config"], "tile_shape": list(tuning["tile_shape"]),
                               "candidates_ms": [[k, v, round(t, 4)] for k, v, t in tuning["timings"]]}},
        "roofline": roof,
        "path_roofline": path,
        "e2e": {"value": _gbs(world, size, ms_e2e), "unit": "GB/s", "h2d_bytes_per_step": moved["h2d"],
                "d2h_bytes_per_step": moved["d2h"], "ms_per_step": ms_e2e, "pcie": pcie, "two_contexts": two,
                "d2h_form": "i32 parents and spans (sign-extended into the caller's i64 arrays on the host "
                            "while later chunks are in flight), u32 tags, u8 kinds"},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clk.summary(),
    }
    if base:
        line["cpu_baseline"] = base
    if parity:
        line["parity"] = parity
    if spec_res:
        line["spec"] = spec_res
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
