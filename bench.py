#!/usr/bin/env python3
"""Benchmark: bit-exact lex+parse of synthetic JSON on B200.

Workload (one step): the full json.alp lex+parse (bytes -> preorder tree
with parents, tags, kinds and spans) of one 256 MiB synthetic JSON document
of nesting depth <= 16, through the C ABI (``alp_parse``).  Inputs are larger
than L2, so no flush is needed between steps.

* ``value``   -- input GB/s with the document resident in HBM (device-timed
                 with CUDA events around the ``alp_parse`` calls).
* ``e2e``     -- the same through ``alp_parse_host``: pinned host bytes in,
                 the whole tree back to pinned host memory, copies inside
                 the timed region.
* ``roofline``-- algorithmic bytes (input + 29 B per output node: i64 parent,
                 u32 tag, u8 kind, i64 start, i64 end) over the step time,
                 against the measured HBM copy bandwidth; plus a per-kernel
                 breakdown from one instrumented step.
* ``cpu_baseline`` -- the CPU oracle (sequential C restatement of the
                 reference's generated lexer and parser) on a bounded sample of
                 the same generator, rank 0 only.

``--impl reference`` times that CPU restatement alone (the reference's own
Futhark/Haskell toolchain is not available) on the same workload shape.
Under torchrun each rank parses its own document (weak scaling, replicas,
no data-path collective); the step time is the max over ranks.
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
SEED = 0xA1FACC00 + 2
METRIC = "input GB/s lex+parse (json.alp, plain scan, bit-exact)"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


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


def cpu_baseline(sample_bytes: int, reps: int):
    """Sequential oracle (lex_int then parse_int restated in C) on a sample."""
    import oracle
    from alpacc_b200 import tables
    tb = tables.load("json", "both")
    o = oracle.Oracle(tb.blob())
    d = make_doc(SEED + 7, sample_bytes).tobytes()
    o.lex_parse(d)  # warm-up
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        r = o.lex_parse(d)
        ts.append(time.perf_counter() - t0)
        assert r is not None
    t = statistics.median(ts)
    return {"value": sample_bytes / t / 1e9, "unit": "GB/s", "cores": 1, "kind": "port",
            "sample": "%d MiB json.alp document (same generator, depth %d), lex+parse, median of %d, 1 thread"
                      % (sample_bytes >> 20, DEPTH, reps)}


def run_reference(args, rank: int, world: int):
    if rank != 0:
        return
    sample = 32 << 20
    import oracle
    from alpacc_b200 import tables
    tb = tables.load("json", "both")
    o = oracle.Oracle(tb.blob())
    d = make_doc(SEED + 7, sample).tobytes()
    for _ in range(args.warmup):
        o.lex_parse(d)
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        r = o.lex_parse(d)
        ts.append(time.perf_counter() - t0)
        assert r is not None
    step = sum(ts) / len(ts)
    v = sample / step / 1e9
    line = {"metric": METRIC, "value": v, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8", "data": "synthetic", "impl": "reference",
            "config": {"workload": "json.alp lex+parse, 256 MiB-document generator (depth <= 16); the CPU "
                                   "restatement runs a 32 MiB sample of it per step",
                       "doc_bytes": sample},
            "cpu_baseline": {"value": v, "unit": "GB/s", "cores": 1, "kind": "port",
                             "sample": "32 MiB json.alp document per step, 1 thread (the restatement is "
                                       "sequential; the reference's Futhark multicore build needs GHC and "
                                       "futhark, absent here)"},
            "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--doc-mib", type=int, default=DOC_BYTES >> 20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    from alpacc_b200 import api, tables

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
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
    ms = ev0.elapsed_time(ev1) / args.steps
    if dist:
        t = torch.tensor([ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()

    # per-kernel breakdown from one instrumented step (outside the timed region)
    g.profile(True)
    step()
    kern = g.timings()
    g.profile(False)

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
    ms_e2e = e0.elapsed_time(e1) / k_e2e
    if dist:
        t = torch.tensor([ms_e2e], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())

    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base = cpu_baseline(64 << 20, 2)

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    peak, peak_kind = _peaks()
    alg_bytes = size + NODE_BYTES * N
    achieved = alg_bytes / (ms * 1e-3) / 1e9
    total_k = sum(t for _, t in kern) or 1.0
    # one mark per kernel, except "a+b" marks that cover two launches
    launches_per_step = sum(1 + k.count("+") for k, _ in kern)
    top = max(kern, key=lambda x: x[1]) if kern else ("", 0.0)
    line = {
        "metric": METRIC,
        "value": world * size / (ms * 1e-3) / 1e9,
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
        "config": {"workload": "json.alp full lex+parse, one %d MiB synthetic JSON document per GPU "
                               "(depth <= %d), bytes -> preorder tree" % (args.doc_mib, DEPTH),
                   "doc_bytes": size, "nodes": N, "nodes_per_byte": N / size, "parallelism": "replicas",
                   "l2": "inputs larger than L2 (no flush needed)"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": None,
                     "scope": "whole alp_parse call: %d input bytes + %d B per node, over the step time"
                              % (size, NODE_BYTES),
                     "dominant_kernel": top[0], "dominant_kernel_ms": top[1],
                     "kernels_ms": {k: round(t, 4) for k, t in kern},
                     "kernel_share": {k: round(t / total_k, 4) for k, t in kern}},
        "e2e": {"value": world * size / (ms_e2e * 1e-3) / 1e9, "unit": "GB/s", "h2d_bytes_per_step": size,
                "d2h_bytes_per_step": NODE_BYTES * N, "ms_per_step": ms_e2e},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clk.summary(),
    }
    if base:
        line["cpu_baseline"] = base
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
