#!/usr/bin/env python
"""Throughput of the lex + LLP-parse path on B200.

Workload (default): one 256 MiB JSON document (grammar ``grammars/json_ext.alp``:
the reference JSON productions with full JSON lexical rules, lookback 1,
lookahead 3, 16-bit token lengths, 32-bit indices), seeded synthetic data.

A step is one pass of the whole path over the document: lexing, pair
expansion, bracket matching, parents, compaction. ``value`` is input GB/s with
the input resident in device memory (CUDA events on the library's stream
around K steps, max over ranks); ``e2e`` is the same through the public host
API: pinned host input -> device -> host result arrays, every step.

``--impl reference`` times the reference's own C backend (oracle/_ref, built
from alpacc's backends/c sources) on the host cores instead: one independent
document per core.

Multi-GPU: replicas only (each rank parses its own document; no collective on
the data path); ``scaling`` is "weak".
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "input GB/s lex+parse at 1 B200 (% HBM peak); serve p99 ms vs per-input launch"
GRAMMAR = os.path.join(REPO, "grammars", "json_ext.alp")
REF_CONFIG = "json_ext_i32"

# Workloads (the default is the headline one). Each: grammar, index width,
# reference configuration, default size, document generator (n, seed), and
# whether the document is meant to be rejected.
WORKLOADS = {
    "json": dict(grammar="json_ext.alp", index32=True, ref="json_ext_i32", size=256 << 20, reject=False,
                 desc="json_ext %d MiB single JSON document per GPU"),
    "sexp": dict(grammar="sexp.alp", index32=False, ref="sexp_i64", size=1 << 30, reject=False,
                 desc="sexp %d MiB single s-expression document per GPU (nesting up to 10000)"),
    "sexp_unbalanced": dict(grammar="sexp.alp", index32=False, ref="sexp_i64", size=1 << 30, reject=True,
                            desc="sexp %d MiB document with 5%% of forms carrying an extra ')' (rejected)"),
    "batch": dict(grammar="json_ext.alp", index32=True, ref="json_ext_i32", size=0, reject=False,
                  desc="4096 JSON documents, log-normal lengths (median 8 KiB, 200 B to 4 MiB; %d MiB)"),
    "serve": dict(grammar="json_ext.alp", index32=True, ref="json_ext_i32", size=0, reject=False,
                  desc="serving trace of JSON requests, Poisson arrivals, log-normal sizes (median 16 KiB, "
                       "64 B to 16 MiB; %d MiB)"),
}

SERVE_RATES = (2000, 5000, 10000, 20000, 50000, 100000)


def _pct(x, q):
    import numpy as np
    return float(np.percentile(np.asarray(x), q)) if len(x) else None


def ours_serve(a, rank, world, local_rank, dist):
    """The served form: per arrival rate, a seeded Poisson trace of at least
    --serve-seconds of JSON requests (drawn from a pool of seeded documents
    with log-normal sizes) replayed in real time from a native client thread
    against alpacc_server (continuous batching, 8 GiB scratch budget), and the
    same trace as one plain alpacc_gpu_parse per request in arrival order;
    p50/p99 latency (scheduled arrival to result) and GB/s per rate."""
    import numpy as np
    import torch

    from alpacc_b200 import workloads as W
    from alpacc_b200.grammar.cache import load_tables
    from alpacc_b200.native import Parser, Server

    torch.cuda.set_device(local_rank)
    wl = WORKLOADS["serve"]
    tables = load_tables(os.path.join(REPO, "grammars", wl["grammar"]), index32=True)
    pool, offs = W.json_batch(a.serve_pool, 16384, 64, 16 << 20, 5 + rank)
    offs = np.asarray(offs, dtype=np.int64)
    sizes = np.diff(offs)
    srv = Server(tables, device=local_rank, workers=2, budget=8 << 30)
    plain = Parser(tables, device=local_rank, max_input=int(sizes.max()))
    # warm-up: every pool document once through both arms (grows their scratch
    # to the largest batch and document before anything is timed)
    warm = np.arange(len(sizes), dtype=np.uint32)
    srv.replay(pool, offs, warm, np.zeros(len(warm)))
    plain.replay(pool, offs, warm, np.zeros(len(warm)))
    rates = [int(r) for r in a.serve_rates.split(",")]
    sweep = []
    total_req = 0
    clocks = ClockSampler(local_rank)
    clocks.start()
    for rate in rates:
        rng = np.random.default_rng(1000 + rate)
        count = max(int(rate * a.serve_seconds), 1000)
        gaps = rng.exponential(1.0 / rate, count)
        arr = np.cumsum(gaps) - gaps[0]
        doc = rng.integers(0, len(sizes), count).astype(np.uint32)
        nbytes = float(sizes[doc].sum())
        lat, st, el = srv.replay(pool, offs, doc, arr)
        plat, pst, pel = plain.replay(pool, offs, doc, arr)
        if (st != 0).any() or (pst != 0).any():
            raise SystemExit("serve: %d served and %d plain requests did not parse" % ((st != 0).sum(), (pst != 0).sum()))
        total_req += count
        sweep.append({"rate_per_s": rate, "requests": count, "arrival_s": float(arr[-1]), "bytes": int(nbytes),
                      "p50_ms": _pct(lat, 50), "p99_ms": _pct(lat, 99), "gbs": nbytes / el / 1e9,
                      "plain_p50_ms": _pct(plat, 50), "plain_p99_ms": _pct(plat, 99), "plain_gbs": nbytes / pel / 1e9})
    clk = clocks.stop()
    stt = srv.stats()
    srv.close()
    if rank != 0:
        return
    top = sweep[-1]
    line = {
        "metric": METRIC, "value": top["gbs"], "unit": "GB/s", "n_gpus": world, "steps": len(rates),
        "warmup": len(warm), "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u8", "data": "synthetic (seeded JSON request pool, seeded Poisson arrivals)",
        "config": dict(workload_config(int(sizes.sum()), world, "serve"), pool=len(sizes), requests=total_req,
                       seconds_per_rate=a.serve_seconds, workers=2, scratch_budget_gib=8,
                       batches=stt["batches"], largest_batch=stt["largest_batch"],
                       max_scratch_held=stt["max_scratch_held"], scratch_share=stt["scratch_share"]),
        "serve": sweep,
        "p99_ms_at_max_rate": top["p99_ms"], "plain_p99_ms_at_max_rate": top["plain_p99_ms"],
        "served_over_plain_at_max_rate": top["gbs"] / top["plain_gbs"],
        "clocks": clk,
        "e2e": {"value": top["gbs"], "unit": "GB/s", "h2d_bytes_per_step": top["bytes"], "d2h_bytes_per_step": None,
                "note": "requests arrive as host buffers and results return to host memory"},
    }
    print(json.dumps(line))


def ours_batch(a, rank, world, local_rank, dist):
    """The batched form: 4096 documents per step through alpacc_gpu_parse_batch
    (host buffers in and out, one launch per stage), against one plain
    alpacc_gpu_parse per document."""
    import numpy as np
    import torch

    from alpacc_b200 import workloads as W
    from alpacc_b200.grammar.cache import load_tables
    from alpacc_b200.native import Parser, Result

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    wl = WORKLOADS["batch"]
    buf, offs = W.json_batch(count=4096, median=8192, lo=200, hi=4 << 20, seed=4 + rank)
    total = len(buf)
    tables = load_tables(os.path.join(REPO, "grammars", wl["grammar"]), index32=True)
    parser = Parser(tables, device=local_rank, max_input=total)
    pin = torch.empty(total, dtype=torch.uint8, pin_memory=True)
    pin.numpy()[:] = np.frombuffer(buf, dtype=np.uint8)
    offs = np.ascontiguousarray(offs, dtype=np.int64)
    d_all = pin.to(dev)
    parser.autotune(d_all.data_ptr(), total)  # launch geometry for this grammar
    ext = torch.cuda.ExternalStream(parser.stream_handle(), device=dev)
    count = len(offs) - 1

    def batched():
        outs = parser.parse_batch_raw(pin.data_ptr(), offs.ctypes.data, count)
        ok = sum(outs[i].valid for i in range(count))
        for i in range(count):
            Parser.free_result(outs[i])
        return ok

    for _ in range(a.warmup):
        accepted = batched()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    for _ in range(a.steps):
        batched()
    e1.record(ext)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = max_over_ranks(dist, e0.elapsed_time(e1), dev)
    value = job_throughput(world, total, a.steps, ms)
    # one plain call per document (the same host buffers)
    for i in range(min(64, count)):
        rc, r = parser.parse_raw(pin.data_ptr() + int(offs[i]), int(offs[i + 1] - offs[i]))
        Parser.free_result(r)
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(ext)
    for i in range(count):
        rc, r = parser.parse_raw(pin.data_ptr() + int(offs[i]), int(offs[i + 1] - offs[i]))
        Parser.free_result(r)
    f1.record(ext)
    torch.cuda.synchronize()
    per_ms = max_over_ranks(dist, f0.elapsed_time(f1), dev)
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u8", "data": "synthetic (seeded JSON generator, log-normal lengths)",
        "config": dict(workload_config(total, world, "batch"), documents=count, accepted=int(accepted),
                       geometry=parser.geometry()),
        "per_input": {"value": job_throughput(world, total, 1, per_ms), "unit": "GB/s", "ms": per_ms,
                      "what": "one alpacc_gpu_parse per document, same host buffers"},
        "speedup_vs_per_input": (job_throughput(world, total, a.steps, ms) / job_throughput(world, total, 1, per_ms)),
        "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": total, "d2h_bytes_per_step": None,
                "note": "the batch entry point takes and returns host buffers: value is end to end"},
        "gpu_launches": parser.counts()["launches"] * a.steps,
        "clocks": clk,
    }
    if not a.no_cpu_baseline:
        from oracle.ref import RefOracle, available
        if available(wl["ref"]):
            ref = RefOracle(wl["ref"])
            t0 = time.perf_counter()
            for i in range(count):
                ref.pipeline(np.frombuffer(buf[offs[i]:offs[i + 1]], dtype=np.uint8))
            t = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": total / t / 1e9, "unit": "GB/s", "cores": 1, "kind": "reference",
                                    "sample": "all %d documents once, reference C backend in memory (%.2fs)"
                                              % (count, t)}
    print(json.dumps(line))


def make_doc(workload, n, seed):
    from alpacc_b200 import workloads as W
    if workload in ("json", "batch", "serve"):
        return W.json_doc(n, seed)
    return W.sexp_doc(n, seed + 1, unbalanced_frac=0.05 if workload == "sexp_unbalanced" else 0.0, max_depth=10000)


def peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = os.path.join("/tmp", "alpacc_clocks_%d_%d.csv" % (os.getpid(), device))

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        # the timed region is short: start it only once sampling is running
        t0 = time.time()
        while time.time() - t0 < 10 and self.proc.poll() is None and os.path.getsize(self.path) == 0:
            time.sleep(0.02)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.06)  # one more sample at the end of the region
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        os.remove(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def algorithmic_bytes(n, T, N, lay):
    """bytes(n) of the whole path: input once plus the compulsory outputs."""
    return n + T * (lay.terminal + lay.index + lay.length) + N * (lay.production + lay.index) + T * lay.index


def kernel_bytes(stage, n, T, B, P, N, lay):
    """Algorithmic bytes of one launch of each kernel: its compulsory inputs
    and outputs (brackets and productions are u32 on the device)."""
    if stage == "lex":
        return n + T * (lay.terminal + lay.index + lay.length)
    if stage == "pairs":
        return T * lay.terminal + 4 * (B + P)
    if stage == "bracket_walk":
        return 4 * B
    if stage == "parent_walk":
        return 4 * P + N * (lay.production + lay.index) + T * lay.index
    return 0


def cpu_baseline_sample(host: bytes, n_sample: int, ref_config: str = REF_CONFIG, workload: str = "json",
                        reps: int = 4):
    """The reference C backend, single thread (it is sequential), on the timed
    document itself when n_sample >= its size, otherwise on a seeded document
    of n_sample bytes from the same generator."""
    from oracle.ref import RefOracle, available
    import numpy as np

    if not available(ref_config):
        return None
    if n_sample >= len(host):
        doc = np.frombuffer(host, dtype=np.uint8)
        what = "the timed %d MiB document itself" % (len(host) >> 20)
    else:
        doc = np.frombuffer(make_doc(workload, n_sample, 2), dtype=np.uint8)
        what = "one %d MiB document of the same generator (seed 2)" % (n_sample >> 20)
    ref = RefOracle(ref_config)
    ref.pipeline(doc[: 1 << 20])  # warm
    times = []
    ok = None
    for _ in range(reps):
        t0 = time.perf_counter()
        ok = ref.pipeline(doc)
        times.append(time.perf_counter() - t0)
    t = statistics.median(times)
    return {"value": len(doc) / t / 1e9, "unit": "GB/s", "cores": 1, "kind": "reference",
            "sample": "%s, lex_string -> parse_test -> compute_parents -> compact_tree in memory, median of %d "
                      "runs (%.2fs each, %.1fs of CPU work), accepted=%s" % (what, reps, t, sum(times), ok[0])}


def max_over_ranks(dist, ms, device=None):
    """The largest of every rank's value: the job takes as long as its slowest rank."""
    if not dist:
        return ms
    import torch

    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world, n, steps, ms_total):
    """Whole-job input GB/s: each of `world` ranks parsed its own n-byte document per step."""
    return world * n * steps / (ms_total / 1e3) / 1e9


def workload_config(n, world, workload="json"):
    wl = WORKLOADS[workload]
    return {"workload": wl["desc"] % (n >> 20), "grammar": wl["grammar"], "bytes": n,
            "index": "i32" if wl["index32"] else "i64", "parallelism": "replicas x%d" % world,
            "l2": "input larger than L2 (no flush)"}


def reference_arm(a, rank, world):
    if rank != 0:
        return
    import multiprocessing as mp

    from oracle.ref import available

    wl = WORKLOADS[a.workload]
    if not available(wl["ref"]):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/lib%s.so is not built" % wl["ref"]}))
        return
    cores = os.cpu_count() or 1
    sample = a.ref_sample
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores, initializer=_pool_init, initargs=(sample, a.workload)) as pool:
        pool.map(_pool_step, range(cores))  # load
        for _ in range(a.warmup):
            pool.map(_pool_step, range(cores))
        t0 = time.perf_counter()
        oks = []
        for _ in range(a.steps):
            oks.extend(pool.map(_pool_step, range(cores)))
        t = time.perf_counter() - t0
    value = a.steps * cores * sample / t / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": 0, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": t / a.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": dict(workload_config(a.size or wl["size"], a.gpus, a.workload),
                       sample="each step: %d independent %d MiB documents of the same generator, one per host "
                              "core (the reference backend parses one document on one thread)" % (cores, sample >> 20)),
        "cpu_baseline": {"value": value, "unit": "GB/s", "cores": cores, "kind": "reference",
                         "sample": "%d independent %d MiB JSON documents per step (one per core), reference C "
                                   "backend in memory; all accepted=%s" % (cores, sample >> 20, all(oks))},
        "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


_POOL = {}


def _pool_init(sample, workload="json"):
    from oracle.ref import RefOracle
    import numpy as np

    pid = os.getpid()
    _POOL["doc"] = np.frombuffer(make_doc(workload, sample, 2 + (pid % 97)), dtype=np.uint8)
    _POOL["ref"] = RefOracle(WORKLOADS[workload]["ref"])


def _pool_step(_):
    return _POOL["ref"].pipeline(_POOL["doc"])[0]


def ours(a, rank, world, local_rank, dist):
    import numpy as np
    import torch

    from alpacc_b200 import wire, workloads as W
    from alpacc_b200.grammar.cache import load_tables
    from alpacc_b200.native import Parser

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    wl = WORKLOADS[a.workload]
    n = a.size if a.size else wl["size"]
    tables = load_tables(os.path.join(REPO, "grammars", wl["grammar"]), index32=wl["index32"])
    lay = wire.Layout.of(tables)
    host = make_doc(a.workload, n, 2 + rank)
    parser = Parser(tables, device=local_rank, max_input=n)
    d_in = torch.frombuffer(bytearray(host), dtype=torch.uint8).to(dev)
    ext = torch.cuda.ExternalStream(parser.stream_handle(), device=dev)
    stages = {k: [] for k in Parser.STAGES}

    def step():
        rc, r = parser.parse_device(d_in.data_ptr(), n)
        return rc, r

    if not a.no_autotune:  # launch geometry for this grammar, tuned on the document (outside the timed region)
        parser.autotune(d_in.data_ptr(), n)
    parser.set_stage_timing(True)  # per-stage device times for the line's stage_ms and roofline
    for _ in range(a.warmup):
        rc, r = step()
    if rc != (1 if wl["reject"] else 0):
        raise SystemExit("warm-up parse returned status %d on the %s workload" % (rc, a.workload))
    T, N = r.num_tokens, r.num_nodes
    info = parser.info()
    # ---- device-resident timing ----
    clocks = ClockSampler(local_rank)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    for _ in range(a.steps):
        rc, r = step()
        for k, v in parser.stage_ms().items():
            stages[k].append(v)
    e1.record(ext)
    torch.cuda.synchronize()
    ms_total = e0.elapsed_time(e1)
    clk = clocks.stop()
    launches_per_call = parser.counts()["launches"]  # kernels the library launched in one timed step
    ms_total = max_over_ranks(dist, ms_total, dev)
    ms_step = ms_total / a.steps
    value = job_throughput(world, n, a.steps, ms_total)

    # ---- end to end: pinned host input, host results ----
    pin = torch.empty(n, dtype=torch.uint8, pin_memory=True)
    pin.numpy()[:] = np.frombuffer(host, dtype=np.uint8)
    for _ in range(max(1, a.warmup)):
        rc2, r2 = parser.parse_raw(pin.data_ptr(), n)
        Parser.free_result(r2)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(ext)
    for _ in range(a.steps):
        rc2, r2 = parser.parse_raw(pin.data_ptr(), n)
        Parser.free_result(r2)
    f1.record(ext)
    torch.cuda.synchronize()
    e2e_ms = f0.elapsed_time(f1)
    e2e_ms = max_over_ranks(dist, e2e_ms, dev)
    e2e = job_throughput(world, n, a.steps, e2e_ms)
    d2h = T * (lay.terminal + lay.index + lay.length) + N * (lay.production + lay.index) + T * lay.index

    if rank != 0:
        return
    peak, peak_kind = peaks()
    mean = {k: (sum(v) / len(v) if v else 0.0) for k, v in stages.items()}
    dom = max(mean, key=lambda k: mean[k])
    st = parser.counts()
    B, P = st.get("B", 0), st.get("P", 0)
    kb = kernel_bytes(dom, n, T, B, P, N, lay)
    achieved = kb / (mean[dom] / 1e3) / 1e9 if mean[dom] > 0 else 0.0
    path_bytes = algorithmic_bytes(n, T, N, lay)
    traffic = committed_traffic(a.workload, dom, n)
    line = {
        "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded JSON generator, one document per rank)",
        "config": dict(workload_config(n, world, a.workload), tokens=T, nodes=N, brackets=B, productions=P,
                       geometry=parser.geometry()),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                     "algorithmic_bytes": kb, "ms": mean[dom]},
        "path_roofline": {"algorithmic_bytes": path_bytes, "achieved": path_bytes / (ms_step / 1e3) / 1e9,
                          "frac": path_bytes / (ms_step / 1e3) / 1e9 / peak},
        "stage_ms": mean,
        "e2e": {"value": e2e, "unit": "GB/s", "h2d_bytes_per_step": n, "d2h_bytes_per_step": d2h,
                "ms_per_step": e2e_ms / a.steps},
        "gpu_launches": launches_per_call * a.steps,
        "clocks": clk,
        "machine": info,
    }
    if not a.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sample(host, a.cpu_sample, wl["ref"], a.workload,
                                                   reps=2 if n > (512 << 20) else 4)
    line["parity"] = record_parity(parser, pin, host, wl["ref"]) if not a.no_parity else None
    print(json.dumps(line))
    if line["parity"] and line["parity"]["match"] is False:
        raise SystemExit("parity failure: the GPU record of the timed document differs from oracle/_ref's")


def record_parity(parser, pin, host: bytes, ref_config: str):
    """Outside the timed region: the SHA-256 of the response record the GPU
    path returns for the timed document (through alpacc_gpu_parse, host
    buffers) against the record the reference's own C backend (oracle/_ref)
    writes for the same bytes."""
    import numpy as np

    from oracle.ref import RefOracle, available

    rc, got, got_size = parser.record_digest_raw(pin.data_ptr(), len(host))
    if not available(ref_config):
        return {"oracle": None, "match": None, "note": "oracle/_ref/lib%s.so is not built" % ref_config}
    t0 = time.perf_counter()
    want, want_size = RefOracle(ref_config).record_digest(np.frombuffer(host, dtype=np.uint8))
    return {"oracle": "oracle/_ref/lib%s.so" % ref_config, "what": "sha256 of the run_case response record",
            "record_bytes": got_size, "valid": rc == 0, "sha256": got[:16], "match": got == want and got_size == want_size,
            "oracle_s": round(time.perf_counter() - t0, 2)}


def committed_traffic(workload: str, kernel: str, n: int):
    """DRAM bytes per launch of `kernel` from the committed ncu summary of the
    same workload family (profiles/traffic.json: bytes of one captured launch
    and the input size it processed), scaled to n bytes of input; None when
    there is no capture for it."""
    p = os.path.join(REPO, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    fam = "sexp" if workload.startswith("sexp") else "json"
    v = d.get(fam, {}).get(kernel)
    if not isinstance(v, dict) or not v.get("input_bytes"):
        return None
    return int(v["bytes_per_launch"] * n / v["input_bytes"])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=0, help="input bytes (default: the workload's size)")
    ap.add_argument("--workload", default="json", choices=sorted(WORKLOADS))
    ap.add_argument("--serve-pool", type=int, default=2048, help="documents in the serve request pool")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch geometry")
    ap.add_argument("--serve-seconds", type=float, default=2.0, help="seconds of arrivals per rate")
    ap.add_argument("--serve-rates", default=",".join(str(r) for r in SERVE_RATES))
    ap.add_argument("--cpu-sample", type=int, default=256 << 20)
    ap.add_argument("--ref-sample", type=int, default=16 << 20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="skip the record comparison with oracle/_ref")
    a = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist

        if a.impl == "ours":
            torch.cuda.set_device(local_rank)
            tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
            dist = tdist
    if a.impl == "reference":
        reference_arm(a, rank, world)
    elif a.workload == "batch":
        ours_batch(a, rank, world, local_rank, dist)
    elif a.workload == "serve":
        ours_serve(a, rank, world, local_rank, dist)
    else:
        ours(a, rank, world, local_rank, dist)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
