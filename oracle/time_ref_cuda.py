"""Times the reference's own CUDA backend on this GPU (a baseline, not the product).

MEASUREMENT INFRASTRUCTURE ONLY. Runs the program ``oracle/build_ref_cuda.py``
assembles (``oracle/_ref/cuda_<config>``: the reference's CUDA templates
around restated constants, compiled for sm_100a) in its own benchmark mode
``--benchmark N --warmup W`` (backends/cuda/cli.cu:877-1060) on the same
seeded document the bench times, framed as its benchmark input expects (u64
count, then per test u64 frame length, u64 n, the bytes). That mode times the
lexer kernel, a device-to-device copy of the terminals and the fused
cooperative parser kernel (kernel-only), and the same plus the input and
result copies (+io), with CUDA events, and prints the mean time and GB/s of
each to stderr. This script samples the SM clocks while it runs and prints one
JSON line with both figures.

Usage: python oracle/time_ref_cuda.py [--config json_ext_i32] [--size BYTES] [--runs 10] [--warmup 3]
"""

from __future__ import annotations

import argparse
import json
import os
import re
import struct
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, REPO)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="json_ext_i32")
    ap.add_argument("--size", type=int, default=256 << 20)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--runs", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    a = ap.parse_args(argv)
    exe = os.path.join(HERE, "_ref", "cuda_%s" % a.config)
    if not os.path.exists(exe):
        print(json.dumps({"impl": "reference-cuda", "unavailable": "%s is not built" % exe}))
        return 0
    from alpacc_b200 import workloads as W
    from bench import ClockSampler

    doc = W.json_doc(a.size, a.seed) if a.config.startswith("json") else W.sexp_doc(a.size, a.seed + 1)
    with tempfile.NamedTemporaryFile(suffix=".bin", delete=False) as f:
        f.write(struct.pack("<QQQ", 1, 8 + len(doc), len(doc)))
        f.write(doc)
        path = f.name
    clocks = ClockSampler(0)
    clocks.start()
    try:
        p = subprocess.run([exe, "--benchmark", str(a.runs), "--warmup", str(a.warmup), "-i", path],
                           capture_output=True, text=True, timeout=600)
    finally:
        clk = clocks.stop()
        os.remove(path)
    out = {"impl": "reference-cuda", "program": os.path.relpath(exe, REPO), "config": a.config, "bytes": len(doc),
           "runs": a.runs, "warmup": a.warmup, "rc": p.returncode, "clocks": clk}
    # "parse_int (cuda, N bytes):\n        XXXus (95% CI: [...]); YYGB/s"
    for label, key in (("cuda", "kernel_only"), ("cuda\\+io", "with_io")):
        m = re.search(r"parse_int \(%s, \d+ bytes\):\s*\n\s*([0-9.]+)\S*s .*?;\s*([0-9.]+)GB/s" % label, p.stderr)
        if m:
            us = float(m.group(1))
            out[key] = {"us": us, "input_gbs": len(doc) / (us * 1e-6) / 1e9, "printed_gbs": float(m.group(2))}
    out["stderr_tail"] = p.stderr[-600:]
    print(json.dumps(out))
    return 0 if p.returncode == 0 else p.returncode


if __name__ == "__main__":
    sys.exit(main())
