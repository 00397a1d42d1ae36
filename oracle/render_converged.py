"""Renders the oracle's converged image of a benchmark workload: test and
measurement infrastructure only (the checker, never the product).

    python oracle/render_converged.py [--workload rings_1080p] [--spp 4096] [--threads N] [--f64]

The image is the running mean of `spp` samples with noise keys from
NOISE_SEED on (disjoint from the keys any timed or tested render uses), saved
as float32 (height*width, 4) to oracle/_cache/<workload>_<spp>spp.npy with a
JSON note beside it; with --f64 the oracle's f64 build (liboracle_f64.so)
renders it, to <workload>_<spp>spp_f64.npy. The render resumes from the last completed 64-sample
dispatch if interrupted. bench.py reads the file, when present, to report
the relative RMSE of the CUDA image against the oracle's converged image
(the metric's "to 1% RMSE vs oracle").
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

CACHE = Path(__file__).resolve().parent / "_cache"
NOISE_SEED = 0x40000000


def cache_path(workload: str, spp: int, f64: bool = False) -> Path:
    return CACHE / f"{workload}_{spp}spp{'_f64' if f64 else ''}.npy"


def render(workload: str, spp: int, threads: int, f64: bool = False) -> Path:
    from oracle.binding import OracleTracer
    from stargaze_b200 import abi
    from stargaze_b200.workloads import WORKLOADS, render_options, upload_workload

    wl = WORKLOADS[workload]()
    out = cache_path(workload, spp, f64)
    partial = out.with_suffix(".partial.npz")
    CACHE.mkdir(exist_ok=True)
    t = OracleTracer((wl.width, wl.height), render_options(wl, spp=abi.MAX_BATCH_SAMPLES, noise_seed=NOISE_SEED),
                     threads=threads, f64=f64)
    upload_workload(t, wl)
    if partial.exists():
        z = np.load(partial)
        t.prepare_frame(wl.frame)  # the history key of the frame; then restore
        t.acc[:] = z["acc"]
        t.samples_ = int(z["samples"])
        t.sequence_ = int(z["samples"])
    start = time.perf_counter()
    while t.samples() < spp:
        t.encode(wl.frame)
        np.savez(partial, acc=t.acc, samples=t.samples())
        done = t.samples()
        print(f"{workload}: {done}/{spp} spp, {time.perf_counter() - start:.0f} s", flush=True)
    np.save(out, t.read_pixels())
    out.with_suffix(".json").write_text(json.dumps({
        "workload": workload, "width": wl.width, "height": wl.height, "spp": spp, "noise_seed": NOISE_SEED,
        "renderer": f"oracle (oracle/oracle.c, {'f64' if f64 else 'f32'}, -ffp-contract=off)",
        "seconds": time.perf_counter() - start,
    }) + "\n")
    partial.unlink(missing_ok=True)
    return out


def main():
    p = argparse.ArgumentParser(description=__doc__)
    p.add_argument("--workload", default="rings_1080p")
    p.add_argument("--spp", type=int, default=4096)
    p.add_argument("--threads", type=int, default=0)
    p.add_argument("--f64", action="store_true", help="render with the oracle's f64 build")
    a = p.parse_args()
    print(render(a.workload, a.spp, a.threads, a.f64))


if __name__ == "__main__":
    main()
