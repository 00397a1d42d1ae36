#!/usr/bin/env python
"""Benchmark of the progressive integrator (one JSON line on rank 0).

A step renders the ring workload (1920x1080, 256 spp: a ringed giant with a
512-bin optical-depth table, a binary star and a moon eclipse) from a fresh
accumulation: four 64-sample dispatches of the reference's encode contract,
through the wavefront integrator (the library default; `--integrator
megakernel` times the per-pixel megakernel instead).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value` is whole-job Msamples/s with the scene resident on the device
(CUDA events around each dispatch, L2 flushed between steps). `e2e` is the
same metric through the public API with the frame handed over from host
memory and the 33 MB accumulation read back to the host every step.
`--impl reference` times the CPU restatement of the reference integrator
(the oracle; the reference's own Rust/WGSL cannot run here) on the host.

After the timed region (one GPU only) further figures of the metric are
measured: `convergence`, the relative RMSE of the 256-spp image against the
oracle's 4096-spp image of the workload (oracle/render_converged.py, when
its cache is present) and against this integrator's own 4096-spp image, and
the samples (and time) each implies for 1 %; `adjoint`, the path-replay
adjoint's time against the forward's at equal spp on the ring scene
(512x512, 64 spp) and on the terrain scene (1920x1080, 256 spp, 1024^2
albedo map), and vertex checkpoints against replay on the latter; the C1
and C3 configurations with their own rooflines; the ring inverse problem.
The line ends with a summary of those figures.
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
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Msamples/s at 1080p to 1% RMSE vs oracle; adjoint/forward time ratio"
UNIT = "Msamples/s"
BATCH = 64

# Algorithmic work model: source-level FP32/INT operations per counted event
# of the integrator (add, mul, div, sqrt, compare, transcendental = 1 each),
# counted from the kernel source (stargaze_b200/csrc/sg_device.cuh,
# sg_kernels.cu). The kernel counts the events themselves.
OPS_PER_EVENT = {
    "vertices": 24,        # loop bookkeeping, closest-hit/ring selection, branch
    "sphere_tests": 40,    # relative_center, a, b, cross, |cross|^2, discriminant
    "sphere_hits": 17,     # sqrt, q, c, two divisions, root selection
    "ring_tests": 70,      # plane denominator, double cross, along, point, annulus
    "light_samples": 86,   # axis, cone width, stratum, sincos, basis, pdf
    "shadow_rays": 12,     # loop overhead of light_visibility
    "ring_events": 120,    # optics, transmission, slab BSDF, MIS, null/scatter
    "surface_events": 110, # normal, outgoing, albedo, cosine bounce, roulette
    "rng_draws": 10,       # LCG step + permutation + float conversion
    # Local landscape (sg_landscape.cuh): an interior quadtree node decodes
    # its Morton index (30) and slab-tests its four children (4 x 25 for
    # t_interval, 4 x 4 for the validity test, 10 for sort and push); a
    # terrain triangle is one Moller-Trumbore test (58) plus its share of the
    # cell's four vertex fetches (12); a group-marker box is one 3-slab
    # interval (27) plus the skip test (7); a primitive test is the
    # translation and rotation into its frame (18) plus the shape test,
    # weighted 5:2 ellipsoids (45) to rocks (150) as in the terrain scene.
    "terrain_nodes": 156,
    "terrain_triangles": 70,
    "prop_boxes": 34,
    "prop_tests": 93,
}
EVENT_ORDER = ["vertices", "sphere_tests", "sphere_hits", "ring_tests", "light_samples", "shadow_rays",
               "ring_events", "surface_events", "rng_draws", "terrain_nodes", "terrain_triangles", "prop_boxes",
               "prop_tests"]
# DRAM traffic of one 64-sample dispatch of the ring workload: an ncu
# capture of one steady-state iteration of the three stage kernels (4 Mi-path
# pool: 655 MB for 4.19 M path extensions) scaled to the dispatch's 183 M
# path extensions (1.38 per sample, counting kernel). Issue-slot fraction of
# the same capture, weighted by the stages' share of the step.
TRAFFIC_BYTES_PER_LAUNCH = 654.6e6 * (1.38 * 1920 * 1080 * 64) / 4.194e6
ISSUE_SLOT_FRACTION = 0.60
L2_FLUSH_BYTES = 256 << 20


def profile_terrain_640x360():
    """Terrain workload at 640x360, 64 spp: two frames (the first also runs
    the terrain-cache kernel)."""
    from stargaze_b200 import PathTracer, workloads as W

    wl, _land = W.terrain_1080p(640, 360, 64)
    t = PathTracer((wl.width, wl.height), W.render_options(wl, 64))
    W.upload_workload(t, wl)
    for r in range(2):
        frame = wl.frame.copy()
        frame.scene_time = float(r)
        t.encode(frame)
    t.read_pixels()


def profile_adjoint_ring_512():
    """Ring workload at 512x512: render 64 spp and run the adjoint, twice."""
    from stargaze_b200 import PathTracer, workloads as W

    wl = W.rings_1080p(512, 512, 64)
    t = PathTracer((wl.width, wl.height), W.render_options(wl, 64))
    W.upload_workload(t, wl)
    dl = np.random.default_rng(0).uniform(0.0, 1.0, (wl.width * wl.height, 4)).astype(np.float32)
    for r in range(2):
        frame = wl.frame.copy()
        frame.scene_time = float(r)
        t.prepare_frame(frame)
        t.encode(frame)
        t.backward(frame, t.tape(), dl)


def profile_adjoint_ring_512_small():
    """As adjoint_ring_512 with a 2 Mi-path pool (about 2.5 GB of path state
    and adjoint slots on the device, small enough for multi-pass captures)."""
    from stargaze_b200 import PathTracer, workloads as W

    wl = W.rings_1080p(512, 512, 64)
    t = PathTracer((wl.width, wl.height), W.render_options(wl, 64))
    W.upload_workload(t, wl)
    t.set_integrator("wavefront", 1 << 21)
    dl = np.random.default_rng(0).uniform(0.0, 1.0, (wl.width * wl.height, 4)).astype(np.float32)
    for r in range(2):
        frame = wl.frame.copy()
        frame.scene_time = float(r)
        t.prepare_frame(frame)
        t.encode(frame)
        t.backward(frame, t.tape(), dl)


def profile_wavefront_rings_1080p():
    """Ring workload at 1920x1080 through the wavefront integrator with a
    4 Mi-path pool (3.4 GB on the device, small enough for multi-pass
    captures): two 64-sample dispatches (the first allocates the pool)."""
    from stargaze_b200 import PathTracer, workloads as W

    wl = W.rings_1080p()
    t = PathTracer((wl.width, wl.height), W.render_options(wl, 64))
    W.upload_workload(t, wl)
    t.set_integrator("wavefront", 1 << 22)
    for r in range(2):
        frame = wl.frame.copy()
        frame.scene_time = float(r)
        t.prepare_frame(frame)
        t.encode(frame)
    t.read_pixels()
    print(t.integrator(), flush=True)


def profile_wavefront_terrain_640x360():
    """Terrain workload at 640x360, 64 spp, through the wavefront integrator
    with a 2 Mi-path pool (about 2 GB on the device with the terrain): two
    frames."""
    from stargaze_b200 import PathTracer, workloads as W

    wl, _land = W.terrain_1080p(640, 360, 64)
    t = PathTracer((wl.width, wl.height), W.render_options(wl, 64))
    W.upload_workload(t, wl)
    t.set_integrator("wavefront", 1 << 21)
    for r in range(2):
        frame = wl.frame.copy()
        frame.scene_time = float(r)
        t.encode(frame)
    t.read_pixels()
    print(t.integrator(), flush=True)


def profile_dispatch_rings_1080p():
    """The bench's own dispatch: ring workload at 1920x1080 with the default
    16 Mi-path pool, two 64-sample dispatches (the first allocates the pool
    and loads the kernels)."""
    from stargaze_b200 import PathTracer, workloads as W

    wl = W.rings_1080p()
    t = PathTracer((wl.width, wl.height), W.render_options(wl, 64))
    W.upload_workload(t, wl)
    for r in range(2):
        frame = wl.frame.copy()
        frame.scene_time = float(r)
        t.prepare_frame(frame)
        t.encode(frame)
    t.read_pixels()
    print(t.integrator(), flush=True)


PROFILE_CASES = {"terrain_640x360": profile_terrain_640x360, "adjoint_ring_512": profile_adjoint_ring_512,
                 "adjoint_ring_512_small": profile_adjoint_ring_512_small,
                 "dispatch_rings_1080p": profile_dispatch_rings_1080p,
                 "wavefront_rings_1080p": profile_wavefront_rings_1080p,
                 "wavefront_terrain_640x360": profile_wavefront_terrain_640x360}


def parse_args():
    p = argparse.ArgumentParser(description=__doc__)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", default="rings_1080p")
    p.add_argument("--integrator", choices=["wavefront", "megakernel"], default="wavefront")
    p.add_argument("--spp", type=int, default=256)
    p.add_argument("--cpu-seconds", type=float, default=12.0, help="bounded CPU-baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-extras", action="store_true", help="skip the convergence and adjoint figures")
    p.add_argument("--profile-case", choices=sorted(PROFILE_CASES),
                   help="run one small case for an ncu capture (profiles/) and exit")
    return p.parse_args()


def measured_hbm_gbs():
    """HBM copy bandwidth measured on this pool's B200s (GB/s), if known."""
    try:
        return float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["hbm_gbs"])
    except (OSError, ValueError, KeyError):
        return None


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            if self.thread is not None:
                self.thread.join(timeout=5)

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(wl, seconds: float, threads: int = 0) -> dict:
    """The oracle (CPU restatement of the reference integrator) on all host
    cores, over a bounded sample of the workload: whole frames of
    8-sample dispatches until `seconds` have elapsed."""
    from oracle.binding import OracleTracer
    from stargaze_b200.workloads import render_options as bench_options

    from stargaze_b200.workloads import upload_workload

    t = OracleTracer((wl.width, wl.height), bench_options(wl, spp=8), threads=threads)
    upload_workload(t, wl)
    rows_per_chunk = max(1, wl.height // 27)
    samples = 0
    start = time.perf_counter()
    y = 0
    frame = wl.frame
    while True:
        y1 = min(y + rows_per_chunk, wl.height)
        t.samples_ = 0
        t.key = None
        t.encode(frame, rows=(y, y1))
        samples += (y1 - y) * wl.width * 8
        y = 0 if y1 >= wl.height else y1
        if time.perf_counter() - start >= seconds:
            break
    elapsed = time.perf_counter() - start
    cores = threads if threads > 0 else (os.cpu_count() or 1)
    return {"value": samples / elapsed / 1e6, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{samples} samples ({wl.width}x{wl.height} frame, 8-sample dispatches, row bands) "
                      f"in {elapsed:.1f} s", "build": oracle_build_flags()}


# Replicas: rank r renders noise keys from RANK_KEY_STRIDE * r on, so ranks
# never share a sample while each renders fewer than RANK_KEY_STRIDE.
RANK_KEY_STRIDE = 1 << 26


def rank_noise_seed(rank: int) -> int:
    return (rank * RANK_KEY_STRIDE) & 0xFFFFFFFF


def max_over_ranks(values, dist, device) -> list[float]:
    """Element-wise maximum of per-rank timings (every rank gets it)."""
    import torch

    if dist is None:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def job_msamples_per_s(world: int, samples_per_step: int, steps: int, total_ms: float) -> float:
    """Whole-job throughput of `world` replicas, timed by the slowest rank."""
    return world * samples_per_step * steps / (total_ms * 1e-3) / 1e6


def relative_rmse(x: np.ndarray, reference: np.ndarray) -> float:
    """sqrt(sum (x - ref)^2 / sum ref^2) over rgb (scripts/benchmark.py:219-232)."""
    d = x[:, :3].astype(np.float64) - reference[:, :3].astype(np.float64)
    return float(np.sqrt((d * d).sum() / (reference[:, :3].astype(np.float64) ** 2).sum()))


CONVERGED_SPP = 4096
CONVERGED_NOISE_SEED = 0x40000000  # keys disjoint from every timed render's


def _to_1pct(err: float, spp: int, ref_spp: int, width: int, height: int, msamples_per_s: float) -> dict:
    """Samples per pixel (and time at `msamples_per_s`) for 1 % relative
    RMSE from the 1/sqrt(spp) law, after removing the reference image's own
    noise: with independent keys err^2 = e^2 (1 + spp / ref_spp)."""
    own = err / np.sqrt(1.0 + spp / ref_spp)
    spp_1pct = spp * (own / 0.01) ** 2
    return {"relative_rmse": err, "spp_to_1pct": spp_1pct,
            "ms_to_1pct": spp_1pct * width * height / (msamples_per_s * 1e6) * 1e3}


def convergence(wl, image: np.ndarray, spp: int, msamples_per_s: float, device: int, stream) -> dict:
    """Relative RMSE (scripts/benchmark.py:219-232) of the `spp`-sample
    image against the oracle's 4096-sample image of the workload (rendered
    once on the host by oracle/render_converged.py, disjoint noise keys) and
    against this integrator's own 4096-sample image, with the spp and time
    each implies for 1 %."""
    from stargaze_b200 import PathTracer
    from stargaze_b200.workloads import render_options, upload_workload

    out = {"spp": spp, "reference_spp": CONVERGED_SPP}
    cached = ROOT / "oracle" / "_cache" / f"{wl.name}_{CONVERGED_SPP}spp.npy"
    if cached.exists():
        oracle_image = np.load(cached)
        out["vs_oracle"] = _to_1pct(relative_rmse(image, oracle_image), spp, CONVERGED_SPP, wl.width, wl.height,
                                    msamples_per_s)
        out["reference"] = f"oracle at {CONVERGED_SPP} spp ({cached.name})"
    else:
        out["reference"] = f"oracle image missing: run oracle/render_converged.py --workload {wl.name}"
    t = PathTracer((wl.width, wl.height), render_options(wl, spp=BATCH, noise_seed=CONVERGED_NOISE_SEED),
                   device=device)
    upload_workload(t, wl)
    frame = wl.frame.copy()
    frame.scene_time = -12345.0
    for _ in range(CONVERGED_SPP // BATCH):
        t.encode(frame, stream)
    own_image = t.read_pixels(stream)
    t.close()
    out["vs_self"] = _to_1pct(relative_rmse(image, own_image), spp, CONVERGED_SPP, wl.width, wl.height,
                              msamples_per_s)
    if cached.exists():
        # Both references are converged estimates of the same image: their
        # distance bounds any bias between the CUDA path and the oracle.
        out["oracle_vs_self_relative_rmse"] = relative_rmse(own_image, oracle_image)
    # The oracle's f64 build at the same noise keys (the same paths, f64
    # arithmetic): the f32 image's distance from it, and the 1 % figures.
    cached_f64 = cached.with_name(f"{wl.name}_{CONVERGED_SPP}spp_f64.npy")
    if cached_f64.exists():
        oracle_f64 = np.load(cached_f64)
        out["vs_oracle_f64"] = _to_1pct(relative_rmse(image, oracle_f64), spp, CONVERGED_SPP, wl.width, wl.height,
                                        msamples_per_s)
        if cached.exists():
            out["oracle_f32_vs_f64_relative_rmse"] = relative_rmse(oracle_image, oracle_f64)
    return out


def timed_forward(t, wl, frame, stream) -> float:
    """Milliseconds (CUDA events on `stream`) to render `wl.spp` samples
    from a fresh accumulation of `frame`."""
    import torch

    t.prepare_frame(frame)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    while t.samples() < wl.spp:
        t.encode(frame, stream)
    b.record(stream)
    stream.synchronize()
    return a.elapsed_time(b)


def adjoint_ratio(wl, device: int, stream, reps: int = 3) -> dict:
    """Forward (spp samples from a fresh accumulation) and path-replay
    adjoint (sg_backward for a seeded d loss / d image) times, CUDA events on
    the launching stream, median over `reps`; the forward with both
    integrators, and both adjoints (staged and per-pixel) on the same tape."""
    import torch

    from stargaze_b200 import PathTracer
    from stargaze_b200.workloads import render_options, upload_workload

    t = PathTracer((wl.width, wl.height), render_options(wl, spp=BATCH), device=device)
    upload_workload(t, wl)
    dl = np.random.default_rng(0).uniform(0.0, 1.0, (wl.width * wl.height, 4)).astype(np.float32)
    fwd, mega, bwd, per_pixel = [], [], [], []
    for r in range(reps + 1):
        frame = wl.frame.copy()
        frame.scene_time = float(-1 - r)
        t.set_integrator("megakernel")
        m = timed_forward(t, wl, frame, stream)
        t.set_integrator("wavefront")
        frame.scene_time = float(-100 - r)
        f = timed_forward(t, wl, frame, stream)
        tape = t.tape()
        e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        e[0].record(stream)
        g = t.backward(frame, tape, dl, stream)  # staged adjoint
        e[1].record(stream)
        t.set_integrator("megakernel")
        e[2].record(stream)
        t.backward(frame, tape, dl, stream)  # per-pixel adjoint kernel
        e[3].record(stream)
        stream.synchronize()
        if r > 0:  # the first round loads the kernels
            fwd.append(f)
            mega.append(m)
            bwd.append(e[0].elapsed_time(e[1]))
            per_pixel.append(e[2].elapsed_time(e[3]))
    # With the forward storing each sample's radiance (sg_set_checkpoints
    # with every beyond the bounce limit: totals only, 16 B per sample),
    # samples whose ring-indirect cap does not bind replay once with every
    # weight known.
    t.set_integrator("wavefront")
    t.set_checkpoints(wl.max_bounces + 1, wl.spp)
    fwd_totals, bwd_totals = [], []
    for r in range(reps + 1):
        frame = wl.frame.copy()
        frame.scene_time = float(-200 - r)
        ft = timed_forward(t, wl, frame, stream)
        tape = t.tape()
        e = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        e[0].record(stream)
        t.backward(frame, tape, dl, stream)
        e[1].record(stream)
        stream.synchronize()
        if r > 0:
            fwd_totals.append(ft)
            bwd_totals.append(e[0].elapsed_time(e[1]))
    t.close()
    f, m, b = statistics.median(fwd), statistics.median(mega), statistics.median(bwd)
    ft, bt = statistics.median(fwd_totals), statistics.median(bwd_totals)
    params = int(sum(v.size for v in wl.ring_tables.values())) + 6 * len(wl.frame.bodies)
    if wl.landscape is not None and wl.landscape.albedo_map is not None:
        params += int(wl.landscape.albedo_map.size)
    return {"workload": wl.name, "width": wl.width, "height": wl.height, "spp": wl.spp, "forward_ms": f,
            "forward_megakernel_ms": m, "backward_ms": b, "backward_per_pixel_ms": statistics.median(per_pixel),
            "ratio": b / f, "forward_plus_adjoint_over_forward": (f + b) / f,
            "with_radiance_totals": {"forward_ms": ft, "backward_ms": bt,
                                     "forward_plus_adjoint_over_plain_forward": (ft + bt) / f},
            "parameters": params, "dropped_entries": int(g.dropped),
            "note": "forward: wavefront; backward: staged adjoint (per-pixel adjoint kernel beside it)"}


def count_ops(lib, wl, opts, frame, device: int, stream, batches: int):
    """Events of one step through the counting variant of the integrator
    (same image and noise keys), and the FP32/INT operations per dispatch
    they imply under OPS_PER_EVENT."""
    import ctypes as C

    from stargaze_b200 import PathTracer
    from stargaze_b200.workloads import upload_workload

    counter = PathTracer((wl.width, wl.height), opts, device=device)
    upload_workload(counter, wl)
    totals = np.zeros(len(EVENT_ORDER), np.uint64)
    ev = (C.c_uint64 * len(EVENT_ORDER))()
    for _ in range(batches):
        view = frame.view()
        status = lib.sg_encode_counted(counter.handle, C.byref(view), C.c_void_p(stream.cuda_stream), ev)
        assert status == 0, status
        totals += np.array(list(ev), np.uint64)
    counter.close()
    ops = float(sum(int(totals[k]) * OPS_PER_EVENT[n] for k, n in enumerate(EVENT_ORDER))) / batches
    return totals, ops


def config_entry(lib, wl, device: int, stream, peak: float, reps: int = 2) -> dict:
    """Another configuration's step (its spp from a fresh accumulation,
    64-sample dispatches, wavefront integrator) with its own roofline."""
    import torch

    from stargaze_b200 import PathTracer
    from stargaze_b200.workloads import render_options, upload_workload

    opts = render_options(wl, spp=BATCH)
    batches = (wl.spp + BATCH - 1) // BATCH
    t = PathTracer((wl.width, wl.height), opts, device=device)
    upload_workload(t, wl)
    times, dispatch_ms = [], []
    for r in range(reps + 1):
        frame = wl.frame.copy()
        frame.scene_time = float(-900 - r)
        t.prepare_frame(frame)
        marks = [torch.cuda.Event(enable_timing=True) for _ in range(batches + 1)]
        marks[0].record(stream)
        for b in range(batches):
            t.encode(frame, stream)
            marks[b + 1].record(stream)
        stream.synchronize()
        if r > 0:
            times.append(marks[0].elapsed_time(marks[-1]))
            dispatch_ms += [marks[b].elapsed_time(marks[b + 1]) for b in range(batches)]
    t.close()
    totals, ops = count_ops(lib, wl, opts, wl.frame.copy(), device, stream, batches)
    ms = statistics.median(times)
    achieved = ops / (statistics.mean(dispatch_ms) * 1e-3)
    return {"workload": wl.name, "width": wl.width, "height": wl.height, "spp": wl.spp,
            "max_bounces": wl.max_bounces, "ms_per_step": ms,
            "msamples_per_s": wl.width * wl.height * wl.spp / (ms * 1e3),
            "roofline": {"bound": "fp32", "achieved": achieved / 1e12, "peak": peak / 1e12, "unit": "TFLOP/s",
                         "frac": achieved / peak, "ops_per_launch": ops,
                         "events_per_launch": {n: int(totals[k]) // batches for k, n in enumerate(EVENT_ORDER)}}}


def checkpoint_comparison(wl, device: int, stream, every: int = 2, reps: int = 2) -> dict:
    """The adjoint with vertex checkpoints every `every` bounces against path
    replay on the same scene and spp: forward and backward times (CUDA
    events, median of `reps`) and the device memory the checkpoints hold."""
    import torch

    from stargaze_b200 import PathTracer
    from stargaze_b200.workloads import render_options, upload_workload

    dl = np.random.default_rng(0).uniform(0.0, 1.0, (wl.width * wl.height, 4)).astype(np.float32)
    out = {"workload": wl.name, "width": wl.width, "height": wl.height, "spp": wl.spp, "every": every}
    for mode in ("replay", "checkpoints"):
        t = PathTracer((wl.width, wl.height), render_options(wl, spp=BATCH), device=device)
        upload_workload(t, wl)
        if mode == "checkpoints":
            t.set_checkpoints(every, wl.spp)
        fwd, bwd, stats = [], [], None
        for r in range(reps + 1):
            frame = wl.frame.copy()
            frame.scene_time = float(-500 - r)
            f = timed_forward(t, wl, frame, stream)
            if mode == "checkpoints":
                stats = t.checkpoint_stats()
            tape = t.tape()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            t.backward(frame, tape, dl, stream)
            b.record(stream)
            stream.synchronize()
            if r > 0:
                fwd.append(f)
                bwd.append(a.elapsed_time(b))
        t.close()
        entry = {"forward_ms": statistics.median(fwd), "backward_ms": statistics.median(bwd)}
        entry["forward_plus_adjoint_ms"] = entry["forward_ms"] + entry["backward_ms"]
        if stats is not None:
            entry["device_bytes"] = stats["device_bytes"]
            entry["records"] = stats["records"]
            entry["records_dropped"] = stats["dropped"]
        else:
            entry["device_bytes"] = 0
        out[mode] = entry
    out["note"] = ("replay: the staged adjoint replays every sample from its noise key; checkpoints: the "
                   "forward stores path state every `every` bounces and each sample's radiance, the "
                   "backward replays segments between checkpoints (device_bytes: what they hold)")
    return out


def integrator_comparison(wl, device: int, stream, reps: int = 3) -> dict:
    """The workload's step (spp samples from a fresh accumulation) with each
    integrator, and the wavefront's time per stage on one more step."""
    from stargaze_b200 import PathTracer
    from stargaze_b200.workloads import render_options, upload_workload

    t = PathTracer((wl.width, wl.height), render_options(wl, spp=BATCH), device=device)
    upload_workload(t, wl)
    out = {}
    for name in ("megakernel", "wavefront"):
        t.set_integrator(name)
        times = []
        for r in range(reps + 1):
            frame = wl.frame.copy()
            frame.scene_time = float(-7 - r)
            ms = timed_forward(t, wl, frame, stream)
            if r > 0:
                times.append(ms)
        out[f"{name}_ms_per_step"] = statistics.median(times)
    out["wavefront_speedup"] = out["megakernel_ms_per_step"] / out["wavefront_ms_per_step"]
    info = t.integrator()
    out["wavefront_pool_paths"] = info["pool_paths"]
    out["wavefront_iterations_per_dispatch"] = info["iterations"]
    t.close()
    return out


def stage_times(tracer, wl, frame, stream, batches: int) -> dict:
    """Milliseconds per wavefront stage over one step (events around every
    stage launch; outside the timed region)."""
    tracer.set_stage_timing(True)
    frame.scene_time = -55.0
    tracer.prepare_frame(frame)
    total = dict.fromkeys(tracer.STAGES, 0.0)
    for _ in range(batches):
        tracer.encode(frame, stream)
        for k, v in tracer.stage_times().items():
            total[k] += v
    tracer.set_stage_timing(False)
    return total


def fp64_sites(wl, device: int, stream, reps: int = 2) -> dict:
    """The FP64 sites against the reference's f32 arithmetic: hit-distance
    error of both at the host-sphere and ring-plane sites against double,
    and the ring workload's time per step with each."""
    import torch

    from stargaze_b200 import PathTracer, precision
    from stargaze_b200.workloads import render_options, upload_workload

    out = {"host_sphere": {}, "ring_plane": {}, "ms_per_step": {}}
    for mode, fp64 in (("f32", False), ("fp64", True)):
        out["host_sphere"][mode] = precision.host_sphere_precision(10**7, fp64, device)
        out["ring_plane"][mode] = precision.ring_plane_precision(wl.frame, 10**6, fp64, wl.ring_tables, device)
        t = PathTracer((wl.width, wl.height), render_options(wl, spp=BATCH), device=device)
        upload_workload(t, wl)
        t.set_fp64_sites(fp64)
        times = []
        for r in range(reps + 1):
            frame = wl.frame.copy()
            frame.scene_time = float(-1 - r)
            t.prepare_frame(frame)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            while t.samples() < wl.spp:
                t.encode(frame, stream)
            b.record(stream)
            stream.synchronize()
            if r > 0:
                times.append(a.elapsed_time(b))
        t.close()
        out["ms_per_step"][mode] = statistics.median(times)
    out["slowdown"] = out["ms_per_step"]["fp64"] / out["ms_per_step"]["f32"]
    out["note"] = ("relative error of the device's hit distance (and ring radius) against the exact "
                   "intersection of the same f32 rays; host sphere 6.4e6 m, camera 2 m up, 1e7 rays grazing "
                   "to nadir; ring plane 1e6 camera rays per ringed body of the ring workload")
    return out


def air_terrain(device: int, stream, reps: int = 1) -> dict:
    """The terrain workload (1080p, 128 spp, 4096^2 cells, 7,000 props) with
    the host's earthlike air (camera-ray single scattering, sky-lit ground,
    extinction of starlight and continuations): time per step with each
    integrator, and without air for comparison."""
    from stargaze_b200 import PathTracer
    from stargaze_b200.workloads import render_options, terrain_1080p, upload_workload, with_air

    wl, land = terrain_1080p(1920, 1080, 128)
    air_frame = with_air(wl.frame.copy(), 1)
    t = PathTracer((wl.width, wl.height), render_options(wl, spp=BATCH), device=device)
    upload_workload(t, wl)
    out = {"workload": "terrain 1920x1080, 128 spp, 4096^2 cells, 7,000 props, earthlike air", "ms_per_step": {}}
    for name, integrator, frame in (("wavefront_air", "wavefront", air_frame), ("megakernel_air", "megakernel", air_frame),
                                    ("wavefront_airless", "wavefront", wl.frame)):
        t.set_integrator(integrator)
        times = []
        for r in range(reps + 1):
            f = frame.copy()
            f.scene_time = float(-300 - r)
            ms = timed_forward(t, wl, f, stream)
            if r > 0:
                times.append(ms)
        out["ms_per_step"][name] = statistics.median(times)
    t.close()
    samples = wl.width * wl.height * wl.spp
    out["msamples_per_s"] = {k: samples / (v * 1e3) for k, v in out["ms_per_step"].items()}
    out["air_cost"] = out["ms_per_step"]["wavefront_air"] / out["ms_per_step"]["wavefront_airless"]
    return out


def oracle_build_flags() -> str:
    """The compile line of the oracle library (oracle/Makefile)."""
    try:
        text = (ROOT / "oracle" / "Makefile").read_text()
        flags = next(line.split("=", 1)[1].strip() for line in text.splitlines() if line.startswith("CFLAGS"))
        return f"gcc {flags}"
    except (OSError, StopIteration):
        return "unknown"


def run_reference(args):
    """The reference integrator's CPU restatement (the oracle) on every host
    core. Each step is one bounded sample of the workload: row bands of the
    frame in 8-sample dispatches for `per_step` seconds. `ms_per_step` is
    that measured wall time; the full 256-spp frame it extrapolates to is
    reported apart."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from stargaze_b200.workloads import WORKLOADS

    wl = WORKLOADS[args.workload](spp=args.spp)
    per_step = max(2.0, min(args.cpu_seconds, 60.0 / max(args.steps + args.warmup, 1)))
    for _ in range(args.warmup):
        cpu_baseline(wl, min(per_step, 2.0))
    values, walls = [], []
    for _ in range(args.steps):
        start = time.perf_counter()
        values.append(cpu_baseline(wl, per_step))
        walls.append((time.perf_counter() - start) * 1e3)
    value = statistics.median(v["value"] for v in values)
    base = values[0]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": statistics.mean(walls),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": wl.name, "width": wl.width, "height": wl.height, "spp": args.spp,
                   "max_bounces": wl.max_bounces,
                   "step": f"a bounded sample of the workload, about {per_step:.1f} s of row bands",
                   "cpu_sample": base["sample"],
                   "full_frame_ms_extrapolated": 1e3 * wl.width * wl.height * args.spp / (value * 1e6)},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": base["cores"], "kind": base["kind"],
                         "sample": base["sample"], "build": oracle_build_flags()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    from stargaze_b200 import PathTracer, abi
    from stargaze_b200._lib import load
    from stargaze_b200.workloads import WORKLOADS
    from stargaze_b200.workloads import render_options as bench_options
    import ctypes as C

    lib = load()
    wl = WORKLOADS[args.workload](spp=args.spp)
    batches = (args.spp + BATCH - 1) // BATCH
    # Disjoint noise sequences per rank: each GPU renders its own full-frame
    # 256-spp estimate (weak scaling, no data-path collective).
    opts = bench_options(wl, spp=BATCH, noise_seed=rank_noise_seed(rank))
    from stargaze_b200.workloads import upload_workload

    tracer = PathTracer((wl.width, wl.height), opts, device=local)
    upload_workload(tracer, wl)
    tracer.set_integrator(args.integrator)
    stream = torch.cuda.Stream()
    frame = wl.frame.copy()

    def step(i):
        frame.scene_time = float(i)  # a new frame time restarts the accumulation
        for _ in range(batches):
            tracer.encode(frame, stream)

    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    # Algorithmic work of one launch (counting kernel, outside timing).
    totals, ops_per_launch = count_ops(lib, wl, opts, frame, local, stream, batches)
    peak = C.c_double()
    assert lib.sg_measure_fp32_peak(local, C.byref(peak)) == 0

    with torch.cuda.stream(stream):
        for i in range(args.warmup):
            step(-1 - i)
        stream.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        launches0 = tracer.launch_count()
        step_ms, launch_ms = [], []
        with ClockSampler(local) as clocks:
            for i in range(args.steps):
                flush.zero_()  # evict the accumulation from L2 between steps
                marks = [torch.cuda.Event(enable_timing=True) for _ in range(batches + 1)]
                marks[0].record(stream)
                frame.scene_time = float(i)
                for b in range(batches):
                    tracer.encode(frame, stream)
                    marks[b + 1].record(stream)
                stream.synchronize()
                launch_ms += [marks[b].elapsed_time(marks[b + 1]) for b in range(batches)]
                step_ms.append(marks[0].elapsed_time(marks[-1]))
        torch.cuda.synchronize()
        launches = tracer.launch_count() - launches0
        if dist:
            dist.barrier()

        # End to end through the public API: frame from host memory, image
        # read back to (pinned) host memory every step.
        host_image = torch.empty((wl.width * wl.height * 4,), dtype=torch.float32, pin_memory=True)
        e2e_ms = []
        for i in range(args.steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            frame.scene_time = float(1000 + i)
            for _ in range(batches):
                tracer.encode(frame, stream)
            status = lib.sg_read_accumulation(tracer.handle, C.c_void_p(host_image.data_ptr()), 0,
                                              C.c_void_p(stream.cuda_stream))
            assert status == 0, status
            b.record(stream)
            stream.synchronize()
            e2e_ms.append(a.elapsed_time(b))
        stages = stage_times(tracer, wl, frame, stream, batches) if args.integrator == "wavefront" else None

    total_ms, e2e_total = max_over_ranks([sum(step_ms), sum(e2e_ms)], dist, "cuda")

    samples_per_step = wl.width * wl.height * args.spp
    value = job_msamples_per_s(world, samples_per_step, args.steps, total_ms)
    e2e_value = job_msamples_per_s(world, samples_per_step, args.steps, e2e_total)
    mean_launch_s = statistics.mean(launch_ms) * 1e-3
    achieved = ops_per_launch / mean_launch_s
    # Queue and result traffic by construction (wavefront): an extension
    # reads 3 and writes 4 float4 (planes 0, 1, 6; planes 1, 6 and two hit
    # planes), a shade vertex reads 7 planes and 2 hit planes and writes 7
    # planes, every sample writes and the resolve reads one float4.
    ev = {n: int(totals[k]) / batches for k, n in enumerate(EVENT_ORDER)}
    queue_bytes = (ev["vertices"] * 7 + (ev["ring_events"] + ev["surface_events"]) * 16) * 16 + \
        wl.width * wl.height * BATCH * 32
    hbm_peak_gbs = measured_hbm_gbs()
    result = None
    if rank == 0:
        base = None
        if world == 1 and not args.no_cpu_baseline:
            base = cpu_baseline(wl, args.cpu_seconds)
        clk = clocks.summary()
        extras = {}
        if world == 1 and not args.no_extras:
            from stargaze_b200 import workloads as W

            image = tracer.read_pixels(stream)
            extras["fp64_sites"] = fp64_sites(wl, local, stream)
            extras["integrators"] = integrator_comparison(wl, local, stream)
            extras["air"] = air_terrain(local, stream)
            extras["configs"] = {"spheres_256": config_entry(lib, W.spheres_256(), local, stream, peak.value),
                                 "terrain_1080p": config_entry(lib, W.WORKLOADS["terrain_1080p"](), local, stream,
                                                               peak.value)}
            extras["convergence"] = convergence(wl, image, args.spp, value, local, stream)
            land_wl, land = W.terrain_1080p(1920, 1080, 256)
            land.albedo_map = np.random.default_rng(1).uniform(0.05, 0.6, (1024, 1024)).astype(np.float32)
            land.map_extent = 2000.0
            terrain = adjoint_ratio(land_wl, local, stream, reps=2)
            checkpoints = checkpoint_comparison(land_wl, local, stream)
            from stargaze_b200 import inverse

            extras["ring_inverse_512"] = {"adam": inverse.ring_inverse(device=local),
                                          "central_differences": inverse.central_difference_check(device=local)}
            ring = adjoint_ratio(W.rings_1080p(512, 512, 64), local, stream)
            extras["adjoint"] = {"terrain_1080p": terrain, "checkpoints_terrain_1080p": checkpoints,
                                 "ring_512": ring, "ratio": ring["ratio"],
                                 "note": "ratio = adjoint time / forward time at equal spp (ring scene)"}
        result = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": wl.name, "width": wl.width, "height": wl.height, "spp": args.spp,
                       "max_bounces": wl.max_bounces, "batches_per_step": batches, "samples_per_step": samples_per_step,
                       "l2": f"flushed ({L2_FLUSH_BYTES >> 20} MiB write) between steps",
                       "parallelism": f"replicas x{world}, disjoint noise sequences",
                       "integrator": args.integrator},
            "roofline": {"bound": "fp32", "achieved": achieved / 1e12, "peak": peak.value / 1e12, "unit": "TFLOP/s",
                         "frac": achieved / peak.value,
                         "traffic": TRAFFIC_BYTES_PER_LAUNCH if wl.name == "rings_1080p" else None,
                         "traffic_note": "scaled from a one-iteration capture by path extensions",
                         "algorithmic_bytes_per_launch": queue_bytes,
                         "queue_hbm_frac": queue_bytes / (statistics.mean(launch_ms) * 1e-3) / (hbm_peak_gbs * 1e9)
                         if hbm_peak_gbs else None,
                         "issue_slot_fraction": ISSUE_SLOT_FRACTION if wl.name == "rings_1080p" else None,
                         "kernel": ("wavefront dispatch (extend, ring and surface stages, resolve)"
                                    if args.integrator == "wavefront" else "trace_kernel (megakernel)"),
                         "ops_per_launch": ops_per_launch,
                         "launch_ms": statistics.mean(launch_ms),
                         "stages_ms_per_step": stages,
                         "events_per_launch": {n: int(totals[k]) // batches for k, n in enumerate(EVENT_ORDER)},
                         "peak_source": "measured FMA-chain kernel (sg_measure_fp32_peak)"},
            "e2e": {"value": e2e_value, "unit": UNIT,
                    "h2d_bytes_per_step": batches * (len(frame.bodies) * 160 + len(frame.ground) * (48 + 32)),
                    "d2h_bytes_per_step": wl.width * wl.height * 16},
            "gpu_launches": int(launches),
            "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"]},
            "cpu_baseline": base,
            **extras,
        }
        if extras:
            # The configs' headline figures once more, last, where a reader of
            # the line's end finds them.
            ring, terrain = extras["adjoint"]["ring_512"], extras["adjoint"]["terrain_1080p"]
            result["summary"] = {
                "C1_msamples_per_s": extras["configs"]["spheres_256"]["msamples_per_s"],
                "C2_msamples_per_s": value, "C2_e2e_msamples_per_s": e2e_value,
                "C2_spp_to_1pct_vs_oracle": extras["convergence"]["vs_oracle"]["spp_to_1pct"]
                if extras["convergence"].get("vs_oracle") else None,
                "C2_spp_to_1pct_vs_oracle_f64": extras["convergence"]["vs_oracle_f64"]["spp_to_1pct"]
                if extras["convergence"].get("vs_oracle_f64") else None,
                "C3_msamples_per_s": extras["configs"]["terrain_1080p"]["msamples_per_s"],
                "C4_forward_plus_adjoint_over_forward": ring["forward_plus_adjoint_over_forward"],
                "C5_forward_plus_adjoint_over_forward": terrain["forward_plus_adjoint_over_forward"],
                "C5_checkpoints_vs_replay_ms": [extras["adjoint"]["checkpoints_terrain_1080p"]["checkpoints"]
                                                ["forward_plus_adjoint_ms"],
                                                extras["adjoint"]["checkpoints_terrain_1080p"]["replay"]
                                                ["forward_plus_adjoint_ms"]],
                "roofline_frac": result["roofline"]["frac"],
                "cpu_baseline_msamples_per_s": base["value"] if base else None,
            }
        print(json.dumps(result), flush=True)
    tracer.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse_args()
    if args.profile_case:
        PROFILE_CASES[args.profile_case]()
        print(f"profile case {args.profile_case}: done", flush=True)
        return 0
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
