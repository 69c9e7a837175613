#!/usr/bin/env python
"""Benchmark of the fastvid intra codec on B200: batched encode+decode of the
96-frame uneven mix, Gpix/s (luma pixels of all frames / step time).

One step = encode every frame of the batch and decode every stream again,
inputs resident in HBM (1.3 GB, above the 126 MB L2, so no flush is needed).
Prints one JSON line (rank 0).  ``--impl reference`` times the CPU restatement
of the reference codec (the reference has no CPU codec of its own) on all host
cores over the same 96 frames.  The line's ``reference_gpu`` object times the
reference's own CUDA codec, built from its sources for sm_100 (oracle/_ref),
through its binding one frame at a time as its public API drives it, beside
this library's single-frame and batched forms on the same frames;
``--impl reference_gpu`` prints that leg alone.

Launch: python bench.py [--gpus N] [--steps K] [--warmup W]
        python -m torch.distributed.run --nproc-per-node N ... bench.py --gpus N
With N > 1 every rank runs its own replica of the batch (weak scaling, no
collective on the data path); times are the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import signal
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = ("mixed96: 32x 1280x720 gray8 q100, 32x 1920x1080 rgb444-8 q90, "
            "16x 3840x2160 rgb444-10 q85, 16x 2048x1080 gray16 q87; "
            "every 4th frame near-flat (noise sd 0.5); tiles in config.tiles")
TILES = {("gray", 8): (64, 64), ("rgb444", 8): (64, 64), ("rgb444", 10): (128, 128), ("gray", 16): (128, 128)}


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=("ours", "reference", "reference_gpu"))
    p.add_argument("--frames", type=int, default=96)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-plain", action="store_true")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    p.add_argument("--cpu-seconds", type=float, default=15.0, help="budget of the CPU-baseline sample")
    p.add_argument("--no-tuning", action="store_true", help="ignore the autotuned table (tiles, launch geometry)")
    p.add_argument("--no-reference-gpu", action="store_true", help="skip the reference GPU leg")
    p.add_argument("--serve-requests", type=int, default=10000,
                   help="requests of the serving leg (the serving mix; 0 skips it)")
    p.add_argument("--serve-rates", default="1000,2000,5000,10000,20000,0",
                   help="offered request rates of the serving leg, per second (0: all at once)")
    p.add_argument("--serve-budget-gb", type=float, default=40.0, help="device-memory budget of the server")
    return p.parse_args()


def _gen(spec):
    from fastvid_b200 import synth

    return synth.frame_from_spec(spec)


def generate(specs, workers):
    import multiprocessing as mp

    if workers <= 1:
        return [_gen(s) for s in specs]
    with mp.get_context("spawn").Pool(workers) as pool:
        return pool.map(_gen, specs, chunksize=1)


def _gen_serving(key):
    from fastvid_b200 import synth

    return synth.serving_frame(*key)


def serving_leg(args, device):
    """The serving mix through fastvid_b200.serve.Server (continuous
    batching) at the offered rates, beside the plain single-frame path on
    the same request sequence; a sample of answers is compared with the
    plain path's."""
    import multiprocessing as mp

    import torch

    import fastvid_b200
    from fastvid_b200 import synth
    from fastvid_b200.codec import header_of
    from fastvid_b200.serve import Server, report, run_open_loop

    per_format = 2
    keys = [(f, i) for f in range(len(synth.SERVING_FORMATS)) for i in range(per_format)]
    with mp.get_context("spawn").Pool(min(8, len(keys))) as pool:
        frames = dict(zip(keys, pool.map(_gen_serving, keys, chunksize=1)))
    dev = {k: tuple(torch.from_numpy(p).to(device) for p in v) for k, v in frames.items()}
    params, streams = {}, {}
    for (f, i), planes in dev.items():
        fmt = synth.SERVING_FORMATS[f][1]
        for q in fmt["qualities"]:
            pr = dict(layout=fmt["layout"], bit_depth=fmt["bit_depth"], quality=q, tile_size=fmt["tile"])
            params[(f, q)] = pr
            st = fastvid_b200.encode(planes, **pr)
            streams[(f, i, q)] = (st, header_of(st))
    specs = synth.serving_specs(args.serve_requests, frames_per_format=per_format)
    items, pixels = [], 0
    for sp in specs:
        f, i, q = sp["format"], sp["frame"], sp["quality"]
        fmt = synth.SERVING_FORMATS[f][1]
        pixels += fmt["width"] * fmt["height"]
        if sp["kind"] == "encode":
            items.append(("encode", dev[(f, i)], params[(f, q)]))
        else:
            items.append(("decode", streams[(f, i, q)][0], {"header": streams[(f, i, q)][1]}))
    sample = set(range(0, len(items), 50))

    def plain(item):
        kind, payload, pr = item
        if kind == "encode":
            return fastvid_b200.encode(payload, **pr)
        return fastvid_b200.decode(payload)

    seen = set()
    for item in items:  # warm every shape of the plain path
        key = (item[0], id(item[1]))
        if key not in seen:
            seen.add(key)
            plain(item)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plain_answers = {}
    for j, item in enumerate(items):
        out = plain(item)
        if j in sample:
            plain_answers[j] = out
    torch.cuda.synchronize()
    plain_s = time.perf_counter() - t0

    def same(a, b):
        if isinstance(a, torch.Tensor):
            return torch.equal(a, b)
        return len(a) == len(b) and all(torch.equal(x, y) for x, y in zip(a, b))

    rates = [float(r) for r in args.serve_rates.split(",") if r.strip()]
    out = {"workload": "serving mix: 0.3 720p gray8, 0.4 1080p rgb8 q{100,90,66}, 0.2 4K rgb10 q{100,96,86}, "
                       "0.1 4K gray16 q{100,87}; 60% encode / 40% decode of streams produced earlier; "
                       f"{per_format} frames per format, inputs resident in HBM",
           "requests": len(items), "luma_pixels": pixels, "plain_gpix_s": pixels / plain_s / 1e9,
           "budget_gb": args.serve_budget_gb, "rates": []}
    exact = True
    import gc

    # kept answers are copied into buffers made before the runs, so the
    # harness allocates nothing while the server runs
    into = {j: (torch.empty_like(a) if isinstance(a, torch.Tensor) else tuple(torch.empty_like(x) for x in a))
            for j, a in plain_answers.items()}
    with Server(device, memory_budget=int(args.serve_budget_gb * (1 << 30)), workers=3) as server:
        run_open_loop(server, items, None)  # grow the resident workspaces to the largest batches
        for rate in rates:
            gc.collect()
            gc.freeze()  # objects made so far are never scanned again: no collector pause mid-run
            n_batches = len(server.batches)
            server.peak_charged = 0
            torch.cuda.reset_peak_memory_stats(device)
            m0 = torch.cuda.memory_stats(device)
            recs, t0, kept = run_open_loop(server, items, rate or None, seed=int(rate), keep=into)
            m1 = torch.cuda.memory_stats(device)
            gc.unfreeze()
            rep = report(recs, t0)
            rep["offered_req_s"] = rate or "all at once"
            rep["allocator"] = {k: m1.get(k, 0) - m0.get(k, 0) for k in ("num_alloc_retries", "num_device_alloc",
                                                                         "num_device_free", "num_sync_all_streams")}
            rep["reserved_gb"] = m1.get("reserved_bytes.all.current", 0) / 2**30
            # the server's own charge (resident workspaces + outputs in flight)
            # against its budget, and the process's peak allocation (which
            # also holds the bench's frames, streams and kept answers)
            rep["server_peak_charged_gb"] = server.peak_charged / 2**30
            rep["process_peak_allocated_gb"] = m1.get("allocated_bytes.all.peak", 0) / 2**30
            runs = server.batch_times[n_batches:]
            sizes = [n for _, n in server.batches[n_batches:]]
            rep["batches"] = len(sizes)
            rep["mean_batch"] = sum(sizes) / max(1, len(sizes))
            rep["longest_batch_ms"] = max((r[1] - r[0]) * 1e3 for r in runs) if runs else 0.0
            rep["longest_batches"] = [dict(ms=round((r[1] - r[0]) * 1e3, 2), kind=r[2], frames=r[3], mpix=r[4] / 1e6,
                                           at_s=round(r[0] - t0, 4))
                                      for r in sorted(runs, key=lambda r: r[0] - r[1])[:3]]
            exact = exact and rep["failed"] == 0 and all(same(kept[j], plain_answers[j]) for j in sample)
            out["rates"].append(rep)
        out["max_concurrent_batches"] = server.max_concurrent
        out["mean_batch"] = sum(n for _, n in server.batches) / max(1, len(server.batches))
    best = max(r["gpix_s"] for r in out["rates"]) if out["rates"] else 0.0
    out["served_over_plain"] = best / out["plain_gpix_s"]
    out["bit_exact_sample"] = f"{len(sample)} answers per rate equal to the plain path's: {exact}"
    out["bit_exact"] = bool(exact)
    return out


def format_sample(specs):
    """One frame of each format."""
    seen, out = set(), []
    for i, s in enumerate(specs):
        key = (s["layout"], s["bit_depth"])
        if key not in seen:
            seen.add(key)
            out.append(i)
    return out


LAYOUT_CODES = {"gray": 0, "yuv422": 1, "rgb444": 2}


def load_reference_gpu():
    """The reference's CUDA codec built from its own sources (oracle/_ref),
    or the reason it is unavailable."""
    ref_dir = os.path.join(ROOT, "oracle", "_ref")
    if not os.path.isdir(ref_dir) or not any(f.startswith("fastvid_ref_C") and f.endswith(".so")
                                             for f in os.listdir(ref_dir)):
        return None, "reference extension not built (oracle/build_ref.py needs the reference sources)"
    sys.path.insert(0, ref_dir)
    try:
        import fastvid_ref_C
    except Exception as exc:  # noqa: BLE001 - report why the leg could not run
        return None, f"reference extension failed to load: {exc}"
    return fastvid_ref_C, None


def event_median(fn, warmup, reps):
    """The reference evaluator's protocol (scripts/evaluate.py:447-476):
    warm-ups, then `reps` calls each between two CUDA events with a
    synchronisation, median milliseconds."""
    import torch

    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    times = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        times.append(a.elapsed_time(b))
    return statistics.median(times)


def plain_and_reference_legs(specs, dev_frames, layouts, depths, quals, tiles, luma, warmup, reps, with_ref,
                             ours=True):
    """Per-frame loops over the whole mix (the reference's list API is such a
    loop, fastvid/__init__.py:44-53): this library's single-frame path and
    the reference's CUDA build, encode and decode timed separately, plus one
    frame of each format alone.  Returns (ours, reference) dicts."""
    import torch

    import fastvid_b200

    def our_enc():
        return [fastvid_b200.encode(f, layout=layouts[i], bit_depth=depths[i], quality=quals[i], tile_size=tiles[i])
                for i, f in enumerate(dev_frames)]

    out = {}
    ref_out = None
    fmt_idx = format_sample(specs)
    fmt_name = {i: autotune_key(specs[i]) for i in fmt_idx}
    if ours:
        streams = our_enc()
        enc = event_median(our_enc, warmup, reps)
        dec = event_median(lambda: [fastvid_b200.decode(s) for s in streams], warmup, reps)
        out = {"enc_ms": enc, "dec_ms": dec, "gpix_s": luma / (enc + dec) / 1e6,
               "enc_gpix_s": luma / enc / 1e6, "dec_gpix_s": luma / dec / 1e6, "per_format_ms": {}}
        for i in fmt_idx:
            f = dev_frames[i]
            e = event_median(lambda: fastvid_b200.encode(f, layout=layouts[i], bit_depth=depths[i],
                                                         quality=quals[i], tile_size=tiles[i]), warmup, reps)
            d = event_median(lambda: fastvid_b200.decode(streams[i]), warmup, reps)
            out["per_format_ms"][fmt_name[i]] = {"encode": e, "decode": d}
    if with_ref:
        ref, why = load_reference_gpu()
        if ref is None:
            return out, {"unavailable": why}
        frames_l = [list(f) for f in dev_frames]

        def ref_enc_one(i):
            return ref.encode(frames_l[i], LAYOUT_CODES[layouts[i]], depths[i], quals[i], 24, 1, tiles[i][0],
                              tiles[i][1])

        def ref_enc():
            return [ref_enc_one(i) for i in range(len(dev_frames))]

        rstreams = ref_enc()
        enc = event_median(ref_enc, warmup, reps)
        dec = event_median(lambda: [ref.decode(s, True) for s in rstreams], warmup, reps)
        ref_out = {"impl": "reference CUDA codec (cuda/csrc) built for sm_100 from its own sources, called "
                           "per frame through its binding _C.encode/_C.decode",
                   "enc_ms": enc, "dec_ms": dec, "gpix_s": luma / (enc + dec) / 1e6,
                   "enc_gpix_s": luma / enc / 1e6, "dec_gpix_s": luma / dec / 1e6, "per_format_ms": {},
                   "protocol": f"{warmup} warm-ups, median of {reps} CUDA-event timed calls"}
        for i in fmt_idx:
            e = event_median(lambda: ref_enc_one(i), warmup, reps)
            d = event_median(lambda: ref.decode(rstreams[i], True), warmup, reps)
            ref_out["per_format_ms"][fmt_name[i]] = {"encode": e, "decode": d}
        if ours:
            same = all(torch.equal(a, b) for a, b in zip(streams, rstreams))
            ref_out["streams_identical_to_ours"] = bool(same)
    return out, ref_out


def copy_floor(device, up_bytes, down_bytes, reps=3):
    """Pinned host<->device copy rates of this box: each direction alone and
    both at once for the given byte counts (the e2e step's transfers); the
    concurrent time is the e2e step's copy floor."""
    import torch

    up_h = torch.empty(up_bytes, dtype=torch.uint8).pin_memory()
    down_h = torch.empty(down_bytes, dtype=torch.uint8).pin_memory()
    up_d = torch.empty(up_bytes, dtype=torch.uint8, device=device)
    down_d = torch.empty(down_bytes, dtype=torch.uint8, device=device)
    s1, s2 = torch.cuda.Stream(device), torch.cuda.Stream(device)

    def timed(fn):
        best = None
        for _ in range(reps):
            torch.cuda.synchronize(device)
            t0 = time.perf_counter()
            fn()
            torch.cuda.synchronize(device)
            dt = (time.perf_counter() - t0) * 1e3
            best = dt if best is None else min(best, dt)
        return best

    def up():
        with torch.cuda.stream(s1):
            up_d.copy_(up_h, non_blocking=True)

    def down():
        with torch.cuda.stream(s2):
            down_h.copy_(down_d, non_blocking=True)

    t_up, t_down = timed(up), timed(down)
    t_both = timed(lambda: (up(), down()))
    return {"h2d_gbs": up_bytes / t_up / 1e6, "d2h_gbs": down_bytes / t_down / 1e6,
            "floor_ms": t_both, "both_gbs": (up_bytes + down_bytes) / t_both / 1e6,
            "how": "pinned copies of the step's byte counts, each direction alone and both at once "
                   "(best of 3, wall clock around a synchronize)"}


def autotune_key(spec):
    return f"{spec['layout']}-{spec['bit_depth']}-{spec['width']}x{spec['height']}"


class Clocks:
    """nvidia-smi sampling of SM clock and throttle reasons during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.send_signal(signal.SIGTERM)
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        return False

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except OSError:
            pass
        finally:
            if self.path:
                try:
                    os.unlink(self.path)
                except OSError:
                    pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[j] for r in rows for j in range(4) if r[5 + j] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def time_oracle(frames, specs, idx, budget_s):
    """Encode+decode the sample frames with the oracle on all host cores."""
    import oracle

    threads = oracle.cpu_threads()
    pixels = sum(specs[i]["width"] * specs[i]["height"] for i in idx)
    reps, total = 0, 0.0
    t_start = time.perf_counter()
    while True:
        t0 = time.perf_counter()
        for i in idx:
            s = specs[i]
            stream = oracle.encode(frames[i], layout=s["layout"], bit_depth=s["bit_depth"], quality=s["quality"],
                                   tile_size=s["tile"], threads=threads)
            oracle.decode(stream, threads=threads)
        total += time.perf_counter() - t0
        reps += 1
        if time.perf_counter() - t_start >= budget_s or reps >= 50:
            break
    return pixels * reps / total / 1e9, threads, reps


def run_reference(args, specs):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    idx = list(range(len(specs)))
    fl = generate(specs, max(1, min(16, os.cpu_count() or 2)))
    for _ in range(max(1, args.warmup)):
        time_oracle(fl, specs, idx, 0.0)
    t0 = time.perf_counter()
    values = []
    for _ in range(args.steps):
        g, threads, reps = time_oracle(fl, specs, idx, 0.0)
        values.append(g)
    elapsed = time.perf_counter() - t0
    value = statistics.median(values)
    sample = f"all {len(idx)} frames of the mix, encode+decode per step, {threads} threads"
    line = {
        "impl": "reference", "metric": "Gpix/s encode+decode", "value": value, "unit": "Gpix/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * elapsed / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u16", "data": "synthetic",
        "config": {"workload": WORKLOAD, "frames": len(specs), "parallelism": "replicas",
                   "tiles": {f"{sp['layout']}-{sp['bit_depth']}-{sp['width']}x{sp['height']}": list(sp["tile"])
                             for sp in specs}},
        "cpu_baseline": {"value": value, "unit": "Gpix/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "Gpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_reference_gpu(args, specs):
    """The reference's CUDA build alone over the mix (one GPU, rank 0)."""
    import numpy as np
    import torch

    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    host = generate(specs, max(1, min(16, os.cpu_count() or 2)))
    dev = [tuple(torch.from_numpy(np.ascontiguousarray(p)).cuda() for p in f) for f in host]
    luma = sum(s["width"] * s["height"] for s in specs)
    _, ref = plain_and_reference_legs(specs, dev, [s["layout"] for s in specs], [s["bit_depth"] for s in specs],
                                      [s["quality"] for s in specs], [s["tile"] for s in specs], luma,
                                      max(1, args.warmup), max(1, args.steps), True, ours=False)
    print(json.dumps({"impl": "reference_gpu", "metric": "Gpix/s encode+decode", "unit": "Gpix/s",
                      "value": ref.get("gpix_s"), "config": {"workload": WORKLOAD, "frames": len(specs)},
                      "reference_gpu": ref}), flush=True)
    return 0


# Algorithmic bytes per sample of each stage (encode: 2 B in + stream out;
# decode: stream in + 2 B out).  A kernel is charged its stage's figure.
ENC_KERNELS = {"enc_init", "enc_predict", "enc_predict_wide", "enc_analyze", "enc_rans", "enc_scan", "enc_prefix",
               "enc_emit"}


def main():
    args = parse_args()
    from fastvid_b200 import synth

    specs = synth.mixed_batch_specs(args.frames)
    from fastvid_b200 import autotune

    table = autotune.load() if autotune.TABLE.exists() and not args.no_tuning else None
    for s in specs:
        s["tile"] = autotune.tile_for(table, s["layout"], s["bit_depth"], s["width"], s["height"],
                                      default=TILES[(s["layout"], s["bit_depth"])])
    args.tuning = ("autotuned table fastvid_b200/tuning/b200.json" if table else "built-in defaults")
    if args.impl == "reference":
        return run_reference(args, specs)
    if args.impl == "reference_gpu":
        return run_reference_gpu(args, specs)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    workers = max(1, min(16, (os.cpu_count() or 2) // max(1, world)))
    host_frames = generate(specs, workers)

    import numpy as np
    import torch

    import fastvid_b200
    from fastvid_b200 import _native
    from fastvid_b200.batch import BatchCodec

    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    if table:
        autotune.apply(table)
    # replicas: one process per GPU; the process group carries only the
    # barrier around timed regions and the max over ranks
    from fastvid_b200.replicas import Replicas

    rep = Replicas("nccl", device)
    barrier = rep.barrier
    max_over_ranks = rep.max

    # inputs resident in HBM, plus pinned host copies for the end-to-end leg
    pinned = [tuple(torch.from_numpy(np.ascontiguousarray(p)).pin_memory() for p in f) for f in host_frames]
    dev_frames = [tuple(p.to(device, non_blocking=True) for p in f) for f in pinned]
    torch.cuda.synchronize()
    layouts = [s["layout"] for s in specs]
    depths = [s["bit_depth"] for s in specs]
    quals = [s["quality"] for s in specs]
    tiles = [s["tile"] for s in specs]
    luma = sum(s["width"] * s["height"] for s in specs)
    samples = sum(p.size for f in host_frames for p in f)
    # the timed steps run the public batched form as shipped: analysis and
    # decode passes replayed from CUDA graphs; a separate eager step (same
    # kernels, one launch each) gives the per-kernel times
    codec = BatchCodec(device)
    eager = BatchCodec(device, use_graphs=False)

    def step(frames_dev):
        streams, heads = codec.encode(frames_dev, layout=layouts, bit_depth=depths, quality=quals, tile_size=tiles,
                                      return_headers=True)
        planes = codec.decode(streams, headers=heads)
        return streams, planes

    for _ in range(max(1, args.warmup)):
        streams, planes = step(dev_frames)
    torch.cuda.synchronize()

    # bit-exactness: lossless frames round trip exactly; every frame's bytes
    # equal the single-frame path's; decodes equal the single-frame decode
    bit_exact = True
    for i, (s, f) in enumerate(zip(specs, dev_frames)):
        if s["quality"] == 100 or (s["bit_depth"] == 8 and s["layout"] == "gray"):
            bit_exact &= all(torch.equal(a, b) for a, b in zip(planes[i], f))
    for i in format_sample(specs):
        plain = fastvid_b200.encode(dev_frames[i], layout=layouts[i], bit_depth=depths[i], quality=quals[i],
                                    tile_size=tiles[i])
        bit_exact &= torch.equal(plain, streams[i])
        bit_exact &= all(torch.equal(a, b) for a, b in zip(fastvid_b200.decode(plain), planes[i]))
    stream_bytes = sum(int(s.numel()) for s in streams)

    # timed region
    barrier()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    launches0 = _native.launch_count() + codec.graph_kernels
    with Clocks(local_rank) as clocks:
        for k in range(args.steps):
            a, b, c = ev[k]
            a.record()
            # the headers come back with the encoder's results, so the
            # decode reads nothing back from the streams
            streams, heads = codec.encode(dev_frames, layout=layouts, bit_depth=depths, quality=quals,
                                          tile_size=tiles, return_headers=True)
            b.record()
            planes = codec.decode(streams, headers=heads)
            c.record()
        torch.cuda.synchronize()
    barrier()
    launches = _native.launch_count() + codec.graph_kernels - launches0  # direct + graph-replayed, all K steps
    # per-kernel times: eager steps, CUDA events around each launch
    eager.decode(eager.encode(dev_frames, layout=layouts, bit_depth=depths, quality=quals, tile_size=tiles))
    torch.cuda.synchronize()
    with _native.KernelProfile() as prof:
        for _ in range(args.steps):
            eager.decode(eager.encode(dev_frames, layout=layouts, bit_depth=depths, quality=quals, tile_size=tiles))
        torch.cuda.synchronize()
    enc_ms = sum(a.elapsed_time(b) for a, b, _ in ev) / args.steps
    dec_ms = sum(b.elapsed_time(c) for _, b, c in ev) / args.steps
    step_ms = max_over_ranks(enc_ms + dec_ms)
    enc_ms = max_over_ranks(enc_ms)
    dec_ms = max_over_ranks(dec_ms)
    value = rep.rate(luma, step_ms) / 1e9

    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_kind = "measured" if "hbm_gbs" in peaks else "fallback"

    kernel_ms = {k: v / args.steps for k, v in prof.ms.items()}
    kernel_launches = {k: v // args.steps for k, v in prof.launches.items()}
    dominant = max(kernel_ms, key=kernel_ms.get)
    enc_bytes = 2 * samples + stream_bytes
    dec_bytes = stream_bytes + 2 * samples
    stage_bytes = enc_bytes if dominant in ENC_KERNELS else dec_bytes
    per_launch_ms = kernel_ms[dominant] / max(1, kernel_launches[dominant])
    per_launch_bytes = stage_bytes / max(1, kernel_launches[dominant])
    achieved = per_launch_bytes / (per_launch_ms / 1e3) / 1e9
    traffic = None
    try:
        tr = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
        rec = tr.get(dominant)
        if rec:
            traffic = rec["bytes_per_sample"] * samples / max(1, kernel_launches[dominant])
    except (OSError, ValueError, KeyError):
        pass
    roofline = {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                "frac": achieved / hbm_peak, "traffic": traffic, "peak_source": peak_kind,
                "algorithmic_bytes_per_launch": per_launch_bytes, "launch_ms": per_launch_ms}
    pipeline = (enc_bytes + dec_bytes) / (step_ms / 1e3) / 1e9
    line = {
        "metric": "Gpix/s encode+decode", "value": value, "unit": "Gpix/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u16",
        "data": "synthetic (seeded integer generator standing in for the unavailable corpus)",
        "config": {"workload": WORKLOAD, "frames": len(specs), "luma_pixels": luma, "samples": samples,
                   "form": "batched (one launch per kernel for the whole batch)",
                   "tiles": {autotune.format_key(sp["layout"], sp["bit_depth"], sp["width"], sp["height"]):
                             list(sp["tile"]) for sp in specs},
                   "tuning": args.tuning, "launch_ctas_per_sm": autotune.launch_settings(),
                   "l2": "inputs 1.3 GB > 126 MB L2 (no flush needed)", "parallelism": f"replicas x{world}"},
        "enc_gpix_s": rep.rate(luma, enc_ms) / 1e9, "dec_gpix_s": rep.rate(luma, dec_ms) / 1e9,
        "enc_ms": enc_ms, "dec_ms": dec_ms, "stream_bytes": stream_bytes, "bit_exact": bool(bit_exact),
        "roofline": roofline,
        "pipeline_roofline": {"achieved": pipeline, "peak": hbm_peak, "unit": "GB/s", "frac": pipeline / hbm_peak,
                              "bytes_per_step": enc_bytes + dec_bytes},
        "kernels_ms_per_step": {k: round(v, 4) for k, v in sorted(kernel_ms.items(), key=lambda kv: -kv[1])},
        "gpu_launches": launches,
        "clocks": clocks.summary(),
    }

    # single-frame (plain, drop-in) path and the reference's own CUDA build on
    # the same frames, one call per frame, the reference evaluator's protocol
    if not args.no_plain:
        plain, ref_gpu = plain_and_reference_legs(specs, dev_frames, layouts, depths, quals, tiles, luma, 5, 20,
                                                  rank == 0 and world == 1 and not args.no_reference_gpu)
        plain_ms = max_over_ranks(plain["enc_ms"] + plain["dec_ms"])
        line["plain_gpix_s"] = rep.rate(luma, plain_ms) / 1e9
        line["plain"] = plain
        line["batched_over_plain"] = line["value"] / line["plain_gpix_s"]
        if ref_gpu is not None:
            if "gpix_s" in ref_gpu:
                ref_gpu["batched_over_reference_gpu"] = line["value"] / ref_gpu["gpix_s"]
                ref_gpu["plain_over_reference_gpu"] = plain["gpix_s"] / ref_gpu["gpix_s"]
                ref_gpu["per_format_plain_over_reference_gpu"] = {
                    k: {op: ref_gpu["per_format_ms"][k][op] / plain["per_format_ms"][k][op]
                        for op in ("encode", "decode")} for k in ref_gpu["per_format_ms"]}
            line["reference_gpu"] = ref_gpu

    # end to end through the public API with host buffers
    if not args.no_e2e:
        out = {}
        # pinned output buffers, allocated once like a streaming caller would
        host_sbuf = torch.empty(2 * stream_bytes, dtype=torch.uint8).pin_memory()
        host_pbuf = torch.empty(samples, dtype=torch.uint16).pin_memory()

        def e2e_step():
            # pinned frames in; streams and decoded planes out in pinned host
            # memory; uploads, kernels and downloads overlap chunk by chunk
            out["streams"], out["planes"] = codec.encode_decode_host(
                pinned, layout=layouts, bit_depth=depths, quality=quals, tile_size=tiles,
                out_streams=host_sbuf, out_planes=host_pbuf)

        e2e_step()
        barrier()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        k_e2e = max(1, min(args.steps, 5))
        for _ in range(k_e2e):
            e2e_step()
        b.record()
        b.synchronize()
        e2e_ms = max_over_ranks(a.elapsed_time(b) / k_e2e)
        frame_bytes = 2 * samples
        link = copy_floor(device, frame_bytes, stream_bytes + frame_bytes)
        line["e2e"] = {"value": rep.rate(luma, e2e_ms) / 1e9, "unit": "Gpix/s",
                       "h2d_bytes_per_step": frame_bytes,
                       "d2h_bytes_per_step": stream_bytes + frame_bytes, "ms_per_step": e2e_ms,
                       "path": "BatchCodec.encode_decode_host: pinned frames in, pinned streams and decoded planes "
                               "out; chunks of at most 32 MB of samples, uploads running ahead into a ring of "
                               "device buffers, encode on the calling stream and decode on a second host thread's "
                               "stream, downloads overlapping the uploads",
                       "link": link, "copy_floor_frac": link["floor_ms"] / e2e_ms}
        roundtrip_ok = all(np.array_equal(o.numpy(), h) for op, hf, s in zip(out["planes"], host_frames, specs)
                           if s["quality"] == 100 for o, h in zip(op, hf))
        roundtrip_ok &= all(torch.equal(out["streams"][i], streams[i].cpu()) for i in format_sample(specs))
        line["bit_exact"] = bool(line["bit_exact"] and roundtrip_ok)

    # CPU baseline: the oracle (restatement of the reference) on all host cores
    if rank == 0 and world == 1 and not args.no_cpu:
        idx = list(range(len(specs)))
        gpix, threads, reps = time_oracle(host_frames, specs, idx, args.cpu_seconds)
        line["cpu_baseline"] = {"value": gpix, "unit": "Gpix/s", "cores": threads, "kind": "port",
                                "sample": f"all {len(idx)} frames of the mix, encode+decode, {reps} reps"}
    # serving form (one GPU): continuous batching at offered rates, p50/p99
    if rank == 0 and world == 1 and args.serve_requests > 0:
        line["serving"] = serving_leg(args, device)
        line["bit_exact"] = bool(line["bit_exact"] and line["serving"]["bit_exact"])
    if rank == 0:
        print(json.dumps(line), flush=True)
    rep.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
