"""The reference evaluator's timing protocol and performance gates, run on
this library's public `fastvid` API.

Protocol (scripts/evaluate.py:447-476, 584-617): `warmups` untimed calls,
then `repetitions` calls (at least 20), each bracketed by a device
synchronisation and timed with CUDA events; the gate statistic is the
median.  A throughput case is a batch of 24 independent frames encoded by
one `encode(list)` call and decoded by one `decode(list)` call (luma
Gpixels/s); a latency case is one frame (median milliseconds).  Defaults
follow the evaluator's command line: quality 90, tile 256x128, 5 warm-ups,
20 repetitions (evaluate.py:772-776).

Gates (evaluate.py:740-755):
* 24 frames of 3840x2160: encode >= 1.5 and decode >= 2.0 Gpixels/s
  (yuv422: 2.0 and 3.0);
* one 1920x1080 rgb444 frame: encode median < 1.0 ms, decode < 0.5 ms.

The evaluator reads its frames from a corpus that is not available here;
seeded synthetic frames of the gated shapes stand in for it (four distinct
frames per format, repeated to 24 -- every frame is coded independently, so
repeats cost the same as new frames).  The quality metrics of the evaluator
(libvship) are out of scope.

Run: python -m fastvid_b200.gates [--warmups 5] [--repetitions 20] [--out report.json]
"""

from __future__ import annotations

import argparse
import json
import statistics
import sys
from typing import Any, Callable, Sequence

THROUGHPUT_FRAMES = 24
# (mode, layout, bit depth, width, height)
CASES = (
    ("throughput", "gray", 10, 3840, 2160),
    ("throughput", "yuv422", 10, 3840, 2160),
    ("throughput", "rgb444", 10, 3840, 2160),
    ("throughput", "rgb444", 8, 3840, 2160),
    ("latency", "rgb444", 8, 1920, 1080),
    ("latency", "rgb444", 10, 1920, 1080),
)


def cuda_samples(operation: Callable[[], Any], warmups: int, repetitions: int, torch) -> tuple[list[float], Any]:
    """Seconds of each timed call (CUDA events, synchronised on both sides)
    and the last call's result."""
    for _ in range(warmups):
        operation()
    torch.cuda.synchronize()
    seconds, result = [], None
    for _ in range(repetitions):
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record()
        result = operation()
        end.record()
        end.synchronize()
        seconds.append(start.elapsed_time(end) / 1e3)
    return seconds, result


def distribution(seconds: Sequence[float]) -> dict[str, Any]:
    """Median (the gate statistic), minimum, 95th percentile (the sample at
    rank floor((n-1)*0.95) of the sorted list) and maximum."""
    ordered = sorted(seconds)
    p95 = ordered[min(len(ordered) - 1, int((len(ordered) - 1) * 0.95))]
    return {"samples_seconds": list(seconds), "median_seconds": statistics.median(seconds),
            "min_seconds": ordered[0], "p95_seconds": p95, "max_seconds": ordered[-1],
            "gate_statistic": "median"}


def performance_failures(result: dict[str, Any]) -> list[str]:
    """The gates a result misses (empty when it passes)."""
    failures: list[str] = []
    perf, fmt = result["performance"], result["format"]
    size = (result["width"], result["height"])
    if perf["mode"] == "throughput" and result["frame_count"] == THROUGHPUT_FRAMES and size == (3840, 2160):
        enc_min, dec_min = (2.0, 3.0) if fmt == "yuv422" else (1.5, 2.0)
        if perf["encode"]["gpps"] < enc_min:
            failures.append(f"encode throughput < {enc_min} GP/s")
        if perf["decode"]["gpps"] < dec_min:
            failures.append(f"decode throughput < {dec_min} GP/s")
    if perf["mode"] == "latency" and size == (1920, 1080) and fmt == "rgb444":
        if perf["encode"]["median_ms"] >= 1.0:
            failures.append("encode latency >= 1.0 ms")
        if perf["decode"]["median_ms"] >= 0.5:
            failures.append("decode latency >= 0.5 ms")
    return failures


def _frame(args):
    from . import synth

    layout, depth, width, height, seed = args
    return synth.make_frame(width, height, layout, depth, seed)


def measure(case, device, warmups: int, repetitions: int, quality: int = 90, tile_size=(256, 128),
            distinct: int = 4) -> dict[str, Any]:
    """One gated case through fastvid.encode / fastvid.decode."""
    import multiprocessing as mp

    import torch

    from . import api as fastvid  # the public fastvid API of this library

    mode, layout, depth, width, height = case
    count = THROUGHPUT_FRAMES if mode == "throughput" else 1
    seeds = [7000 + 97 * i + depth for i in range(min(distinct, count))]
    with mp.get_context("spawn").Pool(len(seeds)) as pool:
        host = pool.map(_frame, [(layout, depth, width, height, s) for s in seeds])
    uniq = [tuple(torch.from_numpy(p).to(device) for p in f) for f in host]
    frames = [uniq[i % len(uniq)] for i in range(count)]
    kw = dict(format=layout, bit_depth=depth, quality=quality, tile_size=tuple(tile_size))
    if count == 1:
        encode_op = lambda: fastvid.encode(frames[0], **kw)  # noqa: E731
    else:
        encode_op = lambda: fastvid.encode(frames, **kw)  # noqa: E731
    streams = encode_op()
    torch.cuda.synchronize()
    decode_op = (lambda: fastvid.decode(streams)) if count == 1 else (lambda: fastvid.decode(list(streams)))  # noqa: E731
    enc_s, _ = cuda_samples(encode_op, warmups, repetitions, torch)
    dec_s, decoded = cuda_samples(decode_op, warmups, repetitions, torch)
    enc, dec = distribution(enc_s), distribution(dec_s)
    pixels = width * height * count
    if mode == "throughput":
        enc["gpps"] = pixels / enc["median_seconds"] / 1e9
        dec["gpps"] = pixels / dec["median_seconds"] / 1e9
    else:
        enc["median_ms"] = enc["median_seconds"] * 1e3
        dec["median_ms"] = dec["median_seconds"] * 1e3
    encoded = [streams] if count == 1 else list(streams)
    out_frames = [decoded] if count == 1 else list(decoded)
    raw = sum(int(p.numel()) * 2 for f in frames for p in f)
    nbytes = sum(int(s.numel()) for s in encoded)
    shapes_ok = all(tuple(a.shape) == tuple(b.shape) and a.dtype == torch.uint16 and a.is_cuda
                    for fo, fi in zip(out_frames, frames) for a, b in zip(fo, fi))
    result = {"format": layout, "bit_depth": depth, "width": width, "height": height, "frame_count": count,
              "distinct_frames": len(uniq), "quality": quality, "tile_size": list(tile_size),
              "correctness": {"decoded_shapes": bool(shapes_ok and len(out_frames) == count)},
              "compression": {"raw_bytes": raw, "encoded_bytes": nbytes, "ratio": raw / nbytes},
              "performance": {"mode": mode, "warmups": warmups, "repetitions": repetitions,
                              "encode": enc, "decode": dec}}
    result["failures"] = performance_failures(result)
    return result


def main(argv=None) -> int:
    p = argparse.ArgumentParser(description="the reference evaluator's performance gates on this GPU")
    p.add_argument("--warmups", type=int, default=5)
    p.add_argument("--repetitions", type=int, default=20)
    p.add_argument("--quality", type=int, default=90)
    p.add_argument("--out", default=None)
    args = p.parse_args(argv)
    if args.repetitions < 20:
        p.error("--repetitions must be at least 20")
    if args.warmups < 1:
        p.error("--warmups must be positive")
    import torch

    device = torch.device("cuda", torch.cuda.current_device())
    results = [measure(c, device, args.warmups, args.repetitions, args.quality) for c in CASES]
    report = {"device": torch.cuda.get_device_name(device), "results": results,
              "passed": all(not r["failures"] and r["correctness"]["decoded_shapes"] for r in results)}
    text = json.dumps(report)
    if args.out:
        with open(args.out, "w") as f:
            f.write(text + "\n")
    summary = [{k: r[k] for k in ("format", "bit_depth", "width", "height", "frame_count", "failures")} |
               {"encode": r["performance"]["encode"].get("gpps", r["performance"]["encode"].get("median_ms")),
                "decode": r["performance"]["decode"].get("gpps", r["performance"]["decode"].get("median_ms"))}
               for r in results]
    print(json.dumps({"passed": report["passed"], "cases": summary}))
    return 0 if report["passed"] else 1


if __name__ == "__main__":
    sys.exit(main())
