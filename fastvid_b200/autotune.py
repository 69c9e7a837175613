"""Autotuner for the batched codec on one GPU.

Three kinds of knob, tuned by measurement and kept in a JSON table:

* Launch geometry -- the CTAs-per-SM cap of the persistent kernels
  (fvb_set_launch_ctas): how many tile wavefronts, analysis warps, rANS
  decode warps... share an SM.  No output byte depends on it.  Chosen by
  coordinate descent over the kernels on the measured encode+decode time of a
  sample batch.
* Wavefront block and warps per tile -- how many of the 32 steps of each
  wavefront block the predictor and reconstruction warps unroll
  (fvb_set_wavefront_block: 4, 8, 16 or 32), and whether one warp or a warp
  pair sweeps a tile's bands (fvb_set_tile_warps: 1 or 2).  No output byte
  depends on either; tuned before the launch caps.
* Tile geometry per frame format (layout, depth, width, height) -- the
  wavefront block each warp sweeps.  The tile size is written into the
  stream header, so it changes the bytes and the compression; the tuner takes
  the fastest candidate whose streams stay within `size_tolerance` of the
  smallest candidate's.  The single-frame path called with the chosen
  tile_size writes the same bytes as the batched path.

The reference has no tuner: its tile size is a caller argument (default
256x128, cuda/fastvid_cuda/__init__.py:8-45) and its launch shapes are fixed.
"""

from __future__ import annotations

import json
import statistics
import time
from pathlib import Path

from . import _native

TABLE = Path(__file__).resolve().parent / "tuning" / "b200.json"

# kernels with a launch-geometry knob worth tuning, and the caps tried
LAUNCH_KNOBS = ("enc_predict", "enc_analyze", "enc_emit", "dec_rans", "dec_other", "dec_reconstruct")
LAUNCH_CANDIDATES = (2, 3, 4, 6, 8, 12, 16)
WAVEFRONT_BLOCKS = (4, 8, 16, 32)
TILE_WARPS = (1, 2)
TILE_CANDIDATES = ((32, 32), (64, 64), (128, 128))


def format_key(layout: str, bit_depth: int, width: int, height: int) -> str:
    return f"{layout}-{bit_depth}-{width}x{height}"


# ---- pure selection rules (no GPU) ------------------------------------------

def choose_tile(results: dict, size_tolerance: float) -> tuple:
    """results: {tile: (ms, stream_bytes)}.  The fastest tile among those
    whose bytes are within (1 + size_tolerance) of the smallest; ties go to
    the smaller stream."""
    smallest = min(b for _, b in results.values())
    ok = {t: v for t, v in results.items() if v[1] <= smallest * (1.0 + size_tolerance)}
    return min(ok, key=lambda t: (ok[t][0], ok[t][1]))


def descend(knobs, candidates, measure, start: dict, rounds: int = 2, min_gain: float = 0.01) -> dict:
    """Coordinate descent: for each knob in turn try every candidate with the
    others fixed, keep a change only if it cuts measure() by min_gain;
    repeat until a round changes nothing (at most `rounds`)."""
    cur = dict(start)
    best = measure(cur)
    for _ in range(rounds):
        changed = False
        for k in knobs:
            for c in candidates:
                if c == cur[k]:
                    continue
                trial = dict(cur, **{k: c})
                t = measure(trial)
                if t < best * (1.0 - min_gain):
                    best, cur, changed = t, trial, True
        if not changed:
            break
    return cur


# ---- table I/O and application ----------------------------------------------

def launch_settings() -> dict:
    lib = _native.load()
    names = _native.kernel_names()
    return {n: lib.fvb_get_launch_ctas(i) for i, n in enumerate(names) if lib.fvb_get_launch_ctas(i) >= 0}


def set_launch(settings: dict) -> None:
    lib = _native.load()
    names = _native.kernel_names()
    for name, value in settings.items():
        _native.check(lib.fvb_set_launch_ctas(names.index(name), int(value)))


def reset_launch() -> None:
    set_launch({n: 0 for n in launch_settings()})


def load(path: Path | str = TABLE) -> dict:
    return json.loads(Path(path).read_text())


def save(table: dict, path: Path | str = TABLE) -> None:
    Path(path).parent.mkdir(parents=True, exist_ok=True)
    Path(path).write_text(json.dumps(table, indent=1, sort_keys=True) + "\n")


def wavefront_block() -> int:
    return int(_native.load().fvb_get_wavefront_block())


def set_wavefront_block(steps: int) -> None:
    _native.check(_native.load().fvb_set_wavefront_block(int(steps)))


def tile_warps() -> int:
    return int(_native.load().fvb_get_tile_warps())


def set_tile_warps(warps: int) -> None:
    _native.check(_native.load().fvb_set_tile_warps(int(warps)))


def decode_overlap() -> int:
    return int(_native.load().fvb_get_decode_overlap())


def set_decode_overlap(on: int) -> None:
    _native.check(_native.load().fvb_set_decode_overlap(int(on)))


def rans_pipeline() -> int:
    return int(_native.load().fvb_get_rans_pipeline())


def set_rans_pipeline(steps: int) -> None:
    _native.check(_native.load().fvb_set_rans_pipeline(int(steps)))


def rans_pipeline_tail() -> int:
    return int(_native.load().fvb_get_rans_pipeline_tail())


def set_rans_pipeline_tail(steps: int) -> None:
    _native.check(_native.load().fvb_set_rans_pipeline_tail(int(steps)))


def apply(table: dict) -> None:
    """Set the table's launch geometry, wavefront block, warps per tile,
    decode overlap and rANS encoder pipelines (process-wide)."""
    set_launch(table.get("launch", {}))
    set_wavefront_block(table.get("wavefront_block", 0))
    set_tile_warps(table.get("tile_warps", 0))
    set_decode_overlap(table.get("decode_overlap", 1))
    set_rans_pipeline(table.get("rans_pipeline", -1))
    set_rans_pipeline_tail(table.get("rans_pipeline_tail", -1))


def tile_for(table: dict | None, layout: str, bit_depth: int, width: int, height: int, default=(256, 128)):
    if table:
        t = table.get("tiles", {}).get(format_key(layout, bit_depth, width, height))
        if t:
            return tuple(t)
    return tuple(default)


# ---- measurement (GPU) --------------------------------------------------------

def _time_batch(codec, frames, params, reps: int) -> tuple[float, int]:
    """Median ms of encode+decode of the batch, and its stream bytes."""
    import torch

    def once():
        streams = codec.encode(frames, **params)
        codec.decode(streams)
        torch.cuda.current_stream(codec.device).synchronize()
        return sum(int(s.numel()) for s in streams)

    nbytes = once()
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        once()
        times.append((time.perf_counter() - t0) * 1e3)
    return statistics.median(times), nbytes


def tune_launch(codec, frames, params, knobs=LAUNCH_KNOBS, candidates=LAUNCH_CANDIDATES, reps: int = 3) -> dict:
    current = launch_settings()
    start = {k: current[k] for k in knobs}

    def measure(setting):
        set_launch(setting)
        return _time_batch(codec, frames, params, reps)[0]

    best = descend(knobs, candidates, measure, start)
    set_launch(best)
    return best


def tune_wavefront_block(codec, frames, params, candidates=WAVEFRONT_BLOCKS, reps: int = 3) -> tuple[int, dict]:
    """The wavefront block with the lowest measured batch time (the launch
    caps as currently set); returns it and every candidate's ms."""
    seen = {}
    for steps in candidates:
        set_wavefront_block(steps)
        seen[steps] = _time_batch(codec, frames, params, reps)[0]
    best = min(seen, key=seen.get)
    set_wavefront_block(best)
    return best, {str(k): round(v, 3) for k, v in seen.items()}


def tune_rans_pipeline(codec, frames, params, reps: int = 3, tail: bool = False) -> tuple[int, dict]:
    """The rANS encoder's fetch scheme (-1 automatic, 0, 8, 16) with the
    lowest batch time, for the first encoder pass or (tail) the later ones;
    the automatic choice wins ties."""
    setter = set_rans_pipeline_tail if tail else set_rans_pipeline
    seen = {}
    for steps in (-1, 0, 8, 16):
        setter(steps)
        seen[steps] = _time_batch(codec, frames, params, reps)[0]
    best = min(seen, key=seen.get)
    setter(best)
    return best, {str(k): round(v, 3) for k, v in seen.items()}


def tune_decode_overlap(codec, frames, params, reps: int = 3) -> tuple[int, dict]:
    """dec_other beside dec_rans (1) or after it (0), whichever is faster;
    measured after the launch caps, which decide how the two share SMs."""
    seen = {}
    for on in (1, 0):
        set_decode_overlap(on)
        seen[on] = _time_batch(codec, frames, params, reps)[0]
    best = min(seen, key=seen.get)
    set_decode_overlap(best)
    return best, {str(k): round(v, 3) for k, v in seen.items()}


def tune_tile_warps(codec, frames, params, candidates=TILE_WARPS, reps: int = 3) -> tuple[int, dict]:
    """One warp or a warp pair per tile, whichever measures faster."""
    seen = {}
    for warps in candidates:
        set_tile_warps(warps)
        seen[warps] = _time_batch(codec, frames, params, reps)[0]
    best = min(seen, key=seen.get)
    set_tile_warps(best)
    return best, {str(k): round(v, 3) for k, v in seen.items()}


def tune_tiles(codec, groups: dict, candidates=TILE_CANDIDATES, size_tolerance: float = 0.02,
               reps: int = 3) -> tuple[dict, dict]:
    """groups: {format_key: (frames, params without tile_size)}.  Returns the
    chosen tile per format and the measurements {format_key: {tile: (ms, bytes)}}."""
    chosen, seen = {}, {}
    for key, (frames, params) in groups.items():
        res = {}
        for tile in candidates:
            res[tuple(tile)] = _time_batch(codec, frames, dict(params, tile_size=tuple(tile)), reps)
        seen[key] = {f"{t[0]}x{t[1]}": [round(v[0], 3), v[1]] for t, v in res.items()}
        chosen[key] = list(choose_tile(res, size_tolerance))
    return chosen, seen


def main(argv=None) -> int:
    import argparse

    import torch

    from . import synth
    from .batch import BatchCodec

    p = argparse.ArgumentParser(description="autotune tile and launch geometry on this GPU")
    p.add_argument("--frames", type=int, default=24, help="frames of the sample mix (the 96-frame mix, scaled)")
    p.add_argument("--size-tolerance", type=float, default=0.02)
    p.add_argument("--reps", type=int, default=3)
    p.add_argument("--out", default=str(TABLE))
    args = p.parse_args(argv)

    specs = synth.mixed_batch_specs(args.frames)
    dev = torch.device("cuda", torch.cuda.current_device())
    codec = BatchCodec(dev, use_graphs=False)
    host = [synth.frame_from_spec(s) for s in specs]
    frames = [tuple(torch.from_numpy(p).to(dev) for p in f) for f in host]
    groups: dict = {}
    for s, f in zip(specs, frames):
        key = format_key(s["layout"], s["bit_depth"], s["width"], s["height"])
        g = groups.setdefault(key, ([], dict(layout=s["layout"], bit_depth=s["bit_depth"], quality=s["quality"])))
        g[0].append(f)
    reset_launch()
    tiles, measured = tune_tiles(codec, groups, size_tolerance=args.size_tolerance, reps=args.reps)
    params = dict(layout=[s["layout"] for s in specs], bit_depth=[s["bit_depth"] for s in specs],
                  quality=[s["quality"] for s in specs],
                  tile_size=[tuple(tiles[format_key(s["layout"], s["bit_depth"], s["width"], s["height"])])
                             for s in specs])
    base_ms = _time_batch(codec, frames, params, args.reps)[0]
    block, block_ms = tune_wavefront_block(codec, frames, params, reps=args.reps)
    warps, warps_ms = tune_tile_warps(codec, frames, params, reps=args.reps)
    pipe, pipe_ms = tune_rans_pipeline(codec, frames, params, reps=args.reps)
    pipe_tail, pipe_tail_ms = tune_rans_pipeline(codec, frames, params, reps=args.reps, tail=True)
    launch = tune_launch(codec, frames, params, reps=args.reps)
    overlap, overlap_ms = tune_decode_overlap(codec, frames, params, reps=args.reps)
    tuned_ms = _time_batch(codec, frames, params, args.reps)[0]
    table = {"device": torch.cuda.get_device_name(dev), "sample": f"{args.frames}-frame mix",
             "size_tolerance": args.size_tolerance, "tiles": tiles, "tile_measurements_ms_bytes": measured,
             "wavefront_block": block, "wavefront_block_ms": block_ms,
             "tile_warps": warps, "tile_warps_ms": warps_ms,
             "rans_pipeline": pipe, "rans_pipeline_ms": pipe_ms,
             "rans_pipeline_tail": pipe_tail, "rans_pipeline_tail_ms": pipe_tail_ms,
             "decode_overlap": overlap, "decode_overlap_ms": overlap_ms,
             "launch": launch, "launch_gain": {"default_ms": round(base_ms, 3), "tuned_ms": round(tuned_ms, 3)}}
    save(table, args.out)
    print(json.dumps(table))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
