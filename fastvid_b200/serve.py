"""Serving form: a request loop with continuous batching under a device
memory budget.

Requests (encode a frame, decode a stream) are submitted from any thread and
answered through futures.  A few worker threads, each with its own CUDA
stream and its own resident workspace, take turns forming batches: a worker
that comes free takes the oldest pending request and every later pending
request of the same kind that still fits the batch limits and the memory
budget, and runs them through the batched kernels (one launch per kernel for
the whole batch).  Requests that arrive while batches are on the GPU are
admitted into the next batch of the next free worker, so their work overlaps
on the device with the batches already running.  Each result is the same as
the single-frame path's for that request alone.

Memory accounting (bytes on the device): each worker's resident workspace
(it grows to the largest batch that worker ran and is kept, so steady state
allocates no workspace) plus the outputs of batches in flight.  A batch is
admitted only if that total stays within the budget; a request that does not
fit an empty server is rejected with MemoryError.  Outputs belong to the
caller once delivered.

The reference has no served form: fastvid.encode/decode of a list loop over
single-frame calls (fastvid/__init__.py:44-53, 59-63).
"""

from __future__ import annotations

import collections
import ctypes
import itertools
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import torch

from . import _native
from ._native import Frame
from .codec import _LAYOUTS_DEFAULT, header_of, plan_decode, plan_encode


@dataclass
class Request:
    kind: str                      # "encode" | "decode"
    payload: object                # planes tuple (encode) or 1-D uint8 stream (decode)
    params: dict
    pixels: int                    # luma pixels (W * H)
    ws_bytes: int                  # workspace of this request alone (a batch needs at most the sum)
    out_bytes: int                 # device bytes of its output (encode: the stream bound)
    future: Future = field(default_factory=Future)
    arrival: float = 0.0
    rid: int = 0


@dataclass
class Done:
    """Timing record of an answered request (results are not kept)."""
    rid: int
    kind: str
    pixels: int
    arrival: float
    done: float
    ok: bool


class CodecBackend:
    """The batched CUDA codec behind a server: one BatchCodec with a
    resident workspace per worker."""

    def __init__(self, device):
        self.device = torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.lib = _native.load()
        self._ws_cache: dict = {}
        self._plans: dict = {}    # request parameters and plane shapes -> Frame

    # ---- sizing (host only) ----
    # A batch runs in its shape bucket's workspace: every count rounded up
    # by at most 25 percent, with small floors; admission charges that bound.
    @staticmethod
    def _bucketed(ws: int) -> int:
        return ws + ws // 4 + (2 << 20)

    def _encode_ws(self, frame: Frame) -> int:
        key = ("e", frame.layout, frame.bit_depth, frame.width, frame.height, frame.tile_w, frame.tile_h)
        ws = self._ws_cache.get(key)
        if ws is None:
            arr = (Frame * 1)(frame)
            v = ctypes.c_int64()
            _native.check(self.lib.fvb_batch_encode_plan(arr, 1, ctypes.byref(v)))
            ws = self._ws_cache[key] = v.value
        return ws

    def _decode_ws(self, frame: Frame) -> int:
        key = ("d", frame.layout, frame.bit_depth, frame.width, frame.height, frame.tile_w, frame.tile_h)
        ws = self._ws_cache.get(key)
        if ws is None:
            arr = (Frame * 1)(frame)
            v = ctypes.c_int64()
            _native.check(self.lib.fvb_batch_decode_plan(arr, 1, ctypes.byref(v)))
            ws = self._ws_cache[key] = v.value
        return ws

    def encode_request(self, planes, *, layout=None, bit_depth=10, quality=90, frame_rate=(24, 1),
                       tile_size=(256, 128)) -> Request:
        planes = (planes,) if isinstance(planes, torch.Tensor) else tuple(planes)
        lay = layout
        if lay is None:
            lay = 0 if len(planes) == 1 else (1 if planes[1].shape[1] != planes[0].shape[1] else 2)
        elif isinstance(lay, str):
            lay = _LAYOUTS_DEFAULT[lay]
        key = ("e", lay, bit_depth, quality, tuple(frame_rate), tuple(tile_size),
               tuple((p.shape, p.dtype, p.device, p.stride()) for p in planes))
        frame = self._plans.get(key)
        if frame is None:
            frame = plan_encode(list(planes), lay, bit_depth, quality, frame_rate[0], frame_rate[1],
                                tile_size[0], tile_size[1])[0]
            if len(self._plans) < 4096:
                self._plans[key] = frame
        params = dict(layout=lay, bit_depth=bit_depth, quality=quality, frame_rate=tuple(frame_rate),
                      tile_size=tuple(tile_size))
        return Request("encode", planes, params, frame.width * frame.height, self._bucketed(self._encode_ws(frame)),
                       frame.max_stream_bytes)

    def decode_request(self, stream: torch.Tensor, header: bytes | None = None,
                       predictor: str = "wavefront") -> Request:
        if predictor not in ("wavefront", "serial"):
            raise ValueError("predictor must be 'wavefront' or 'serial'")
        if header is None:
            header = header_of(stream)
        header = bytes(header[:32])
        key = ("d", header, stream.numel(), stream.dtype, stream.dim())
        frame = self._plans.get(key)
        if frame is None:
            frame = plan_decode(stream, header=header)[0]
            if len(self._plans) < 4096:
                self._plans[key] = frame
        return Request("decode", stream, dict(predictor=predictor, header=header), frame.width * frame.height,
                       self._bucketed(self._decode_ws(frame)), 2 * frame.samples)

    # ---- execution (worker threads) ----
    def make_worker_codec(self):
        from .batch import BatchCodec

        # Eager launches (one per kernel per batch, sized by the batch's
        # shape bucket).  Workers do not capture CUDA graphs: torch's capture
        # entry synchronizes the device and empties the allocator's cache,
        # which is not safe beside the other workers' batches in flight; a
        # full-size serving run that captured inside the workers hit an
        # illegal memory access.
        return BatchCodec(self.device, use_graphs=False, resident_workspace=True, max_cached_shapes=32)

    def resident_bytes(self, codec) -> int:
        return codec.workspace_bytes()

    def largest_workspace(self, max_pixels: int) -> int:
        """Workspace bytes (bucket-rounded) of the largest batch a worker may
        run: max_pixels luma pixels of rgb444 (three samples per pixel, the
        most samples per pixel) in 64x64 tiles, encode or decode, whichever
        needs more.  (Batches of smaller tiles hold more shard records and
        rANS scratch and may still grow the workspace.)"""
        side = 4096
        height = max(1, -(-max_pixels // side))
        frame = Frame()
        ws = ctypes.c_int64()
        _native.check(self.lib.fvb_encode_plan(side, height, 2, 16, 90, 24, 1, 64, 64, ctypes.byref(frame),
                                               ctypes.byref(ws)))
        arr = (Frame * 1)(frame)
        dws = ctypes.c_int64()
        _native.check(self.lib.fvb_batch_decode_plan(arr, 1, ctypes.byref(dws)))
        return self._bucketed(max(ws.value, dws.value))

    def presize(self, codec, nbytes: int) -> int:
        """Allocate the worker's resident workspace up front; returns its bytes."""
        codec._workspace(nbytes)
        return codec.workspace_bytes()

    def release(self, codec):
        codec.release_workspace()

    def run(self, codec, kind: str, reqs: list[Request]) -> list:
        if kind == "encode":
            out = codec.encode([r.payload for r in reqs], layout=[r.params["layout"] for r in reqs],
                               bit_depth=[r.params["bit_depth"] for r in reqs],
                               quality=[r.params["quality"] for r in reqs],
                               frame_rate=[r.params["frame_rate"] for r in reqs],
                               tile_size=[r.params["tile_size"] for r in reqs])
        else:
            out = codec.decode([r.payload for r in reqs], predictor=reqs[0].params["predictor"],
                               headers=[r.params["header"] for r in reqs])
        torch.cuda.current_stream(self.device).synchronize()  # answers are complete when delivered
        return out

    def warm(self, nbytes: int):
        """Allocate and free `nbytes` on the calling worker's stream, so the
        caching allocator serves that worker's later outputs from cached
        memory: growing the pool mid-run (cudaMalloc) stalled single batches
        for tens of milliseconds."""
        if nbytes > 0:
            block = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
            del block

    def stream(self):
        return torch.cuda.Stream(self.device)

    def bind(self, stream):
        torch.cuda.set_device(self.device)
        torch.cuda.set_stream(stream)


class Server:
    """Continuous-batching request loop on one device.

    workers: batches that may be on the GPU at once (one CUDA stream each).
    memory_budget: device bytes for resident workspaces plus the outputs of
    batches in flight.  max_batch_frames / max_batch_pixels bound one batch.
    """

    def __init__(self, device=None, *, memory_budget: int = 40 << 30, workers: int = 3,
                 max_batch_frames: int = 64, max_batch_pixels: int = 200_000_000, backend=None,
                 warm_bytes: int | None = None):
        """warm_bytes: device memory each worker allocates and frees once at
        start on its own stream (default: half the budget shared among the
        workers, at most 8 GiB each), so outputs come from the allocator's
        cache.
        Each worker also allocates its resident workspace for the largest
        batch it may run (max_batch_pixels) at start when all workers' fit
        in half the budget, so the workspace never grows mid-run."""
        self.backend = backend if backend is not None else CodecBackend(device if device is not None else "cuda")
        self.budget = int(memory_budget)
        self.warm_bytes = (min(8 << 30, self.budget // (2 * workers)) if warm_bytes is None else int(warm_bytes))
        self.presize_bytes = 0
        if hasattr(self.backend, "largest_workspace"):
            need = self.backend.largest_workspace(max_batch_pixels)
            if need * workers <= self.budget // 2:
                self.presize_bytes = need
        self.max_frames = max_batch_frames
        self.max_pixels = max_batch_pixels
        self._pending: collections.deque[Request] = collections.deque()
        self._cv = threading.Condition()
        self._closing = False
        self._broken: BaseException | None = None
        self._resident = [0] * workers       # workspace bytes held per worker
        self._inflight = 0                   # output bytes of batches running
        self._running = 0                    # batches on the GPU
        self.completed: list[Done] = []    # one record per answer, in answer order
        self._rids = itertools.count()
        self.batches: list[tuple[str, int]] = []  # (kind, size) of every batch run
        self.batch_times: list[tuple[float, float, str, int, int]] = []  # (start, end, kind, size, pixels)
        self.max_concurrent = 0
        self.peak_charged = 0  # largest resident + in-flight bytes charged against the budget
        self._threads = [threading.Thread(target=self._worker, args=(i,), daemon=True) for i in range(workers)]
        for t in self._threads:
            t.start()

    # ---- submission ----
    def _submit(self, req: Request) -> Future:
        req.arrival = time.perf_counter()
        req.rid = next(self._rids)
        req.future.rid = req.rid
        if req.ws_bytes + req.out_bytes > self.budget:
            req.future.set_exception(MemoryError(
                f"request needs {req.ws_bytes + req.out_bytes} device bytes, above the server budget "
                f"of {self.budget}"))
            return req.future
        with self._cv:
            if self._closing:
                raise RuntimeError("server is closed")
            if self._broken is not None:
                raise RuntimeError(f"serving worker failed: {self._broken!r}")
            self._pending.append(req)
            self._cv.notify_all()
        return req.future

    def submit_encode(self, planes, **params) -> Future:
        """Encode one frame (CUDA uint16 planes, the fastvid_cuda.encode
        arguments); the future yields the 1-D CUDA uint8 stream."""
        return self._submit(self.backend.encode_request(planes, **params))

    def submit_decode(self, stream, header: bytes | None = None, predictor: str = "wavefront") -> Future:
        """Decode one stream; the future yields the tuple of planes.  `header`
        (the stream's first 32 bytes) saves a device read when known."""
        return self._submit(self.backend.decode_request(stream, header, predictor))

    def close(self, wait: bool = True):
        with self._cv:
            self._closing = True
            self._cv.notify_all()
        if wait:
            for t in self._threads:
                t.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- scheduling ----
    def _take_batch(self, w: int):
        """Pop the next batch for worker w, or None if nothing fits yet.
        Called with the lock held."""
        head = self._pending[0]
        kind = head.kind
        key = head.params.get("predictor")
        others = sum(self._resident) - self._resident[w]
        chosen, ws, out, pixels = [], 0, 0, 0
        for req in self._pending:
            if req.kind != kind or req.params.get("predictor") != key:
                continue
            if len(chosen) >= self.max_frames or (chosen and pixels + req.pixels > self.max_pixels):
                break
            need = others + max(self._resident[w], ws + req.ws_bytes) + self._inflight + out + req.out_bytes
            if need > self.budget:
                break
            chosen.append(req)
            ws += req.ws_bytes
            out += req.out_bytes
            pixels += req.pixels
        if not chosen:
            return None
        ids = {id(r) for r in chosen}
        self._pending = collections.deque(r for r in self._pending if id(r) not in ids)
        self._resident[w] = max(self._resident[w], ws)  # reserved before the workspace grows
        self._inflight += out
        self._running += 1
        self.max_concurrent = max(self.max_concurrent, self._running)
        self.peak_charged = max(self.peak_charged, sum(self._resident) + self._inflight)
        return kind, chosen, out

    def _worker(self, w: int):
        try:
            self._serve(w)
        except BaseException as exc:  # a worker that cannot go on fails what it would have answered
            with self._cv:
                self._broken = exc
                pending, self._pending = list(self._pending), collections.deque()
                self._cv.notify_all()
            for r in pending:
                if not r.future.done():
                    r.future.set_exception(RuntimeError(f"serving worker failed: {exc!r}"))

    def _serve(self, w: int):
        stream = self.backend.stream()
        self.backend.bind(stream)
        if hasattr(self.backend, "warm"):
            self.backend.warm(self.warm_bytes)
        codec = self.backend.make_worker_codec()
        if self.presize_bytes:
            held = self.backend.presize(codec, self.presize_bytes)
            with self._cv:
                self._resident[w] = held
                self.peak_charged = max(self.peak_charged, sum(self._resident) + self._inflight)
        while True:
            release = False
            with self._cv:
                batch = None
                while batch is None:
                    if self._pending:
                        batch = self._take_batch(w)
                        if batch is not None:
                            break
                        if self._running == 0 and self._resident[w] > 0:
                            # nothing runs and the oldest request does not fit
                            # beside the idle workers' workspaces: give this
                            # one back (a request that fits an empty server
                            # is then always admitted)
                            self._resident[w] = 0
                            release = True
                            break
                    elif self._closing:
                        return
                    self._cv.wait()
            if release:
                self.backend.release(codec)
                with self._cv:
                    self._cv.notify_all()
                continue
            kind, reqs, out = batch
            t_start = time.perf_counter()
            self._run(codec, kind, reqs)
            t_end = time.perf_counter()
            with self._cv:
                self.batch_times.append((t_start, t_end, kind, len(reqs), sum(r.pixels for r in reqs)))
                self._inflight -= out
                self._running -= 1
                self._resident[w] = max(self.backend.resident_bytes(codec), 0)
                self.peak_charged = max(self.peak_charged, sum(self._resident) + self._inflight)
                self.batches.append((kind, len(reqs)))
                self._cv.notify_all()

    def _run(self, codec, kind: str, reqs: list[Request]):
        try:
            results = self.backend.run(codec, kind, reqs)
        except Exception:
            if len(reqs) == 1:
                self._finish(reqs[0], exc=_current_exception())
                return
            # a failing frame fails its batch: answer every request alone
            for r in reqs:
                try:
                    (res,) = self.backend.run(codec, kind, [r])
                except Exception:
                    self._finish(r, exc=_current_exception())
                else:
                    self._finish(r, res)
            return
        for r, res in zip(reqs, results):
            self._finish(r, res)

    def _finish(self, req: Request, result=None, exc=None):
        rec = Done(req.rid, req.kind, req.pixels, req.arrival, time.perf_counter(), exc is None)
        with self._cv:
            self.completed.append(rec)
        if exc is not None:
            req.future.set_exception(exc)
        else:
            req.future.set_result(result)


def _current_exception():
    import sys

    return sys.exc_info()[1]


# ---- latency / throughput report --------------------------------------------

def percentile(values, q: float) -> float:
    """Nearest-rank percentile of a non-empty sequence (q in 0..100)."""
    v = sorted(values)
    k = max(0, min(len(v) - 1, int(-(-q * len(v) // 100)) - 1))
    return v[k]


def report(records: list[Done], t0: float) -> dict:
    lat = [(r.done - r.arrival) * 1e3 for r in records]
    end = max(r.done for r in records)
    pixels = sum(r.pixels for r in records)
    return {
        "requests": len(records),
        "failed": sum(not r.ok for r in records),
        "gpix_s": pixels / (end - t0) / 1e9,
        "p50_ms": percentile(lat, 50),
        "p99_ms": percentile(lat, 99),
        "max_ms": max(lat),
        "wall_s": end - t0,
    }


def run_open_loop(server: Server, items, rate: float | None, seed: int = 0, keep=()):
    """Submit `items` -- (kind, payload, params) -- at Poisson arrivals of
    `rate` per second (None: all at once).  Answers are dropped as they come
    in, except those whose item index is in `keep`: a set of indices (the
    answer is copied into new device memory) or a dict {index: destination}
    of tensors (or tuples of tensors) of the answers' shapes, allocated
    before the run, that the answer is copied into -- so keeping answers
    allocates nothing while the server runs.  Returns (records of these
    requests in item order, t0, {index: kept answer})."""
    import random

    rng = random.Random(seed)
    into = dict(keep) if isinstance(keep, dict) else {}
    keep = set(keep)
    kept: dict = {}
    rids = []
    remaining = [len(items)]
    lock = threading.Lock()
    all_done = threading.Event()

    def answered(_f):
        with lock:
            remaining[0] -= 1
            if remaining[0] == 0:
                all_done.set()

    def copy(answer, dst=None):
        # an answer is a view of its batch's output arena; a copy lets the
        # arena go back to the allocator (the callback runs on the worker's
        # thread, so the copy is ordered on the worker's stream before any
        # reuse of the arena)
        if isinstance(answer, torch.Tensor):
            if dst is None:
                return answer.clone()
            if dst.shape != answer.shape or dst.dtype != answer.dtype:
                raise ValueError("kept answer does not match its destination")
            return dst.copy_(answer)
        if isinstance(answer, tuple):
            return tuple(copy(a, None if dst is None else d) for a, d in zip(answer, dst or (None,) * len(answer)))
        return answer

    devices = set()

    def keeper(i):
        def done(f):
            if f.exception() is None:
                res = f.result()
                kept[i] = copy(res, into.get(i))
                for a in (res if isinstance(res, tuple) else (res,)):
                    if isinstance(a, torch.Tensor) and a.is_cuda:
                        devices.add(a.device)
        return done

    t0 = time.perf_counter()
    t = t0
    for i, (kind, payload, params) in enumerate(items):
        if rate:
            t += rng.expovariate(rate)
            delay = t - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
        fut = server.submit_encode(payload, **params) if kind == "encode" else server.submit_decode(payload, **params)
        rids.append(fut.rid)
        if i in keep:
            fut.add_done_callback(keeper(i))
        fut.add_done_callback(answered)  # answers are released with their futures
    if items:
        all_done.wait()
    for dev in devices:  # the kept copies are complete on return
        torch.cuda.synchronize(dev)
    want = set(rids)
    with server._cv:
        got = {r.rid: r for r in server.completed if r.rid in want}
    return [got[r] for r in rids], t0, kept
