"""Batched encode/decode: every frame of a batch in one launch of each kernel.

The reference batches with a Python loop of single-frame calls
(fastvid/__init__.py:44-53, 63), each paying its own host synchronisations.
Here a batch of frames of any mix of sizes, layouts and depths goes through
one persistent launch per kernel: the predictor and reconstruction kernels
drain a device work queue of tiles from all frames, the analysis, rANS and
emission kernels cover every shard of every frame, and the frame policy runs
on the device.  Launches are sized by a shape bucket -- the batch's frame,
tile, shard and sample counts rounded up to steps of at most 25 percent
(fvb_batch_bucket) -- and the kernels read the batch's actual counts from the
workspace, so the analysis passes and the decode of a bucket are captured
once as CUDA graphs and replayed for every batch that falls into it, whatever
its mix of frames.  The host waits once per batch (the stream lengths), then
launches emission into one exact-size arena.  Streams are byte-identical to
the single-frame path frame by frame.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import torch

from . import _native
from ._native import Bucket, Frame
from .codec import _LAYOUTS_DEFAULT, plan_encode, plan_decode, plane_views


def _per_frame(value, n, name):
    if isinstance(value, (list, tuple)) and len(value) == n and not (
            name in ("tile_size", "frame_rate") and len(value) == 2 and isinstance(value[0], int)):
        return list(value)
    return [value] * n


@dataclass
class _Slot:
    """Cached resources of one shape bucket (encode or decode)."""
    bucket: Bucket
    ws_bytes: int
    workspace: torch.Tensor
    results: torch.Tensor            # pinned int64 [bucket.frames, 2]
    wavefront: bool = True
    headers: torch.Tensor | None = None  # encode: pinned uint8 [bucket.frames * 32], written by a kernel
    graph: torch.cuda.CUDAGraph | None = None
    stream: torch.cuda.Stream | None = None
    kernels: int = 0                 # kernel launches captured in the graph


class BatchCodec:
    """Batched encoder/decoder bound to one CUDA device.

    Resources (workspace, pinned result buffer, CUDA graph) are cached per
    shape bucket, so steady-state calls of batches falling into a seen bucket
    allocate nothing but their outputs and issue one graph launch for all
    analysis passes (and one for the whole decode).
    """

    def __init__(self, device=None, use_graphs: bool = True, max_cached_shapes: int = 8,
                 resident_workspace: bool = False):
        """resident_workspace: every batch shape shares one device workspace
        that grows to the largest batch seen and is kept (a server's
        steady state allocates no workspace); otherwise each cached shape
        owns its own."""
        dev = torch.device(device) if device is not None else torch.device("cuda")
        if dev.type != "cuda":
            raise RuntimeError("BatchCodec needs a CUDA device")
        self.device = dev if dev.index is not None else torch.device("cuda", torch.cuda.current_device())
        self.use_graphs = use_graphs
        self.max_cached = max_cached_shapes
        self._enc: dict = {}
        self._dec: dict = {}
        self._plans: dict = {}
        self._dec_plans: dict = {}
        self._hdr_scratch = None
        self.lib = _native.load()
        self.resident = resident_workspace
        self._ws_buf: torch.Tensor | None = None
        self._pin_buf: torch.Tensor | None = None
        self.graph_kernels = 0  # kernels run by graph replays (launch_count() sees only direct launches)

    def _pinned_heads(self, n: int) -> torch.Tensor:
        """Pinned host buffer for n gathered 32-byte headers: the gather
        kernel writes it directly, so the read does not queue behind
        downloads in flight on other streams."""
        buf = getattr(self, "_heads_pin", None)
        if buf is None or buf.numel() < 32 * n:
            buf = torch.empty(max(32 * n, 4096), dtype=torch.uint8).pin_memory()
            self._heads_pin = buf
        return buf[:32 * n]

    def workspace_bytes(self) -> int:
        """Device bytes of the resident workspace (0 when not resident)."""
        return self._ws_buf.numel() if self._ws_buf is not None else 0

    def _results(self, n: int) -> torch.Tensor:
        """Pinned int64 [n, 2] status/length buffer (shared by every shape
        in resident mode, where calls run one at a time)."""
        if not self.resident:
            return torch.zeros((n, 2), dtype=torch.int64).pin_memory()
        if self._pin_buf is None or self._pin_buf.size(0) < n:
            self._pin_buf = torch.zeros((max(n, 64), 2), dtype=torch.int64).pin_memory()
        return self._pin_buf[:n]

    def release_workspace(self):
        """Drop the resident workspace (and the shapes cached on it)."""
        self._enc.clear()
        self._dec.clear()
        self._ws_buf = None

    def _workspace(self, nbytes: int) -> torch.Tensor:
        if not self.resident:
            return torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        if self._ws_buf is None or self._ws_buf.numel() < nbytes:
            # cached shapes (and their graphs) point into the old buffer;
            # calls return only once their work is done, so nothing uses it
            self._enc.clear()
            self._dec.clear()
            self._ws_buf = None
            self._ws_buf = torch.empty(max(nbytes, 1 << 20), dtype=torch.uint8, device=self.device)
        return self._ws_buf[:nbytes]

    # ---- buckets ----------------------------------------------------------
    def _frame_array(self, frames_py: list[Frame]):
        return (Frame * len(frames_py))(*frames_py)

    def _slot(self, cache: dict, arr, n: int, decode: bool, wavefront: bool = True) -> _Slot:
        bucket = Bucket()
        _native.check(self.lib.fvb_batch_bucket(arr, n, ctypes.byref(bucket)))
        key = (decode, wavefront) + bucket.key()
        slot = cache.get(key)
        if slot is not None:
            return slot
        ws = ctypes.c_int64()
        plan = self.lib.fvb_bucket_decode_plan if decode else self.lib.fvb_bucket_encode_plan
        _native.check(plan(ctypes.byref(bucket), ctypes.byref(ws)))
        workspace = self._workspace(ws.value)
        slot = _Slot(bucket, ws.value, workspace, self._results(bucket.frames), wavefront,
                     headers=None if decode else torch.empty(32 * bucket.frames, dtype=torch.uint8).pin_memory())
        if len(cache) >= self.max_cached:
            cache.pop(next(iter(cache)))
        cache[key] = slot
        return slot

    def _run_slot(self, slot: _Slot, enqueue, cur, graphs: bool = True) -> None:
        """Run `enqueue(stream_handle)` for this slot: captured as a graph on
        the slot's first use (after one eager run), replayed afterwards;
        launched directly when the codec or the call (`graphs`) says so."""
        if not (self.use_graphs and graphs):
            enqueue(cur.cuda_stream)
            return
        if slot.graph is None:
            slot.stream = torch.cuda.Stream(self.device)
            slot.stream.wait_stream(cur)
            # one eager run first (it sets kernel attributes), then capture
            with torch.cuda.stream(slot.stream):
                enqueue(slot.stream.cuda_stream)
            slot.stream.synchronize()
            graph = torch.cuda.CUDAGraph()
            k0 = _native.launch_count()
            # thread-local capture: other threads (serving workers) may keep
            # launching and allocating on their own streams meanwhile
            with torch.cuda.graph(graph, stream=slot.stream, capture_error_mode="thread_local"):
                enqueue(slot.stream.cuda_stream)
            slot.kernels = _native.launch_count() - k0
            slot.graph = graph
        else:
            slot.stream.wait_stream(cur)
            with torch.cuda.stream(slot.stream):
                slot.graph.replay()
            self.graph_kernels += slot.kernels
        cur.wait_stream(slot.stream)

    # ---- encode -----------------------------------------------------------
    @staticmethod
    def _enc_shape(f: Frame) -> tuple:
        return (f.layout, f.bit_depth, f.quality, f.width, f.height, f.tile_w, f.tile_h, f.fps_num, f.fps_den)

    def encode(self, frames, *, layout=None, bit_depth=10, quality=90, frame_rate=(24, 1), tile_size=(256, 128),
               arena: torch.Tensor | None = None, return_headers: bool = False, graphs: bool = True):
        """Encode a list of frames (each a tuple of CUDA uint16 planes).

        Scalar arguments apply to every frame; lists give one value per frame.
        `arena`: a device uint8 buffer the streams are written into when it
        is large enough (the caller keeps it alive and unused meanwhile).
        Returns a list of 1-D CUDA uint8 streams (views of one arena); with
        `return_headers`, also the streams' 32-byte headers (bytes), which
        decode(streams, headers=...) takes instead of reading them back.
        `graphs=False` launches directly even when the codec uses graphs (a
        capture must not meet another thread's work on the device).
        """
        frames = [tuple(f) if not isinstance(f, torch.Tensor) else (f,) for f in frames]
        n = len(frames)
        if n == 0:
            return []
        layouts = _per_frame(layout, n, "layout")
        depths = _per_frame(bit_depth, n, "bit_depth")
        qualities = _per_frame(quality, n, "quality")
        rates = _per_frame(frame_rate, n, "frame_rate")
        tiles = _per_frame(tile_size, n, "tile_size")
        plans, shapes, ptrs, pitches = [], [], [], []
        for i, planes in enumerate(frames):
            lay = layouts[i]
            if lay is None:
                lay = 0 if len(planes) == 1 else (1 if planes[1].shape[1] != planes[0].shape[1] else 2)
            elif isinstance(lay, str):
                lay = _LAYOUTS_DEFAULT[lay]
            # plan cache: the planes' shapes, strides, dtype and device index
            # decide every check of plan_encode
            key = (lay, depths[i], qualities[i], tuple(rates[i]), tuple(tiles[i]),
                   tuple((p.shape, p.stride(), p.dtype, p.get_device()) for p in planes))
            hit = self._plans.get(key)
            if hit is not None:
                frame, pit, shape = hit
                views = planes
            else:
                frame, _, views, pit = plan_encode(list(planes), lay, depths[i], qualities[i], rates[i][0],
                                                   rates[i][1], tiles[i][0], tiles[i][1])
                if views[0].device != self.device:
                    raise RuntimeError("all frames of a batch must be on the codec's device")
                shape = self._enc_shape(frame)
                if all(v is p for v, p in zip(views, planes)):  # no copy was needed: cacheable
                    self._plans[key] = (frame, pit, shape)
            plans.append(frame)
            shapes.append(shape)
            for v in views:
                ptrs.append(v.data_ptr())
            ptrs.extend((0,) * (3 - len(views)))
            pitches.extend(pit)
            pitches.extend((0,) * (3 - len(pit)))
        with torch.cuda.device(self.device):
            arr = self._frame_array(plans)
            slot = self._slot(self._enc, arr, n, decode=False)
            bucket = ctypes.byref(slot.bucket)
            cur = torch.cuda.current_stream(self.device)
            p_arr = (ctypes.c_void_p * (3 * n))(*ptrs)
            q_arr = (ctypes.c_int64 * (3 * n))(*pitches)
            _native.check(self.lib.fvb_bucket_encode_prepare(bucket, arr, n, p_arr, q_arr, slot.workspace.data_ptr(),
                                                             slot.ws_bytes, cur.cuda_stream))
            def enqueue(h):
                _native.check(self.lib.fvb_bucket_encode_enqueue(bucket, slot.workspace.data_ptr(), slot.ws_bytes,
                                                                 slot.results.data_ptr(), h))
                _native.check(self.lib.fvb_bucket_encode_headers(bucket, slot.workspace.data_ptr(), slot.ws_bytes,
                                                                 slot.headers.data_ptr(), h))

            self._run_slot(slot, enqueue, cur, graphs)
            cur.synchronize()
            res = slot.results[:n].tolist()
            for i, (status, _) in enumerate(res):
                if status:
                    raise RuntimeError(f"frame {i}: CUDA encoder analysis failed (status {status})")
            lengths = [length for _, length in res]
            total = sum(lengths)
            if arena is not None and arena.dtype == torch.uint8 and arena.device == self.device \
                    and arena.numel() >= total:
                arena = arena.narrow(0, 0, total)
            else:
                arena = torch.empty(total, dtype=torch.uint8, device=self.device)
            outs, off, base = [], 0, arena.data_ptr()
            for length in lengths:
                outs.append(base + off)
                off += length
            o_arr = (ctypes.c_void_p * n)(*outs)
            _native.check(self.lib.fvb_bucket_encode_emit(bucket, arr, n, slot.workspace.data_ptr(), slot.ws_bytes,
                                                          o_arr, cur.cuda_stream))
            views, off = [], 0  # made while the GPU emits
            for length in lengths:
                views.append(arena.narrow(0, off, length))
                off += length
            if return_headers:
                raw = slot.headers[:32 * n].numpy().tobytes()
                return views, [raw[32 * i:32 * i + 32] for i in range(n)]
        return views

    # ---- decode -----------------------------------------------------------
    @staticmethod
    def _dec_shape(f: Frame) -> tuple:
        return (f.layout, f.bit_depth, f.quality, f.flags, f.width, f.height, f.tile_w, f.tile_h)

    def decode(self, streams, predictor="wavefront", headers=None, arena: torch.Tensor | None = None,
               graphs: bool = True):
        """Decode a list of 1-D uint8 streams; returns a list of plane tuples.
        `headers`: the streams' first 32 bytes when the caller has them
        (saves reading them back from the device).  `arena`: a device
        uint16 buffer the planes are written into when it is large enough.
        `graphs=False` launches directly even when the codec uses graphs."""
        if predictor not in ("wavefront", "serial"):
            raise ValueError("predictor must be 'wavefront' or 'serial'")
        n = len(streams)
        if n == 0:
            return []
        dev_streams, host_heads = [], []
        for s in streams:
            if s.dtype != torch.uint8 or s.dim() != 1:
                raise RuntimeError("encoded must be a one-dimensional uint8 tensor")
            if s.numel() < 32:
                raise RuntimeError("truncated Fastvid header")
            s = s.contiguous()
            if s.device == self.device:
                dev_streams.append(s)
                host_heads.append(None)
            elif not s.is_cuda:
                # a host stream: its header is read here, its bytes uploaded
                # without blocking (ordered before the decode on this stream)
                host_heads.append(bytes(s[:32].numpy().tobytes()))
                with torch.cuda.device(self.device):
                    dev_streams.append(s.to(self.device, non_blocking=s.is_pinned()))
            else:
                dev_streams.append(s.to(self.device))
                host_heads.append(None)
        if headers is None and all(h is not None for h in host_heads):
            headers = host_heads
        with torch.cuda.device(self.device):
            cur = torch.cuda.current_stream(self.device)
            need = ((16 * n + 255) // 256) * 256 + 32 * n
            if self._hdr_scratch is None or self._hdr_scratch.numel() < need:
                self._hdr_scratch = torch.empty(max(need, 1 << 16), dtype=torch.uint8, device=self.device)
            s_arr = (ctypes.c_void_p * n)(*[s.data_ptr() for s in dev_streams])
            l_arr = (ctypes.c_int64 * n)(*[s.numel() for s in dev_streams])
            if headers is not None and len(headers) == n and all(len(h) >= 32 for h in headers):
                raw = b"".join(bytes(h[:32]) for h in headers)
            else:
                heads = self._pinned_heads(n)
                _native.check(self.lib.fvb_gather_headers(s_arr, l_arr, n, self._hdr_scratch.data_ptr(),
                                                          self._hdr_scratch.numel(), heads.data_ptr(),
                                                          cur.cuda_stream))
                raw = heads.numpy().tobytes()
            plans, shapes, sizes = [], [], []
            for i, s in enumerate(dev_streams):
                header = raw[32 * i:32 * i + 32]
                key = (header, s.numel())
                hit = self._dec_plans.get(key)
                if hit is None:
                    frame = plan_decode(s, header=header)[0]
                    cw = frame.plane_width[1] if frame.planes == 3 else 0
                    # (frame, shape key, samples, planes, width, chroma width, luma and chroma samples)
                    hit = (frame, self._dec_shape(frame), frame.samples, frame.planes, frame.width, cw,
                           frame.width * frame.height, cw * frame.height)
                    if len(self._dec_plans) < 65536:
                        self._dec_plans[key] = hit
                plans.append(hit)
                shapes.append(hit[1])
                sizes.append(hit[2])
            arr = self._frame_array([h[0] for h in plans])
            wavefront = predictor == "wavefront"
            slot = self._slot(self._dec, arr, n, decode=True, wavefront=wavefront)
            bucket = ctypes.byref(slot.bucket)
            total = sum(sizes)
            if arena is not None and arena.dtype == torch.uint16 and arena.device == self.device \
                    and arena.numel() >= total:
                arena = arena.narrow(0, 0, total)
            else:
                arena = torch.empty(total, dtype=torch.uint16, device=self.device)
            # plane pointers by arithmetic (Y, then Cb, then Cr of each frame);
            # the tensor views are made while the GPU decodes
            ptrs, pitches, off, base = [], [], 0, arena.data_ptr()
            for _, _, samples, planes_n, width, cw, y, c in plans:
                if planes_n == 3:
                    ptrs.extend((base + 2 * off, base + 2 * (off + y), base + 2 * (off + y + c)))
                    pitches.extend((width, cw, cw))
                else:
                    ptrs.extend((base + 2 * off, 0, 0))
                    pitches.extend((width, 0, 0))
                off += samples
            p_arr = (ctypes.c_void_p * (3 * n))(*ptrs)
            q_arr = (ctypes.c_int64 * (3 * n))(*pitches)
            _native.check(self.lib.fvb_bucket_decode_prepare(bucket, arr, n, s_arr, l_arr, p_arr, q_arr,
                                                             slot.workspace.data_ptr(), slot.ws_bytes,
                                                             cur.cuda_stream))
            self._run_slot(slot, lambda h: _native.check(self.lib.fvb_bucket_decode_enqueue(
                bucket, 1 if wavefront else 0, slot.workspace.data_ptr(), slot.ws_bytes, slot.results.data_ptr(),
                h)), cur, graphs)
            out_planes = []
            off = 0
            for f, _, samples, *_ in plans:
                out_planes.append(tuple(plane_views(arena.narrow(0, off, samples), f)))
                off += samples
            cur.synchronize()
            for i, (status, _) in enumerate(slot.results[:n].tolist()):
                if status:
                    raise RuntimeError(f"frame {i}: malformed entropy payload (CUDA status {status})")
        return out_planes


    # ---- host buffers, pipelined ------------------------------------------
    def encode_host(self, frames, *, chunk: int = 16, out: torch.Tensor | None = None, **params):
        """Encode frames held in (preferably pinned) host memory; returns the
        streams in pinned host memory: views of `out` (a pinned uint8 tensor
        the caller allocates once and reuses -- pinning memory costs far more
        than the copies) while it has room, else of new pinned buffers.

        The batch runs in chunks of `chunk` frames: chunk i+2 is copied to the
        device and chunk i-1's streams are copied back while chunk i is
        encoded, on two copy streams beside the compute stream, so transfers
        in both directions overlap the kernels.  Other arguments as encode();
        per-frame lists are split with the frames.  Streams are identical to
        encode()'s.
        """
        n = len(frames)
        if n == 0:
            return []
        frames = [tuple(f) if not isinstance(f, torch.Tensor) else (f,) for f in frames]
        per = {k: _per_frame(v, n, k) for k, v in params.items()}
        with torch.cuda.device(self.device):
            comp = torch.cuda.current_stream(self.device)
            h2d, d2h = torch.cuda.Stream(self.device), torch.cuda.Stream(self.device)
            h2d.wait_stream(comp)
            d2h.wait_stream(comp)
            bounds = list(range(0, n, chunk)) + [n]
            staged: dict = {}

            def stage(i):
                lo, hi = bounds[i], bounds[i + 1]
                with torch.cuda.stream(h2d):
                    dev = [tuple(p.to(self.device, non_blocking=True) for p in f) for f in frames[lo:hi]]
                    ev = torch.cuda.Event()
                    ev.record(h2d)
                staged[i] = (dev, ev)

            res, cursor = [], 0
            nchunks = len(bounds) - 1
            for i in range(min(2, nchunks)):
                stage(i)
            for i in range(nchunks):
                dev, ev = staged.pop(i)
                comp.wait_event(ev)
                for f in dev:
                    for p in f:
                        p.record_stream(comp)
                lo, hi = bounds[i], bounds[i + 1]
                streams = self.encode(dev, **{k: v[lo:hi] for k, v in per.items()})
                if i + 2 < nchunks:
                    stage(i + 2)
                done = torch.cuda.Event()
                done.record(comp)
                total = sum(int(s.numel()) for s in streams)
                if out is not None and cursor + total <= out.numel():
                    host = out.narrow(0, cursor, total)
                    cursor += total
                else:
                    host = torch.empty(total, dtype=torch.uint8, pin_memory=True)
                arena = streams[0]._base if streams[0]._base is not None else streams[0]
                with torch.cuda.stream(d2h):
                    d2h.wait_event(done)
                    arena.record_stream(d2h)
                    host.copy_(arena.narrow(0, 0, total), non_blocking=True)
                off = 0
                for st in streams:
                    res.append(host.narrow(0, off, st.numel()))
                    off += st.numel()
            d2h.synchronize()
        return res

    def decode_host(self, streams, *, chunk: int = 16, predictor: str = "wavefront",
                    out: torch.Tensor | None = None):
        """Decode streams held in (preferably pinned) host memory; returns
        each frame's planes in pinned host memory -- views of `out` (a pinned
        uint16 tensor reused across calls) while it has room -- pipelined
        like encode_host (uploads of chunk i+2 and downloads of chunk i-1
        overlap the decode of chunk i)."""
        n = len(streams)
        if n == 0:
            return []
        with torch.cuda.device(self.device):
            comp = torch.cuda.current_stream(self.device)
            h2d, d2h = torch.cuda.Stream(self.device), torch.cuda.Stream(self.device)
            h2d.wait_stream(comp)
            d2h.wait_stream(comp)
            bounds = list(range(0, n, chunk)) + [n]
            staged: dict = {}

            def stage(i):
                lo, hi = bounds[i], bounds[i + 1]
                with torch.cuda.stream(h2d):
                    dev = [s.to(self.device, non_blocking=True) for s in streams[lo:hi]]
                    ev = torch.cuda.Event()
                    ev.record(h2d)
                heads = [bytes(s[:32].numpy().tobytes()) if (not s.is_cuda and s.numel() >= 32) else None
                         for s in streams[lo:hi]]
                staged[i] = (dev, ev, heads)

            res, cursor = [], 0
            nchunks = len(bounds) - 1
            for i in range(min(2, nchunks)):
                stage(i)
            for i in range(nchunks):
                dev, ev, heads = staged.pop(i)
                comp.wait_event(ev)
                for s in dev:
                    s.record_stream(comp)
                planes = self.decode(dev, predictor=predictor,
                                     headers=heads if all(h is not None for h in heads) else None)
                if i + 2 < nchunks:
                    stage(i + 2)
                done = torch.cuda.Event()
                done.record(comp)
                first = planes[0][0]
                arena = first._base if first._base is not None else first
                total = sum(p.numel() for f in planes for p in f)
                if out is not None and cursor + total <= out.numel():
                    host = out.narrow(0, cursor, total)
                    cursor += total
                else:
                    host = torch.empty(total, dtype=torch.uint16, pin_memory=True)
                with torch.cuda.stream(d2h):
                    d2h.wait_event(done)
                    arena.record_stream(d2h)
                    host.copy_(arena.reshape(-1).narrow(0, 0, total), non_blocking=True)
                off = 0
                for f in planes:
                    views = []
                    for p in f:
                        views.append(host.narrow(0, off, p.numel()).view(p.shape))
                        off += p.numel()
                    res.append(tuple(views))
            d2h.synchronize()
        return res


    def headers(self, streams) -> list[bytes]:
        """The 32-byte header of each stream (shorter streams: their bytes):
        CPU streams read in place, this device's streams with one gather
        kernel for all of them, which writes pinned host memory directly."""
        out: list = [None] * len(streams)
        dev = []
        for i, s in enumerate(streams):
            if s.is_cuda and s.device == self.device:
                dev.append(i)
            else:
                out[i] = bytes(s[:32].cpu().numpy().tobytes())
        if dev:
            n = len(dev)
            with torch.cuda.device(self.device):
                cur = torch.cuda.current_stream(self.device)
                need = ((16 * n + 255) // 256) * 256 + 32 * n
                if self._hdr_scratch is None or self._hdr_scratch.numel() < need:
                    self._hdr_scratch = torch.empty(max(need, 1 << 16), dtype=torch.uint8, device=self.device)
                s_arr = (ctypes.c_void_p * n)(*[streams[i].contiguous().data_ptr() for i in dev])
                l_arr = (ctypes.c_int64 * n)(*[streams[i].numel() for i in dev])
                heads = self._pinned_heads(n)
                _native.check(self.lib.fvb_gather_headers(s_arr, l_arr, n, self._hdr_scratch.data_ptr(),
                                                          self._hdr_scratch.numel(), heads.data_ptr(),
                                                          cur.cuda_stream))
                raw = heads.numpy().tobytes()
            for k, i in enumerate(dev):
                out[i] = raw[32 * k:32 * k + min(32, streams[i].numel())]
        return out


    def encode_decode_host(self, frames, *, chunk: int = 32, chunk_bytes: int = 32 << 20,
                           ring_bytes: int = 8 << 30, predictor: str = "wavefront",
                           out_streams: torch.Tensor | None = None, out_planes: torch.Tensor | None = None,
                           **params):
        """Encode frames held in (preferably pinned) host memory and decode
        the streams again -- the round trip a codec evaluation makes -- with
        the streams and the decoded planes delivered in pinned host memory
        (views of `out_streams` / `out_planes` while they have room).

        The frames go through in chunks of consecutive frames, each closed
        once it holds `chunk` frames or its next frame would take it above
        `chunk_bytes` of samples (a larger frame is a chunk of its own).
        Two host threads drive the GPU: this one uploads the chunks as far
        ahead as the ring of device buffers allows and encodes chunk i on
        the calling stream; a decode thread decodes the
        encoded chunks on a stream of its own, through a second codec (its
        own shape buckets and workspaces), and downloads each chunk's
        streams and planes.  So the encoder's wait for its stream lengths
        and the decoder's wait for its status words overlap instead of
        adding up (the headers come with the encoder's results).  Both
        threads launch directly: a graph capture on one thread must not meet
        the other thread's work on the device (a capture invalidated that
        way was seen).  Uploads, kernels and downloads of different chunks
        run at once on the two copy streams and the two compute streams.  Device buffers are resident: a ring of slots, each
        an upload buffer, a stream arena and a plane arena for one chunk
        (about 6 bytes per sample), as many as `ring_bytes` holds (at least
        two, at most one per chunk), kept by the codec and reused chunk
        after chunk (events order each reuse after the download of the
        chunk that last used the slot), so the pipeline makes no allocation
        once warm.  The streams stay on the device between the encode and the
        decode.  Streams equal encode()'s and planes decode()'s.  Returns
        (streams, planes), one entry per frame."""
        import queue
        import threading

        n = len(frames)
        if n == 0:
            return [], []
        frames = [tuple(f) if not isinstance(f, torch.Tensor) else (f,) for f in frames]
        per = {k: _per_frame(v, n, k) for k, v in params.items()}
        bounds = _chunk_bounds([2 * sum(p.numel() for p in f) for f in frames], chunk, chunk_bytes)
        nchunks = len(bounds) - 1
        chunk_samples = [sum(p.numel() for f in frames[lo:hi] for p in f) for lo, hi in zip(bounds, bounds[1:])]
        max_samples = max(chunk_samples)
        slots = max(2, min(nchunks, ring_bytes // (6 * max_samples + (64 << 10))))
        ahead = slots - 1
        decoder = self._decode_partner()
        out_s: list = [None] * n
        out_p: list = [None] * n
        with torch.cuda.device(self.device):
            comp = torch.cuda.current_stream(self.device)
            ring = self._ring(slots, max_samples)
            h2d, d2h, dstream = ring["h2d"], ring["d2h"], ring["dec"]
            for st in (h2d, d2h, dstream):
                st.wait_stream(comp)
            staged: dict = {}
            freed = [None] * slots        # event: the slot's upload buffer was last read (encode done)
            drained = [None] * nchunks    # event: chunk i's arenas were last read (download done)
            drained_ready = [threading.Event() for _ in range(nchunks)]
            work: queue.Queue = queue.Queue()
            failure: list = []

            def stage(i):
                lo, hi = bounds[i], bounds[i + 1]
                k = i % slots
                buf = ring["up"][k]
                with torch.cuda.stream(h2d):
                    if freed[k] is not None:
                        h2d.wait_event(freed[k])
                    dev, off = [], 0
                    for f in frames[lo:hi]:
                        planes = []
                        for p in f:
                            v = buf.narrow(0, off, p.numel()).view(p.shape)
                            v.copy_(p, non_blocking=True)
                            planes.append(v)
                            off += p.numel()
                        dev.append(tuple(planes))
                    ev = torch.cuda.Event()
                    ev.record(h2d)
                staged[i] = (dev, ev)

            def host_slice(buf, cursor, count, dtype):
                if buf is not None and cursor + count <= buf.numel():
                    return buf.narrow(0, cursor, count), cursor + count
                return torch.empty(count, dtype=dtype, pin_memory=True), cursor

            def decode_side():
                cur_s = cur_p = 0
                try:
                    with torch.cuda.device(self.device), torch.cuda.stream(dstream):
                        while True:
                            item = work.get()
                            if item is None:
                                return
                            i, streams, heads, enc_done = item
                            k = i % slots
                            lo = bounds[i]
                            dstream.wait_event(enc_done)
                            if i >= slots:  # the plane arena's last download
                                dstream.wait_event(drained[i - slots])
                            s_src = streams[0]._base if streams[0]._base is not None else streams[0]
                            own_arena = s_src.data_ptr() != ring["streams"][k].data_ptr()
                            if own_arena:  # the ring slot was too small: an arena of its own
                                s_src.record_stream(dstream)
                                s_src.record_stream(d2h)
                            planes = decoder.decode(streams, predictor=predictor, headers=heads,
                                                    arena=ring["planes"][k], graphs=False)
                            done = torch.cuda.Event()
                            done.record(dstream)
                            s_total = sum(int(st.numel()) for st in streams)
                            p_total = sum(p.numel() for f in planes for p in f)
                            p_src = planes[0][0]._base if planes[0][0]._base is not None else planes[0][0]
                            hs, cur_s = host_slice(out_streams, cur_s, s_total, torch.uint8)
                            hp, cur_p = host_slice(out_planes, cur_p, p_total, torch.uint16)
                            with torch.cuda.stream(d2h):
                                d2h.wait_event(done)
                                if p_src.data_ptr() != ring["planes"][k].data_ptr():
                                    p_src.record_stream(d2h)
                                hs.copy_(s_src.reshape(-1).narrow(0, 0, s_total), non_blocking=True)
                                hp.copy_(p_src.reshape(-1).narrow(0, 0, p_total), non_blocking=True)
                                dr = torch.cuda.Event()
                                dr.record(d2h)
                            drained[i] = dr
                            drained_ready[i].set()
                            off = 0
                            for j, st in enumerate(streams):
                                out_s[lo + j] = hs.narrow(0, off, st.numel())
                                off += st.numel()
                            off = 0
                            for j, f in enumerate(planes):
                                views = []
                                for p in f:
                                    views.append(hp.narrow(0, off, p.numel()).view(p.shape))
                                    off += p.numel()
                                out_p[lo + j] = tuple(views)
                except BaseException as exc:  # reported by the calling thread
                    failure.append(exc)
                    for e in drained_ready:
                        e.set()
                    while work.get() is not None:
                        pass

            worker = threading.Thread(target=decode_side, name="fastvid-roundtrip-decode", daemon=True)
            worker.start()
            try:
                for i in range(min(ahead, nchunks)):
                    stage(i)
                for i in range(nchunks):
                    dev, ev = staged.pop(i)
                    k = i % slots
                    comp.wait_event(ev)
                    if i >= slots:  # the stream arena: decoded and downloaded
                        drained_ready[i - slots].wait()
                        if failure:
                            break
                        comp.wait_event(drained[i - slots])
                    lo, hi = bounds[i], bounds[i + 1]
                    streams, heads = self.encode(dev, arena=ring["streams"][k], return_headers=True, graphs=False,
                                                 **{kk: v[lo:hi] for kk, v in per.items()})
                    enc_done = torch.cuda.Event()
                    enc_done.record(comp)
                    freed[k] = enc_done
                    work.put((i, streams, heads, enc_done))
                    if i + ahead < nchunks:
                        stage(i + ahead)
            finally:
                work.put(None)
                worker.join()
            if failure:
                torch.cuda.synchronize(self.device)
                raise failure[0]
            d2h.synchronize()
            comp.wait_stream(d2h)
            comp.wait_stream(dstream)
        return out_s, out_p

    def _decode_partner(self) -> "BatchCodec":
        """A second codec on this device for the round trip's decode thread
        (its own shape buckets, workspaces and header scratch)."""
        p = getattr(self, "_partner", None)
        if p is None:
            p = BatchCodec(self.device, use_graphs=self.use_graphs, max_cached_shapes=self.max_cached)
            self._partner = p
        return p

    def _ring(self, slots: int, samples: int) -> dict:
        """Resident buffers of the host round trip: `slots` upload slots and
        plane arenas of `samples` uint16, stream arenas of 2 * `samples` +
        64 KiB bytes (a chunk whose streams are larger -- possible only for
        near-incompressible 16-bit content -- gets an arena of its own), and
        the two copy streams and the decode thread's compute stream."""
        r = getattr(self, "_ring_bufs", None)
        if r is None or r["slots"] < slots or r["samples"] < samples:
            r = {"slots": slots, "samples": samples,
                 "up": [torch.empty(samples, dtype=torch.uint16, device=self.device) for _ in range(slots)],
                 "streams": [torch.empty(2 * samples + (64 << 10), dtype=torch.uint8, device=self.device)
                             for _ in range(slots)],
                 "planes": [torch.empty(samples, dtype=torch.uint16, device=self.device) for _ in range(slots)],
                 "h2d": torch.cuda.Stream(self.device), "d2h": torch.cuda.Stream(self.device),
                 "dec": torch.cuda.Stream(self.device)}
            self._ring_bufs = r
        return r


def _chunk_bounds(sizes: list[int], max_frames: int, max_bytes: int) -> list[int]:
    """Chunk boundaries over consecutive items: a chunk closes at
    `max_frames` items or before the item that would take it above
    `max_bytes` (an item larger than that is a chunk of its own)."""
    bounds, acc = [0], 0
    for i, b in enumerate(sizes):
        if i > bounds[-1] and (acc + b > max_bytes or i - bounds[-1] >= max_frames):
            bounds.append(i)
            acc = 0
        acc += b
    bounds.append(len(sizes))
    return bounds


_default: dict = {}


def default_codec(device=None) -> BatchCodec:
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    codec = _default.get(dev)
    if codec is None:
        codec = BatchCodec(dev)
        _default[dev] = codec
    return codec


def encode_batch(frames, **kwargs):
    """Encode a list of frames with the per-device default BatchCodec."""
    if not frames:
        return []
    first = frames[0][0] if not isinstance(frames[0], torch.Tensor) else frames[0]
    return default_codec(first.device).encode(frames, **kwargs)


def decode_batch(streams, predictor="wavefront"):
    """Decode a list of streams with the per-device default BatchCodec."""
    if not streams:
        return []
    dev = next((s.device for s in streams if s.is_cuda), None)
    return default_codec(dev).decode(streams, predictor)


def stream_headers(streams) -> list[bytes]:
    """Headers of a list of streams (see BatchCodec.headers)."""
    if not streams:
        return []
    cuda = [s for s in streams if s.is_cuda]
    if not cuda:
        return [bytes(s[:32].numpy().tobytes()) for s in streams]
    return default_codec(cuda[0].device).headers(streams)
