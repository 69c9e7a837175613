"""Single-frame encode/decode over the C ABI (the drop-in path).

``encode_frame`` / ``decode_frame`` have the contract of the reference
binding ``_C.encode`` / ``_C.decode`` (cuda/csrc/fastvid_cuda.cpp:359-378):
same arguments, same validation order and messages, ``RuntimeError`` on every
failure.  torch tensors serve only as device buffers; all codec work runs in
libfastvid_b200.so.
"""

from __future__ import annotations

import ctypes
import operator
import threading

import torch

from . import _native
from ._native import Frame

_U32_MAX = 0xFFFFFFFF
_LAYOUTS_DEFAULT = {"gray": 0, "yuv422": 1, "rgb444": 2}


def _fail(msg: str):
    raise RuntimeError(msg)


def _i64(value) -> int:
    return operator.index(value)


def _stream_handle(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def _plane_view(plane: torch.Tensor) -> tuple[torch.Tensor, int]:
    """A plane with unit column stride and its row pitch in elements."""
    if plane.stride(1) != 1 or plane.stride(0) < plane.size(1) or plane.storage_offset() < 0:
        plane = plane.contiguous()
    pitch = plane.stride(0) if plane.size(0) > 1 else plane.size(1)
    return plane, max(pitch, plane.size(1))


def plan_encode(planes, layout, bit_depth, quality, fps_numerator, fps_denominator, tile_width, tile_height):
    """Validate like encode.cu:695-725 and return (frame, workspace_bytes, planes, pitches)."""
    layout = _i64(layout)
    bit_depth = _i64(bit_depth)
    quality = _i64(quality)
    fps_numerator = _i64(fps_numerator)
    fps_denominator = _i64(fps_denominator)
    tile_width = _i64(tile_width)
    tile_height = _i64(tile_height)
    if not (0 <= layout <= 2):
        _fail("layout must be gray, yuv422, or rgb444")
    if len(planes) != (1 if layout == 0 else 3):
        _fail("plane count does not match layout")
    if bit_depth not in (8, 10, 12, 16):
        _fail("bit_depth must be 8, 10, 12, or 16")
    if not (1 <= quality <= 100):
        _fail("quality must be in 1..=100")
    if not (0 < fps_numerator <= _U32_MAX and 0 < fps_denominator <= _U32_MAX):
        _fail("frame-rate components must be nonzero u32 values")
    if not (0 < tile_width <= 0xFFFF and 0 < tile_height <= 0xFFFF):
        _fail("tile dimensions must be nonzero u16 values")
    first = planes[0]
    if not first.is_cuda:
        _fail("encoder input planes must be CUDA tensors")
    if first.dtype != torch.uint16 or first.dim() != 2:
        _fail("encoder planes must be two-dimensional uint16 tensors")
    device = first.device
    height, width = first.shape
    if not (0 < width <= _U32_MAX and 0 < height <= _U32_MAX):
        _fail("frame dimensions must be nonzero u32 values")
    secondary = (width + 1) // 2 if layout == 1 else width
    views, pitches = [], []
    for index, plane in enumerate(planes):
        if plane.device != device:
            _fail("all planes must use the same CUDA device")
        if plane.dtype != torch.uint16 or plane.dim() != 2:
            _fail("encoder planes must be two-dimensional uint16 tensors")
        expected = width if index == 0 else secondary
        if plane.size(0) != height or plane.size(1) != expected:
            _fail("plane dimensions do not match declared layout")
        view, pitch = _plane_view(plane)
        views.append(view)
        pitches.append(pitch)
    lib = _native.load()
    frame = Frame()
    ws = ctypes.c_int64()
    _native.check(lib.fvb_encode_plan(width, height, layout, bit_depth, quality, fps_numerator,
                                      fps_denominator, tile_width, tile_height, ctypes.byref(frame),
                                      ctypes.byref(ws)))
    return frame, ws.value, views, pitches


def encode_frame(planes, layout, bit_depth, quality, fps_numerator=24, fps_denominator=1,
                 tile_width=256, tile_height=128) -> torch.Tensor:
    """Encode CUDA uint16 planes to one stream (a 1-D CUDA uint8 tensor)."""
    planes = list(planes)
    if not planes:
        _fail("plane count does not match layout")
    frame, ws_bytes, views, pitches = plan_encode(planes, layout, bit_depth, quality, fps_numerator,
                                                  fps_denominator, tile_width, tile_height)
    device = views[0].device
    lib = _native.load()
    with torch.cuda.device(device):
        workspace = torch.empty(ws_bytes, dtype=torch.uint8, device=device)
        ptrs = (ctypes.c_void_p * 3)(*[v.data_ptr() for v in views] + [0] * (3 - len(views)))
        pit = (ctypes.c_int64 * 3)(*pitches + [0] * (3 - len(pitches)))
        stream = _stream_handle(device)
        length = ctypes.c_int64()
        _native.check(lib.fvb_encode_analyze(ctypes.byref(frame), ptrs, pit, workspace.data_ptr(), ws_bytes,
                                             stream, ctypes.byref(length)))
        out = torch.empty(length.value, dtype=torch.uint8, device=device)
        _native.check(lib.fvb_encode_emit(ctypes.byref(frame), workspace.data_ptr(), ws_bytes, out.data_ptr(),
                                          length.value, stream))
        # the workspace must outlive the asynchronous emission on this stream
        workspace.record_stream(torch.cuda.current_stream(device))
    return out


def header_of(encoded: torch.Tensor) -> bytes:
    head = encoded[:32]
    if head.is_cuda:
        head = head.cpu()
    return bytes(head.contiguous().numpy().tobytes())


def plan_decode(encoded: torch.Tensor, header: bytes | None = None):
    """Validate like fastvid_cuda.cpp:142-183; returns (frame, workspace_bytes)."""
    if encoded.dtype != torch.uint8:
        _fail("encoded must have dtype uint8")
    if encoded.dim() != 1:
        _fail("encoded must be one-dimensional")
    if not torch.cuda.is_available():
        _fail("CUDA is required")
    size = encoded.numel()
    if size < 32:
        _fail("truncated Fastvid header")
    if header is None:
        header = header_of(encoded)
    lib = _native.load()
    frame = Frame()
    ws = ctypes.c_int64()
    buf = ctypes.create_string_buffer(header, 32)
    _native.check(lib.fvb_decode_plan(buf, 32, size, ctypes.byref(frame), ctypes.byref(ws)))
    return frame, ws.value


def plane_views(output: torch.Tensor, frame: Frame):
    """Planes as views of one contiguous uint16 buffer, Y then Cb then Cr (decode.cu:720-729)."""
    w, h = frame.width, frame.height
    y = w * h
    planes = [output.narrow(0, 0, y).view(h, w)]
    if frame.planes == 3:
        cw = frame.plane_width[1]
        c = cw * h
        planes.append(output.narrow(0, y, c).view(h, cw))
        planes.append(output.narrow(0, y + c, c).view(h, cw))
    return planes


_STAGE_CHUNK = 1 << 20
_staging = threading.local()


def _upload(host: torch.Tensor, device: torch.device) -> torch.Tensor:
    """Copy a CPU stream to the device on the current stream without
    blocking on the transfer.  A pinned tensor is copied directly; a pageable
    one goes through two pinned 1 MiB staging halves kept per thread: the
    host fills one half while the other is in flight, so host copying and
    the transfer overlap.  The caller's decode waits for its status word,
    which orders these copies before the staging is reused."""
    out = torch.empty(host.numel(), dtype=torch.uint8, device=device)
    if host.is_pinned() or host.numel() <= 4096:
        out.copy_(host, non_blocking=host.is_pinned())
        return out
    per_device = getattr(_staging, "by_device", None)
    if per_device is None:
        per_device = _staging.by_device = {}
    stage = per_device.get(device.index)
    if stage is None:
        stage = per_device[device.index] = (torch.empty(2 * _STAGE_CHUNK, dtype=torch.uint8).pin_memory(),
                                            [torch.cuda.Event(), torch.cuda.Event()])
    buf, events = stage
    stream = torch.cuda.current_stream(device)
    # (the previous call's transfers ended before it returned: its decode
    # waited for its status word on this stream)
    for k, lo in enumerate(range(0, host.numel(), _STAGE_CHUNK)):
        n = min(_STAGE_CHUNK, host.numel() - lo)
        half = buf.narrow(0, (k & 1) * _STAGE_CHUNK, n)
        events[k & 1].synchronize()  # this half's previous transfer has landed (no-op before its first use)
        half.copy_(host.narrow(0, lo, n))
        out.narrow(0, lo, n).copy_(half, non_blocking=True)
        events[k & 1].record(stream)
    return out


def decode_frame(encoded: torch.Tensor, wavefront: bool = True):
    """Decode one stream (CPU or CUDA uint8) to a list of CUDA uint16 planes.

    A CPU stream is validated from its host header (fastvid_cuda.cpp:142-183)
    and uploaded without blocking (see _upload), so the host plans the frame
    and allocates its outputs while the bytes are in flight; the device
    metadata parse then runs on the uploaded copy."""
    frame, ws_bytes = plan_decode(encoded)
    if encoded.is_cuda:
        device = encoded.device
        stream_dev = encoded.contiguous()
    else:
        device = torch.device("cuda", torch.cuda.current_device())
        with torch.cuda.device(device):
            stream_dev = _upload(encoded.contiguous(), device)
    lib = _native.load()
    with torch.cuda.device(device):
        output = torch.empty(frame.samples, dtype=torch.uint16, device=device)
        workspace = torch.empty(ws_bytes, dtype=torch.uint8, device=device)
        planes = plane_views(output, frame)
        ptrs = (ctypes.c_void_p * 3)(*[p.data_ptr() for p in planes] + [0] * (3 - len(planes)))
        pit = (ctypes.c_int64 * 3)(*[p.size(1) for p in planes] + [0] * (3 - len(planes)))
        _native.check(lib.fvb_decode(ctypes.byref(frame), stream_dev.data_ptr(), stream_dev.numel(), ptrs, pit,
                                     1 if wavefront else 0, workspace.data_ptr(), ws_bytes,
                                     _stream_handle(device)))
    return planes


class _CModule:
    """Stand-in for the reference's pybind module ``fastvid_cuda._C``."""

    @staticmethod
    def encode(planes, layout, bit_depth, quality, fps_numerator=24, fps_denominator=1, tile_width=256,
               tile_height=128):
        return encode_frame(planes, layout, bit_depth, quality, fps_numerator, fps_denominator, tile_width,
                            tile_height)

    @staticmethod
    def decode(encoded, wavefront=True):
        return decode_frame(encoded, wavefront)


_C = _CModule()
