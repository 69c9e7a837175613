"""GPU test of the allocation-free decode entry point, fvb_decode_noalloc.

Some callers cannot allocate device memory at the moment they decode:
plug-ins that a host application hands pre-allocated frame buffers while it
owns the device heap, real-time pipelines that forbid allocation once they
run (cudaMalloc and cudaFree can block and synchronise the device), and
components held to a device-memory budget enforced elsewhere.  They call
fvb_decode_noalloc, whose scratch is a fixed array inside the library.  Its
planes must equal, exactly, those of fvb_decode (the entry point that takes a
caller-allocated workspace), on consecutive calls that share that array.

This file is collected last, so a run that stops at the first failure has
already run every other test.
"""

import ctypes

import numpy as np
import pytest
import torch

import fastvid_b200
from fastvid_b200 import _native, synth
from fastvid_b200._native import Frame
from fastvid_b200.codec import plane_views

pytestmark = pytest.mark.gpu


def _plan(stream: torch.Tensor) -> Frame:
    lib = _native.load()
    frame = Frame()
    ws = ctypes.c_int64()
    header = ctypes.create_string_buffer(bytes(stream[:32].cpu().numpy().tobytes()), 32)
    _native.check(lib.fvb_decode_plan(header, 32, stream.numel(), ctypes.byref(frame), ctypes.byref(ws)))
    return frame


def _decode_noalloc(stream: torch.Tensor, frame: Frame | None = None):
    """Decode through fvb_decode_noalloc into caller-owned planes."""
    lib = _native.load()
    frame = frame or _plan(stream)
    out = torch.empty(frame.samples, dtype=torch.uint16, device=stream.device)
    planes = plane_views(out, frame)
    ptrs = (ctypes.c_void_p * 3)(*[p.data_ptr() for p in planes] + [0] * (3 - len(planes)))
    pitches = (ctypes.c_int64 * 3)(*[p.size(1) for p in planes] + [0] * (3 - len(planes)))
    rc = lib.fvb_decode_noalloc(ctypes.byref(frame), stream.data_ptr(), stream.numel(), ptrs, pitches, 1,
                                torch.cuda.current_stream(stream.device).cuda_stream)
    return rc, planes


def _encode(width, height, layout, depth, quality, tile, seed):
    planes = synth.make_frame(width, height, layout, depth, seed)
    cuda_planes = tuple(torch.from_numpy(np.ascontiguousarray(p)).cuda() for p in planes)
    return fastvid_b200.encode(cuda_planes, layout=layout, bit_depth=depth, quality=quality, tile_size=tile)


def test_noalloc_decode_matches_workspace_decode_on_consecutive_calls(cuda):
    streams = [
        _encode(1920, 1080, "rgb444", 8, 90, (64, 64), 101),   # 6.2 M samples
        _encode(3840, 2160, "gray", 16, 87, (128, 128), 104),  # 8.3 M samples: fits with u16 folded symbols
        _encode(640, 360, "yuv422", 10, 80, (128, 128), 102),
        _encode(1280, 720, "gray", 16, 87, (128, 128), 103),
    ]
    for _ in range(2):  # consecutive calls share the array; no state may leak between them
        for stream in streams:
            rc, got = _decode_noalloc(stream)
            assert rc == 0, _native.last_error()
            expected = fastvid_b200.decode(stream)  # fvb_decode, workspace allocated by the caller
            assert len(got) == len(expected)
            for a, b in zip(got, expected):
                assert torch.equal(a, b)  # integer codec: exact


def test_noalloc_decode_rejects_frames_beyond_its_scratch(cuda):
    lib = _native.load()
    assert lib.fvb_decode_noalloc_capacity() == 32 << 20
    # 8.3 M samples of a lossless 16-bit frame: u32 folded symbols, beyond the array
    stream = _encode(3840, 2160, "gray", 16, 100, (128, 128), 104)
    rc, _ = _decode_noalloc(stream)
    assert rc != 0
    assert "allocation-free decode" in _native.last_error()
    stream = _encode(3840, 2160, "rgb444", 8, 90, (128, 128), 106)  # 24.9 M samples
    rc, _ = _decode_noalloc(stream)
    assert rc != 0
    assert "allocation-free decode" in _native.last_error()


def test_noalloc_decode_leaves_no_state_behind_after_a_rejected_stream(cuda):
    """A malformed stream decoded through the shared array fails, and the
    next valid decode through the same array is still exact."""
    good = _encode(640, 360, "rgb444", 10, 90, (64, 64), 105)
    frame = _plan(good)
    truncated = good[:-5].clone()  # the last tile's payload no longer ends at the stream end
    rc, _ = _decode_noalloc(truncated, frame)
    assert rc == 10, _native.last_error()
    corrupt = good.clone()
    mid = good.numel() // 2
    corrupt[mid:mid + 64] ^= 0x5A  # damage entropy payload bytes
    rc_corrupt, _ = _decode_noalloc(corrupt, frame)
    assert rc_corrupt in (0, 1, 2, 3, 4, 5, 11)
    for _ in range(2):
        rc, got = _decode_noalloc(good)
        assert rc == 0, _native.last_error()
        for a, b in zip(got, fastvid_b200.decode(good)):
            assert torch.equal(a, b)


def test_noalloc_decode_rejects_a_host_stream_without_launching(cuda):
    lib = _native.load()
    good = _encode(320, 180, "gray", 10, 90, (64, 64), 106)
    host = good.cpu()
    frame = _plan(good)
    out = torch.empty(frame.samples, dtype=torch.uint16, device=good.device)
    ptrs = (ctypes.c_void_p * 3)(out.data_ptr(), 0, 0)
    pitches = (ctypes.c_int64 * 3)(frame.width, 0, 0)
    before = lib.fvb_launch_count()
    rc = lib.fvb_decode_noalloc(ctypes.byref(frame), host.data_ptr(), host.numel(), ptrs, pitches, 1,
                                torch.cuda.current_stream(good.device).cuda_stream)
    assert rc == -1 and "device memory" in _native.last_error()
    assert lib.fvb_launch_count() == before
