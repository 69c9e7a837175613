"""CPU tests of the C-ABI library: it loads, exports every declared symbol,
and its host-side validation matches the reference's (no GPU calls)."""

import ctypes
import re
from pathlib import Path

import pytest

import oracle
from fastvid_b200 import _native
from fastvid_b200._native import Frame

HEADER = Path(__file__).resolve().parent.parent / "include" / "fastvid_b200.h"


def _declared():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int|int64_t|const char\*)\s+(fvb_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    lib = _native.load()
    names = _declared()
    assert len(names) >= 14
    for name in names:
        assert hasattr(lib, name), name
        assert name in _native.SIGNATURES, name
    assert lib.fvb_abi_version() == _native.ABI_VERSION == 2


def _plan(width, height, layout, depth, quality, fps=(24, 1), tile=(256, 128)):
    lib = _native.load()
    frame = Frame()
    ws = ctypes.c_int64()
    rc = lib.fvb_encode_plan(width, height, layout, depth, quality, fps[0], fps[1], tile[0], tile[1],
                             ctypes.byref(frame), ctypes.byref(ws))
    return rc, frame, ws.value


@pytest.mark.parametrize("args,message", [
    ((64, 64, 3, 8, 90), "layout must be gray, yuv422, or rgb444"),
    ((64, 64, 0, 9, 90), "bit_depth must be 8, 10, 12, or 16"),
    ((64, 64, 0, 8, 0), "quality must be in 1..=100"),
    ((64, 64, 0, 8, 101), "quality must be in 1..=100"),
])
def test_encode_plan_rejects_like_reference(args, message):
    rc, _, _ = _plan(*args)
    assert rc != 0
    assert _native.last_error() == message


def test_encode_plan_rejects_bad_rates_and_tiles():
    assert _plan(64, 64, 0, 8, 90, fps=(0, 1))[0] != 0
    assert _native.last_error() == "frame-rate components must be nonzero u32 values"
    assert _plan(64, 64, 0, 8, 90, tile=(0, 8))[0] != 0
    assert _native.last_error() == "tile dimensions must be nonzero u16 values"
    assert _plan(64, 64, 0, 8, 90, tile=(65536, 8))[0] != 0
    assert _plan(0, 64, 0, 8, 90)[0] != 0
    assert _native.last_error() == "frame dimensions must be nonzero u32 values"
    assert _plan(4096, 4096, 0, 8, 90, tile=(1, 1))[0] != 0
    assert _native.last_error() == "too many tiles"


@pytest.mark.parametrize("w,h,layout,depth,q,tile", [
    (67, 35, 0, 8, 100, (256, 128)), (263, 133, 1, 10, 90, (256, 128)), (3840, 2160, 2, 10, 85, (128, 128)),
    (1920, 1080, 2, 8, 90, (64, 64)), (301, 203, 1, 10, 80, (67, 35)), (9, 7, 0, 10, 80, (1, 3)),
    (3840, 2160, 0, 16, 87, (128, 128)), (1300, 90, 0, 12, 95, (600, 40)),
])
def test_plan_geometry_matches_oracle(w, h, layout, depth, q, tile):
    rc, frame, ws = _plan(w, h, layout, depth, q, tile=tile)
    assert rc == 0
    assert (frame.tiles, frame.shards, frame.samples) == oracle.geometry(w, h, layout, tile)
    assert frame.step == oracle.quantization_step(layout, depth, q)
    assert frame.prefix_bytes == 32 + 32 * frame.tiles
    assert ws > 0 and frame.max_stream_bytes > frame.prefix_bytes


def _header(layout=1, quality=90, flags=2, width=263, height=133, tile=(256, 128), fps=(24, 1), tiles=None):
    import struct

    if tiles is None:
        tiles = oracle.geometry(width, height, layout, tile)[0]
    return struct.pack("<4sBBBBIIHHIII", b"FVID", 1, layout, quality, flags, width, height, tile[0], tile[1],
                       fps[0], fps[1], tiles)


def _decode_plan(header, size=None):
    lib = _native.load()
    frame = Frame()
    ws = ctypes.c_int64()
    buf = ctypes.create_string_buffer(header, len(header))
    rc = lib.fvb_decode_plan(buf, len(header), size if size is not None else 1 << 20, ctypes.byref(frame),
                             ctypes.byref(ws))
    return rc, frame


@pytest.mark.parametrize("mutate,message", [
    (lambda h: b"XVID" + h[4:], "bad Fastvid magic"),
    (lambda h: h[:4] + bytes([7]) + h[5:], "unsupported Fastvid bitstream version"),
    (lambda h: h[:5] + bytes([3]) + h[6:], "unknown pixel layout"),
    (lambda h: h[:6] + bytes([0]) + h[7:], "quality is out of range"),
    (lambda h: h[:7] + bytes([3]) + h[8:], "unsupported high-bit depth"),
    (lambda h: h[:7] + bytes([0x82]) + h[8:], "invalid gray16 refinement flag"),
    (lambda h: h[:7] + bytes([0x42]) + h[8:], "invalid gray MED flag"),
    (lambda h: h[:28] + bytes([1, 0, 0, 0]), "tile count does not match dimensions"),
])
def test_decode_plan_rejects_like_reference(mutate, message):
    rc, _ = _decode_plan(mutate(_header()))
    assert rc != 0
    assert _native.last_error() == message


def test_decode_plan_accepts_valid_header_and_checks_directory_size():
    header = _header()
    rc, frame = _decode_plan(header)
    assert rc == 0
    assert frame.layout == 1 and frame.bit_depth == 10 and frame.step == 3
    assert _decode_plan(header, size=32)[0] != 0
    assert _native.last_error() == "truncated tile directory"
    assert _decode_plan(header[:20], size=20)[0] != 0
    assert _native.last_error() == "truncated Fastvid header"


def test_host_pointers_are_rejected_before_any_launch():
    """The single-frame entry points check that the stream and the planes are
    device (or managed) memory; a host buffer returns FVB_ERR_ARGUMENT and
    nothing is launched (on a CPU-only machine too)."""
    import numpy as np

    lib = _native.load()
    planes = (np.arange(67 * 35, dtype=np.uint16).reshape(35, 67) % 256,)
    stream = oracle.encode(planes, layout="gray", bit_depth=8, quality=100)
    rc, frame = _decode_plan(stream[:32], size=len(stream))
    assert rc == 0
    host_stream = ctypes.create_string_buffer(stream, len(stream))
    out = np.zeros(frame.samples, dtype=np.uint16)
    ptrs = (ctypes.c_void_p * 3)(out.ctypes.data, 0, 0)
    pitches = (ctypes.c_int64 * 3)(67, 0, 0)
    before = lib.fvb_launch_count()
    rc = lib.fvb_decode(ctypes.byref(frame), ctypes.addressof(host_stream), len(stream), ptrs, pitches, 1,
                        None, 0, None)
    assert rc == -1 and _native.last_error() == "encoded stream must be device memory"
    rc = lib.fvb_decode_noalloc(ctypes.byref(frame), ctypes.addressof(host_stream), len(stream), ptrs, pitches,
                                1, None)
    assert rc == -1 and _native.last_error() == "encoded stream must be device memory"
    rc, enc_frame, ws = _plan(67, 35, 0, 8, 100)
    assert rc == 0
    src = np.ascontiguousarray(planes[0])
    length = ctypes.c_int64()
    rc = lib.fvb_encode_analyze(ctypes.byref(enc_frame), (ctypes.c_void_p * 3)(src.ctypes.data, 0, 0),
                                (ctypes.c_int64 * 3)(67, 0, 0), None, ws, None, ctypes.byref(length))
    assert rc == -1 and _native.last_error() == "input planes must be device memory"
    assert lib.fvb_launch_count() == before


def test_batch_bucket_rounds_counts_up_by_at_most_a_quarter():
    """fvb_batch_bucket: every count of the batch rounded up to m * 2^e with
    m in 4..8 (so within 25 percent), small floors, exact passes and wide flag."""
    from fastvid_b200._native import Bucket

    lib = _native.load()
    frames = []
    for w, h, layout, depth, q, tile in [(1920, 1080, 2, 8, 90, (64, 64)), (2048, 1080, 0, 16, 87, (128, 128)),
                                         (1280, 720, 0, 8, 100, (64, 64)), (301, 203, 1, 10, 80, (67, 35))]:
        rc, frame, _ = _plan(w, h, layout, depth, q, tile=tile)
        assert rc == 0
        frames.append(frame)
    arr = (Frame * len(frames))(*frames)
    b = Bucket()
    assert lib.fvb_batch_bucket(arr, len(frames), ctypes.byref(b)) == 0
    tiles = sum(f.tiles for f in frames)
    shards = sum(f.shards for f in frames)
    samples = sum(f.samples for f in frames)
    for actual, cap in ((len(frames), b.frames), (tiles, b.tiles), (shards, b.shards), (samples, b.samples)):
        assert actual <= cap
        if actual >= 8:
            assert cap <= actual * 1.25
            e = cap.bit_length() - 3
            assert cap % (1 << max(e, 0)) == 0 and 4 <= cap >> max(e, 0) <= 8
    # the gray16 q87 frame may try a refined step (a losing trial is not
    # re-run: the first pass's records are kept)
    assert b.passes == 2
    assert b.frames_p[1] >= 1 and b.frames_p[2] == 0
    gray16 = frames[1]
    assert b.samples_p[1] >= gray16.samples and b.prefix_p[1] >= gray16.prefix_bytes
    assert b.wide == 0
    ws = ctypes.c_int64()
    assert lib.fvb_bucket_encode_plan(ctypes.byref(b), ctypes.byref(ws)) == 0 and ws.value > 0
    exact = ctypes.c_int64()
    assert lib.fvb_batch_encode_plan(arr, len(frames), ctypes.byref(exact)) == 0
    assert exact.value <= ws.value <= 1.3 * exact.value + (4 << 20)
    b.passes = 0
    assert lib.fvb_bucket_encode_plan(ctypes.byref(b), ctypes.byref(ws)) == -1
    assert _native.last_error() == "invalid bucket"


def test_bucket_folded_symbol_width():
    """Folded symbols are held as u16 unless a frame is 16-bit lossless: the
    bucket records it, the workspace shrinks by 2 bytes per sample, and a u32
    capacity still takes a batch that would fit u16."""
    from fastvid_b200._native import Bucket

    lib = _native.load()

    def bucket(specs):
        frames = []
        for w, h, layout, depth, q in specs:
            rc, frame, _ = _plan(w, h, layout, depth, q)
            assert rc == 0
            frames.append(frame)
        arr = (Frame * len(frames))(*frames)
        b = Bucket()
        assert lib.fvb_batch_bucket(arr, len(frames), ctypes.byref(b)) == 0
        exact = ctypes.c_int64()
        assert lib.fvb_batch_encode_plan(arr, len(frames), ctypes.byref(exact)) == 0
        return b, exact.value, arr

    b8, ws8, _ = bucket([(640, 360, 0, 8, 100), (320, 200, 2, 12, 100)])
    assert b8.fold16 == 1
    b16, _, _ = bucket([(640, 360, 0, 16, 99), (320, 200, 1, 16, 50)])
    assert b16.fold16 == 1
    bl, wsl, arr = bucket([(640, 360, 0, 8, 100), (320, 200, 2, 16, 100)])
    assert bl.fold16 == 0
    b8b, ws8b, _ = bucket([(640, 360, 0, 8, 100), (320, 200, 2, 16, 99)])
    assert b8b.fold16 == 1 and wsl - ws8b >= 2 * (640 * 360 + 3 * 320 * 200)
    # the u16 bucket refuses the lossless 16-bit batch; a u32 one takes a u16 batch
    ws = ctypes.c_int64()
    assert lib.fvb_bucket_encode_plan(ctypes.byref(b8b), ctypes.byref(ws)) == 0
    b8b.fold16 = 0
    assert lib.fvb_bucket_encode_plan(ctypes.byref(b8b), ctypes.byref(ws)) == 0
