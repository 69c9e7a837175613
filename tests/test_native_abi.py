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
    assert lib.fvb_abi_version() == 1


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
