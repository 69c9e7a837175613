"""ctypes binding of the CPU oracle (test infrastructure only).

The oracle is a plain-C restatement of the reference fastvid codec
(fastvid_oracle.c).  Only tests/, __graft_entry__.smoke() and the CPU-baseline
leg of bench.py may import this package, and only as the checker.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / "liboracle.so"
_lib = None

LAYOUTS = {"gray": 0, "yuv422": 1, "rgb444": 2}


class OracleError(RuntimeError):
    """Rejection reported by the oracle (same meaning as the reference's RuntimeError)."""


def build() -> Path:
    """Compile liboracle.so with gcc (seconds)."""
    subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)
    return _LIB_PATH


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not _LIB_PATH.exists():
        build()
    lib = ctypes.CDLL(str(_LIB_PATH))
    i64, i32, p = ctypes.c_int64, ctypes.c_int, ctypes.c_void_p
    lib.fvo_encode.argtypes = [p, i64, i64, i32, i32, i32, i64, i64, i64, i64, i32,
                               ctypes.POINTER(p), ctypes.POINTER(i64), ctypes.c_char_p, i32]
    lib.fvo_encode.restype = i32
    lib.fvo_decode.argtypes = [p, i64, i32, i32, ctypes.POINTER(p), ctypes.POINTER(i64),
                               ctypes.POINTER(i64), ctypes.POINTER(i64), ctypes.POINTER(i32),
                               ctypes.POINTER(i32), ctypes.c_char_p, i32]
    lib.fvo_decode.restype = i32
    lib.fvo_predict.argtypes = [p, i64, i64, i32, i32, i64, i64, i32, i32, p, p]
    lib.fvo_predict.restype = i32
    lib.fvo_analyze.argtypes = [p, i64, i64, i32, i64, i64, i32, p]
    lib.fvo_analyze.restype = i32
    lib.fvo_geometry.argtypes = [i64, i64, i32, i64, i64, ctypes.POINTER(i64),
                                 ctypes.POINTER(i64), ctypes.POINTER(i64)]
    lib.fvo_geometry.restype = i32
    lib.fvo_quantization_step.argtypes = [i32, i32, i32]
    lib.fvo_quantization_step.restype = ctypes.c_int32
    lib.fvo_refined_gray16_step.argtypes = [i32]
    lib.fvo_refined_gray16_step.restype = ctypes.c_int32
    lib.fvo_free.argtypes = [p]
    _lib = lib
    return lib


def _layout_code(layout) -> int:
    return LAYOUTS[layout] if isinstance(layout, str) else int(layout)


def concat_planes(planes) -> np.ndarray:
    arrays = [np.ascontiguousarray(np.asarray(pl, dtype=np.uint16)).reshape(-1) for pl in planes]
    return np.ascontiguousarray(np.concatenate(arrays))


def quantization_step(layout, bit_depth: int, quality: int) -> int:
    return int(_load().fvo_quantization_step(_layout_code(layout), bit_depth, quality))


def refined_gray16_step(quality: int) -> int:
    return int(_load().fvo_refined_gray16_step(quality))


def geometry(width, height, layout, tile_size=(256, 128)):
    lib = _load()
    t, s, n = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
    if lib.fvo_geometry(width, height, _layout_code(layout), tile_size[0], tile_size[1],
                        ctypes.byref(t), ctypes.byref(s), ctypes.byref(n)):
        raise OracleError("too many tiles")
    return t.value, s.value, n.value


def encode(planes, *, layout, bit_depth=10, quality=90, frame_rate=(24, 1),
           tile_size=(256, 128), threads=1) -> bytes:
    """Encode numpy/uint16 planes; returns the stream bytes or raises OracleError."""
    lib = _load()
    planes = list(planes)
    height, width = np.asarray(planes[0]).shape
    flat = concat_planes(planes)
    out = ctypes.c_void_p()
    out_len = ctypes.c_int64()
    msg = ctypes.create_string_buffer(256)
    rc = lib.fvo_encode(flat.ctypes.data, width, height, _layout_code(layout), bit_depth, quality,
                        frame_rate[0], frame_rate[1], tile_size[0], tile_size[1], threads,
                        ctypes.byref(out), ctypes.byref(out_len), msg, 256)
    if rc:
        raise OracleError(msg.value.decode())
    try:
        return ctypes.string_at(out.value, out_len.value)
    finally:
        lib.fvo_free(out)


def decode(stream, threads=1):
    """Decode stream bytes; returns a tuple of (H, W) uint16 numpy planes."""
    lib = _load()
    data = np.frombuffer(bytes(stream), dtype=np.uint8)
    if data.size == 0:
        data = np.zeros(1, dtype=np.uint8)[:0]
    out = ctypes.c_void_p()
    n, w, h = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
    layout, depth = ctypes.c_int(), ctypes.c_int()
    msg = ctypes.create_string_buffer(256)
    buf = np.ascontiguousarray(data)
    rc = lib.fvo_decode(buf.ctypes.data if buf.size else None, len(bytes(stream)), 1, threads,
                        ctypes.byref(out), ctypes.byref(n), ctypes.byref(w), ctypes.byref(h),
                        ctypes.byref(layout), ctypes.byref(depth), msg, 256)
    if rc:
        raise OracleError(msg.value.decode())
    try:
        flat = np.ctypeslib.as_array(ctypes.cast(out.value, ctypes.POINTER(ctypes.c_uint16)),
                                     shape=(n.value,)).copy()
    finally:
        lib.fvo_free(out)
    return split_planes(flat, w.value, h.value, layout.value)


def split_planes(flat: np.ndarray, width: int, height: int, layout: int):
    y = width * height
    if layout == 0:
        return (flat[:y].reshape(height, width),)
    cw = (width + 1) // 2 if layout == 1 else width
    c = cw * height
    return (flat[:y].reshape(height, width), flat[y:y + c].reshape(height, cw),
            flat[y + c:y + 2 * c].reshape(height, cw))


def predict(planes, *, layout, bit_depth, tile_size, step, use_med):
    """Folded residuals (tile-raster order, uint32) and reconstructed samples."""
    lib = _load()
    planes = list(planes)
    height, width = np.asarray(planes[0]).shape
    flat = concat_planes(planes)
    folded = np.zeros(flat.size, dtype=np.uint32)
    recon = np.zeros(flat.size, dtype=np.uint16)
    st = lib.fvo_predict(flat.ctypes.data, width, height, _layout_code(layout), bit_depth,
                         tile_size[0], tile_size[1], step, int(use_med), folded.ctypes.data,
                         recon.ctypes.data)
    return folded, recon, st


def analyze(folded, *, width, height, layout, tile_size, force_order0):
    """Per-shard analysis rows: mode, parameter, body, record, lane_bytes[4]."""
    lib = _load()
    _, shards, _ = geometry(width, height, layout, tile_size)
    out = np.zeros((shards, 8), dtype=np.int64)
    f = np.ascontiguousarray(folded, dtype=np.uint32)
    st = lib.fvo_analyze(f.ctypes.data, width, height, _layout_code(layout), tile_size[0],
                         tile_size[1], int(force_order0), out.ctypes.data)
    return out, st


def cpu_threads() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
