"""ctypes binding of libfastvid_b200.so (include/fastvid_b200.h).

The shared library is the product's compute path; there is no fallback.  If
it is missing it is built once with nvcc (fastvid_b200/build.py); if that is
impossible the import fails loudly.
"""

from __future__ import annotations

import ctypes
import threading
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libfastvid_b200.so"

c_i32, c_i64, c_p = ctypes.c_int32, ctypes.c_int64, ctypes.c_void_p


class Frame(ctypes.Structure):
    """Mirror of ``fvb_frame``."""

    _fields_ = [
        ("layout", c_i32), ("bit_depth", c_i32), ("quality", c_i32), ("flags", c_i32),
        ("width", c_i64), ("height", c_i64), ("tile_w", c_i64), ("tile_h", c_i64),
        ("fps_num", c_i64), ("fps_den", c_i64),
        ("tiles", c_i64), ("shards", c_i64), ("samples", c_i64),
        ("plane_width", c_i64 * 3),
        ("planes", c_i32), ("step", c_i32),
        ("prefix_bytes", c_i64), ("max_stream_bytes", c_i64),
    ]

    def copy(self) -> "Frame":
        other = Frame()
        ctypes.memmove(ctypes.byref(other), ctypes.byref(self), ctypes.sizeof(Frame))
        return other


ABI_VERSION = 2  # FVB_ABI_VERSION of include/fastvid_b200.h (2: fvb_bucket.fold16)


class Bucket(ctypes.Structure):
    """Mirror of ``fvb_bucket``: a capacity that a batch fits (see the header)."""

    _fields_ = [
        ("frames", c_i64), ("tiles", c_i64), ("shards", c_i64), ("samples", c_i64), ("prefix", c_i64),
        ("frames_p", c_i64 * 3), ("tiles_p", c_i64 * 3), ("shards_p", c_i64 * 3),
        ("samples_p", c_i64 * 3), ("prefix_p", c_i64 * 3),
        ("passes", c_i32), ("wide", c_i32), ("fold16", c_i32), ("pad", c_i32),
    ]

    def key(self) -> tuple:
        return (self.frames, self.tiles, self.shards, self.samples, self.prefix, tuple(self.frames_p),
                tuple(self.tiles_p), tuple(self.shards_p), tuple(self.samples_p), tuple(self.prefix_p), self.passes,
                self.wide, self.fold16)


# exported symbol -> (argtypes, restype)
SIGNATURES = {
    "fvb_abi_version": ([], c_i32),
    "fvb_last_error": ([], ctypes.c_char_p),
    "fvb_launch_count": ([], c_i64),
    "fvb_kernel_count": ([], c_i32),
    "fvb_kernel_name": ([c_i32], ctypes.c_char_p),
    "fvb_set_launch_ctas": ([c_i32, c_i32], c_i32),
    "fvb_get_launch_ctas": ([c_i32], c_i32),
    "fvb_set_wavefront_block": ([c_i32], c_i32),
    "fvb_get_wavefront_block": ([], c_i32),
    "fvb_set_tile_warps": ([c_i32], c_i32),
    "fvb_get_tile_warps": ([], c_i32),
    "fvb_set_decode_overlap": ([c_i32], c_i32),
    "fvb_get_decode_overlap": ([], c_i32),
    "fvb_set_rans_pipeline": ([c_i32], c_i32),
    "fvb_get_rans_pipeline": ([], c_i32),
    "fvb_set_rans_pipeline_tail": ([c_i32], c_i32),
    "fvb_get_rans_pipeline_tail": ([], c_i32),
    "fvb_profile_begin": ([], c_i32),
    "fvb_profile_end": ([c_p, c_p, c_i32], c_i32),
    "fvb_encode_plan": ([c_i64, c_i64, c_i32, c_i32, c_i32, c_i64, c_i64, c_i64, c_i64,
                         ctypes.POINTER(Frame), ctypes.POINTER(c_i64)], c_i32),
    "fvb_encode_analyze": ([ctypes.POINTER(Frame), c_p, c_p, c_p, c_i64, c_p, ctypes.POINTER(c_i64)], c_i32),
    "fvb_encode_emit": ([ctypes.POINTER(Frame), c_p, c_i64, c_p, c_i64, c_p], c_i32),
    "fvb_decode_plan": ([c_p, c_i64, c_i64, ctypes.POINTER(Frame), ctypes.POINTER(c_i64)], c_i32),
    "fvb_decode": ([ctypes.POINTER(Frame), c_p, c_i64, c_p, c_p, c_i32, c_p, c_i64, c_p], c_i32),
    "fvb_batch_encode_plan": ([ctypes.POINTER(Frame), c_i32, ctypes.POINTER(c_i64)], c_i32),
    "fvb_batch_encode_prepare": ([ctypes.POINTER(Frame), c_i32, c_p, c_p, c_p, c_i64, c_p], c_i32),
    "fvb_batch_encode_enqueue": ([ctypes.POINTER(Frame), c_i32, c_p, c_i64, c_p, c_p], c_i32),
    "fvb_batch_encode_emit": ([ctypes.POINTER(Frame), c_i32, c_p, c_i64, c_p, c_p], c_i32),
    "fvb_decode_noalloc_capacity": ([], c_i64),
    "fvb_decode_noalloc": ([ctypes.POINTER(Frame), c_p, c_i64, c_p, c_p, c_i32, c_p], c_i32),
    "fvb_gather_headers": ([c_p, c_p, c_i32, c_p, c_i64, c_p, c_p], c_i32),
    "fvb_batch_decode_plan": ([ctypes.POINTER(Frame), c_i32, ctypes.POINTER(c_i64)], c_i32),
    "fvb_batch_decode_prepare": ([ctypes.POINTER(Frame), c_i32, c_p, c_p, c_p, c_p, c_p, c_i64, c_p], c_i32),
    "fvb_batch_decode_enqueue": ([ctypes.POINTER(Frame), c_i32, c_i32, c_p, c_i64, c_p, c_p], c_i32),
    "fvb_batch_bucket": ([ctypes.POINTER(Frame), c_i32, ctypes.POINTER(Bucket)], c_i32),
    "fvb_bucket_encode_plan": ([ctypes.POINTER(Bucket), ctypes.POINTER(c_i64)], c_i32),
    "fvb_bucket_decode_plan": ([ctypes.POINTER(Bucket), ctypes.POINTER(c_i64)], c_i32),
    "fvb_bucket_encode_prepare": ([ctypes.POINTER(Bucket), ctypes.POINTER(Frame), c_i32, c_p, c_p, c_p, c_i64, c_p],
                                  c_i32),
    "fvb_bucket_encode_enqueue": ([ctypes.POINTER(Bucket), c_p, c_i64, c_p, c_p], c_i32),
    "fvb_bucket_encode_emit": ([ctypes.POINTER(Bucket), ctypes.POINTER(Frame), c_i32, c_p, c_i64, c_p, c_p], c_i32),
    "fvb_bucket_encode_headers": ([ctypes.POINTER(Bucket), c_p, c_i64, c_p, c_p], c_i32),
    "fvb_bucket_decode_prepare": ([ctypes.POINTER(Bucket), ctypes.POINTER(Frame), c_i32, c_p, c_p, c_p, c_p, c_p,
                                   c_i64, c_p], c_i32),
    "fvb_bucket_decode_enqueue": ([ctypes.POINTER(Bucket), c_i32, c_p, c_i64, c_p, c_p], c_i32),
}

_lib = None
_lock = threading.Lock()


def load():
    """Load (building once if absent) and return the ctypes library."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not LIB_PATH.exists():
            from . import build as _build

            _build.build()
        lib = ctypes.CDLL(str(LIB_PATH))
        for name, (argtypes, restype) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = argtypes
            fn.restype = restype
        if lib.fvb_abi_version() != ABI_VERSION:
            raise RuntimeError(f"{LIB_PATH} has ABI version {lib.fvb_abi_version()}, expected {ABI_VERSION}: "
                               "rebuild it (python -m fastvid_b200.build)")
        _lib = lib
    return _lib


def last_error() -> str:
    msg = load().fvb_last_error()
    return msg.decode() if msg else ""


def kernel_names() -> list[str]:
    lib = load()
    return [lib.fvb_kernel_name(i).decode() for i in range(lib.fvb_kernel_count())]


class KernelProfile:
    """Context manager: per-kernel device time (ms) and launch counts of the
    library's launches issued by this thread inside the block."""

    def __enter__(self):
        check(load().fvb_profile_begin())
        self.ms = {}
        self.launches = {}
        return self

    def __exit__(self, *exc):
        lib = load()
        n = lib.fvb_kernel_count()
        ms = (ctypes.c_double * n)()
        cnt = (c_i64 * n)()
        check(lib.fvb_profile_end(ms, cnt, n))
        for i, name in enumerate(kernel_names()):
            if cnt[i]:
                self.ms[name] = ms[i]
                self.launches[name] = cnt[i]
        return False


def launch_count() -> int:
    return int(load().fvb_launch_count())


def check(rc: int) -> None:
    if rc != 0:
        raise RuntimeError(last_error() or f"fastvid_b200 error {rc}")
