"""Public codec API over frames and batches (mirror of the reference's
``fastvid`` package, fastvid/__init__.py:24-87).

``encode`` / ``decode`` accept one frame (a tuple of planes) or one stream,
or a sequence of them.  The reference turns a sequence into a Python loop of
single-frame calls (fastvid/__init__.py:44-53, 63); here a sequence goes
through the batched form (fastvid_b200.batch), one launch of each kernel for
all frames, with byte-identical results frame by frame.
"""

from __future__ import annotations

import struct
from collections.abc import Sequence

import torch

from . import decode as _decode
from . import encode as _encode
from .batch import decode_batch, encode_batch, stream_headers

_LAYOUT_TO_FORMAT = {0: "gray", 1: "yuv422", 2: "rgb444"}


def _is_frame(value) -> bool:
    return (isinstance(value, (tuple, list)) and bool(value)
            and all(isinstance(plane, torch.Tensor) for plane in value))


def encode(frame, *, format: str, bit_depth: int, quality: int = 90, tile_size: tuple[int, int] = (256, 128)):
    """Encode one frame or a sequence of independent frames."""
    if _is_frame(frame):
        return _encode(frame, layout=format, bit_depth=bit_depth, quality=quality, tile_size=tile_size)
    if not isinstance(frame, Sequence):
        raise TypeError("frame must be planar tensors or a sequence of frames")
    frames = list(frame)
    if not frames:
        return []
    return encode_batch(frames, layout=format, bit_depth=bit_depth, quality=quality, tile_size=tile_size)


def decode(encoded):
    """Decode one independent stream or a sequence of streams."""
    if isinstance(encoded, torch.Tensor):
        return _decode(encoded)
    if not isinstance(encoded, Sequence):
        raise TypeError("encoded must be a byte tensor or a sequence of byte tensors")
    streams = list(encoded)
    if not streams:
        return []
    # host-resident streams join the batch: uploaded without blocking, their
    # headers read on the host
    return [tuple(planes) for planes in decode_batch(streams)]


def inspect(encoded) -> dict[str, int | str]:
    """Self-described frame metadata and exact overhead accounting (fastvid/__init__.py:66-87)."""
    if not isinstance(encoded, torch.Tensor) or encoded.dtype != torch.uint8 or encoded.ndim != 1:
        raise TypeError("encoded must be a one-dimensional uint8 tensor")
    return _describe(bytes(encoded[:32].cpu().numpy()))


def inspect_batch(streams) -> list[dict[str, int | str]]:
    """inspect() of every stream of a sequence (no reference counterpart: the
    reference inspects one stream per call).  The headers of the device
    streams come back with one gather kernel and one copy for all of them;
    the same checks and errors as inspect()."""
    streams = list(streams)
    for s in streams:
        if not isinstance(s, torch.Tensor) or s.dtype != torch.uint8 or s.ndim != 1:
            raise TypeError("encoded must be a one-dimensional uint8 tensor")
    return [_describe(h) for h in stream_headers(streams)]


def _describe(header: bytes) -> dict[str, int | str]:
    if len(header) != 32 or header[:4] != b"FVID" or header[4] != 1:
        raise ValueError("not a Fastvid supported stream")
    layout = header[5]
    if layout not in _LAYOUT_TO_FORMAT:
        raise ValueError("unknown pixel layout")
    width, height = struct.unpack_from("<II", header, 8)
    tile_count = struct.unpack_from("<I", header, 28)[0]
    return {
        "width": width,
        "height": height,
        "format": _LAYOUT_TO_FORMAT[layout],
        "bit_depth": (header[7] & 0x3F) + 8,
        "frame_count": 1,
        "metadata_bytes": 32 + tile_count * 32,
        "container_overhead_bytes": 0,
    }


__all__ = ["decode", "encode", "inspect", "inspect_batch"]
