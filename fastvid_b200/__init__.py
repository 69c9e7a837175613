"""fastvid_b200 -- B200-native (sm_100a) fastvid intra codec.

Drop-in for the reference ``fastvid_cuda`` module
(cuda/fastvid_cuda/__init__.py:8-58): ``encode`` and ``decode`` keep its
signature, argument normalisation and errors, and produce byte-identical
streams / bit-exact planes.  ``fastvid_b200.api`` mirrors the public
``fastvid`` package (encode/decode/inspect over frames and batches), and
``fastvid_b200.batch`` / ``fastvid_b200.serve`` are the batched and served forms.
"""

from __future__ import annotations

import torch

from .codec import _C

_LAYOUTS = {"gray": 0, "yuv422": 1, "rgb444": 2}


def encode(planes, *, layout=None, bit_depth=10, quality=90, frame_rate=(24, 1), tile_size=(256, 128)):
    """Encode one CUDA uint16 grayscale or planar frame to a 1-D CUDA uint8 stream.

    ``planes`` is ``(Y,)`` or ``(Y, Cb, Cr)``; the layout is inferred from the
    plane shapes when not given (cuda/fastvid_cuda/__init__.py:24-33).
    """
    if isinstance(planes, torch.Tensor):
        planes = (planes,)
    else:
        planes = tuple(planes)
    if layout is None:
        layout = 0 if len(planes) == 1 else (1 if planes[1].shape[1] != planes[0].shape[1] else 2)
    elif isinstance(layout, str):
        layout = _LAYOUTS[layout]
    fps_numerator, fps_denominator = frame_rate
    tile_width, tile_height = tile_size
    return _C.encode(list(planes), layout, bit_depth, quality, fps_numerator, fps_denominator, tile_width,
                     tile_height)


def decode(encoded, predictor="wavefront"):
    """Decode one stream (1-D uint8, CPU or CUDA) to a tuple of CUDA uint16 planes."""
    if predictor not in ("wavefront", "serial"):
        raise ValueError("predictor must be 'wavefront' or 'serial'")
    return tuple(_C.decode(encoded, predictor == "wavefront"))


__all__ = ["decode", "encode"]
