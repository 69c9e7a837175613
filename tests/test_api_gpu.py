"""The public ``fastvid`` API (fastvid/__init__.py:24-87) on a B200 against
the oracle: single frames and lists (the batched form), host and device
streams mixed in one list, ``inspect`` and ``inspect_batch``, and a host
stream larger than the staging chunk."""

import numpy as np
import pytest
import torch

import fastvid
import fastvid_b200
import oracle
from fastvid_b200 import synth
from fastvid_b200.api import inspect_batch

pytestmark = pytest.mark.gpu

FRAMES = [(200, 120, 11), (67, 35, 12), (321, 77, 13)]


def _frames(layout, depth):
    return [synth.make_frame(w, h, layout, depth, seed) for w, h, seed in FRAMES]


def _cuda(planes):
    return tuple(torch.from_numpy(np.ascontiguousarray(p)).cuda() for p in planes)


@pytest.mark.parametrize("layout,depth,quality", [("gray", 8, 100), ("yuv422", 10, 90), ("rgb444", 16, 70)])
def test_list_encode_and_decode_match_oracle(cuda, layout, depth, quality):
    host = _frames(layout, depth)
    streams = fastvid.encode([_cuda(f) for f in host], format=layout, bit_depth=depth, quality=quality,
                             tile_size=(64, 64))
    assert isinstance(streams, list) and len(streams) == len(host)
    expected = [oracle.encode(f, layout=layout, bit_depth=depth, quality=quality, tile_size=(64, 64)) for f in host]
    for got, exp in zip(streams, expected):
        assert bytes(got.cpu().numpy().tobytes()) == exp
    decoded = fastvid.decode(streams)
    # host and device streams in one list go through the batch as well
    mixed = fastvid.decode([s.cpu() if i % 2 else s for i, s in enumerate(streams)])
    for got, got_mixed, exp in zip(decoded, mixed, expected):
        ref = oracle.decode(exp)
        assert isinstance(got, tuple) and len(got) == len(ref)
        for a, b, c in zip(got, got_mixed, ref):
            assert np.array_equal(a.cpu().numpy(), c) and np.array_equal(b.cpu().numpy(), c)


def test_inspect_and_inspect_batch_match_the_stream_headers(cuda):
    host = _frames("yuv422", 12)
    streams = fastvid.encode([_cuda(f) for f in host], format="yuv422", bit_depth=12, quality=85,
                             tile_size=(32, 48))
    singles = [fastvid.inspect(s) for s in streams]
    assert inspect_batch(streams) == singles
    assert inspect_batch([s.cpu() for s in streams]) == singles
    for (w, h, _), info in zip(FRAMES, singles):
        tiles = oracle.geometry(w, h, "yuv422", (32, 48))[0]
        assert info == {"width": w, "height": h, "format": "yuv422", "bit_depth": 12, "frame_count": 1,
                        "metadata_bytes": 32 + 32 * tiles, "container_overhead_bytes": 0}
    with pytest.raises(TypeError):
        fastvid.inspect([streams[0]])
    with pytest.raises(ValueError):
        fastvid.inspect(torch.zeros(64, dtype=torch.uint8, device="cuda"))


def test_host_stream_above_the_staging_chunk_decodes_like_device_stream(cuda):
    planes = synth.make_frame(1920, 1080, "rgb444", 10, 14, sigma=(40, 1))
    stream = fastvid_b200.encode(_cuda(planes), layout="rgb444", bit_depth=10, quality=100, tile_size=(128, 128))
    assert stream.numel() > 2 << 20  # three or more staging chunks
    host = stream.cpu()
    for a, b, p in zip(fastvid_b200.decode(host), fastvid_b200.decode(stream), planes):
        assert torch.equal(a, b)
        assert np.array_equal(a.cpu().numpy(), p)  # lossless
