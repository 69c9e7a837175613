"""The folded-symbol intermediate held as u16 (every frame of a batch below
bit depth 16 or quality 100) against the oracle:

* 16-bit streams whose symbols exceed 16 bits: a lossless 16-bit stream
  (symbols up to 2 * 65535) with its quality byte lowered below 100 is still
  a valid stream (the decoder accepts symbols up to 2 * max_sample), and is
  decoded through the u16 intermediate with saturated symbols; the planes
  must equal the oracle's decode of the same bytes;
* a batch mixing u16-eligible frames with a lossless 16-bit frame (u32),
  and the same u16-eligible frames alone (u16), give identical streams;
* a u32 bucket forced onto a u16-eligible batch gives identical streams.
"""

import numpy as np
import pytest
import torch

import oracle
from fastvid_b200 import _native
from fastvid_b200.batch import BatchCodec

pytestmark = pytest.mark.gpu


def _noise(layout, width, height, seed):
    rng = np.random.default_rng(seed)
    widths = {"gray": [width], "yuv422": [width, (width + 1) // 2, (width + 1) // 2], "rgb444": [width] * 3}[layout]
    return tuple(rng.integers(0, 65536, size=(height, w), dtype=np.uint16) for w in widths)


def _cuda(planes):
    return tuple(torch.from_numpy(np.ascontiguousarray(p)).cuda() for p in planes)


@pytest.mark.parametrize("layout", ["gray", "yuv422", "rgb444"])
@pytest.mark.parametrize("quality", [99, 50])
def test_wide_symbols_of_a_16bit_stream_decode_like_the_oracle(cuda, layout, quality):
    planes = _noise(layout, 150, 70, 7)
    # uniform 16-bit noise: about a quarter of the residuals exceed 2^15 in
    # magnitude, so their folded symbols exceed 16 bits
    row = planes[0][0].astype(np.int64)
    assert np.count_nonzero(np.abs(np.diff(row)) > 32767) > 0
    lossless = bytearray(oracle.encode(planes, layout=layout, bit_depth=16, quality=100, tile_size=(64, 32)))
    assert lossless[6] == 100
    lossless[6] = quality  # quality byte: step 12 (yuv422) or 44 (gray, rgb444) at 99
    stream = bytes(lossless)
    expected = oracle.decode(stream)
    codec = BatchCodec("cuda", use_graphs=False)
    dev = torch.frombuffer(bytearray(stream), dtype=torch.uint8).cuda()
    # alone (u16 intermediate) and beside an 8-bit frame (still u16)
    other = oracle.encode(tuple(p >> 8 for p in _noise("gray", 64, 40, 3)), layout="gray", bit_depth=8, quality=100)
    for batch in ([dev], [dev, torch.frombuffer(bytearray(other), dtype=torch.uint8).cuda()]):
        decoded = codec.decode(batch)
        for got, ref in zip(decoded[0], expected):
            assert np.array_equal(got.cpu().numpy(), ref)
    # the serial predictor reads the u16 intermediate too
    decoded = codec.decode([dev], predictor="serial")
    for got, ref in zip(decoded[0], expected):
        assert np.array_equal(got.cpu().numpy(), ref)


def _encode(codec, frames):
    return codec.encode([_cuda(f["planes"]) for f in frames], layout=[f["layout"] for f in frames],
                        bit_depth=[f["bit_depth"] for f in frames], quality=[f["quality"] for f in frames],
                        tile_size=[(64, 64)] * len(frames))


def _frames():
    rng = np.random.default_rng(11)
    out = []
    for layout, depth, quality in [("gray", 8, 100), ("rgb444", 10, 85), ("yuv422", 16, 90), ("gray", 16, 87),
                                   ("gray", 12, 100)]:
        planes = tuple((p >> (16 - depth)).astype(np.uint16) for p in _noise(layout, 130, 66, int(rng.integers(1 << 30))))
        # smooth the noise so predicted frames carry the usual small symbols
        planes = tuple(np.cumsum(p.astype(np.int64) % 7 - 3, axis=1).clip(0, (1 << depth) - 1).astype(np.uint16)
                       for p in planes)
        out.append(dict(planes=planes, layout=layout, bit_depth=depth, quality=quality))
    for f in out:
        f["oracle"] = oracle.encode(f["planes"], layout=f["layout"], bit_depth=f["bit_depth"], quality=f["quality"],
                                    tile_size=(64, 64))
    return out


def test_u16_and_u32_batches_give_the_same_streams(cuda):
    frames = _frames()
    lossless16 = dict(planes=_noise("gray", 90, 50, 5), layout="gray", bit_depth=16, quality=100)
    lossless16["oracle"] = oracle.encode(lossless16["planes"], layout="gray", bit_depth=16, quality=100,
                                         tile_size=(64, 64))
    codec = BatchCodec("cuda", use_graphs=False)
    for batch in (frames, frames + [lossless16], [lossless16] + frames[:2]):
        streams = _encode(codec, batch)
        for f, s in zip(batch, streams):
            assert bytes(s.cpu().numpy()) == f["oracle"]
        decoded = codec.decode(streams)
        for f, planes in zip(batch, decoded):
            for got, ref in zip(planes, oracle.decode(f["oracle"])):
                assert np.array_equal(got.cpu().numpy(), ref)
    keys = [k for k in codec._enc] + [k for k in codec._dec]
    assert {k[-1] for k in keys} == {0, 1}  # both intermediate widths ran


class _U32Buckets:
    """The library with every bucket widened to the u32 intermediate."""

    def __init__(self, lib):
        self._lib = lib

    def fvb_batch_bucket(self, arr, n, bucket_ref):
        rc = self._lib.fvb_batch_bucket(arr, n, bucket_ref)
        bucket_ref._obj.fold16 = 0
        return rc

    def __getattr__(self, name):
        return getattr(self._lib, name)


def test_u32_bucket_serves_a_u16_batch(cuda):
    frames = _frames()
    codec = BatchCodec("cuda", use_graphs=False)
    codec.lib = _U32Buckets(_native.load())
    streams = _encode(codec, frames)
    for f, s in zip(frames, streams):
        assert bytes(s.cpu().numpy()) == f["oracle"]
    decoded = codec.decode(streams)
    for f, planes in zip(frames, decoded):
        for got, ref in zip(planes, oracle.decode(f["oracle"])):
            assert np.array_equal(got.cpu().numpy(), ref)
    assert all(k[-1] == 0 for k in list(codec._enc) + list(codec._dec))
