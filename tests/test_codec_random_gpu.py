"""Parity of the sm_100a path with the oracle over a seeded sweep of random
small frames: odd sizes and tile shapes, every layout and depth, qualities
from 1 to 100.  Each frame is encoded and decoded alone through the
fastvid_cuda-compatible API and all of them together in one mixed batch;
the stream bytes and decoded planes must equal the oracle's."""

import numpy as np
import pytest
import torch

import fastvid_b200
import oracle
from fastvid_b200 import synth
from fastvid_b200.batch import BatchCodec

pytestmark = pytest.mark.gpu


def _cases(n=48, seed=20261204):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        layout = ("gray", "yuv422", "rgb444")[i % 3]
        depth = (8, 10, 12, 16)[(i // 3) % 4]
        w, h = int(rng.integers(1, 300)), int(rng.integers(1, 200))
        tile = (int(rng.choice([2, 7, 16, 33, 64, 100, 256])), int(rng.choice([1, 5, 16, 31, 64, 128])))
        q = int(rng.choice([100, int(rng.integers(1, 100))]))
        out.append(dict(layout=layout, bit_depth=depth, width=w, height=h, tile=tile, quality=q, seed=900 + i))
    return out


CASES = _cases()


def _frame(c):
    return synth.make_frame(c["width"], c["height"], c["layout"], c["bit_depth"], c["seed"])


def test_random_frames_alone_match_the_oracle(cuda):
    for c in CASES:
        planes = _frame(c)
        kw = dict(layout=c["layout"], bit_depth=c["bit_depth"], quality=c["quality"], tile_size=c["tile"])
        expected = oracle.encode(planes, **kw)
        got = fastvid_b200.encode(tuple(torch.from_numpy(p).to(cuda) for p in planes), **kw)
        assert bytes(got.cpu().numpy()) == expected, c
        for a, b in zip(fastvid_b200.decode(got), oracle.decode(expected)):
            assert np.array_equal(a.cpu().numpy(), b), c


def test_random_frames_in_one_batch_match_the_oracle(cuda):
    frames = [tuple(torch.from_numpy(p).to(cuda) for p in _frame(c)) for c in CASES]
    codec = BatchCodec(cuda)
    streams = codec.encode(frames, layout=[c["layout"] for c in CASES], bit_depth=[c["bit_depth"] for c in CASES],
                           quality=[c["quality"] for c in CASES], tile_size=[c["tile"] for c in CASES])
    decoded = codec.decode(streams)
    for c, s, planes in zip(CASES, streams, decoded):
        expected = oracle.encode(_frame(c), layout=c["layout"], bit_depth=c["bit_depth"], quality=c["quality"],
                                 tile_size=c["tile"])
        assert bytes(s.cpu().numpy()) == expected, c
        for a, b in zip(planes, oracle.decode(expected)):
            assert np.array_equal(a.cpu().numpy(), b), c
