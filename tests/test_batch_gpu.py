"""GPU parity tests of the batched form (one launch per kernel for a whole
batch of mixed frames).

Every frame of a mixed batch -- all layouts and depths, frames that take the
gray10 MED re-run and the gray16 step refinements, ragged tiles, tiles of one
column -- must encode to exactly the bytes the oracle writes for it alone and
decode to exactly the oracle's planes, whatever the frames' order in the batch
and whether the batch runs eagerly or from a captured CUDA graph.
"""

import random

import numpy as np
import pytest
import torch

import oracle
from fastvid_b200 import synth
from fastvid_b200.batch import BatchCodec

pytestmark = pytest.mark.gpu

# (width, height, layout, depth, quality, tile, noise sd)
SPECS = [
    (320, 200, "gray", 16, 87, (64, 64), (40, 1)),     # a refined-step trial that loses
    (300, 170, "gray", 10, 85, (128, 64), (3, 1)),     # MED re-run candidate
    (263, 133, "rgb444", 10, 90, (256, 128), (3, 1)),
    (301, 203, "yuv422", 8, 80, (67, 35), (2, 1)),
    (67, 35, "gray", 8, 100, (256, 128), (3, 1)),
    (200, 120, "gray", 16, 100, (64, 32), (1, 2)),     # lossless gray16: one pass
    (150, 90, "gray", 10, 100, (32, 32), (1, 2)),
    (96, 64, "rgb444", 8, 90, (64, 64), (1, 2)),
    (9, 7, "gray", 10, 80, (1, 3), (2, 1)),
    (257, 129, "gray", 12, 95, (600, 40), (3, 1)),
    (128, 96, "gray", 16, 60, (128, 128), (1, 2)),
    (160, 100, "yuv422", 10, 85, (64, 64), (3, 1)),
]


def _frames():
    frames = []
    for i, (w, h, layout, depth, q, tile, sd) in enumerate(SPECS):
        planes = synth.make_frame(w, h, layout, depth, 500 + i, sigma=sd)
        frames.append(dict(planes=planes, layout=layout, bit_depth=depth, quality=q, tile=tile))
    return frames


@pytest.fixture(scope="module")
def mixed():
    frames = _frames()
    for f in frames:
        f["oracle"] = oracle.encode(f["planes"], layout=f["layout"], bit_depth=f["bit_depth"],
                                    quality=f["quality"], tile_size=f["tile"], threads=4)
    return frames


def _encode(codec, frames):
    return codec.encode([tuple(torch.from_numpy(p).cuda() for p in f["planes"]) for f in frames],
                        layout=[f["layout"] for f in frames], bit_depth=[f["bit_depth"] for f in frames],
                        quality=[f["quality"] for f in frames], tile_size=[f["tile"] for f in frames])


def test_mixed_batch_streams_equal_the_oracle(cuda, mixed):
    codec = BatchCodec("cuda", use_graphs=False)
    streams = _encode(codec, mixed)
    for i, (f, s) in enumerate(zip(mixed, streams)):
        assert bytes(s.cpu().numpy()) == f["oracle"], i


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_frame_order_does_not_change_any_stream(cuda, mixed, seed):
    order = list(range(len(mixed)))
    random.Random(seed).shuffle(order)
    codec = BatchCodec("cuda", use_graphs=False)
    streams = _encode(codec, [mixed[i] for i in order])
    for pos, i in enumerate(order):
        assert bytes(streams[pos].cpu().numpy()) == mixed[i]["oracle"], (pos, i)


def test_graph_replays_equal_eager(cuda, mixed):
    codec = BatchCodec("cuda", use_graphs=True)
    for _ in range(2):  # capture, then replay
        streams = _encode(codec, mixed)
        for f, s in zip(mixed, streams):
            assert bytes(s.cpu().numpy()) == f["oracle"]


def test_single_frames_equal_their_batch(cuda, mixed):
    codec = BatchCodec("cuda", use_graphs=False)
    for f in mixed[:4]:
        (s,) = _encode(codec, [f])
        assert bytes(s.cpu().numpy()) == f["oracle"]


@pytest.mark.parametrize("predictor", ["wavefront", "serial"])
def test_mixed_batch_decodes_equal_the_oracle(cuda, mixed, predictor):
    codec = BatchCodec("cuda", use_graphs=False)
    streams = [torch.frombuffer(bytearray(f["oracle"]), dtype=torch.uint8).cuda() for f in mixed]
    decoded = codec.decode(streams, predictor=predictor)
    for f, planes in zip(mixed, decoded):
        want = oracle.decode(f["oracle"])
        assert len(planes) == len(want)
        for got, ref in zip(planes, want):
            assert np.array_equal(got.cpu().numpy(), ref)


def test_failing_frame_is_reported_at_its_own_index(cuda, mixed):
    # a gray8 frame with a sample above 255, placed ahead of frames the
    # encoder lays out first (gray16, gray10)
    bad = dict(mixed[4])
    planes = [p.copy() for p in bad["planes"]]
    planes[0][3, 5] = 300
    bad["planes"] = tuple(planes)
    frames = [mixed[2], bad, mixed[0], mixed[1]]
    codec = BatchCodec("cuda", use_graphs=False)
    with pytest.raises(RuntimeError, match=r"^frame 1: "):
        _encode(codec, frames)
    streams = _encode(codec, [mixed[2], mixed[4], mixed[0], mixed[1]])
    for s, f in zip(streams, [mixed[2], mixed[4], mixed[0], mixed[1]]):
        assert bytes(s.cpu().numpy()) == f["oracle"]


@pytest.mark.parametrize("chunk", [1, 3, 16])
def test_host_pipelines_equal_the_device_path(cuda, mixed, chunk):
    codec = BatchCodec("cuda")
    host = [tuple(torch.from_numpy(p).pin_memory() for p in f["planes"]) for f in mixed]
    params = dict(layout=[f["layout"] for f in mixed], bit_depth=[f["bit_depth"] for f in mixed],
                  quality=[f["quality"] for f in mixed], tile_size=[f["tile"] for f in mixed])
    streams = codec.encode_host(host, chunk=chunk, **params)
    assert all(not s.is_cuda and s.is_pinned() for s in streams)
    for f, s in zip(mixed, streams):
        assert bytes(s.numpy()) == f["oracle"]
    planes = codec.decode_host(streams, chunk=chunk)
    for f, got in zip(mixed, planes):
        want = oracle.decode(f["oracle"])
        assert len(got) == len(want)
        for g, w in zip(got, want):
            assert not g.is_cuda and np.array_equal(g.numpy(), w)


def test_batches_of_one_bucket_replay_one_graph(cuda):
    """Two batches of different frames whose counts fall into the same shape
    bucket share one captured graph per direction, and each still writes the
    oracle's bytes and planes."""
    codec = BatchCodec(cuda)
    base = [(640, 360, "rgb444", 8, 90, (64, 64)), (600, 352, "rgb444", 8, 90, (64, 64))]
    batches = []
    for seed, (w, h, layout, depth, q, tile) in enumerate(base):
        frames = [dict(planes=synth.make_frame(w, h, layout, depth, 900 + 10 * seed + k), layout=layout,
                       bit_depth=depth, quality=q, tile=tile) for k in range(3)]
        batches.append(frames)
    for frames in batches + batches:
        streams = _encode(codec, frames)
        planes = codec.decode(streams)
        for f, st, pl in zip(frames, streams, planes):
            exp = oracle.encode(f["planes"], layout=f["layout"], bit_depth=f["bit_depth"], quality=f["quality"],
                                tile_size=f["tile"])
            assert bytes(st.cpu().numpy().tobytes()) == exp
            for a, b in zip(pl, oracle.decode(exp)):
                assert np.array_equal(a.cpu().numpy(), b)
    assert len(codec._enc) == 1 and len(codec._dec) == 1  # one bucket each way
    assert codec.graph_kernels > 0  # later batches replayed the captured graphs


def test_host_round_trip_matches_device_batch(cuda, mixed):
    """encode_decode_host (pinned frames in, streams and planes out, copies
    overlapping the kernels chunk by chunk) returns the oracle's streams and
    planes, with a chunk size that splits the batch unevenly and an output
    buffer too small for all of it."""
    codec = BatchCodec(cuda)
    pinned = [tuple(torch.from_numpy(np.ascontiguousarray(p)).pin_memory() for p in f["planes"]) for f in mixed]
    total_bytes = sum(len(f["oracle"]) for f in mixed)
    out_s = torch.empty(total_bytes // 2, dtype=torch.uint8).pin_memory()  # later chunks get new buffers
    streams, planes = codec.encode_decode_host(pinned, chunk=5, layout=[f["layout"] for f in mixed],
                                               bit_depth=[f["bit_depth"] for f in mixed],
                                               quality=[f["quality"] for f in mixed],
                                               tile_size=[f["tile"] for f in mixed], out_streams=out_s)
    assert len(streams) == len(planes) == len(mixed)
    for f, st, pl in zip(mixed, streams, planes):
        assert not st.is_cuda and bytes(st.numpy().tobytes()) == f["oracle"]
        for a, b in zip(pl, oracle.decode(f["oracle"])):
            assert not a.is_cuda and np.array_equal(a.numpy(), b)


@pytest.mark.parametrize("block", [4, 8, 16, 32])
def test_wavefront_knobs_keep_the_bytes(cuda, mixed, block):
    """Every wavefront block, and warp pairs per tile (tiles of one band or
    of fewer than 66 columns stay on one warp), write the oracle's streams
    and decode to the oracle's planes: the knobs change only the schedule."""
    from fastvid_b200 import autotune

    before = (autotune.wavefront_block(), autotune.tile_warps())
    extra = [dict(planes=synth.make_frame(w, h, "gray", 10, 700 + w, sigma=(3, 1)), layout="gray", bit_depth=10,
                  quality=90, tile=tile) for w, h, tile in ((300, 257, (128, 256)), (97, 95, (97, 40)),
                                                             (65, 200, (65, 100)), (130, 33, (130, 33)))]
    for f in extra:
        f["oracle"] = oracle.encode(f["planes"], layout=f["layout"], bit_depth=f["bit_depth"], quality=f["quality"],
                                    tile_size=f["tile"])
    frames = mixed + extra
    try:
        for warps in (1, 2):
            autotune.set_wavefront_block(block)
            autotune.set_tile_warps(warps)
            codec = BatchCodec(cuda, use_graphs=False)
            streams = _encode(codec, frames)
            planes = codec.decode(streams)
            for f, st, pl in zip(frames, streams, planes):
                assert bytes(st.cpu().numpy().tobytes()) == f["oracle"], (block, warps)
                for a, b in zip(pl, oracle.decode(f["oracle"])):
                    assert np.array_equal(a.cpu().numpy(), b), (block, warps)
    finally:
        autotune.set_wavefront_block(before[0])
        autotune.set_tile_warps(before[1])


@pytest.mark.parametrize("pipe,tail", [(8, 16), (16, 8), (0, 16)])
def test_rans_pipeline_keeps_the_bytes(cuda, mixed, pipe, tail):
    """The pipelined rANS encoder fetch, in the first pass and in the
    later passes of the frame policy, writes the oracle's streams."""
    from fastvid_b200 import autotune

    before = autotune.rans_pipeline(), autotune.rans_pipeline_tail()
    try:
        autotune.set_rans_pipeline(pipe)
        autotune.set_rans_pipeline_tail(tail)
        codec = BatchCodec(cuda, use_graphs=False)
        for f, st in zip(mixed, _encode(codec, mixed)):
            assert bytes(st.cpu().numpy().tobytes()) == f["oracle"], (pipe, tail)
    finally:
        autotune.set_rans_pipeline(before[0])
        autotune.set_rans_pipeline_tail(before[1])


def test_encoder_returns_the_stream_headers(cuda, mixed):
    """encode(..., return_headers=True) hands back each stream's 32-byte
    header (written by a kernel into pinned memory with the results), the
    final pass's flags included; decoding with them equals decoding
    without."""
    for graphs in (False, True):
        codec = BatchCodec(cuda, use_graphs=graphs)
        frames = [tuple(torch.from_numpy(p).cuda() for p in f["planes"]) for f in mixed]
        kw = dict(layout=[f["layout"] for f in mixed], bit_depth=[f["bit_depth"] for f in mixed],
                  quality=[f["quality"] for f in mixed], tile_size=[f["tile"] for f in mixed])
        for _ in range(2):  # eager, then (graphs) a replay
            streams, heads = codec.encode(frames, return_headers=True, **kw)
            assert len(heads) == len(streams)
            for f, st, h in zip(mixed, streams, heads):
                assert h == f["oracle"][:32] == bytes(st[:32].cpu().numpy().tobytes())
            with_heads = codec.decode(streams, headers=heads)
            without = codec.decode(streams)
            for a, b in zip(with_heads, without):
                assert all(torch.equal(x, y) for x, y in zip(a, b))

