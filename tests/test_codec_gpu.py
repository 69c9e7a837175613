"""GPU parity tests of the sm_100a path (called through the C ABI).

* the reference test suite (cuda/tests/test_codec.py) against fastvid_b200;
* every golden case: stream bytes identical to the reference's (SHA-256),
  decodes identical to the reference's, for wavefront and serial
  reconstruction and for CUDA- and CPU-resident streams;
* malformed streams: random mutations are accepted or rejected exactly as
  the oracle accepts or rejects them, with identical planes when accepted.
"""

import hashlib
import json
import struct
import sys
import zlib
from pathlib import Path

import numpy as np
import pytest
import torch

import fastvid_b200
import oracle
from fastvid_b200 import synth

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))
import cases as golden_cases  # noqa: E402

RECORDS = json.loads((GOLDEN / "reference_streams.json").read_text())["cases"]
ALL = golden_cases.all_cases()


def _cuda(planes):
    return tuple(torch.from_numpy(np.ascontiguousarray(p)).cuda() for p in planes)


def _sha_planes(planes) -> str:
    h = hashlib.sha256()
    for p in planes:
        arr = p.cpu().numpy() if isinstance(p, torch.Tensor) else p
        h.update(np.ascontiguousarray(arr, dtype=np.uint16).astype("<u2").tobytes())
    return h.hexdigest()


def _source_planes(layout, width, height, bit_depth, pattern="polynomial"):
    return tuple(torch.from_numpy(p) for p in synth.reference_pattern(layout, width, height, bit_depth, pattern))


def _shard_modes(stream):
    tile_count = struct.unpack_from("<I", stream, 28)[0]
    modes = set()
    for tile in range(tile_count):
        entry = 32 + tile * 32
        width, height = struct.unpack_from("<II", stream, entry + 12)
        cursor = struct.unpack_from("<Q", stream, entry + 20)[0]
        tile_end = cursor + struct.unpack_from("<I", stream, entry + 28)[0]
        decoded = 0
        while decoded < width * height:
            modes.add(stream[cursor])
            cursor += 3 + struct.unpack_from("<H", stream, cursor + 1)[0]
            decoded += min(4096, width * height - decoded)
        assert cursor == tile_end
    return modes


# ---- the reference suite, against fastvid_b200 --------------------------------

@pytest.mark.parametrize("layout", ("gray", "yuv422", "rgb444"))
@pytest.mark.parametrize("bit_depth", (8, 10, 12, 16))
def test_q100_roundtrip_is_exact_and_emits_version_one(cuda, layout, bit_depth):
    source = _source_planes(layout, 67, 35, bit_depth)
    cuda_source = tuple(plane.cuda() for plane in source)
    first = fastvid_b200.encode(cuda_source, layout=layout, bit_depth=bit_depth, quality=100)
    second = fastvid_b200.encode(cuda_source, layout=layout, bit_depth=bit_depth, quality=100)
    assert first.is_cuda and first.dtype == torch.uint8
    assert bytes(first.cpu().numpy()) == bytes(second.cpu().numpy())
    assert int(first[4].item()) == 1
    for placement in (first.cpu(), first):
        for predictor in ("wavefront", "serial"):
            actual = fastvid_b200.decode(placement, predictor=predictor)
            assert len(actual) == len(source)
            for result, expected in zip(actual, source):
                assert result.is_cuda and result.dtype == torch.uint16
                assert torch.equal(result.cpu(), expected)


def test_lossy_stream_is_deterministic_and_exercises_entropy_modes(cuda):
    selected_modes = set()
    for quality, pattern in ((90, "ramp"), (100, "zero"), (100, "polynomial")):
        source = _source_planes("yuv422", 263, 133, 10, pattern)
        stream = fastvid_b200.encode(tuple(p.cuda() for p in source), layout="yuv422", bit_depth=10, quality=quality)
        selected_modes.update(_shard_modes(bytes(stream.cpu().numpy())))
        wavefront = fastvid_b200.decode(stream, predictor="wavefront")
        serial = fastvid_b200.decode(stream, predictor="serial")
        assert all(torch.equal(a, b) for a, b in zip(wavefront, serial))
    assert 0 in selected_modes
    assert 18 in selected_modes
    assert any(1 <= mode <= 17 for mode in selected_modes)


def test_decode_rejects_other_versions_and_malformed_streams(cuda):
    source = _source_planes("yuv422", 263, 133, 10)
    stream = bytearray(fastvid_b200.encode(tuple(p.cuda() for p in source), layout="yuv422", bit_depth=10,
                                           quality=100).cpu().numpy())
    first_payload = struct.unpack_from("<Q", stream, 32 + 20)[0]
    mutations = []
    m = bytearray(stream)
    m[4] = 7
    mutations.append(m)
    m = bytearray(stream)
    m[32 + 3] = 1
    mutations.append(m)
    m = bytearray(stream)
    struct.pack_into("<Q", m, 32 + 20, first_payload + 1)
    mutations.append(m)
    m = bytearray(stream)
    m[first_payload] = 255
    mutations.append(m)
    mutations.append(bytearray(stream[:-1]))
    mutations.append(bytearray(stream + b"\x00"))
    for malformed in mutations:
        with pytest.raises(RuntimeError):
            fastvid_b200.decode(torch.frombuffer(malformed, dtype=torch.uint8).cuda())


# ---- golden parity -----------------------------------------------------------

@pytest.mark.parametrize("case", ALL, ids=lambda c: c["name"])
def test_stream_bytes_match_reference(cuda, case):
    rec = RECORDS[case["name"]]
    planes = case["make"]()
    stream = fastvid_b200.encode(_cuda(planes), layout=case["layout"], bit_depth=case["bit_depth"],
                                 quality=case["quality"], tile_size=case["tile"])
    data = bytes(stream.cpu().numpy().tobytes())
    assert len(data) == rec["stream_len"]
    assert hashlib.sha256(data).hexdigest() == rec["stream_sha256"]
    if not case["big"]:
        assert data == oracle.encode(planes, layout=case["layout"], bit_depth=case["bit_depth"],
                                     quality=case["quality"], tile_size=case["tile"], threads=4)
    for predictor in ("wavefront", "serial"):
        decoded = fastvid_b200.decode(stream, predictor=predictor)
        assert _sha_planes(decoded) == rec["decoded_sha256"], predictor
    if not case["big"]:
        decoded_host = fastvid_b200.decode(stream.cpu())
        assert _sha_planes(decoded_host) == rec["decoded_sha256"]


def test_config_3a_gray16_4k_refines_to_step_417(cuda):
    """3840x2160 gray16 q87: the reference's frame policy refines the step
    from 556 to 417 (header flag 0x80, encode.cu:826-840); so does this one."""
    rec = RECORDS["cfg_gray16_4k_step417"]
    assert rec["flags"] == 0x88  # refined gray16 (0x80) | depth 16 (0x08), as the reference wrote it
    case = golden_cases.case_map()["cfg_gray16_4k_step417"]
    stream = fastvid_b200.encode(_cuda(case["make"]()), layout="gray", bit_depth=16, quality=87,
                                 tile_size=(128, 128))
    from fastvid_b200.codec import plan_decode

    frame, _ = plan_decode(stream)
    assert stream[7].item() == 0x88 and frame.step == 417 and frame.flags == 0x80


def test_pitched_and_strided_planes_encode_like_contiguous(cuda):
    planes = synth.make_frame(301, 97, "rgb444", 10, 77)
    base = fastvid_b200.encode(_cuda(planes), layout="rgb444", bit_depth=10, quality=88, tile_size=(64, 32))
    padded = []
    for p in planes:
        big = torch.zeros((p.shape[0], p.shape[1] + 13), dtype=torch.uint16, device="cuda")
        big[:, 5:5 + p.shape[1]] = torch.from_numpy(p).cuda()
        padded.append(big[:, 5:5 + p.shape[1]])
    got = fastvid_b200.encode(tuple(padded), layout="rgb444", bit_depth=10, quality=88, tile_size=(64, 32))
    assert torch.equal(base, got)
    transposed = [torch.from_numpy(np.ascontiguousarray(p.T)).cuda().T for p in planes]
    got_t = fastvid_b200.encode(tuple(transposed), layout="rgb444", bit_depth=10, quality=88, tile_size=(64, 32))
    assert torch.equal(base, got_t)


def test_encode_on_side_stream_matches(cuda):
    planes = _cuda(synth.make_frame(640, 360, "rgb444", 8, 78))
    base = fastvid_b200.encode(planes, layout="rgb444", bit_depth=8, quality=90, tile_size=(64, 64))
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        got = fastvid_b200.encode(planes, layout="rgb444", bit_depth=8, quality=90, tile_size=(64, 64))
        dec = fastvid_b200.decode(got)
    side.synchronize()
    assert torch.equal(base, got)
    assert all(torch.equal(a, b) for a, b in zip(dec, fastvid_b200.decode(base)))


def test_encoder_rejects_samples_above_depth(cuda):
    planes = _cuda(synth.make_frame(64, 64, "gray", 10, 79))
    bad = planes[0].clone()
    bad[3, 7] = 1024
    with pytest.raises(RuntimeError, match="status 1"):
        fastvid_b200.encode((bad,), layout="gray", bit_depth=10, quality=100)


def test_encoder_argument_errors(cuda):
    plane = torch.zeros((16, 16), dtype=torch.uint16, device="cuda")
    with pytest.raises(RuntimeError, match="bit_depth must be 8, 10, 12, or 16"):
        fastvid_b200.encode((plane,), layout="gray", bit_depth=9)
    with pytest.raises(RuntimeError, match="plane count does not match layout"):
        fastvid_b200.encode((plane,), layout="rgb444", bit_depth=8)
    with pytest.raises(RuntimeError, match="encoder input planes must be CUDA tensors"):
        fastvid_b200.encode((plane.cpu(),), layout="gray", bit_depth=8)
    with pytest.raises(RuntimeError, match="two-dimensional uint16"):
        fastvid_b200.encode((plane.to(torch.int16),), layout="gray", bit_depth=8)
    with pytest.raises(RuntimeError, match="plane dimensions do not match declared layout"):
        fastvid_b200.encode((plane, plane, plane[:, :8]), layout="rgb444", bit_depth=8)
    with pytest.raises(ValueError):
        fastvid_b200.decode(torch.zeros(40, dtype=torch.uint8), predictor="diagonal")


# ---- malformed streams: accept/reject exactly like the oracle -----------------

def _mutations(stream: bytes, rng: np.random.Generator, count: int):
    out = []
    n = len(stream)
    for _ in range(count):
        kind = int(rng.integers(0, 5))
        b = bytearray(stream)
        if kind == 0:  # flip a bit in the payload
            i = int(rng.integers(32, n))
            b[i] ^= 1 << int(rng.integers(0, 8))
        elif kind == 1:  # random byte in the payload
            b[int(rng.integers(32, n))] = int(rng.integers(0, 256))
        elif kind == 2:  # truncate
            b = b[:int(rng.integers(32, n))]
        elif kind == 3:  # append
            b += bytes(rng.integers(0, 256, size=int(rng.integers(1, 5))).astype(np.uint8))
        else:  # corrupt the directory
            i = int(rng.integers(32, min(n, 32 + 32 * struct.unpack_from("<I", stream, 28)[0])))
            b[i] ^= 1 << int(rng.integers(0, 8))
        out.append(bytes(b))
    return out


@pytest.mark.parametrize("name", ["ref_yuv42210_67x35_q90", "ref_rgb4448_67x35_q90", "ref_gray16_67x35_q50",
                                  "ref_yuv422_10_263x133_ramp_q90", "flat_gray8", "tiles_1x3_gray10",
                                  "ref_gray12_67x35_q100", "zero_rgb12"])
def test_mutated_streams_accepted_or_rejected_like_oracle(cuda, name):
    case = golden_cases.case_map()[name]
    stream = oracle.encode(case["make"](), layout=case["layout"], bit_depth=case["bit_depth"],
                           quality=case["quality"], tile_size=case["tile"])
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    accepted = rejected = 0
    for bad in _mutations(stream, rng, 60):
        try:
            expected = oracle.decode(bad)
        except oracle.OracleError:
            expected = None
        tensor = torch.frombuffer(bytearray(bad), dtype=torch.uint8).cuda()
        if expected is None:
            with pytest.raises(RuntimeError):
                fastvid_b200.decode(tensor)
            rejected += 1
        else:
            got = fastvid_b200.decode(tensor)
            assert all(np.array_equal(g.cpu().numpy(), e) for g, e in zip(got, expected))
            accepted += 1
    assert rejected > 0


def _sparse_gray8(width, height, seed):
    rng = np.random.default_rng(seed)
    plane = np.full((height, width), 128, dtype=np.uint16)
    idx = rng.integers(0, width * height, size=width * height // 40)
    plane.flat[idx] = rng.integers(0, 256, size=idx.size)
    return (plane,)


@pytest.mark.parametrize("kind", ["zero_run", "rice"])
def test_mutated_zero_run_and_rice_payloads_like_oracle(cuda, kind):
    """Mutations aimed at the payload of frames whose shards are zero-run
    (sparse content) or Rice (noise): the warp-parallel zero-run parser and
    the shared-memory Rice lanes accept or reject exactly as the serial
    oracle does, and decode what they accept identically."""
    if kind == "zero_run":
        planes = _sparse_gray8(200, 96, 5)
    else:
        planes = synth.make_frame(200, 96, "gray", 8, 6, sigma=(3, 1))
    tile = (64, 64)
    folded, _, _ = oracle.predict(planes, layout="gray", bit_depth=8, tile_size=tile, step=1, use_med=0)
    rows, _ = oracle.analyze(folded, width=200, height=96, layout="gray", tile_size=tile, force_order0=False)
    modes = rows[:, 0]
    assert ((modes == 0).sum() if kind == "zero_run" else ((modes >= 1) & (modes <= 17)).sum()) >= len(modes) // 2
    stream = oracle.encode(planes, layout="gray", bit_depth=8, quality=100, tile_size=tile)
    rng = np.random.default_rng(17 if kind == "zero_run" else 18)
    payload0 = 32 + 32 * struct.unpack_from("<I", stream, 28)[0]
    accepted = rejected = 0
    for _ in range(160):
        b = bytearray(stream)
        for _ in range(int(rng.integers(1, 3))):
            i = int(rng.integers(payload0, len(b)))
            b[i] = int(rng.integers(0, 256)) if rng.random() < 0.5 else b[i] ^ (1 << int(rng.integers(0, 8)))
        try:
            expected = oracle.decode(bytes(b))
        except oracle.OracleError:
            expected = None
        tensor = torch.frombuffer(bytearray(b), dtype=torch.uint8).cuda()
        if expected is None:
            with pytest.raises(RuntimeError):
                fastvid_b200.decode(tensor)
            rejected += 1
        else:
            got = fastvid_b200.decode(tensor)
            assert all(np.array_equal(g.cpu().numpy(), e) for g, e in zip(got, expected))
            accepted += 1
    assert rejected > 0 and accepted > 0
