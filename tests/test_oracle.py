"""CPU tests of the oracle: pinned to the reference's own outputs.

reference_streams.json holds, per case, the SHA-256 of the stream the
reference CUDA encoder produced on a B200 and of the planes its decoder
returned (made by tests/golden/make_golden.py).  The oracle must reproduce
both exactly; the reference test suite's properties (cuda/tests/test_codec.py)
are checked on the oracle as well.
"""

import hashlib
import json
import struct
from pathlib import Path

import numpy as np
import pytest

import oracle
from fastvid_b200 import synth

GOLDEN = Path(__file__).resolve().parent / "golden"

import sys  # noqa: E402

sys.path.insert(0, str(GOLDEN))
import cases as golden_cases  # noqa: E402

RECORDS = json.loads((GOLDEN / "reference_streams.json").read_text())["cases"]
SMALL = [c for c in golden_cases.all_cases() if not c["big"]]
BIG = [c for c in golden_cases.all_cases() if c["big"]]


def _planes_sha(planes) -> str:
    h = hashlib.sha256()
    for p in planes:
        h.update(np.ascontiguousarray(p, dtype=np.uint16).astype("<u2").tobytes())
    return h.hexdigest()


def _encode(case, threads=4):
    planes = case["make"]()
    stream = oracle.encode(planes, layout=case["layout"], bit_depth=case["bit_depth"], quality=case["quality"],
                           tile_size=case["tile"], threads=threads)
    return planes, stream


@pytest.mark.parametrize("case", SMALL + BIG, ids=lambda c: c["name"])
def test_oracle_matches_reference_golden(case):
    rec = RECORDS[case["name"]]
    planes, stream = _encode(case, threads=8)
    assert _planes_sha(planes) == rec["input_sha256"], "input generator drifted"
    assert len(stream) == rec["stream_len"]
    assert hashlib.sha256(stream).hexdigest() == rec["stream_sha256"]
    decoded = oracle.decode(stream, threads=8)
    assert _planes_sha(decoded) == rec["decoded_sha256"]
    stored = GOLDEN / "streams" / f"{case['name']}.bin"
    if stored.exists():
        assert stored.read_bytes() == stream


def test_reference_refined_config_3a_at_full_size():
    """The reference's own 3840x2160 gray16 q87 stream is refined to step 417
    (flag 0x80); the oracle's bytes for it are checked by the golden test."""
    rec = RECORDS["cfg_gray16_4k_step417"]
    assert rec["flags"] == 0x88
    assert oracle.refined_gray16_step(87) == 417 and oracle.quantization_step("gray", 16, 87) == 556


def _shard_modes(stream):
    """cuda/tests/test_codec.py:33-49"""
    tile_count = struct.unpack_from("<I", stream, 28)[0]
    modes = set()
    for tile in range(tile_count):
        entry = 32 + tile * 32
        width, height = struct.unpack_from("<II", stream, entry + 12)
        cursor = struct.unpack_from("<Q", stream, entry + 20)[0]
        tile_end = cursor + struct.unpack_from("<I", stream, entry + 28)[0]
        decoded = 0
        while decoded < width * height:
            mode = stream[cursor]
            body_length = struct.unpack_from("<H", stream, cursor + 1)[0]
            modes.add(mode)
            cursor += 3 + body_length
            decoded += min(4096, width * height - decoded)
        assert cursor == tile_end
    return modes


@pytest.mark.parametrize("layout", ("gray", "yuv422", "rgb444"))
@pytest.mark.parametrize("bit_depth", (8, 10, 12, 16))
def test_oracle_q100_roundtrip_is_exact(layout, bit_depth):
    source = synth.reference_pattern(layout, 67, 35, bit_depth)
    first = oracle.encode(source, layout=layout, bit_depth=bit_depth, quality=100)
    second = oracle.encode(source, layout=layout, bit_depth=bit_depth, quality=100)
    assert first == second and first[4] == 1
    for got, exp in zip(oracle.decode(first), source):
        assert np.array_equal(got, exp)


def test_oracle_exercises_entropy_modes():
    selected = set()
    for quality, pattern in ((90, "ramp"), (100, "zero"), (100, "polynomial")):
        source = synth.reference_pattern("yuv422", 263, 133, 10, pattern)
        selected |= _shard_modes(oracle.encode(source, layout="yuv422", bit_depth=10, quality=quality))
    assert 0 in selected and 18 in selected and any(1 <= m <= 17 for m in selected)


def test_oracle_covers_rans_and_policies():
    modes = set()
    flags = set()
    for case in SMALL:
        _, stream = _encode(case)
        modes |= _shard_modes(stream)
        flags.add(stream[7] & 0xC0)
    assert 19 in modes
    assert {0x00, 0x40, 0x80} <= flags


def test_oracle_rejects_malformed_streams():
    """The six mutations of test_codec.py:89-115, on the oracle."""
    source = synth.reference_pattern("yuv422", 263, 133, 10)
    stream = bytearray(oracle.encode(source, layout="yuv422", bit_depth=10, quality=100))
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
    for bad in mutations:
        with pytest.raises(oracle.OracleError):
            oracle.decode(bytes(bad))


def test_oracle_steps_match_reference_policy():
    # encode.cu:71-89
    assert oracle.quantization_step("gray", 8, 50) == 1
    assert oracle.quantization_step("rgb444", 8, 90) == 3
    assert oracle.quantization_step("rgb444", 10, 85) == 7
    assert oracle.quantization_step("gray", 16, 87) == 556
    assert oracle.refined_gray16_step(87) == 417
    assert oracle.quantization_step("yuv422", 10, 90) == 3
    assert oracle.quantization_step("yuv422", 16, 90) == 108


def test_oracle_planted_mistake_is_caught():
    """A wrong byte planted in an oracle stream is detected by the golden check."""
    case = next(c for c in SMALL if c["name"] == "ref_rgb44410_67x35_q90")
    _, stream = _encode(case)
    bad = bytearray(stream)
    bad[-1] ^= 0x01
    assert hashlib.sha256(bytes(bad)).hexdigest() != RECORDS[case["name"]]["stream_sha256"]
