"""CPU tests of the autotuner's selection rules and of the launch-geometry
knob of the C ABI (host-side state only, no kernel launch)."""

import pytest

from fastvid_b200 import _native, autotune


def test_choose_tile_takes_the_fastest_within_the_size_tolerance():
    res = {(32, 32): (1.0, 1100), (64, 64): (1.5, 1010), (128, 128): (2.0, 1000)}
    assert autotune.choose_tile(res, 0.02) == (64, 64)   # 32x32 is 10% larger
    assert autotune.choose_tile(res, 0.2) == (32, 32)
    assert autotune.choose_tile(res, 0.0) == (128, 128)
    tie = {(32, 32): (1.0, 1005), (64, 64): (1.0, 1000)}
    assert autotune.choose_tile(tie, 0.01) == (64, 64)   # equal time: the smaller stream


def test_descend_finds_the_separable_optimum():
    target = {"a": 6, "b": 3}
    calls = []

    def cost(s):
        calls.append(dict(s))
        return 10 + (s["a"] - target["a"]) ** 2 + (s["b"] - target["b"]) ** 2

    best = autotune.descend(("a", "b"), (2, 3, 4, 6, 8), cost, {"a": 2, "b": 8})
    assert best == target
    assert len(calls) < 30


def test_descend_keeps_the_start_without_a_real_gain():
    best = autotune.descend(("a",), (1, 2, 3), lambda s: 100.0 - 0.1 * s["a"], {"a": 1}, min_gain=0.01)
    assert best == {"a": 1}


def test_launch_knob_round_trip_and_rejections():
    lib = _native.load()
    names = _native.kernel_names()
    before = autotune.launch_settings()
    assert set(autotune.LAUNCH_KNOBS) <= set(before)
    try:
        autotune.set_launch({"enc_predict": 3, "dec_rans": 12})
        now = autotune.launch_settings()
        assert now["enc_predict"] == 3 and now["dec_rans"] == 12
        autotune.reset_launch()
        assert autotune.launch_settings() == before
        assert lib.fvb_set_launch_ctas(names.index("enc_rans"), 4) != 0
        assert _native.last_error() == "kernel has no launch-geometry knob"
        assert lib.fvb_get_launch_ctas(names.index("enc_rans")) == -1
        assert lib.fvb_set_launch_ctas(names.index("enc_predict"), 65) != 0
        with pytest.raises(RuntimeError):
            autotune.set_launch({"enc_scan": 2})
    finally:
        autotune.reset_launch()


def test_table_round_trip(tmp_path):
    table = {"tiles": {autotune.format_key("gray", 8, 1280, 720): [32, 32]}, "launch": {"enc_emit": 6}}
    path = tmp_path / "t.json"
    autotune.save(table, path)
    assert autotune.load(path) == table
    assert autotune.tile_for(table, "gray", 8, 1280, 720) == (32, 32)
    assert autotune.tile_for(table, "gray", 8, 640, 480, default=(64, 64)) == (64, 64)
    try:
        autotune.apply(table)
        assert autotune.launch_settings()["enc_emit"] == 6
    finally:
        autotune.reset_launch()


def test_wavefront_block_knob_round_trip_and_rejections():
    lib = _native.load()
    before = autotune.wavefront_block()
    try:
        for steps in autotune.WAVEFRONT_BLOCKS:
            autotune.set_wavefront_block(steps)
            assert autotune.wavefront_block() == steps
        for bad in (1, 3, 12, 64, -8):
            assert lib.fvb_set_wavefront_block(bad) == -1
            assert "wavefront block" in _native.last_error()
        autotune.set_wavefront_block(0)
        assert autotune.wavefront_block() == 8  # the default
        autotune.apply({"launch": {}, "wavefront_block": 16})
        assert autotune.wavefront_block() == 16
    finally:
        autotune.set_wavefront_block(before)


def test_tile_warps_knob_round_trip_and_rejections():
    lib = _native.load()
    before = autotune.tile_warps()
    try:
        for warps in autotune.TILE_WARPS:
            autotune.set_tile_warps(warps)
            assert autotune.tile_warps() == warps
        for bad in (3, 4, -1):
            assert lib.fvb_set_tile_warps(bad) == -1
            assert "warps per tile" in _native.last_error()
        autotune.set_tile_warps(0)
        assert autotune.tile_warps() == 1  # the default
        autotune.apply({"launch": {}, "tile_warps": 2})
        assert autotune.tile_warps() == 2
    finally:
        autotune.set_tile_warps(before)


def test_decode_overlap_knob_round_trip_and_rejections():
    lib = _native.load()
    before = autotune.decode_overlap()
    try:
        for on in (0, 1):
            autotune.set_decode_overlap(on)
            assert autotune.decode_overlap() == on
        assert lib.fvb_set_decode_overlap(2) == -1 and "decode overlap" in _native.last_error()
        autotune.apply({"launch": {}, "decode_overlap": 0})
        assert autotune.decode_overlap() == 0
    finally:
        autotune.set_decode_overlap(before)


def test_rans_pipeline_knob_round_trip_and_rejections():
    lib = _native.load()
    before = autotune.rans_pipeline(), autotune.rans_pipeline_tail()
    try:
        for steps in (0, 8, 16):
            autotune.set_rans_pipeline(steps)
            autotune.set_rans_pipeline_tail(16 - steps if steps else 8)
            assert autotune.rans_pipeline() == steps
            assert autotune.rans_pipeline_tail() == (16 - steps if steps else 8)
        for bad in (4, 32, -2):
            assert lib.fvb_set_rans_pipeline(bad) == -1 and "rANS pipeline" in _native.last_error()
            assert lib.fvb_set_rans_pipeline_tail(bad) == -1 and "rANS pipeline" in _native.last_error()
        autotune.apply({"launch": {}, "rans_pipeline": 8, "rans_pipeline_tail": 16})
        assert autotune.rans_pipeline() == 8 and autotune.rans_pipeline_tail() == 16
        autotune.apply({"launch": {}})  # the automatic choice by default
        assert autotune.rans_pipeline() == -1 and autotune.rans_pipeline_tail() == -1
    finally:
        autotune.set_rans_pipeline(before[0])
        autotune.set_rans_pipeline_tail(before[1])
