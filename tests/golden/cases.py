"""Golden parity cases: inputs and coding parameters.

Each case names a deterministic input (the reference test suite's own
patterns, cuda/tests/test_codec.py:9-30, or the seeded synthetic frames of
fastvid_b200.synth) and the arguments of one encode call.  make_golden.py
encodes and decodes every case with the reference CUDA build and records the
results in reference_streams.json; the tests check the oracle and the sm_100a
path against those records.
"""

from __future__ import annotations

from fastvid_b200 import synth

LAYOUTS = ("gray", "yuv422", "rgb444")
DEPTHS = (8, 10, 12, 16)


def _case(name, layout, depth, quality, tile, make, big=False):
    return dict(name=name, layout=layout, bit_depth=depth, quality=quality, tile=tile, make=make, big=big)


def all_cases():
    cases = []
    # the reference suite's q100 matrix (test_codec.py:52-68) plus lossy variants
    for layout in LAYOUTS:
        for depth in DEPTHS:
            for q in (100, 90, 50):
                cases.append(_case(f"ref_{layout}{depth}_67x35_q{q}", layout, depth, q, (256, 128),
                                   lambda layout=layout, depth=depth: synth.reference_pattern(layout, 67, 35, depth)))
    # the entropy-mode test (test_codec.py:71-86)
    for q, pattern in ((90, "ramp"), (100, "zero"), (100, "polynomial")):
        cases.append(_case(f"ref_yuv422_10_263x133_{pattern}_q{q}", "yuv422", 10, q, (256, 128),
                           lambda pattern=pattern: synth.reference_pattern("yuv422", 263, 133, 10, pattern)))
    # benchmark workloads at full size
    for name, c in synth.CONFIGS.items():
        cases.append(_case(f"cfg_{name}", c["layout"], c["bit_depth"], c["quality"], c["tile"],
                           lambda name=name: synth.config_frame(name), big=c["width"] * c["height"] > 3_000_000))
    # serving-mix qualities: RGB8 steps 1/3/7, RGB10 steps 1/3/7, gray16 lossless
    for q in (100, 90, 66):
        cases.append(_case(f"mix_rgb8_720p_q{q}", "rgb444", 8, q, (64, 64),
                           lambda: synth.make_frame(1280, 720, "rgb444", 8, 21, sigma=(3, 1))))
    for q in (100, 96, 86):
        cases.append(_case(f"mix_rgb10_1080p_q{q}", "rgb444", 10, q, (128, 128),
                           lambda: synth.make_frame(1920, 1080, "rgb444", 10, 22, sigma=(4, 1))))
    cases.append(_case("mix_rgb10_4k_q96", "rgb444", 10, 96, (128, 128),
                       lambda: synth.make_frame(3840, 2160, "rgb444", 10, 23, sigma=(4, 1)), big=True))
    cases.append(_case("mix_gray16_2k_q100", "gray", 16, 100, (128, 128),
                       lambda: synth.make_frame(2048, 1080, "gray", 16, 24, sigma=(40, 1), amplitude=20000,
                                                mean=32768, rects=20)))
    # frame policies (encode.cu:812-847)
    cases.append(_case("policy_gray10_med", "gray", 10, 90, (64, 64),
                       lambda: synth.make_frame(640, 360, "gray", 10, 31, sigma=(60, 1))))
    cases.append(_case("policy_gray10_nomed", "gray", 10, 90, (64, 64),
                       lambda: synth.make_frame(640, 360, "gray", 10, 32, sigma=(1, 1))))
    cases.append(_case("policy_gray16_direct_noisy", "gray", 16, 87, (128, 128),
                       lambda: synth.make_frame(640, 360, "gray", 16, 33, sigma=(3000, 1), amplitude=20000,
                                                mean=32768)))
    cases.append(_case("policy_gray16_direct_smooth", "gray", 16, 70, (128, 128),
                       lambda: synth.make_frame(640, 360, "gray", 16, 34, sigma=(0, 1), amplitude=2000,
                                                mean=32768, rects=2)))
    cases.append(_case("policy_gray16_probe", "gray", 16, 87, (128, 128),
                       lambda: synth.make_frame(960, 540, "gray", 16, 35, sigma=(40, 1), amplitude=20000,
                                                mean=32768, rects=20)))
    # tile geometry
    cases.append(_case("tiles_32_rgb8", "rgb444", 8, 90, (32, 32),
                       lambda: synth.make_frame(300, 200, "rgb444", 8, 41)))
    cases.append(_case("tiles_odd_yuv422_10", "yuv422", 10, 80, (67, 35),
                       lambda: synth.make_frame(301, 203, "yuv422", 10, 42)))
    cases.append(_case("tiles_wide_gray12", "gray", 12, 95, (600, 40),
                       lambda: synth.make_frame(1300, 90, "gray", 12, 43)))
    cases.append(_case("tiles_tall_gray8", "gray", 8, 100, (64, 700),
                       lambda: synth.make_frame(200, 700, "gray", 8, 44)))
    cases.append(_case("tiles_1x3_gray10", "gray", 10, 80, (1, 3),
                       lambda: synth.make_frame(9, 7, "gray", 10, 45)))
    cases.append(_case("tiles_256x128_yuv422_16", "yuv422", 16, 90, (256, 128),
                       lambda: synth.make_frame(777, 333, "yuv422", 16, 46)))
    cases.append(_case("tiny_1x1_gray8", "gray", 8, 100, (256, 128),
                       lambda: synth.make_frame(1, 1, "gray", 8, 47)))
    cases.append(_case("tiny_3x1_rgb16", "rgb444", 16, 70, (256, 128),
                       lambda: synth.make_frame(3, 1, "rgb444", 16, 48)))
    cases.append(_case("tiny_2x5_yuv422_12", "yuv422", 12, 100, (256, 128),
                       lambda: synth.make_frame(2, 5, "yuv422", 12, 49)))
    # zero-run / flat content
    cases.append(_case("flat_gray8", "gray", 8, 100, (64, 64),
                       lambda: synth.make_frame(256, 256, "gray", 8, 51, sigma=(1, 2), amplitude=0, rects=3)))
    cases.append(_case("flat_rgb10_q90", "rgb444", 10, 90, (128, 128),
                       lambda: synth.make_frame(512, 256, "rgb444", 10, 52, sigma=(1, 2), amplitude=4, rects=3)))
    cases.append(_case("zero_rgb12", "rgb444", 12, 100, (64, 64),
                       lambda: synth.reference_pattern("rgb444", 200, 100, 12, "zero")))
    return cases


def case_map():
    return {c["name"]: c for c in all_cases()}
