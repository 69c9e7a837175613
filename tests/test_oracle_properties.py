"""Property tests of the oracle over random small frames (hypothesis):
encoding is deterministic, the decoder returns the source's plane shapes,
and every decoded sample lies within half a quantization step of its source
-- the quantizer rounds residuals to the nearest multiple of the step with
reconstruction in the loop (encode.cu:128-193), so the error never exceeds
floor(step / 2), and quality 100 (step 1) is exact."""

import numpy as np
from hypothesis import given, settings
from hypothesis import strategies as st

import oracle
from fastvid_b200 import synth


@settings(max_examples=60, deadline=None)
@given(layout=st.sampled_from(["gray", "yuv422", "rgb444"]), depth=st.sampled_from([8, 10, 12, 16]),
       width=st.integers(1, 90), height=st.integers(1, 60), quality=st.integers(1, 100),
       tile=st.tuples(st.sampled_from([2, 8, 16, 33, 64, 256]), st.sampled_from([1, 8, 16, 31, 128])),
       seed=st.integers(0, 1 << 16))
def test_roundtrip_error_within_half_a_step(layout, depth, width, height, quality, tile, seed):
    planes = synth.make_frame(width, height, layout, depth, seed)
    kw = dict(layout=layout, bit_depth=depth, quality=quality, tile_size=tile)
    stream = oracle.encode(planes, **kw)
    assert stream == oracle.encode(planes, **kw)
    refined = bool(stream[7] & 0x80)
    step = oracle.refined_gray16_step(quality) if refined else oracle.quantization_step(layout, depth, quality)
    decoded = oracle.decode(stream)
    assert len(decoded) == len(planes)
    for got, src in zip(decoded, planes):
        assert got.shape == src.shape
        err = np.abs(got.astype(np.int64) - src.astype(np.int64))
        assert int(err.max(initial=0)) <= step // 2
        if step == 1:
            assert np.array_equal(got, src)
