"""CPU tests of the evaluator's protocol and gates (fastvid_b200.gates):
the timing distribution, each gate's threshold and the command-line rules
of the reference evaluator (scripts/evaluate.py:460-476, 740-755, 791-796)."""

import pytest

from fastvid_b200 import gates


def _result(mode, fmt, w, h, frames, enc, dec):
    key = "gpps" if mode == "throughput" else "median_ms"
    return {"format": fmt, "width": w, "height": h, "frame_count": frames,
            "performance": {"mode": mode, "encode": {key: enc}, "decode": {key: dec}}}


def test_distribution_median_and_nearest_rank_p95():
    s = [float(v) for v in range(20, 0, -1)]      # 20 samples, unsorted
    d = gates.distribution(s)
    assert d["median_seconds"] == 10.5
    assert d["min_seconds"] == 1.0 and d["max_seconds"] == 20.0
    assert d["p95_seconds"] == 19.0              # sorted[int(19 * 0.95)] = sorted[18]
    assert d["gate_statistic"] == "median"
    assert gates.distribution([4.0])["p95_seconds"] == 4.0


@pytest.mark.parametrize("fmt,enc,dec,expected", [
    ("rgb444", 1.5, 2.0, []),
    ("rgb444", 1.49, 2.0, ["encode throughput < 1.5 GP/s"]),
    ("gray", 1.6, 1.99, ["decode throughput < 2.0 GP/s"]),
    ("yuv422", 1.9, 2.9, ["encode throughput < 2.0 GP/s", "decode throughput < 3.0 GP/s"]),
    ("yuv422", 2.0, 3.0, []),
])
def test_throughput_gates_at_24_frames_of_4k(fmt, enc, dec, expected):
    assert gates.performance_failures(_result("throughput", fmt, 3840, 2160, 24, enc, dec)) == expected


def test_throughput_gates_apply_only_to_24_frames_of_4k():
    assert gates.performance_failures(_result("throughput", "rgb444", 3840, 2160, 23, 0.1, 0.1)) == []
    assert gates.performance_failures(_result("throughput", "rgb444", 1920, 1080, 24, 0.1, 0.1)) == []


@pytest.mark.parametrize("enc,dec,expected", [
    (0.99, 0.49, []),
    (1.0, 0.49, ["encode latency >= 1.0 ms"]),
    (0.5, 0.5, ["decode latency >= 0.5 ms"]),
])
def test_latency_gates_on_one_1080p_rgb444_frame(enc, dec, expected):
    assert gates.performance_failures(_result("latency", "rgb444", 1920, 1080, 1, enc, dec)) == expected
    assert gates.performance_failures(_result("latency", "gray", 1920, 1080, 1, 9.0, 9.0)) == []


def test_command_line_rules_of_the_evaluator():
    with pytest.raises(SystemExit):
        gates.main(["--repetitions", "19"])
    with pytest.raises(SystemExit):
        gates.main(["--warmups", "0"])


def test_gated_cases_cover_every_gate():
    modes = {(m, f, w, h) for m, f, _, w, h in gates.CASES}
    assert ("latency", "rgb444", 1920, 1080) in modes
    for f in ("gray", "yuv422", "rgb444"):
        assert ("throughput", f, 3840, 2160) in modes
