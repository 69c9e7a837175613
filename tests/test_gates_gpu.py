"""The evaluator's protocol (fastvid_b200.gates.measure) on a B200: a
latency case and a 24-frame 4K throughput case through the public fastvid
API, with the decoded planes' shapes checked and the gates evaluated."""

import pytest
import torch

from fastvid_b200 import gates

pytestmark = pytest.mark.gpu


def test_latency_case_reports_median_ms_and_gates():
    r = gates.measure(("latency", "rgb444", 8, 1920, 1080), torch.device("cuda", 0), warmups=2, repetitions=5)
    perf = r["performance"]
    assert r["correctness"]["decoded_shapes"]
    assert len(perf["encode"]["samples_seconds"]) == 5
    assert perf["encode"]["median_ms"] > 0 and perf["decode"]["median_ms"] > 0
    assert r["failures"] == gates.performance_failures(r)


def test_throughput_case_of_24_4k_frames():
    r = gates.measure(("throughput", "yuv422", 10, 3840, 2160), torch.device("cuda", 0), warmups=1,
                      repetitions=3, distinct=1)
    assert r["frame_count"] == 24 and r["correctness"]["decoded_shapes"]
    assert r["performance"]["encode"]["gpps"] > 0 and r["performance"]["decode"]["gpps"] > 0
    assert r["failures"] == gates.performance_failures(r)
