"""The multi-GPU bench path on CPU: one process per rank over gloo, as
torchrun launches them (RANK / LOCAL_RANK / WORLD_SIZE, rendezvous on
127.0.0.1).  The replicas share no data; what crosses ranks is the barrier
around a timed region and the max over ranks of its time, from which the
whole-job rate is computed -- fastvid_b200.replicas, which bench.py runs
over NCCL on GPUs."""

import json
import os
import socket
import subprocess
import sys
import time

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RANK_SCRIPT = r"""
import json, sys
sys.path.insert(0, sys.argv[1])
from fastvid_b200.replicas import Replicas
mode = sys.argv[2]
rep = Replicas("gloo", timeout_s=20)
if mode == "leave" and rep.rank == 1:
    sys.exit(0)          # this rank leaves between steps, before the barrier
try:
    rep.barrier()
    ms = 10.0 + 5.0 * rep.rank   # rank 1 is the slower one
    m = rep.max(ms)
    rep.barrier()
    print(json.dumps({"rank": rep.rank, "world": rep.world, "max_ms": m,
                      "rate": rep.rate(1000.0, m), "leader": rep.leader}), flush=True)
    rep.close()
except Exception as exc:
    print(json.dumps({"rank": rep.rank, "error": type(exc).__name__}), flush=True)
    sys.exit(3)
"""


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _launch(world: int, mode: str):
    port = _free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(r),
                   LOCAL_RANK=str(r), WORLD_SIZE=str(world))
        procs.append(subprocess.Popen([sys.executable, "-c", RANK_SCRIPT, ROOT, mode], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    out = []
    for p in procs:
        try:
            o, e = p.communicate(timeout=120)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
        out.append((p.returncode, o, e))
    return out


def test_two_ranks_agree_on_the_slowest_time_and_the_whole_job_rate():
    res = _launch(2, "run")
    for rc, o, e in res:
        assert rc == 0, e
    lines = sorted((json.loads(o.strip().splitlines()[-1]) for _, o, _ in res), key=lambda d: d["rank"])
    for d in lines:
        assert d["world"] == 2
        assert d["max_ms"] == 15.0                      # the max over ranks, on every rank
        assert d["rate"] == pytest.approx(2 * 1000.0 / 0.015)  # all ranks' units over the slowest time
    assert [d["leader"] for d in lines] == [True, False]


def test_a_rank_that_leaves_ends_the_others_wait_with_an_error():
    t0 = time.perf_counter()
    res = _launch(2, "leave")
    assert res[1][0] == 0
    rc0, o0, e0 = res[0]
    assert rc0 != 0                          # rank 0 did not go on as if nothing happened
    assert time.perf_counter() - t0 < 100    # and did not wait for good


def test_single_process_needs_no_process_group():
    from fastvid_b200.replicas import Replicas

    rep = Replicas("gloo", env={})
    assert rep.world == 1 and rep.leader and rep.dist is None
    rep.barrier()
    assert rep.max(3.5) == 3.5
    assert rep.rate(264e6, 10.0) == pytest.approx(26.4e9)
    rep.close()


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "1"], env=env, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ""
