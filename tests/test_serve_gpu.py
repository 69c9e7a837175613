"""GPU tests of the serving form: requests of every serving format, encode and
decode, submitted from two threads while earlier batches run, must each get
exactly the answer they get alone -- the oracle's stream bytes for an encode,
the oracle's planes for a decode -- and the server must actually batch and
overlap them, within its memory budget."""

import random
import threading

import numpy as np
import pytest
import torch

import fastvid_b200
import oracle
from fastvid_b200 import synth
from fastvid_b200.serve import Server

pytestmark = pytest.mark.gpu

SCALE = 8  # serving formats at 1/8 size: 160x90 .. 480x270


@pytest.fixture(scope="module")
def pool():
    items = []
    for fmt, (_, f) in enumerate(synth.SERVING_FORMATS):
        for q in f["qualities"]:
            planes = synth.serving_frame(fmt, 0, scale=SCALE)
            params = dict(layout=f["layout"], bit_depth=f["bit_depth"], quality=q, tile_size=f["tile"])
            stream = oracle.encode(planes, **params, threads=4)
            items.append(dict(planes=planes, params=params, stream=stream, decoded=oracle.decode(stream)))
    return items


def _requests(pool, count, seed):
    rng = random.Random(seed)
    return [(rng.random() < 0.6, rng.randrange(len(pool))) for _ in range(count)]


def _submit_all(server, pool, reqs, threads=2, seed=0):
    futs = [None] * len(reqs)
    dev = [dict(planes=tuple(torch.from_numpy(p).cuda() for p in it["planes"]),
                stream=torch.frombuffer(bytearray(it["stream"]), dtype=torch.uint8).cuda()) for it in pool]

    def feed(part):
        rng = random.Random(seed + part)
        for i in range(part, len(reqs), threads):
            enc, k = reqs[i]
            if enc:
                futs[i] = server.submit_encode(dev[k]["planes"], **pool[k]["params"])
            else:
                futs[i] = server.submit_decode(dev[k]["stream"])
            if rng.random() < 0.3:
                threading.Event().wait(rng.random() * 0.003)

    ts = [threading.Thread(target=feed, args=(p,)) for p in range(threads)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    return [f.result(timeout=120) for f in futs]


def _check(pool, reqs, results):
    for (enc, k), res in zip(reqs, results):
        if enc:
            assert bytes(res.cpu().numpy()) == pool[k]["stream"], k
        else:
            assert len(res) == len(pool[k]["decoded"])
            for got, want in zip(res, pool[k]["decoded"]):
                assert np.array_equal(got.cpu().numpy(), want), k


def test_mixed_requests_equal_their_answers_alone(cuda, pool):
    reqs = _requests(pool, 48, seed=1)
    with Server("cuda", memory_budget=2 << 30, workers=3, max_batch_frames=6) as server:
        results = _submit_all(server, pool, reqs)
    _check(pool, reqs, results)
    assert max(n for _, n in server.batches) > 1  # arrivals were batched
    assert server.max_concurrent >= 2             # and overlapped on the device
    # alone: one request at a time through a one-worker server, and the
    # single-frame path, give the same answers
    with Server("cuda", workers=1) as alone:
        for (enc, k), res in list(zip(reqs, results))[:12]:
            it = pool[k]
            if enc:
                planes = tuple(torch.from_numpy(p).cuda() for p in it["planes"])
                solo = alone.submit_encode(planes, **it["params"]).result(timeout=60)
                assert torch.equal(solo, res)
                assert torch.equal(fastvid_b200.encode(planes, **it["params"]), res)
            else:
                stream = torch.frombuffer(bytearray(it["stream"]), dtype=torch.uint8).cuda()
                solo = alone.submit_decode(stream).result(timeout=60)
                assert all(torch.equal(a, b) for a, b in zip(solo, res))


def test_small_budget_still_answers_everything(cuda, pool):
    reqs = _requests(pool, 24, seed=2)
    big = max(range(len(pool)), key=lambda k: pool[k]["planes"][0].size * len(pool[k]["planes"]))
    # room for about one of the largest requests at a time
    probe = Server("cuda", workers=1)
    planes = tuple(torch.from_numpy(p).cuda() for p in pool[big]["planes"])
    r = probe.backend.encode_request(planes, **pool[big]["params"])
    probe.close()
    budget = 2 * (r.ws_bytes + r.out_bytes)
    with Server("cuda", memory_budget=budget, workers=3, max_batch_frames=16) as server:
        results = _submit_all(server, pool, reqs, seed=7)
        with pytest.raises(MemoryError, match="above the server budget"):
            server.submit_encode(torch.zeros((1080, 1920), dtype=torch.uint16, device="cuda"), layout="gray",
                                 bit_depth=8, quality=100, tile_size=(64, 64)).result(timeout=10)
    _check(pool, reqs, results)


def test_bad_request_fails_alone(cuda, pool):
    it = pool[0]
    good = tuple(torch.from_numpy(p).cuda() for p in it["planes"])
    bad = tuple(p.clone() for p in good)
    bad[0][1, 1] = (1 << it["params"]["bit_depth"])  # above the bit depth
    with Server("cuda", workers=1, max_batch_frames=8) as server:
        futs = [server.submit_encode(good, **it["params"]) for _ in range(3)]
        futs.insert(1, server.submit_encode(bad, **it["params"]))
        with pytest.raises(RuntimeError):
            futs[1].result(timeout=60)
        for i in (0, 2, 3):
            assert bytes(futs[i].result(timeout=60).cpu().numpy()) == it["stream"]
