"""Generate golden fixtures by running the reference CUDA codec.

Runs on a GPU host.  It imports the reference extension compiled from the
reference's own sources by oracle/build_ref.py (module fastvid_ref_C in
oracle/_ref/), encodes and decodes every case of cases.py through the
reference binding (_C.encode / _C.decode, cuda/csrc/fastvid_cuda.cpp:359-378),
and writes:
  reference_streams.json   per case: stream SHA-256, length, header byte 7,
                           SHA-256 of the decoded planes (uint16 LE, Y Cb Cr)
  streams/<case>.bin       the stream itself for cases below 64 KiB

Usage: python tests/golden/make_golden.py [--out DIR] [--only CASE ...]
Only valid inputs are given to the reference.
"""

from __future__ import annotations

import argparse
import hashlib
import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE))

import numpy as np  # noqa: E402
import torch  # noqa: E402

import cases as golden_cases  # noqa: E402

LAYOUT = {"gray": 0, "yuv422": 1, "rgb444": 2}


def load_reference():
    sys.path.insert(0, str(ROOT / "oracle" / "_ref"))
    import fastvid_ref_C  # noqa: F401

    return fastvid_ref_C


def sha(data: bytes) -> str:
    return hashlib.sha256(data).hexdigest()


def planes_sha(planes) -> str:
    h = hashlib.sha256()
    for p in planes:
        h.update(np.ascontiguousarray(np.asarray(p, dtype=np.uint16)).astype("<u2").tobytes())
    return h.hexdigest()


def main() -> int:
    parser = argparse.ArgumentParser()
    parser.add_argument("--out", default=str(HERE))
    parser.add_argument("--only", action="append", default=[],
                        help="record only these cases and merge them into the existing file")
    args = parser.parse_args()
    out = Path(args.out)
    (out / "streams").mkdir(parents=True, exist_ok=True)
    ref = load_reference()
    records = {}
    if args.only:
        records = json.loads((out / "reference_streams.json").read_text())["cases"]
    for case in golden_cases.all_cases():
        if args.only and case["name"] not in args.only:
            continue
        planes = case["make"]()
        cuda_planes = [torch.from_numpy(np.ascontiguousarray(p)).cuda() for p in planes]
        tw, th = case["tile"]
        stream = ref.encode(cuda_planes, LAYOUT[case["layout"]], case["bit_depth"], case["quality"], 24, 1, tw, th)
        torch.cuda.synchronize()
        data = bytes(stream.cpu().numpy().tobytes())
        decoded = ref.decode(stream, True)
        dec_np = [d.cpu().numpy() for d in decoded]
        rec = dict(stream_sha256=sha(data), stream_len=len(data), flags=data[7],
                   decoded_sha256=planes_sha(dec_np), input_sha256=planes_sha(planes))
        if len(data) < 65536:
            (out / "streams" / f"{case['name']}.bin").write_bytes(data)
        records[case["name"]] = rec
        print(case["name"], rec["stream_len"], hex(rec["flags"]), flush=True)
    meta = dict(generator="reference CUDA extension built from cuda/csrc by oracle/build_ref.py",
                device=torch.cuda.get_device_name(0), torch=torch.__version__)
    (out / "reference_streams.json").write_text(json.dumps(dict(meta=meta, cases=records), indent=1, sort_keys=True))
    return 0


if __name__ == "__main__":
    sys.exit(main())
