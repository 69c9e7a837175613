"""Drop-in ``fastvid`` public package backed by fastvid_b200: encode/decode
over frames and batches (batches through the batched form) and inspect."""

from fastvid_b200.api import decode, encode, inspect

__all__ = ["decode", "encode", "inspect"]
