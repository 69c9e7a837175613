"""Drop-in ``fastvid_cuda`` module backed by fastvid_b200 (sm_100a).

Code written against the reference binding (``from fastvid_cuda import
encode, decode``, or ``fastvid_cuda._C``) runs unchanged on this package.
"""

from fastvid_b200 import decode, encode
from fastvid_b200.codec import _C

__all__ = ["decode", "encode", "_C"]
