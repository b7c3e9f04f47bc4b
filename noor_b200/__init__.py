"""B200-native Noor render path: C-ABI library (libnoor_b200.so, sm_100a)
plus the host-side glue (scene generation, payload building, rendering).

Importing the package loads the in-tree shared library and fails loudly if it
has not been built; there is no CPU fallback for any render routine.
"""
from . import _capi
from ._capi import NoorError, call, lib

lib()

__all__ = ["NoorError", "call", "lib"]
