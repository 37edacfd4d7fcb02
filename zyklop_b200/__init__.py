"""zyklop_b200 — B200 (sm_100a) Groth16 / BN254 prover.

The product is the C-ABI shared library ``libzyklop_b200.so`` built in this
directory (declared in ``include/zyklop_b200.h``).  This package only loads it
through ctypes and adds thin helpers for device buffers (torch tensors are
used as plain device memory).  There is no CPU fallback: importing the
binding fails loudly when the library has not been built.
"""
from ._lib import (  # noqa: F401
    LIB_PATH,
    ZkError,
    lib,
    version,
)
