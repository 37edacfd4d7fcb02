"""ctypes binding of the reference's own sm_100a build (oracle/_ref/, built
by oracle/refbuild/Makefile from the reference sources).  Test
infrastructure: the reference's msm_g1 / msm_g2_device / ntt and groth16Prove
run on the same inputs as the library so results can be compared bit for bit.
"""
import ctypes
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PRIMS = os.path.join(ROOT, "oracle", "_ref", "libzkref_prims.so")
PROVE = os.path.join(ROOT, "oracle", "_ref", "libzkref_prove.so")

INTER = os.path.join(ROOT, "oracle", "_ref", "libzkref_inter.so")

_prims = None
_prove = None
_inter = None
u64p = ctypes.POINTER(ctypes.c_uint64)


def prims():
    global _prims
    if _prims is None:
        if not os.path.exists(PRIMS):
            return None
        L = ctypes.CDLL(PRIMS)
        for name in ("zkref_msm_g1_device", "zkref_msm_g2_device"):
            fn = getattr(L, name)
            fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, u64p]
            fn.restype = ctypes.c_int
        L.zkref_ntt_device.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.zkref_ntt_device.restype = ctypes.c_int
        _prims = L
    return _prims


def prove_lib():
    global _prove
    if _prove is None:
        if not os.path.exists(PROVE):
            return None
        L = ctypes.CDLL(PROVE)
        L.zkref_prove_files.argtypes = [ctypes.c_char_p, ctypes.c_char_p, u64p]
        L.zkref_prove_files.restype = ctypes.c_int
        L.zkref_proof_json.argtypes = [u64p, ctypes.c_char_p, ctypes.c_size_t]
        L.zkref_proof_json.restype = ctypes.c_int
        if hasattr(L, "zkref_proof_calldata"):
            L.zkref_proof_calldata.argtypes = [u64p, ctypes.c_void_p, ctypes.c_size_t]
            L.zkref_proof_calldata.restype = ctypes.c_int
        _prove = L
    return _prove


def inter_lib():
    """The reference prover's steps one by one (oracle/refbuild/ref_inter.cu)."""
    global _inter
    if _inter is None:
        if not os.path.exists(INTER):
            return None
        L = ctypes.CDLL(INTER)
        L.zkref_intermediates.argtypes = [ctypes.c_char_p, ctypes.c_char_p] + \
            [ctypes.c_void_p] * 10 + [ctypes.POINTER(ctypes.c_int)]
        L.zkref_intermediates.restype = ctypes.c_int
        _inter = L
    return _inter


def intermediates(zkey, wtns, domain):
    """The reference's A.w, B.w, coset evaluations, h and MSM results for a
    proof of (zkey, wtns), in the keys Circuit.trace() uses."""
    import numpy as np
    L = inter_lib()
    if L is None:
        return None
    out = {k: np.zeros((domain, 4), np.uint64) for k in ("aw", "bw", "ea", "eb", "ec", "h")}
    for k, n in (("msm_a", 8), ("msm_b2", 16), ("msm_c", 8), ("msm_h", 8)):
        out[k] = np.zeros(n, np.uint64)
    inf = (ctypes.c_int * 4)()
    order = ("aw", "bw", "ea", "eb", "ec", "h", "msm_a", "msm_b2", "msm_c", "msm_h")
    rc = L.zkref_intermediates(str(zkey).encode(), str(wtns).encode(),
                               *[ctypes.c_void_p(out[k].ctypes.data) for k in order], inf)
    assert rc == 0
    out["inf"] = [int(x) for x in inf]
    return out
