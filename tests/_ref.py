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

_prims = None
_prove = None
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
        _prove = L
    return _prove
