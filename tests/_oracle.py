"""ctypes binding of the CPU oracle (oracle/_build/liboracle.so).

The oracle is the checker for the CUDA library: tests compare the library's
results with it, and nothing in the product uses it.
"""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_build", "liboracle.so")

P = 0x30644E72E131A029B85045B68181585D97816A916871CA8D3C208C16D87CFD47
R = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
MONT = 1 << 256

_lib = None


def _u64p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    lib = ctypes.CDLL(LIB)
    u64p = ctypes.POINTER(ctypes.c_uint64)
    u8p = ctypes.POINTER(ctypes.c_uint8)
    sz = ctypes.c_size_t
    i = ctypes.c_int
    for name in ("orc_f_mul", "orc_f_add", "orc_f_sub"):
        getattr(lib, name).argtypes = [i, u64p, u64p, u64p]
    for name in ("orc_f_neg", "orc_f_sqr", "orc_f_inv", "orc_f_inv_normal", "orc_f_encode", "orc_f_decode"):
        getattr(lib, name).argtypes = [i, u64p, u64p]
    lib.orc_f_pow.argtypes = [i, u64p, u64p, u64p]
    lib.orc_f_batch.argtypes = [i, i, u64p, u64p, u64p, sz]
    for name in ("orc_g1_add", "orc_g1_mul", "orc_g2_add", "orc_g2_mul"):
        getattr(lib, name).argtypes = [u64p, u64p, u64p]
        getattr(lib, name).restype = i
    lib.orc_g1_on_curve.argtypes = [u64p]
    lib.orc_g2_on_curve.argtypes = [u64p]
    lib.orc_g1_generator.argtypes = [u64p]
    lib.orc_g2_generator.argtypes = [u64p]
    for name in ("orc_msm_g1", "orc_msm_g2"):
        getattr(lib, name).argtypes = [u64p, u64p, u64p, sz, u64p, i]
        getattr(lib, name).restype = i
    lib.orc_ntt.argtypes = [u64p, i, i, i]
    lib.orc_hpoly.argtypes = [u64p, u64p, i, u64p, i]
    lib.orc_spmv.argtypes = [u8p, sz, u64p, ctypes.c_uint32, ctypes.c_uint32, u64p, u64p]
    lib.orc_prove.argtypes = [u8p, sz, u8p, sz, u64p, u64p, u64p, i]
    lib.orc_prove.restype = i
    lib.orc_prove_intermediates.argtypes = [u8p, sz, u8p, sz, u64p, u64p, u64p, i]
    lib.orc_prove_intermediates.restype = i
    lib.orc_pairing.argtypes = [u64p, u64p, u64p]
    lib.orc_verify.argtypes = [u8p, sz, u64p, u64p, ctypes.c_uint32]
    lib.orc_verify.restype = i
    _lib = Oracle(lib)
    return _lib


# ------------------------------------------------------------ conversions

def limbs(x, n=4):
    return np.array([(x >> (64 * i)) & 0xFFFFFFFFFFFFFFFF for i in range(n)], dtype=np.uint64)


def to_int(a):
    a = np.asarray(a, dtype=np.uint64).reshape(-1)
    v = 0
    for i, x in enumerate(a):
        v |= int(x) << (64 * i)
    return v


def arr(values, n=4):
    """list of ints -> (len, n) uint64 array"""
    out = np.zeros((len(values), n), dtype=np.uint64)
    for k, v in enumerate(values):
        out[k] = limbs(v, n)
    return out


def ints(a):
    a = np.asarray(a, dtype=np.uint64).reshape(-1, 4)
    return [to_int(row) for row in a]


def mont(x, m):
    return (x * MONT) % m


def unmont(x, m):
    return (x * pow(MONT, -1, m)) % m


class Oracle:
    FP, FR = 0, 1

    def __init__(self, lib):
        self.lib = lib

    def f2(self, op, which, a, b):
        r = np.zeros(4, np.uint64)
        getattr(self.lib, "orc_f_" + op)(which, _u64p(r), _u64p(limbs(a)), _u64p(limbs(b)))
        return to_int(r)

    def f1(self, op, which, a):
        r = np.zeros(4, np.uint64)
        getattr(self.lib, "orc_f_" + op)(which, _u64p(r), _u64p(limbs(a)))
        return to_int(r)

    def batch(self, which, op, a, b=None):
        a = np.ascontiguousarray(a, dtype=np.uint64)
        r = np.zeros_like(a)
        bp = _u64p(np.ascontiguousarray(b, dtype=np.uint64)) if b is not None else None
        self.lib.orc_f_batch(which, op, _u64p(r), _u64p(a), bp, a.shape[0])
        return r

    def g1_mul(self, p, k):
        r = np.zeros(8, np.uint64)
        self.lib.orc_g1_mul(_u64p(r), _u64p(np.ascontiguousarray(p, np.uint64)), _u64p(limbs(k)))
        return r

    def g1_add(self, p, q):
        r = np.zeros(8, np.uint64)
        self.lib.orc_g1_add(_u64p(r), _u64p(np.ascontiguousarray(p, np.uint64)),
                            _u64p(np.ascontiguousarray(q, np.uint64)))
        return r

    def g2_mul(self, p, k):
        r = np.zeros(16, np.uint64)
        self.lib.orc_g2_mul(_u64p(r), _u64p(np.ascontiguousarray(p, np.uint64)), _u64p(limbs(k)))
        return r

    def g2_add(self, p, q):
        r = np.zeros(16, np.uint64)
        self.lib.orc_g2_add(_u64p(r), _u64p(np.ascontiguousarray(p, np.uint64)),
                            _u64p(np.ascontiguousarray(q, np.uint64)))
        return r

    def g1_gen(self):
        r = np.zeros(8, np.uint64)
        self.lib.orc_g1_generator(_u64p(r))
        return r

    def g2_gen(self):
        r = np.zeros(16, np.uint64)
        self.lib.orc_g2_generator(_u64p(r))
        return r

    def msm_g1(self, px, py, sc, threads=0):
        px, py, sc = (np.ascontiguousarray(x, np.uint64) for x in (px, py, sc))
        r = np.zeros(8, np.uint64)
        inf = self.lib.orc_msm_g1(_u64p(px), _u64p(py), _u64p(sc), sc.size // 4, _u64p(r), threads)
        return r, inf

    def msm_g2(self, px, py, sc, threads=0):
        px, py, sc = (np.ascontiguousarray(x, np.uint64) for x in (px, py, sc))
        r = np.zeros(16, np.uint64)
        inf = self.lib.orc_msm_g2(_u64p(px), _u64p(py), _u64p(sc), sc.size // 4, _u64p(r), threads)
        return r, inf

    def ntt(self, a, log_n, inverse, threads=0):
        a = np.ascontiguousarray(a, np.uint64).copy()
        self.lib.orc_ntt(_u64p(a), log_n, 1 if inverse else 0, threads)
        return a

    def hpoly(self, aw, bw, log_n, threads=0):
        aw = np.ascontiguousarray(aw, np.uint64)
        bw = np.ascontiguousarray(bw, np.uint64)
        h = np.zeros_like(aw)
        self.lib.orc_hpoly(_u64p(aw), _u64p(bw), log_n, _u64p(h), threads)
        return h

    def pairing(self, p, q):
        out = np.zeros(48, np.uint64)
        self.lib.orc_pairing(_u64p(out), _u64p(np.ascontiguousarray(p, np.uint64)),
                             _u64p(np.ascontiguousarray(q, np.uint64)))
        return out

    def prove(self, zkey: bytes, wtns: bytes, r=None, s=None, threads=0):
        proof = np.zeros(32, np.uint64)
        zb = np.frombuffer(zkey, np.uint8)
        wb = np.frombuffer(wtns, np.uint8)
        rp = _u64p(limbs(r)) if r is not None else None
        sp = _u64p(limbs(s)) if s is not None else None
        rc = self.lib.orc_prove(zb.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), zb.size,
                                wb.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), wb.size,
                                rp, sp, _u64p(proof), threads)
        if rc:
            raise RuntimeError(f"orc_prove failed: {rc}")
        return proof

    def intermediates(self, zkey: bytes, wtns: bytes, domain: int, threads=0):
        aw = np.zeros((domain, 4), np.uint64)
        bw = np.zeros((domain, 4), np.uint64)
        h = np.zeros((domain, 4), np.uint64)
        zb = np.frombuffer(zkey, np.uint8)
        wb = np.frombuffer(wtns, np.uint8)
        rc = self.lib.orc_prove_intermediates(
            zb.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), zb.size,
            wb.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), wb.size,
            _u64p(aw), _u64p(bw), _u64p(h), threads)
        if rc:
            raise RuntimeError(f"orc_prove_intermediates failed: {rc}")
        return aw, bw, h

    def verify(self, zkey: bytes, proof, publics):
        zb = np.frombuffer(zkey, np.uint8)
        pub = arr(publics) if len(publics) else np.zeros((1, 4), np.uint64)
        return self.lib.orc_verify(zb.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), zb.size,
                                   _u64p(np.ascontiguousarray(proof, np.uint64)), _u64p(pub),
                                   len(publics))
