"""Host-side convenience wrappers over the C ABI.

Inputs/outputs are numpy uint64 arrays shaped (n, 4) for field elements,
(n, 4) / (n, 8) for G1 / G2 affine coordinates (SoA, like the reference's
msm_g1(d_Px, d_Py, d_scalars, N, ...)).  Device memory comes from torch,
used only as an allocator; every computation runs in libzyklop_b200.so.
"""
import ctypes

import numpy as np

from ._lib import check, lib

FP, FR = 0, 1
OPS = {"mul": 0, "add": 1, "sub": 2, "sqr": 3, "neg": 4, "inv": 5, "encode": 6, "decode": 7}


def _torch():
    import torch
    return torch


def to_device(a):
    torch = _torch()
    a = np.ascontiguousarray(a, dtype=np.uint64)
    return torch.from_numpy(a.view(np.int64).copy()).cuda()


def to_host(t, shape=None):
    a = t.cpu().numpy().view(np.uint64)
    return a.reshape(shape) if shape is not None else a


def empty_device(n_u64):
    torch = _torch()
    return torch.empty(max(int(n_u64), 4), dtype=torch.int64, device="cuda")


def ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def field_op(field, op, a, b=None, ctx=None):
    a = np.ascontiguousarray(a, dtype=np.uint64).reshape(-1, 4)
    n = a.shape[0]
    da = to_device(a)
    db = to_device(np.ascontiguousarray(b, dtype=np.uint64).reshape(-1, 4)) if b is not None else None
    out = empty_device(4 * n)
    check(lib().zk_field_op(ctx, field, OPS[op] if isinstance(op, str) else op, ptr(out), ptr(da),
                            ptr(db) if db is not None else None, n))
    return to_host(out)[: 4 * n].reshape(n, 4)


def ntt(a, log_n, inverse=False, ctx=None):
    a = np.ascontiguousarray(a, dtype=np.uint64).reshape(-1, 4)
    d = to_device(a)
    check(lib().zk_ntt(ctx, ptr(d), log_n, 1 if inverse else 0))
    return to_host(d).reshape(-1, 4)


def hpoly(aw, bw, log_n, ctx=None):
    da, db = to_device(aw), to_device(bw)
    dh = empty_device(4 << log_n)
    check(lib().zk_hpoly(ctx, ptr(da), ptr(db), log_n, ptr(dh)))
    return to_host(dh)[: 4 << log_n].reshape(-1, 4)


def _msm(fn, width, px, py, scalars, ctx=None):
    sc = np.ascontiguousarray(scalars, dtype=np.uint64).reshape(-1, 4)
    n = sc.shape[0]
    dx, dy, ds = to_device(px), to_device(py), to_device(sc)
    out = np.zeros(width, dtype=np.uint64)
    inf = ctypes.c_int(0)
    check(fn(ctx, ptr(dx), ptr(dy), ptr(ds), n,
             out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), ctypes.byref(inf)))
    return out, bool(inf.value)


def msm_g1(px, py, scalars, ctx=None):
    """sum k_i P_i on G1 -> (x[4] ++ y[4] affine Montgomery, is_infinity)"""
    return _msm(lib().zk_msm_g1, 8, px, py, scalars, ctx)


def msm_g2(px, py, scalars, ctx=None):
    """sum k_i Q_i on G2 -> (x.a0, x.a1, y.a0, y.a1 affine Montgomery, is_infinity)"""
    return _msm(lib().zk_msm_g2, 16, px, py, scalars, ctx)


def msm_set_config(group, c=0, k0=32, k1=16, chunk=16, ctx=None):
    check(lib().zk_msm_set_config(ctx, group, c, k0, k1, chunk))


def mul_generator(group, scalars, ctx=None, keep_on_device=False):
    """k_i * G for the standard generator of G1 (group 1) or G2 (group 2)."""
    sc = np.ascontiguousarray(scalars, dtype=np.uint64).reshape(-1, 4)
    n = sc.shape[0]
    w = 4 if group == 1 else 8
    ds = to_device(sc)
    dx, dy = empty_device(w * n), empty_device(w * n)
    check(lib().zk_mul_generator(ctx, group, ptr(ds), n, ptr(dx), ptr(dy)))
    if keep_on_device:
        return dx, dy
    return to_host(dx)[: w * n].reshape(n, w), to_host(dy)[: w * n].reshape(n, w)
