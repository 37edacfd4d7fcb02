"""Host-side convenience wrappers over the C ABI.

Inputs/outputs are numpy uint64 arrays shaped (n, 4) for field elements,
(n, 4) / (n, 8) for G1 / G2 affine coordinates (SoA, like the reference's
msm_g1(d_Px, d_Py, d_scalars, N, ...)).  Device memory comes from torch,
used only as an allocator; every computation runs in libzyklop_b200.so.
"""
import ctypes

import numpy as np

from ._lib import ZkError, check, lib

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


def msm_set_config(group, c=0, k0=0, k1=16, chunk=0, ctx=None):
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


# ------------------------------------------------------------------ Groth16
from ._lib import SynthParams, ZkeyHeader  # noqa: E402

_u64p = ctypes.POINTER(ctypes.c_uint64)


def synth_circuit(zkey_path, wtns_path, log_domain, n_public=8, n_private_inputs=8, nnz=(2, 2),
                  witness="uniform", seed=1, ctx=None):
    """Write a seeded synthetic circuit + CRS (zkey) and its witness (wtns)."""
    p = SynthParams(log_domain, n_public, n_private_inputs, nnz[0], nnz[1],
                    {"uniform": 0, "circom": 1}[witness], seed)
    check(lib().zk_synth_circuit(ctx, ctypes.byref(p), str(zkey_path).encode(),
                                 str(wtns_path).encode()))


def read_wtns(path):
    """canonical witness values of a wtns file -> (n, 4) uint64"""
    data = open(path, "rb").read()
    assert data[:4] == b"wtns"
    ns = int.from_bytes(data[8:12], "little")
    pos, n_vars, values = 12, None, None
    for _ in range(ns):
        t = int.from_bytes(data[pos:pos + 4], "little")
        size = int.from_bytes(data[pos + 4:pos + 12], "little")
        pos += 12
        if t == 1:
            n_vars = int.from_bytes(data[pos + 36:pos + 40], "little")
        elif t == 2:
            values = data[pos:pos + size]
        pos += size
    return np.frombuffer(values, dtype=np.uint64)[: 4 * n_vars].reshape(n_vars, 4).copy()


class Circuit:
    """A zkey resident on the device (zk_circuit_load_file / zk_prove)."""

    def __init__(self, zkey_path, ctx=None):
        h = ctypes.c_void_p()
        check(lib().zk_circuit_load_file(ctx, str(zkey_path).encode(), ctypes.byref(h)))
        self.handle = h
        a, b, c = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        check(lib().zk_circuit_info(h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        self.n_vars, self.n_public, self.domain = a.value, b.value, c.value

    def set_scalar_dist(self, dist):
        """-1: detect from each host witness; 0 uniform; 1 skewed"""
        check(lib().zk_circuit_set_scalar_dist(self.handle, dist))

    def precompute(self, c_g1=0, c_g2=0):
        check(lib().zk_circuit_precompute(self.handle, c_g1, c_g2))

    def prove(self, witness, r=None, s=None):
        w = np.ascontiguousarray(witness, dtype=np.uint64).reshape(-1, 4)
        proof = np.zeros(32, dtype=np.uint64)
        rr = np.array([(r >> (64 * i)) & (2**64 - 1) for i in range(4)], np.uint64) if r is not None else None
        ss = np.array([(s >> (64 * i)) & (2**64 - 1) for i in range(4)], np.uint64) if s is not None else None
        check(lib().zk_prove(self.handle, w.ctypes.data_as(ctypes.c_void_p), w.shape[0],
                             rr.ctypes.data_as(ctypes.c_void_p) if rr is not None else None,
                             ss.ctypes.data_as(ctypes.c_void_p) if ss is not None else None,
                             proof.ctypes.data_as(_u64p)))
        return proof

    def prove_device(self, d_witness, n, r=None, s=None):
        proof = np.zeros(32, dtype=np.uint64)
        check(lib().zk_prove_device(self.handle, ptr(d_witness), n, None, None,
                                    proof.ctypes.data_as(_u64p)))
        return proof

    def intermediates(self, witness):
        w = np.ascontiguousarray(witness, dtype=np.uint64).reshape(-1, 4)
        aw = np.zeros((self.domain, 4), np.uint64)
        bw = np.zeros((self.domain, 4), np.uint64)
        h = np.zeros((self.domain, 4), np.uint64)
        proof = np.zeros(32, dtype=np.uint64)
        check(lib().zk_prove_intermediates(self.handle, w.ctypes.data_as(ctypes.c_void_p),
                                           w.shape[0], aw.ctypes.data_as(ctypes.c_void_p),
                                           bw.ctypes.data_as(ctypes.c_void_p),
                                           h.ctypes.data_as(ctypes.c_void_p),
                                           proof.ctypes.data_as(_u64p)))
        return aw, bw, h, proof

    def trace(self, witness):
        """Every intermediate of the unblinded proof (zk_prove_traced): a dict
        of A.w, B.w, the odd-coset evaluations of A, B, C, h (domain x 4
        arrays), the four MSM results (msm_a, msm_b2, msm_c, msm_h), their
        infinity flags and the proof."""
        from ._lib import ProveTrace
        w = np.ascontiguousarray(witness, dtype=np.uint64).reshape(-1, 4)
        bufs = {k: np.zeros((self.domain, 4), np.uint64) for k in ("aw", "bw", "ea", "eb", "ec", "h")}
        t = ProveTrace()
        for k, b in bufs.items():
            setattr(t, k, b.ctypes.data)
        proof = np.zeros(32, dtype=np.uint64)
        check(lib().zk_prove_traced(self.handle, w.ctypes.data_as(ctypes.c_void_p), w.shape[0],
                                    ctypes.byref(t), proof.ctypes.data_as(_u64p)))
        out = dict(bufs)
        for k, n in (("msm_a", 8), ("msm_b2", 16), ("msm_c", 8), ("msm_h", 8)):
            out[k] = np.array(list(getattr(t, k)), dtype=np.uint64)
        out["inf"] = [int(x) for x in t.inf]
        out["proof"] = proof
        return out

    def close(self):
        if self.handle:
            lib().zk_circuit_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def prove_files(zkey_path, wtns_path, ctx=None):
    proof = np.zeros(32, dtype=np.uint64)
    check(lib().zk_groth16_prove_files(ctx, str(zkey_path).encode(), str(wtns_path).encode(),
                                       proof.ctypes.data_as(_u64p)))
    return proof


def prove_mem(zkey: bytes, wtns: bytes, ctx=None):
    proof = np.zeros(32, dtype=np.uint64)
    check(lib().zk_groth16_prove_mem(ctx, zkey, len(zkey), wtns, len(wtns),
                                     proof.ctypes.data_as(_u64p)))
    return proof


def read_zkey_header(path):
    h = ZkeyHeader()
    check(lib().zk_read_zkey_header(str(path).encode(), ctypes.byref(h)))
    return h


def proof_to_json(proof):
    buf = ctypes.create_string_buffer(4096)
    p = np.ascontiguousarray(proof, dtype=np.uint64)
    check(lib().zk_proof_to_json(p.ctypes.data_as(_u64p), buf, 4096))
    return buf.value.decode()


def proof_to_calldata(proof):
    out = (ctypes.c_uint8 * 256)()
    p = np.ascontiguousarray(proof, dtype=np.uint64)
    check(lib().zk_proof_to_calldata(p.ctypes.data_as(_u64p), out, 256))
    return bytes(out)


def public_json(wtns_path, n_public):
    size = 64 + 96 * (n_public + 1)
    buf = ctypes.create_string_buffer(size)
    check(lib().zk_public_json(str(wtns_path).encode(), n_public, buf, size))
    return buf.value.decode()


class MsmTable:
    """Fixed-base MSM table (zk_msm_table_create / zk_msm_table_run)."""

    def __init__(self, group, px, py, c=0, ctx=None):
        self.group = group
        self.dx, self.dy = to_device(px), to_device(py)
        h = ctypes.c_void_p()
        n = np.asarray(px).shape[0]
        check(lib().zk_msm_table_create(ctx, group, ptr(self.dx), ptr(self.dy), n, c,
                                        ctypes.byref(h)))
        self.handle = h

    def run(self, scalars):
        sc = np.ascontiguousarray(scalars, dtype=np.uint64).reshape(-1, 4)
        ds = to_device(sc)
        out = np.zeros(8 if self.group == 1 else 16, dtype=np.uint64)
        inf = ctypes.c_int(0)
        check(lib().zk_msm_table_run(self.handle, ptr(ds), sc.shape[0],
                                     out.ctypes.data_as(_u64p), ctypes.byref(inf)))
        return out, bool(inf.value)

    def close(self):
        if self.handle:
            lib().zk_msm_table_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def prove_batch(circuits, witnesses, inflight=3, rs=None, ss=None, on_device=False, ctx=None):
    """Prove many jobs with several proofs in flight (zk_prove_batch).

    circuits: Circuit objects (same context); witnesses: (n, 4) uint64 arrays
    (or device tensors with on_device=True).  rs / ss: optional lists of ints.
    Returns a (count, 32) uint64 array of proofs."""
    count = len(circuits)
    handles = (ctypes.c_void_p * count)(*[c.handle.value for c in circuits])
    if on_device:
        wptrs = [w.data_ptr() for w in witnesses]
        ns = [w.numel() // 4 for w in witnesses]
    else:
        ws = [np.ascontiguousarray(w, dtype=np.uint64).reshape(-1, 4) for w in witnesses]
        wptrs = [w.ctypes.data for w in ws]
        ns = [w.shape[0] for w in ws]
    wp = (ctypes.c_void_p * count)(*wptrs)
    nw = (ctypes.c_size_t * count)(*ns)
    proofs = np.zeros((count, 32), dtype=np.uint64)
    rb = sb = None
    if rs is not None:
        rb = np.array([[(x >> (64 * i)) & (2**64 - 1) for i in range(4)] for x in rs], np.uint64)
        sb = np.array([[(x >> (64 * i)) & (2**64 - 1) for i in range(4)] for x in ss], np.uint64)
    check(lib().zk_prove_batch(ctx, count, handles, wp, nw, 1 if on_device else 0,
                               rb.ctypes.data_as(ctypes.c_void_p) if rb is not None else None,
                               sb.ctypes.data_as(ctypes.c_void_p) if sb is not None else None,
                               proofs.ctypes.data_as(_u64p), inflight))
    return proofs


def set_graphs(on, ctx=None):
    check(lib().zk_ctx_set_graphs(ctx, 1 if on else 0))


BATCH_AUTO, BATCH_INFLIGHT, BATCH_FUSED = 0, 1, 2


def set_batch_mode(mode, group=16, ctx=None):
    """0: fused when every circuit has tables, else in-flight; 1: in-flight
    pipelines; 2: fused groups of up to `group` proofs"""
    check(lib().zk_ctx_set_batch_mode(ctx, mode, group))


# ------------------------------------------------------------- autotuning
UNIFORM, SKEWED = 0, 1


def table_c_default(log_n):
    """fixed-base window bits used when nothing is tuned for the size"""
    return min(max(log_n, 8), 20)


def autotune_msm(group, log_n, dist=UNIFORM, fixed_c=0, ctx=None):
    """Time MSM settings at 2^log_n points; the fastest is recorded in ctx."""
    from ._lib import TuneResult
    r = TuneResult()
    check(lib().zk_autotune_msm(ctx, group, log_n, dist, fixed_c, ctypes.byref(r)))
    return r.as_dict()


def autotune_table_c(group, log_n, dist=UNIFORM, max_table_bytes=0, ctx=None):
    from ._lib import TuneResult
    r = TuneResult()
    check(lib().zk_autotune_table_c(ctx, group, log_n, dist, max_table_bytes, ctypes.byref(r)))
    return r.as_dict()


def autotune_ntt(log_n, ctx=None):
    from ._lib import TuneResult
    r = TuneResult()
    check(lib().zk_autotune_ntt(ctx, log_n, ctypes.byref(r)))
    return r.as_dict()


def tune_export(ctx=None):
    n = ctypes.c_size_t()
    check(lib().zk_tune_export(ctx, None, 0, ctypes.byref(n)))
    buf = ctypes.create_string_buffer(n.value + 1)
    check(lib().zk_tune_export(ctx, buf, n.value + 1, ctypes.byref(n)))
    return buf.value.decode()


def tune_import(text, ctx=None):
    check(lib().zk_tune_import(ctx, text.encode()))


def set_scalar_dist(dist, ctx=None):
    check(lib().zk_ctx_set_scalar_dist(ctx, dist))


def _limbs(x):
    return np.array([(x >> (64 * i)) & (2**64 - 1) for i in range(4)], np.uint64)


class Server:
    """Continuous-batching proof server (zk_server_*).

    submit() queues a proof and returns a ticket at once; wait(ticket) returns
    (proof, latency_ms).  The server keeps each submitted witness alive until
    its ticket is waited for."""

    def __init__(self, max_inflight=4, reserve_bytes=0, ctx=None):
        h = ctypes.c_void_p()
        check(lib().zk_server_create(ctx, max_inflight, reserve_bytes, ctypes.byref(h)))
        self.handle = h
        self._keep = {}

    def submit(self, circuit, witness, r=None, s=None):
        w = np.ascontiguousarray(witness, dtype=np.uint64).reshape(-1, 4)
        rb = _limbs(r) if r is not None else None
        sb = _limbs(s) if s is not None else None
        t = ctypes.c_uint64()
        check(lib().zk_server_submit(self.handle, circuit.handle, w.ctypes.data_as(_u64p),
                                     w.shape[0],
                                     rb.ctypes.data_as(ctypes.c_void_p) if rb is not None else None,
                                     sb.ctypes.data_as(ctypes.c_void_p) if sb is not None else None,
                                     ctypes.byref(t)))
        self._keep[t.value] = w
        return t.value

    def wait(self, ticket, timeout_ms=-1):
        proof = np.zeros(32, dtype=np.uint64)
        lat = ctypes.c_double()
        try:
            check(lib().zk_server_wait(self.handle, ticket, timeout_ms, proof.ctypes.data_as(_u64p),
                                       ctypes.byref(lat)))
        except ZkError as e:
            if e.code != 7:  # ZK_ETIMEOUT keeps the ticket
                self._keep.pop(ticket, None)
            raise
        self._keep.pop(ticket, None)
        return proof, lat.value

    def stats(self):
        v = [ctypes.c_uint64() for _ in range(4)]
        check(lib().zk_server_stats(self.handle, *[ctypes.byref(x) for x in v]))
        return dict(zip(("completed", "failed", "peak_inflight", "admission_waits"),
                        [x.value for x in v]))

    def set_policy(self, policy, max_wait_ms=500):
        """0: arrival order; 1: smallest circuit first with aging"""
        check(lib().zk_server_set_policy(self.handle, policy, max_wait_ms))

    def cancel_queued(self):
        n = ctypes.c_uint64()
        check(lib().zk_server_cancel_queued(self.handle, ctypes.byref(n)))
        return n.value

    def close(self):
        if self.handle is not None and self.handle.value:
            check(lib().zk_server_destroy(self.handle))
            self.handle = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
