"""ctypes binding of libzyklop_b200.so (signatures of include/zyklop_b200.h)."""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libzyklop_b200.so")

_lib = None

u64p = ctypes.POINTER(ctypes.c_uint64)
u8p = ctypes.POINTER(ctypes.c_uint8)
c_int_p = ctypes.POINTER(ctypes.c_int)
sz = ctypes.c_size_t


class ZkError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"zyklop_b200 error {code}: {msg}")
        self.code = code


# name -> (restype, argtypes)
SIGNATURES = {
    "zk_version": (ctypes.c_char_p, []),
    "zk_last_error": (ctypes.c_char_p, []),
    "zk_ctx_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "zk_ctx_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "zk_ctx_sync": (ctypes.c_int, [ctypes.c_void_p]),
    "zk_ctx_set_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "zk_release_cached_memory": (ctypes.c_int, [ctypes.c_void_p]),
    "zk_launch_count": (ctypes.c_int, [ctypes.POINTER(ctypes.c_uint64)]),
    "zk_memory_stats": (ctypes.c_int, [ctypes.c_int, ctypes.c_void_p]),
    "zk_ctx_set_profiling": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "zk_ctx_profile": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "zk_imad_probe": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]),
    "zk_int_probe": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    "zk_field_op": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                   ctypes.c_void_p, ctypes.c_void_p, sz]),
    "zk_ntt": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int]),
    "zk_hpoly": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                ctypes.c_void_p]),
    "zk_msm_g1": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                 sz, u64p, c_int_p]),
    "zk_msm_g2": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                 sz, u64p, c_int_p]),
    "zk_msm_g1_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, sz,
                                         u64p, c_int_p, ctypes.c_void_p]),
    "zk_msm_table_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                           ctypes.c_void_p, sz, ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_void_p)]),
    "zk_msm_table_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, sz, u64p, c_int_p]),
    "zk_msm_table_free": (ctypes.c_int, [ctypes.c_void_p]),
    "zk_circuit_precompute": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "zk_msm_set_config": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int]),
    "zk_msm_scratch_bytes": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, sz,
                                            ctypes.POINTER(ctypes.c_size_t)]),
    "zk_mul_generator": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, sz,
                                        ctypes.c_void_p, ctypes.c_void_p]),
    "zk_circuit_load_file": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p,
                                            ctypes.POINTER(ctypes.c_void_p)]),
    "zk_circuit_load_mem": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, sz,
                                           ctypes.POINTER(ctypes.c_void_p)]),
    "zk_circuit_free": (ctypes.c_int, [ctypes.c_void_p]),
    "zk_circuit_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32),
                                       ctypes.POINTER(ctypes.c_uint32),
                                       ctypes.POINTER(ctypes.c_uint32)]),
    "zk_prove": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, sz, ctypes.c_void_p,
                                ctypes.c_void_p, u64p]),
    "zk_prove_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, sz, ctypes.c_void_p,
                                       ctypes.c_void_p, u64p]),
    "zk_prove_intermediates": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, sz,
                                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                              u64p]),
    "zk_prove_traced": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, sz, ctypes.c_void_p,
                                       u64p]),
    "zk_prove_batch": (ctypes.c_int, [ctypes.c_void_p, sz, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                      ctypes.c_void_p, u64p, ctypes.c_int]),
    "zk_ctx_set_graphs": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "zk_ctx_set_prove_streams": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "zk_ctx_set_batch_mode": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "zk_autotune_msm": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_void_p]),
    "zk_autotune_table_c": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           sz, ctypes.c_void_p]),
    "zk_autotune_ntt": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "zk_tune_export": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, sz,
                                      ctypes.POINTER(ctypes.c_size_t)]),
    "zk_tune_import": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p]),
    "zk_ctx_set_scalar_dist": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "zk_circuit_set_scalar_dist": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "zk_server_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, sz,
                                        ctypes.POINTER(ctypes.c_void_p)]),
    "zk_server_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, u64p, sz, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)]),
    "zk_server_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, u64p,
                                      ctypes.POINTER(ctypes.c_double)]),
    "zk_server_stats": (ctypes.c_int, [ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_uint64)] * 4),
    "zk_server_set_policy": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "zk_server_cancel_queued": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)]),
    "zk_server_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "zk_groth16_prove_files": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_char_p,
                                              u64p]),
    "zk_groth16_prove_mem": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, sz, ctypes.c_void_p,
                                            sz, u64p]),
    "zk_read_zkey_header": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_void_p]),
    "zk_proof_to_json": (ctypes.c_int, [u64p, ctypes.c_char_p, sz]),
    "zk_proof_to_calldata": (ctypes.c_int, [u64p, ctypes.c_void_p, sz]),
    "zk_public_json": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_uint32, ctypes.c_char_p, sz]),
    "zk_synth_circuit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p,
                                        ctypes.c_char_p]),
}


class ZkeyHeader(ctypes.Structure):
    _fields_ = [("n_constraints", ctypes.c_uint32), ("n_vars", ctypes.c_uint32),
                ("n_public", ctypes.c_uint32), ("domain_size", ctypes.c_uint32),
                ("log_domain", ctypes.c_int32), ("prime", ctypes.c_uint64 * 4)]


class MemoryStats(ctypes.Structure):
    """zk_memory_stats_t"""
    _fields_ = [("device_allocations", ctypes.c_uint64),
                ("device_allocated_bytes", ctypes.c_uint64),
                ("pinned_allocations", ctypes.c_uint64),
                ("pool_reserved_bytes", ctypes.c_uint64), ("pool_used_bytes", ctypes.c_uint64)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


def memory_stats(device=0):
    s = MemoryStats()
    check(lib().zk_memory_stats(device, ctypes.byref(s)))
    return s.as_dict()


class ProveTrace(ctypes.Structure):
    """zk_prove_trace: buffer pointers in, MSM results out."""
    _fields_ = [("aw", ctypes.c_void_p), ("bw", ctypes.c_void_p), ("ea", ctypes.c_void_p),
                ("eb", ctypes.c_void_p), ("ec", ctypes.c_void_p), ("h", ctypes.c_void_p),
                ("msm_a", ctypes.c_uint64 * 8), ("msm_b2", ctypes.c_uint64 * 16),
                ("msm_c", ctypes.c_uint64 * 8), ("msm_h", ctypes.c_uint64 * 8),
                ("inf", ctypes.c_int32 * 4)]


class TuneResult(ctypes.Structure):
    _fields_ = [("c", ctypes.c_int), ("k0", ctypes.c_int), ("k1", ctypes.c_int),
                ("chunk", ctypes.c_int), ("table_c", ctypes.c_int), ("pass_bits", ctypes.c_int),
                ("ms", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class SynthParams(ctypes.Structure):
    _fields_ = [("log_domain", ctypes.c_uint32), ("n_public", ctypes.c_uint32),
                ("n_private_inputs", ctypes.c_uint32), ("nnz_min", ctypes.c_uint32),
                ("nnz_max", ctypes.c_uint32), ("witness_kind", ctypes.c_uint32),
                ("seed", ctypes.c_uint64)]


def lib():
    """Load the library (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `make -C zyklop_b200/csrc` "
            "(or __graft_entry__.build()); there is no CPU fallback")
    L = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(rc):
    if rc != 0:
        raise ZkError(rc, lib().zk_last_error().decode())
    return rc


def version():
    return lib().zk_version().decode()


class Profile(ctypes.Structure):
    KINDS = ("accum_g1", "accum_g2", "ntt_pass", "spmv")
    _fields_ = [("ms", ctypes.c_double * 4), ("launches", ctypes.c_double * 4),
                ("units", ctypes.c_double * 4)]
