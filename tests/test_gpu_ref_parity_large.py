"""Bit-exact parity with the reference's own sm_100a build at the benchmarked
sizes, step by step.

  * Whole proofs of 2^16, 2^20 (2 nonzeros per A/B row, uniform witness)
    and 2^22 constraints (1-4 nonzeros, circom-like witness): every
    intermediate the reference's prover computes -- A.w and B.w from
    readAndComputeMVM (src/groth16.cu:737-861), the odd-coset evaluations of
    A, B, C and h from computeHPoly (src/groth16.cu:1037-1128), the four MSM
    results (src/groth16.cu:1329-1389) -- and the proof of groth16Prove
    (src/groth16.cu:1143-1397), against the library's resident, fixed-base
    and one-shot proofs.
  * The primitive sweep: G1 MSM at 2^20, 2^22 and 2^24 points, G2 MSM at
    2^18 and 2^20 (points k_i G, uniform scalars), NTT and INTT at 2^20,
    2^22 and 2^24 (msm_g1 include/msm_g1.cuh:918, msm_g2_device
    include/msm_g2.cuh:669, ntt include/ntt_bn254.cuh:418).

The reference side runs from oracle/_ref (built by oracle/refbuild/Makefile
from the reference sources); each test skips when its library is absent.
"""
import ctypes

import numpy as np
import pytest

import _ref

pytestmark = pytest.mark.gpu

CIRCUITS = {
    # name: (log_domain, witness kind, nnz range, seed)
    "c16": (16, "circom", (1, 4), 21),
    "u20": (20, "uniform", (2, 2), 1),
    "c22": (22, "circom", (1, 4), 2),
}


@pytest.fixture(scope="module")
def api():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from zyklop_b200 import api as A
    return A


@pytest.fixture(scope="module")
def files(api, tmp_path_factory):
    d = tmp_path_factory.mktemp("large")
    out = {}

    def get(name):
        if name not in out:
            lg, kind, nnz, seed = CIRCUITS[name]
            z, w = d / f"{name}.zkey", d / f"{name}.wtns"
            api.synth_circuit(z, w, lg, n_public=8, n_private_inputs=8, nnz=nnz, witness=kind,
                              seed=seed)
            out[name] = (str(z), str(w))
        return out[name]
    return get


@pytest.mark.parametrize("name", ["c16", "u20", "c22"])
def test_every_intermediate_matches_reference(api, files, name):
    if _ref.inter_lib() is None or _ref.prove_lib() is None:
        pytest.skip("reference sm_100a build (oracle/_ref) not present")
    z, w = files(name)
    c = api.Circuit(z)
    wit = api.read_wtns(w)
    mine = c.trace(wit)
    theirs = _ref.intermediates(z, w, c.domain)
    for key in ("aw", "bw", "ea", "eb", "ec", "h", "msm_a", "msm_b2", "msm_c", "msm_h", "inf"):
        assert np.array_equal(np.asarray(mine[key]), np.asarray(theirs[key])), key
    ref_proof = np.zeros(32, np.uint64)
    assert _ref.prove_lib().zkref_prove_files(
        z.encode(), w.encode(), ref_proof.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))) == 0
    assert np.array_equal(mine["proof"], ref_proof)
    # the same proof through every path a caller has
    assert np.array_equal(c.prove(wit), ref_proof)
    assert np.array_equal(api.prove_files(z, w), ref_proof)
    c.precompute()
    assert np.array_equal(c.prove(wit), ref_proof)
    assert np.array_equal(c.prove_device(api.to_device(wit), wit.shape[0]), ref_proof)
    c.close()


def generator_multiples(api, group, n, seed):
    """n points k_i G (device SoA) with seeded k_i below 2^252, and n uniform
    scalars below 2^252 (device)."""
    rng = np.random.default_rng(seed)
    k = rng.integers(0, 2**63, size=(n, 4), dtype=np.uint64)
    k[:, 3] &= np.uint64((1 << 60) - 1)
    px, py = api.mul_generator(group, k, keep_on_device=True)
    s = rng.integers(0, 2**63, size=(n, 4), dtype=np.uint64)
    s[:, 3] &= np.uint64((1 << 60) - 1)
    return px, py, api.to_device(s)


def run_both(api, group, px, py, sc, n):
    from zyklop_b200._lib import check, lib
    L = _ref.prims()
    width = 8 if group == 1 else 16
    mine, theirs = np.zeros(width, np.uint64), np.zeros(width, np.uint64)
    inf = ctypes.c_int()
    fn = lib().zk_msm_g1 if group == 1 else lib().zk_msm_g2
    check(fn(None, api.ptr(px), api.ptr(py), api.ptr(sc), n,
             mine.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), ctypes.byref(inf)))
    rfn = L.zkref_msm_g1_device if group == 1 else L.zkref_msm_g2_device
    tinf = rfn(api.ptr(px), api.ptr(py), api.ptr(sc), n,
               theirs.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)))
    return mine, bool(inf.value), theirs, bool(tinf)


@pytest.mark.parametrize("group,logs", [(1, (20, 22, 24)), (2, (18, 20))])
def test_msm_sweep_matches_reference(api, group, logs):
    if _ref.prims() is None:
        pytest.skip("reference sm_100a build (oracle/_ref) not present")
    import torch
    px, py, sc = generator_multiples(api, group, 1 << max(logs), 90 + group)
    for lg in logs:
        mine, minf, theirs, tinf = run_both(api, group, px, py, sc, 1 << lg)
        assert minf == tinf and not minf, lg
        assert np.array_equal(mine, theirs), lg
    del px, py, sc
    torch.cuda.empty_cache()


@pytest.mark.parametrize("log_n,inverse", [(20, False), (20, True), (22, False), (22, True),
                                           (24, False), (24, True)])
def test_ntt_sweep_matches_reference(api, log_n, inverse):
    L = _ref.prims()
    if L is None:
        pytest.skip("reference sm_100a build (oracle/_ref) not present")
    import torch
    n = 1 << log_n
    g = torch.Generator(device="cuda")
    g.manual_seed(log_n * 2 + inverse)
    buf = torch.randint(0, 2**62, (n, 4), dtype=torch.int64, device="cuda", generator=g)
    buf[:, 3] &= (1 << 58) - 1  # below r, read as Montgomery elements
    ref = buf.clone()
    from zyklop_b200._lib import check, lib
    check(lib().zk_ntt(None, api.ptr(buf), log_n, 1 if inverse else 0))
    assert L.zkref_ntt_device(api.ptr(ref), log_n, 1 if inverse else 0) == 0
    torch.cuda.synchronize()
    assert torch.equal(buf, ref)
    del buf, ref
    torch.cuda.empty_cache()
