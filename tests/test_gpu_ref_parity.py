"""Bit-exact parity with the reference's own sm_100a build on the same inputs.

The reference's msm_g1 (include/msm_g1.cuh:918), msm_g2_device
(include/msm_g2.cuh:669) and ntt (include/ntt_bn254.cuh:418) are compiled
from the reference sources into oracle/_ref/ and run on the same device
buffers as the library.  Skipped when that build is absent.
"""
import ctypes

import numpy as np
import pytest

import _ref
from test_gpu_primitives import point_pool, scalars, tile_points

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    L = _ref.prims()
    if L is None:
        pytest.skip("reference sm_100a build (oracle/_ref) not present")
    return L


@pytest.fixture(scope="module")
def api():
    from zyklop_b200 import api as A
    return A


def ref_msm(ref, fn, width, px, py, sc):
    from zyklop_b200.api import ptr, to_device
    dx, dy, ds = to_device(px), to_device(py), to_device(sc)
    out = np.zeros(width, np.uint64)
    inf = fn(ptr(dx), ptr(dy), ptr(ds), sc.shape[0], out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)))
    return out, bool(inf)


@pytest.mark.parametrize("log_n,kind", [(12, "uniform"), (16, "uniform"), (16, "circom"),
                                        (18, "uniform")])
def test_msm_g1_matches_reference(api, oracle, ref, log_n, kind):
    rng = np.random.default_rng(log_n * 3 + len(kind))
    n = 1 << log_n
    xs, ys = point_pool(oracle, 1, 512)
    px, py = tile_points(xs, ys, n)
    sc = scalars(rng, n, kind) if n <= 4096 else None
    if sc is None:
        sc = rng.integers(0, 2**63, size=(n, 4), dtype=np.uint64) * np.uint64(2) + np.uint64(1)
        sc[:, 3] &= np.uint64(0x0FFFFFFFFFFFFFFF)
        if kind == "circom":
            u = rng.random(n)
            sc[u < 0.55] = 0
            sc[u < 0.275, 0] = 1
            small = (u >= 0.55) & (u < 0.70)
            sc[small, 1:] = 0
    mine, minf = api.msm_g1(px, py, sc)
    theirs, tinf = ref_msm(ref, ref.zkref_msm_g1_device, 8, px, py, sc)
    assert minf == tinf
    assert np.array_equal(mine, theirs)


@pytest.mark.parametrize("log_n", [10, 13])
def test_msm_g2_matches_reference(api, oracle, ref, log_n):
    rng = np.random.default_rng(log_n)
    n = 1 << log_n
    xs, ys = point_pool(oracle, 2, 128)
    px, py = tile_points(xs, ys, n)
    sc = scalars(rng, n)
    mine, minf = api.msm_g2(px, py, sc)
    theirs, tinf = ref_msm(ref, ref.zkref_msm_g2_device, 16, px, py, sc)
    assert minf == tinf
    assert np.array_equal(mine, theirs)


@pytest.mark.parametrize("log_n,inverse", [(12, False), (12, True), (16, False), (16, True)])
def test_ntt_matches_reference(api, ref, log_n, inverse):
    from zyklop_b200.api import ptr, to_device, to_host
    rng = np.random.default_rng(log_n + inverse)
    n = 1 << log_n
    a = rng.integers(0, 2**63, size=(n, 4), dtype=np.uint64)
    a[:, 3] &= np.uint64(0x0FFFFFFFFFFFFFFF)
    d = to_device(a)
    assert ref.zkref_ntt_device(ptr(d), log_n, 1 if inverse else 0) == 0
    theirs = to_host(d).reshape(-1, 4)
    assert np.array_equal(api.ntt(a, log_n, inverse), theirs)
