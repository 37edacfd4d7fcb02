"""zk_msm_g1_noalloc: the G1 MSM for callers that cannot allocate device memory.

Such callers (a plugin whose host application has given all device memory to
its own pool allocator, or a latency-critical loop that cannot take
cudaMalloc's implicit synchronization) get an entry point whose scratch is a
fixed 24 MiB __device__ array inside the library, limited to 2^16 points.
These tests call it through the C ABI and compare it with the allocating
zk_msm_g1 on the same inputs (exact equality: the result is an affine point,
integer arithmetic, tolerance zero), twice in a row with different inputs so
that leftovers of the first call cannot leak into the second.  The file is
named to be collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

R = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
MAX_POINTS = 1 << 16


@pytest.fixture(scope="module")
def api():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from zyklop_b200 import api as A
    return A


def scalars(rng, n):
    out = np.zeros((n, 4), np.uint64)
    for i in range(n):
        k = int.from_bytes(rng.bytes(32), "little") % R
        out[i] = [(k >> (64 * j)) & (2**64 - 1) for j in range(4)]
    return out


def noalloc(api, dx, dy, ds, n, stream=None):
    from zyklop_b200._lib import lib
    out = np.zeros(8, np.uint64)
    inf = ctypes.c_int(-1)
    rc = lib().zk_msm_g1_noalloc(api.ptr(dx), api.ptr(dy), api.ptr(ds), n,
                                 out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                 ctypes.byref(inf), stream)
    return rc, out, inf.value


def test_noalloc_matches_zk_msm_g1_two_calls(api):
    rng = np.random.default_rng(2024)
    # distinct bases k_i * G built on the device, random scalars
    for n in (MAX_POINTS, 3000, 200):
        base = scalars(rng, n)
        px, py = api.mul_generator(1, base)
        sc = scalars(rng, n)
        dx, dy, ds = api.to_device(px), api.to_device(py), api.to_device(sc)
        rc, got, inf = noalloc(api, dx, dy, ds, n)
        assert rc == 0
        want, winf = api.msm_g1(px, py, sc)
        assert np.array_equal(got, want)
        assert bool(inf) == winf


def test_noalloc_rejects_more_than_max_points(api):
    from zyklop_b200._lib import lib
    d = api.empty_device(4)
    rc, _, _ = noalloc(api, d, d, d, MAX_POINTS + 1)
    assert rc == 1  # ZK_EINVAL
    assert b"maximum" in lib().zk_last_error()


def test_noalloc_allocates_nothing(api):
    """The property the entry point exists for: once a device has made its
    first call, further calls (other sizes, another stream) leave the device's
    free memory, the library's allocation count and its memory pool exactly
    as they were."""
    import torch
    from zyklop_b200._lib import memory_stats
    rng = np.random.default_rng(77)
    inputs = []
    for n in (4096, 50000):
        px, py = api.mul_generator(1, scalars(rng, n))
        sc = scalars(rng, n)
        want, winf = api.msm_g1(px, py, sc)
        inputs.append((n, api.to_device(px), api.to_device(py), api.to_device(sc), want, winf))
    side = torch.cuda.Stream()
    torch.cuda.synchronize()
    n, dx, dy, ds, want, _ = inputs[0]
    assert noalloc(api, dx, dy, ds, n)[0] == 0  # warm-up: the scratch array is placed
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    stats0 = memory_stats(torch.cuda.current_device())
    for n, dx, dy, ds, want, winf in inputs:
        for stream in (None, ctypes.c_void_p(side.cuda_stream)):
            rc, got, inf = noalloc(api, dx, dy, ds, n, stream)
            assert rc == 0
            assert np.array_equal(got, want) and bool(inf) == winf
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert memory_stats(torch.cuda.current_device()) == stats0


def test_noalloc_empty_input_is_infinity(api):
    d = api.empty_device(4)
    rc, out, inf = noalloc(api, d, d, d, 0)
    assert rc == 0 and inf == 1
    assert not out.any()  # (0, 0) encodes infinity, like the reference


def test_noalloc_refuses_a_capturing_stream(api):
    """The call synchronizes its stream, so it refuses to run inside a CUDA
    graph capture (and the capture stays intact)."""
    import torch
    from zyklop_b200._lib import lib
    d = api.empty_device(4 * 16)
    assert noalloc(api, d, d, d, 0)[0] == 0  # the device's first call happens outside capture
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        g.capture_begin()
        rc, _, _ = noalloc(api, d, d, d, 16, ctypes.c_void_p(s.cuda_stream))
        g.capture_end()
    assert rc == 9  # ZK_ENOTSUP
    assert b"captur" in lib().zk_last_error()
