"""GPU parity of the field, NTT, H-polynomial and MSM primitives.

Bit-exact against (1) the reference's own golden vectors (tests/golden, the
same checks as test/unit/test_fp_bn254.cu, test_fr_bn254.cu, test_ntt.cu,
test_msm.cu, test_msm_g2.cu) and (2) the CPU oracle on seeded inputs at sizes
the oracle finishes in seconds, plus size-independent properties at larger
sizes (NTT round trips, MSM linearity).
"""
import json
import os

import numpy as np
import pytest

from _oracle import MONT, P, R, arr, ints, limbs, mont, to_int, unmont

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)


def H(x):
    return int(x, 16)


@pytest.fixture(scope="module")
def api():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from zyklop_b200 import api as A
    return A


def rand_fe(rng, n, m):
    return [int.from_bytes(rng.bytes(32), "little") % m for _ in range(n)]


# ---------------------------------------------------------------- fields
FPV = load("fp_vectors.json")
FRV = load("fr_vectors.json")


@pytest.mark.parametrize("op", ["add", "sub", "mul"])
def test_fp_binary_golden(api, op):
    vec = FPV["fp_" + op]
    got = api.field_op(0, op, arr([H(v[0]) for v in vec]), arr([H(v[1]) for v in vec]))
    assert ints(got) == [H(v[2]) for v in vec]


@pytest.mark.parametrize("op", ["neg", "sqr"])
def test_fp_unary_golden(api, op):
    vec = FPV["fp_" + op]
    got = api.field_op(0, op, arr([H(v[0]) for v in vec]))
    assert ints(got) == [H(v[1]) for v in vec]


def test_fp_inverse_golden(api):
    # canonical inverse = decode(inv(encode(a))) (test_fp_bn254.cu:255-280)
    vec = FPV["fp_inv"]
    a = arr([H(v[0]) for v in vec])
    got = api.field_op(0, "decode", api.field_op(0, "inv", api.field_op(0, "encode", a)))
    assert ints(got) == [H(v[1]) for v in vec]


@pytest.mark.parametrize("op,key", [("add", "frAdd"), ("sub", "frSub"), ("mul", "frMul")])
def test_fr_binary_golden(api, op, key):
    vec = FRV["ops"][key]
    got = api.field_op(1, op, arr([H(v["a"]) for v in vec]), arr([H(v["b"]) for v in vec]))
    assert ints(got) == [H(v["r"]) for v in vec]


@pytest.mark.parametrize("op,key", [("neg", "frNeg"), ("sqr", "frSqr"), ("inv", "frInv")])
def test_fr_unary_golden(api, op, key):
    vec = FRV["ops"][key]
    got = api.field_op(1, op, arr([H(v["a"]) for v in vec]))
    assert ints(got) == [H(v["r"]) for v in vec]


def test_fr_encode_decode_golden(api):
    vec = FRV["ops"]["frRoundTrip"]
    enc = api.field_op(1, "encode", arr([H(v["x"]) for v in vec]))
    assert ints(enc) == [H(v["x_enc"]) for v in vec]
    assert ints(api.field_op(1, "decode", enc)) == [H(v["x_dec"]) for v in vec]


def test_field_random_vs_oracle(api, oracle):
    rng = np.random.default_rng(7)
    for which, m in ((0, P), (1, R)):
        a = arr(rand_fe(rng, 4096, m))
        b = arr(rand_fe(rng, 4096, m))
        for op, code in (("mul", 0), ("add", 1), ("sub", 2), ("sqr", 3), ("neg", 4)):
            got = api.field_op(which, op, a, b if code < 3 else None)
            exp = oracle.batch(which, code, a, b if code < 3 else None)
            assert np.array_equal(got, exp), (which, op)
    # edge values: 0, 1, m-1 (Montgomery), all limbs maxed below m
    edges = arr([0, 1, P - 1, mont(1, P), mont(P - 1, P), P - 2])
    got = api.field_op(0, "mul", edges, edges[::-1].copy())
    assert np.array_equal(got, oracle.batch(0, 0, edges, edges[::-1].copy()))


# ------------------------------------------------------------------- NTT
NTTV = load("ntt_vectors.json")


@pytest.mark.parametrize("case", range(len(NTTV)))
def test_ntt_golden(api, case):
    v = NTTV[case]
    inp = [mont(H(x), R) for x in v["input"]]
    exp = [mont(H(x), R) for x in v["expected"]]
    # the reference test: INTT(expected) == input (test_ntt.cu:129-146)
    assert ints(api.ntt(arr(exp), v["log_n"], inverse=True)) == inp
    assert ints(api.ntt(arr(inp), v["log_n"], inverse=False)) == exp


@pytest.mark.parametrize("log_n", [1, 5, 8, 9, 12, 16, 17])
def test_ntt_vs_oracle(api, oracle, log_n):
    rng = np.random.default_rng(log_n)
    a = arr(rand_fe(rng, 1 << log_n, R))
    assert np.array_equal(api.ntt(a, log_n, False), oracle.ntt(a, log_n, False))
    assert np.array_equal(api.ntt(a, log_n, True), oracle.ntt(a, log_n, True))


@pytest.mark.parametrize("log_n", [20, 22])
def test_ntt_roundtrip_large(api, log_n):
    rng = np.random.default_rng(100 + log_n)
    n = 1 << log_n
    # uniform 254-bit limbs reduced below r by clearing the top bits
    a = rng.integers(0, 2**63, size=(n, 4), dtype=np.uint64)
    a[:, 3] &= np.uint64(0x0FFFFFFFFFFFFFFF)
    f = api.ntt(a, log_n, False)
    assert not np.array_equal(f, a)
    assert np.array_equal(api.ntt(f, log_n, True), a)


@pytest.mark.parametrize("log_n", [1, 4, 10, 13])
def test_hpoly_vs_oracle(api, oracle, log_n):
    rng = np.random.default_rng(200 + log_n)
    n = 1 << log_n
    aw = arr(rand_fe(rng, n, R))
    bw = arr(rand_fe(rng, n, R))
    assert np.array_equal(api.hpoly(aw, bw, log_n), oracle.hpoly(aw, bw, log_n))


# ------------------------------------------------------------------- MSM
M1 = load("msm_g1_vectors.json")
M2 = load("msm_g2_vectors.json")


@pytest.mark.parametrize("case", range(len(M1)))
def test_msm_g1_golden(api, case):
    v = M1[case]
    out, inf = api.msm_g1(arr([H(x) for x in v["px"]]), arr([H(x) for x in v["py"]]),
                          arr([H(x) for x in v["scalars"]]))
    assert not inf
    assert to_int(out[:4]) == H(v["out"][0]) and to_int(out[4:]) == H(v["out"][1]), v["label"]


def g2_arr(pairs):
    return np.concatenate([arr([H(a), H(b)]).reshape(1, 8) for a, b in pairs])


@pytest.mark.parametrize("case", range(len(M2)))
def test_msm_g2_golden(api, case):
    v = M2[case]
    out, inf = api.msm_g2(g2_arr(v["px"]), g2_arr(v["py"]), arr([H(x) for x in v["scalars"]]))
    assert inf == v["infinity"]
    if not inf:
        assert [to_int(out[4 * i:4 * i + 4]) for i in range(4)] == [H(x) for x in v["out"]]


_POOL = {}


def point_pool(oracle, group, n):
    """n distinct random multiples of the generator (affine Montgomery, SoA)."""
    key = (group, n)
    if key not in _POOL:
        rng = np.random.default_rng(1234 + group)
        g = oracle.g1_gen() if group == 1 else oracle.g2_gen()
        w = 4 if group == 1 else 8
        xs = np.zeros((n, w), np.uint64)
        ys = np.zeros((n, w), np.uint64)
        for i in range(n):
            k = int.from_bytes(rng.bytes(32), "little") % R
            p = oracle.g1_mul(g, k) if group == 1 else oracle.g2_mul(g, k)
            xs[i], ys[i] = p[:w], p[w:]
        _POOL[key] = (xs, ys)
    return _POOL[key]


def tile_points(xs, ys, n):
    reps = (n + xs.shape[0] - 1) // xs.shape[0]
    return np.tile(xs, (reps, 1))[:n].copy(), np.tile(ys, (reps, 1))[:n].copy()


def scalars(rng, n, kind="uniform"):
    if kind == "uniform":
        return arr([int.from_bytes(rng.bytes(32), "little") % R for _ in range(n)])
    if kind == "circom":  # 55% {0,1}, 15% < 2^64, 30% uniform
        out = []
        for _ in range(n):
            u = rng.random()
            if u < 0.55:
                out.append(int(rng.integers(0, 2)))
            elif u < 0.70:
                out.append(int(rng.integers(0, 2**63)) * 2 + 1)
            else:
                out.append(int.from_bytes(rng.bytes(32), "little") % R)
        return arr(out)
    if kind == "ones":
        return arr([1] * n)
    if kind == "same":
        k = int.from_bytes(rng.bytes(32), "little") % R
        return arr([k] * n)
    if kind == "max":  # 256-bit values, not reduced: the full integer is used
        return arr([2**256 - 1 - i for i in range(n)])
    raise ValueError(kind)


@pytest.mark.parametrize("n,kind", [(0, "uniform"), (1, "uniform"), (7, "uniform"),
                                    (1000, "uniform"), (4096, "uniform"), (20000, "uniform"),
                                    (5000, "circom"), (3000, "ones"), (3000, "same"),
                                    (500, "max")])
def test_msm_g1_vs_oracle(api, oracle, n, kind):
    rng = np.random.default_rng(n + len(kind))
    xs, ys = point_pool(oracle, 1, 512)
    px, py = tile_points(xs, ys, max(n, 1))
    sc = scalars(rng, n, kind) if n else np.zeros((0, 4), np.uint64)
    out, inf = api.msm_g1(px[:max(n, 1)], py[:max(n, 1)], sc)
    exp, einf = oracle.msm_g1(px[:n], py[:n], sc) if n else (np.zeros(8, np.uint64), 1)
    assert inf == bool(einf)
    assert np.array_equal(out, exp)


def test_msm_g1_infinity_points_and_zero_scalars(api, oracle):
    rng = np.random.default_rng(5)
    xs, ys = point_pool(oracle, 1, 512)
    px, py = xs.copy(), ys.copy()
    px[::3] = 0
    py[::3] = 0  # (0,0) points are skipped (msm_g1.cuh:232-245)
    sc = scalars(rng, 512)
    sc[1::5] = 0
    out, inf = api.msm_g1(px, py, sc)
    exp, einf = oracle.msm_g1(px, py, sc)
    assert np.array_equal(out, exp) and inf == bool(einf)
    zero = np.zeros_like(sc)
    out, inf = api.msm_g1(px, py, zero)
    assert inf and not out.any()
    # P + (-P) cancels to infinity
    nsc = np.stack([limbs(5), limbs(R - 5)])
    out, inf = api.msm_g1(np.stack([xs[0], xs[0]]), np.stack([ys[0], ys[0]]), nsc)
    assert inf


@pytest.mark.parametrize("c", [8, 11, 13, 16])
def test_msm_g1_window_sizes(api, oracle, c):
    rng = np.random.default_rng(c)
    xs, ys = point_pool(oracle, 1, 512)
    px, py = tile_points(xs, ys, 3000)
    sc = scalars(rng, 3000)
    exp, _ = oracle.msm_g1(px, py, sc)
    try:
        api.msm_set_config(1, c=c, k0=8, k1=4, chunk=8)
        out, _ = api.msm_g1(px, py, sc)
    finally:
        api.msm_set_config(1)
    assert np.array_equal(out, exp)


def test_msm_g1_linearity_large(api, oracle):
    # size-independent property at 2^20: MSM(k) + MSM(k') == MSM(k + k')
    rng = np.random.default_rng(99)
    n = 1 << 20
    xs, ys = point_pool(oracle, 1, 512)
    px, py = tile_points(xs, ys, n)
    k1 = rng.integers(0, 2**63, size=(n, 4), dtype=np.uint64)
    k2 = rng.integers(0, 2**63, size=(n, 4), dtype=np.uint64)
    k1[:, 3] >>= np.uint64(2)
    k2[:, 3] >>= np.uint64(2)
    s = k1 + k2  # no limb overflow: each limb < 2^64 and top limbs < 2^62
    carry = np.zeros(n, dtype=np.uint64)
    s = np.zeros_like(k1)
    for j in range(4):
        t = k1[:, j].astype(object) + k2[:, j].astype(object) + carry.astype(object)
        s[:, j] = np.array([int(x) & (2**64 - 1) for x in t], dtype=np.uint64)
        carry = np.array([int(x) >> 64 for x in t], dtype=np.uint64)
    a, _ = api.msm_g1(px, py, k1)
    b, _ = api.msm_g1(px, py, k2)
    c, _ = api.msm_g1(px, py, s)
    assert np.array_equal(oracle.g1_add(a, b), c)


@pytest.mark.parametrize("n,kind", [(1, "uniform"), (300, "uniform"), (2000, "uniform"),
                                    (1500, "circom"), (700, "same")])
def test_msm_g2_vs_oracle(api, oracle, n, kind):
    rng = np.random.default_rng(50 + n)
    xs, ys = point_pool(oracle, 2, 128)
    px, py = tile_points(xs, ys, n)
    sc = scalars(rng, n, kind)
    out, inf = api.msm_g2(px, py, sc)
    exp, einf = oracle.msm_g2(px, py, sc)
    assert inf == bool(einf)
    assert np.array_equal(out, exp)


@pytest.mark.parametrize("group", [1, 2])
def test_mul_generator_vs_oracle(api, oracle, group):
    rng = np.random.default_rng(group)
    ks = [0, 1, 2, R - 1] + [int.from_bytes(rng.bytes(32), "little") % R for _ in range(60)]
    px, py = api.mul_generator(group, arr(ks))
    g = oracle.g1_gen() if group == 1 else oracle.g2_gen()
    w = 4 if group == 1 else 8
    for i, k in enumerate(ks):
        exp = oracle.g1_mul(g, k) if group == 1 else oracle.g2_mul(g, k)
        assert np.array_equal(np.concatenate([px[i], py[i]]), exp), (group, i)


@pytest.mark.parametrize("group,n,c", [(1, 1, 0), (1, 100, 8), (1, 5000, 0), (1, 1 << 16, 0),
                                       (1, 3000, 13), (2, 50, 0), (2, 3000, 0), (2, 2048, 11)])
def test_fixed_base_table_matches_windowed(api, oracle, group, n, c):
    """zk_msm_table (precomputed 2^(cw) multiples, one shared bucket set) gives
    the same affine point as the windowed MSM, including for scalars >= r
    (reduced mod r against points of order r), for partial scalar vectors and
    with a base at infinity; window counts cover whole and partial chunks of
    the table build's shared inversions."""
    rng = np.random.default_rng(group * 1000 + n)
    base = scalars(rng, n)
    if n > 10:
        base[5] = 0  # a point at infinity, (0, 0), among the bases
    px, py = api.mul_generator(group, base)
    sc = scalars(rng, n)
    if n >= 4:
        over = int.from_bytes(rng.bytes(32), "little") % R
        sc[1] = limbs(over + R)        # >= r
        sc[2] = limbs(2**256 - 1)      # maximal 256-bit integer
        sc[3] = 0
    t = api.MsmTable(group, px, py, c=c)
    got, ginf = t.run(sc)
    want, winf = (api.msm_g1 if group == 1 else api.msm_g2)(px, py, sc)
    assert ginf == winf and np.array_equal(got, want)
    if n > 10:
        k = n // 2  # fewer scalars than table points: the rest count as zero
        got, _ = t.run(sc[:k])
        want, _ = (api.msm_g1 if group == 1 else api.msm_g2)(px[:k], py[:k], sc[:k])
        assert np.array_equal(got, want)
    t.close()
