"""Pins the CPU oracle against the reference's own golden vectors.

The fixtures in tests/golden/ are the reference's unit-test vectors
(test/unit/test_vectors*.json), re-encoded by tests/golden/make_fixtures.py.
Each check mirrors the reference test that consumes the same vectors:
  Fp ops + G1 curve    test/unit/test_fp_bn254.cu:465-612
  Fr ops               test/unit/test_fr_bn254.cu:655-693
  NTT (inverse only)   test/unit/test_ntt.cu:129-146
  G1 MSM               test/unit/test_msm.cu:131-172
  G2 MSM               test/unit/test_msm_g2.cu
"""
import json
import os

import numpy as np
import pytest

from _oracle import MONT, P, R, arr, ints, limbs, mont, to_int, unmont

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)


FP = load("fp_vectors.json")
FR = load("fr_vectors.json")
NTT = load("ntt_vectors.json")
MSM1 = load("msm_g1_vectors.json")
MSM2 = load("msm_g2_vectors.json")


def H(x):
    return int(x, 16)


@pytest.mark.parametrize("op,code", [("fp_add", 1), ("fp_sub", 2), ("fp_mul", 0)])
def test_fp_binary(oracle, op, code):
    vec = FP[op]
    a = arr([H(v[0]) for v in vec])
    b = arr([H(v[1]) for v in vec])
    got = ints(oracle.batch(0, code, a, b))
    assert got == [H(v[2]) for v in vec]


@pytest.mark.parametrize("op,code", [("fp_neg", 4), ("fp_sqr", 3)])
def test_fp_unary(oracle, op, code):
    vec = FP[op]
    got = ints(oracle.batch(0, code, arr([H(v[0]) for v in vec])))
    assert got == [H(v[1]) for v in vec]


def test_fp_inv_normal(oracle):
    for a, r in FP["fp_inv"]:
        assert oracle.f1("inv_normal", 0, H(a)) == H(r)


def test_g1_affine_add(oracle):
    for v in FP["curve_g1"]:
        p1 = np.concatenate([limbs(mont(H(v["p1"][0]), P)), limbs(mont(H(v["p1"][1]), P))])
        p2 = np.concatenate([limbs(mont(H(v["p2"][0]), P)), limbs(mont(H(v["p2"][1]), P))])
        r = oracle.g1_add(p1, p2)
        assert unmont(to_int(r[:4]), P) == H(v["r"][0]), v["note"]
        assert unmont(to_int(r[4:]), P) == H(v["r"][1]), v["note"]


def test_g1_scalar_mul(oracle):
    g = oracle.g1_gen()
    for v in FP["curve_g1_mul"]:
        r = oracle.g1_mul(g, H(v["scalar"]))
        assert unmont(to_int(r[:4]), P) == H(v["r"][0]), v["note"]
        assert unmont(to_int(r[4:]), P) == H(v["r"][1]), v["note"]


@pytest.mark.parametrize("op,code", [("frAdd", 1), ("frSub", 2), ("frMul", 0)])
def test_fr_binary(oracle, op, code):
    vec = FR["ops"][op]
    got = ints(oracle.batch(1, code, arr([H(v["a"]) for v in vec]), arr([H(v["b"]) for v in vec])))
    assert got == [H(v["r"]) for v in vec]


@pytest.mark.parametrize("op,code", [("frNeg", 4), ("frSqr", 3), ("frInv", 5)])
def test_fr_unary(oracle, op, code):
    vec = FR["ops"][op]
    got = ints(oracle.batch(1, code, arr([H(v["a"]) for v in vec])))
    assert got == [H(v["r"]) for v in vec]


def test_fr_inv_normal_and_roundtrip(oracle):
    for v in FR["ops"]["frInvNormal"]:
        assert oracle.f1("inv_normal", 1, H(v["a"])) == H(v["r"])
    for v in FR["ops"]["frRoundTrip"]:
        assert oracle.f1("encode", 1, H(v["x"])) == H(v["x_enc"])
        assert oracle.f1("decode", 1, H(v["x_enc"])) == H(v["x_dec"])
    assert oracle.f1("encode", 1, 1) == H(FR["ops"]["frMontEncode_1"][0]["expected_R_Fr"])


def test_fr_ntt_butterfly_and_pow(oracle):
    for v in FR["ops"]["frNTT_CT"]:
        t = oracle.f2("mul", 1, H(v["b"]), H(v["omega"]))
        assert oracle.f2("add", 1, H(v["a"]), t) == H(v["a_out"])
        assert oracle.f2("sub", 1, H(v["a"]), t) == H(v["b_out"])
    for v in FR["ops"]["frPow"]:
        e = int(v["exp"])
        assert e < 2**256
        r = np.zeros(4, np.uint64)
        import ctypes
        u64p = ctypes.POINTER(ctypes.c_uint64)
        oracle.lib.orc_f_pow(1, r.ctypes.data_as(u64p), limbs(H(v["base"])).ctypes.data_as(u64p),
                             limbs(e).ctypes.data_as(u64p))
        assert to_int(r) == H(v["r"])


@pytest.mark.parametrize("case", range(len(NTT)))
def test_ntt_vectors(oracle, case):
    v = NTT[case]
    n = 1 << v["log_n"]
    inp = [mont(H(x), R) for x in v["input"]]
    exp = [mont(H(x), R) for x in v["expected"]]
    assert len(inp) == n
    # the reference checks INTT(expected) == input in Montgomery form
    assert ints(oracle.ntt(arr(exp), v["log_n"], True)) == inp
    # and the forward transform is the natural-order DFT
    assert ints(oracle.ntt(arr(inp), v["log_n"], False)) == exp


@pytest.mark.parametrize("case", range(len(MSM1)))
def test_msm_g1_vectors(oracle, case):
    v = MSM1[case]
    r, inf = oracle.msm_g1(arr([H(x) for x in v["px"]]), arr([H(x) for x in v["py"]]),
                           arr([H(x) for x in v["scalars"]]))
    assert not inf
    assert to_int(r[:4]) == H(v["out"][0]) and to_int(r[4:]) == H(v["out"][1]), v["label"]


@pytest.mark.parametrize("case", range(len(MSM2)))
def test_msm_g2_vectors(oracle, case):
    v = MSM2[case]
    px = np.concatenate([arr([H(a), H(b)]).reshape(1, 8) for a, b in v["px"]])
    py = np.concatenate([arr([H(a), H(b)]).reshape(1, 8) for a, b in v["py"]])
    r, inf = oracle.msm_g2(px, py, arr([H(x) for x in v["scalars"]]))
    if v["infinity"]:
        assert inf == 1
    else:
        assert inf == 0
        assert [to_int(r[4 * i:4 * i + 4]) for i in range(4)] == [H(x) for x in v["out"]], v["label"]


def test_pairing_bilinear(oracle):
    g1, g2 = oracle.g1_gen(), oracle.g2_gen()
    e = oracle.pairing(g1, g2)
    one = np.zeros(48, np.uint64)
    one[:4] = limbs(mont(1, P))
    assert not np.array_equal(e, one)
    a, b = 0x1234567, 0x7654321
    lhs = oracle.pairing(oracle.g1_mul(g1, a), oracle.g2_mul(g2, b))
    # e(aP, bQ) == e(P, Q)^(ab): compare against repeated pairing products
    rhs = oracle.pairing(oracle.g1_mul(g1, a * b % R), g2)
    assert np.array_equal(lhs, rhs)
    rhs2 = oracle.pairing(g1, oracle.g2_mul(g2, a * b % R))
    assert np.array_equal(lhs, rhs2)
