"""Autotuner: tuned settings are recorded per (group, size, distribution),
survive export / import, and never change a result (MSMs and whole proofs
stay equal to the oracle's)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from zyklop_b200 import api as A
    return A


@pytest.fixture
def ctx(api):
    from zyklop_b200._lib import check, lib
    h = ctypes.c_void_p()
    check(lib().zk_ctx_create(0, ctypes.byref(h)))
    yield h
    check(lib().zk_ctx_destroy(h))


def rand_scalars(rng, n, skewed):
    s = rng.integers(0, 2**63, size=(n, 4), dtype=np.uint64)
    s[:, 3] &= np.uint64((1 << 60) - 1)
    if skewed:
        k = rng.random(n)
        s[k < 0.55] = 0
        s[k < 0.55, 0] = rng.integers(0, 2, size=int((k < 0.55).sum()), dtype=np.uint64)
        mid = (k >= 0.55) & (k < 0.7)
        s[mid, 1:] = 0
    return s


@pytest.mark.parametrize("group,dist", [(1, 0), (1, 1), (2, 0)])
def test_autotune_msm_keeps_results(api, oracle, ctx, group, dist):
    lg = 12
    n = 1 << lg
    rng = np.random.default_rng(40 + group + 2 * dist)
    px, py = api.mul_generator(group, rand_scalars(rng, n, False), ctx=ctx)
    sc = rand_scalars(rng, n, dist == 1)
    msm = api.msm_g1 if group == 1 else api.msm_g2
    before = msm(px, py, sc, ctx=ctx)
    r = api.autotune_msm(group, lg, dist, ctx=ctx)
    assert max(4, lg - 6) <= r["c"] <= lg - 1 and r["ms"] > 0
    api.set_scalar_dist(dist, ctx=ctx)
    after = msm(px, py, sc, ctx=ctx)
    assert np.array_equal(before[0], after[0]) and before[1] == after[1]
    want, _ = (oracle.msm_g1 if group == 1 else oracle.msm_g2)(px, py, sc)
    assert np.array_equal(after[0], want)
    text = api.tune_export(ctx=ctx)
    assert text.startswith(f"msm {group} {lg} {dist} 0 {r['c']} ")


def test_autotune_fixed_table_and_ntt(api, ctx):
    lg = 12
    t = api.autotune_table_c(1, lg, 0, max_table_bytes=64 << 20, ctx=ctx)
    assert 8 <= t["table_c"] <= lg + 2
    f = api.autotune_msm(1, lg, 0, fixed_c=t["table_c"], ctx=ctx)
    assert f["k0"] in (16, 32, 64, 128, 256) and f["chunk"] in (4, 8, 16, 32, 64)
    nt = api.autotune_ntt(lg, ctx=ctx)
    assert 4 <= nt["pass_bits"] <= 8
    text = api.tune_export(ctx=ctx)
    assert f"table 1 {lg} 0 {t['table_c']}" in text


def test_tune_import_roundtrip_and_rejects(api, ctx):
    from zyklop_b200 import ZkError
    text = "msm 1 20 1 0 15 128 16 32\ntable 2 20 0 18\nntt 20 7\n"
    api.tune_import(text, ctx=ctx)
    assert sorted(api.tune_export(ctx=ctx).splitlines()) == sorted(text.splitlines())
    for bad in ("msm 1 20 1 0 3 64 16 16", "msm 1 20 1 0 15 64 16 12", "ntt 20 9",
                "table 3 20 0 18", "bogus 1 2 3", "msm 1 20"):
        with pytest.raises(ZkError) as e:
            api.tune_import(bad, ctx=ctx)
        assert e.value.code == 1
    assert sorted(api.tune_export(ctx=ctx).splitlines()) == sorted(text.splitlines())


def test_tuned_proofs_equal_oracle(api, oracle, ctx, tmp_path):
    """Tune every MSM size a 2^12 circuit uses (both distributions, windowed
    and fixed-base) and the NTT; proofs stay bit-identical to the oracle."""
    z, w = tmp_path / "t.zkey", tmp_path / "t.wtns"
    api.synth_circuit(z, w, 12, n_public=8, n_private_inputs=8, nnz=(1, 4), witness="circom",
                      seed=77)
    zb, wb = open(z, "rb").read(), open(w, "rb").read()
    want = oracle.prove(zb, wb)
    wit = api.read_wtns(w)
    for dist in (0, 1):
        api.autotune_msm(1, 12, dist, ctx=ctx)
        api.autotune_msm(2, 12, dist, ctx=ctx)
    api.autotune_ntt(12, ctx=ctx)
    c = api.Circuit(z, ctx=ctx)
    assert np.array_equal(c.prove(wit), want)
    t1 = api.autotune_table_c(1, 12, 1, ctx=ctx)["table_c"]
    api.autotune_table_c(2, 12, 1, ctx=ctx)
    c.precompute(0, 0)
    for dist in (0, 1):
        api.autotune_msm(1, 12, dist, fixed_c=t1, ctx=ctx)
    assert np.array_equal(c.prove(wit), want)
    c.set_scalar_dist(0)  # forcing the other distribution's settings changes nothing
    assert np.array_equal(c.prove(wit), want)
    c.close()
