"""End-to-end Groth16 parity on seeded synthetic circuits.

Checks, on the same zkey / wtns files:
  * the synthetic CRS is sound: the oracle's proofs pass the pairing check;
  * the library's unblinded proof is bit-identical to the oracle's, and so
    are the pipeline intermediates (A.w, B.w, h);
  * blinded proofs equal the oracle's blinded proofs and verify;
  * the library's proof equals the reference's own sm_100a build
    (groth16Prove, src/groth16.cu:1143) and the CLI writes byte-identical
    proof.json / public.json (src/main.cu);
  * malformed inputs come back as status codes.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import _ref
from _oracle import R

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CIRCUITS = {
    # name: (log_domain, witness kind, nnz range, seed)
    "u10": (10, "uniform", (2, 2), 11),
    "c10": (10, "circom", (1, 4), 12),
    "u16": (16, "uniform", (2, 2), 13),
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
    d = tmp_path_factory.mktemp("circuits")
    out = {}
    for name, (lg, kind, nnz, seed) in CIRCUITS.items():
        z, w = d / f"{name}.zkey", d / f"{name}.wtns"
        api.synth_circuit(z, w, lg, n_public=8, n_private_inputs=8, nnz=nnz, witness=kind, seed=seed)
        out[name] = (str(z), str(w))
    return out


def blob(path):
    with open(path, "rb") as f:
        return f.read()


def publics(api, wtns, l):
    w = api.read_wtns(wtns)
    return [int.from_bytes(w[i].tobytes(), "little") for i in range(1, l + 1)]


@pytest.mark.parametrize("name", ["u10", "c10"])
def test_synthetic_crs_is_sound(api, oracle, files, name):
    z, w = files[name]
    zb, wb = blob(z), blob(w)
    pub = publics(api, w, 8)
    proof = oracle.prove(zb, wb)
    assert oracle.verify(zb, proof, pub) == 1
    blinded = oracle.prove(zb, wb, r=12345, s=67890)
    assert oracle.verify(zb, blinded, pub) == 1
    bad = proof.copy()
    bad[24:32] = blinded[24:32]  # mismatched C
    assert oracle.verify(zb, bad, pub) == 0
    assert oracle.verify(zb, proof, [pub[0] + 1] + pub[1:]) == 0


@pytest.mark.parametrize("name", ["u10", "c10", "u16"])
def test_prove_matches_oracle(api, oracle, files, name):
    z, w = files[name]
    c = api.Circuit(z)
    mine = c.prove(api.read_wtns(w))
    assert np.array_equal(mine, oracle.prove(blob(z), blob(w)))


@pytest.mark.parametrize("name", ["u10", "c10", "u16"])
def test_precomputed_circuit_gives_identical_proofs(api, oracle, files, name):
    """Fixed-base tables change how the MSMs run, not what they compute."""
    z, w = files[name]
    c = api.Circuit(z)
    wit = api.read_wtns(w)
    plain = c.prove(wit)
    c.precompute()
    assert np.array_equal(c.prove(wit), plain)
    r, s = 0x1234567890ABCDEF, 0xFEDCBA0987654321
    blinded = c.prove(wit, r=r, s=s)
    assert np.array_equal(blinded, oracle.prove(blob(z), blob(w), r=r, s=s))
    c2 = api.Circuit(z)
    c2.precompute(c_g1=11, c_g2=9)
    assert np.array_equal(c2.prove(wit), plain)


@pytest.mark.parametrize("name", ["u10", "c10"])
def test_intermediates_match_oracle(api, oracle, files, name):
    z, w = files[name]
    c = api.Circuit(z)
    aw, bw, h, proof = c.intermediates(api.read_wtns(w))
    oaw, obw, oh = oracle.intermediates(blob(z), blob(w), c.domain)
    assert np.array_equal(aw, oaw)
    assert np.array_equal(bw, obw)
    assert np.array_equal(h, oh)


@pytest.mark.parametrize("name", ["u10", "c10"])
def test_blinded_matches_oracle_and_verifies(api, oracle, files, name):
    z, w = files[name]
    rng = np.random.default_rng(3)
    r = int.from_bytes(rng.bytes(32), "little") % R
    s = int.from_bytes(rng.bytes(32), "little") % R
    c = api.Circuit(z)
    mine = c.prove(api.read_wtns(w), r=r, s=s)
    assert np.array_equal(mine, oracle.prove(blob(z), blob(w), r=r, s=s))
    assert oracle.verify(blob(z), mine, publics(api, w, 8)) == 1
    # blinding changes the proof but not its validity
    assert not np.array_equal(mine, c.prove(api.read_wtns(w)))


def test_entry_points_agree(api, files):
    z, w = files["u10"]
    c = api.Circuit(z)
    wit = api.read_wtns(w)
    a = c.prove(wit)
    assert np.array_equal(a, api.prove_files(z, w))
    assert np.array_equal(a, api.prove_mem(blob(z), blob(w)))
    d = api.to_device(wit)
    assert np.array_equal(a, c.prove_device(d, wit.shape[0]))
    # repeated proofs on the resident circuit are identical
    assert np.array_equal(a, c.prove(wit))


@pytest.mark.parametrize("name", ["u10", "c10", "u16"])
def test_matches_reference_prover(api, files, name):
    L = _ref.prove_lib()
    if L is None:
        pytest.skip("reference sm_100a build (oracle/_ref) not present")
    z, w = files[name]
    theirs = np.zeros(32, np.uint64)
    assert L.zkref_prove_files(z.encode(), w.encode(),
                               theirs.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))) == 0
    assert np.array_equal(api.prove_files(z, w), theirs)
    buf = ctypes.create_string_buffer(4096)
    L.zkref_proof_json(theirs.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), buf, 4096)
    assert api.proof_to_json(theirs) == buf.value.decode()


def test_cli_matches_reference_cli(api, files, tmp_path):
    ref_cli = os.path.join(ROOT, "oracle", "_ref", "prover")
    my_cli = os.path.join(ROOT, "zyklop_b200", "bin", "prover")
    z, w = files["u10"]
    mine = subprocess.run([my_cli, z, w, str(tmp_path / "p1.json"), str(tmp_path / "q1.json")],
                          capture_output=True, text=True, timeout=300)
    assert mine.returncode == 0, mine.stderr
    assert blob(tmp_path / "p1.json").decode() == api.proof_to_json(api.prove_files(z, w)) + "\n"
    usage = subprocess.run([my_cli, z], capture_output=True, text=True, timeout=60)
    assert usage.returncode == 1 and "Usage" in usage.stderr
    if not os.path.exists(ref_cli):
        pytest.skip("reference CLI not built")
    ref = subprocess.run([ref_cli, z, w, str(tmp_path / "p2.json"), str(tmp_path / "q2.json")],
                         capture_output=True, text=True, timeout=300)
    assert ref.returncode == 0, ref.stderr
    assert blob(tmp_path / "p1.json") == blob(tmp_path / "p2.json")
    assert blob(tmp_path / "q1.json") == blob(tmp_path / "q2.json")


def test_cli_blinded_proof_verifies(api, oracle, files, tmp_path):
    my_cli = os.path.join(ROOT, "zyklop_b200", "bin", "prover")
    z, w = files["c10"]
    out = subprocess.run([my_cli, z, w, str(tmp_path / "p.json"), str(tmp_path / "q.json"),
                          "--blind", "7", "--repeat", "3"], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr
    import json
    pj = json.loads(blob(tmp_path / "p.json"))
    from _oracle import P, limbs, mont
    def m(x):
        return limbs(mont(int(x), P))
    proof = np.concatenate([m(pj["pi_a"][0]), m(pj["pi_a"][1]), m(pj["pi_b"][0][0]),
                            m(pj["pi_b"][0][1]), m(pj["pi_b"][1][0]), m(pj["pi_b"][1][1]),
                            m(pj["pi_c"][0]), m(pj["pi_c"][1])])
    pub = [int(x) for x in json.loads(blob(tmp_path / "q.json"))]
    assert pub == publics(api, w, 8)
    assert oracle.verify(blob(z), proof, pub) == 1


def test_calldata_layout(api, files):
    z, w = files["u10"]
    proof = api.prove_files(z, w)
    cd = api.proof_to_calldata(proof)
    from _oracle import P, to_int, unmont
    def be(i):
        return int.from_bytes(cd[32 * i:32 * i + 32], "big")
    assert be(0) == unmont(to_int(proof[0:4]), P) and be(1) == unmont(to_int(proof[4:8]), P)
    assert be(2) == unmont(to_int(proof[12:16]), P) and be(3) == unmont(to_int(proof[8:12]), P)
    assert be(6) == unmont(to_int(proof[24:28]), P)


def test_header_and_public_json(api, files):
    z, w = files["u10"]
    h = api.read_zkey_header(z)
    assert (h.domain_size, h.log_domain, h.n_public) == (1024, 10, 8)
    text = api.public_json(w, 8)
    assert text.startswith("[\n") and text.count(",") == 7


def test_malformed_inputs_are_status_codes(api, files, tmp_path):
    from zyklop_b200 import ZkError
    z, w = files["u10"]
    data = blob(z)
    (tmp_path / "trunc.zkey").write_bytes(data[: len(data) // 2])
    with pytest.raises(ZkError) as e:
        api.prove_files(tmp_path / "trunc.zkey", w)
    assert e.value.code == 5  # ZK_EFORMAT
    (tmp_path / "magic.zkey").write_bytes(b"zkez" + data[4:])
    with pytest.raises(ZkError) as e:
        api.prove_files(tmp_path / "magic.zkey", w)
    assert e.value.code == 5
    with pytest.raises(ZkError) as e:
        api.prove_files(tmp_path / "missing.zkey", w)
    assert e.value.code == 4  # ZK_EIO
    c = api.Circuit(z)
    with pytest.raises(ZkError) as e:
        c.prove(api.read_wtns(w)[:10])
    assert e.value.code == 6  # ZK_EWITNESS
    # a section-4 entry naming a signal beyond nVars: rejected by the
    # resident load and by the one-shot call (which checks it after proving)
    bad = bytearray(data)
    off = section_offset(data, 4)
    bad[off + 4 + 8:off + 4 + 12] = (0xFFFFFFF0).to_bytes(4, "little")  # entry 0, signal
    (tmp_path / "sig.zkey").write_bytes(bytes(bad))
    with pytest.raises(ZkError) as e:
        api.Circuit(tmp_path / "sig.zkey")
    assert e.value.code == 5
    with pytest.raises(ZkError) as e:
        api.prove_files(tmp_path / "sig.zkey", w)
    assert e.value.code == 5
    # a witness with fewer values than the circuit's nVars, one-shot
    wb = bytearray(blob(w))
    o1 = section_offset(bytes(wb), 1)
    wb[o1 + 36:o1 + 40] = (10).to_bytes(4, "little")
    (tmp_path / "short.wtns").write_bytes(bytes(wb))
    with pytest.raises(ZkError) as e:
        api.prove_files(z, tmp_path / "short.wtns")
    assert e.value.code == 6
    # the context stays usable after the failures
    assert np.array_equal(c.prove(api.read_wtns(w)), api.prove_files(z, w))


def section_offset(data, kind):
    """Byte offset of the first section of `kind` in a snarkjs BinFile."""
    pos = 12
    for _ in range(int.from_bytes(data[8:12], "little")):
        t = int.from_bytes(data[pos:pos + 4], "little")
        size = int.from_bytes(data[pos + 4:pos + 12], "little")
        if t == kind:
            return pos + 12
        pos += 12 + size
    raise KeyError(kind)


@pytest.mark.parametrize("graphs", [False, True])
@pytest.mark.parametrize("inflight", [1, 3])
def test_batch_matches_single_proofs(api, oracle, files, graphs, inflight):
    """A batch over mixed circuits gives, job for job, the proofs zk_prove gives."""
    names = ["u10", "c10", "u16", "u10", "c10", "u16", "c10"]
    circ = {nm: api.Circuit(files[nm][0]) for nm in set(names)}
    wits = {nm: api.read_wtns(files[nm][1]) for nm in set(names)}
    single = {nm: circ[nm].prove(wits[nm]) for nm in circ}
    try:
        api.set_graphs(graphs)
        proofs = api.prove_batch([circ[nm] for nm in names], [wits[nm] for nm in names],
                                 inflight=inflight)
        for k, nm in enumerate(names):
            assert np.array_equal(proofs[k], single[nm]), (k, nm)
        # blinded batch equals the oracle's blinded proofs
        rs = [11 + k for k in range(3)]
        ss = [101 + k for k in range(3)]
        sub = names[:3]
        bp = api.prove_batch([circ[nm] for nm in sub], [wits[nm] for nm in sub],
                             inflight=inflight, rs=rs, ss=ss)
        for k, nm in enumerate(sub):
            z, w = files[nm]
            assert np.array_equal(bp[k], oracle.prove(blob(z), blob(w), r=rs[k], s=ss[k]))
        # a second replay of the captured graphs gives the same proofs
        again = api.prove_batch([circ[nm] for nm in names], [wits[nm] for nm in names],
                                inflight=inflight)
        assert np.array_equal(again, proofs)
    finally:
        api.set_graphs(False)


def test_batch_rejects_short_witness_and_recovers(api, files):
    from zyklop_b200 import ZkError
    z, w = files["u10"]
    c = api.Circuit(z)
    wit = api.read_wtns(w)
    with pytest.raises(ZkError) as e:
        api.prove_batch([c, c], [wit, wit[:5]])
    assert e.value.code == 6
    assert np.array_equal(api.prove_batch([c], [wit])[0], c.prove(wit))


@pytest.mark.parametrize("graphs", [False, True])
def test_server_results_same_alone_and_in_mix(api, oracle, files, graphs):
    """Proofs from the continuous-batching server equal the proofs each job
    gives alone, whatever else is in flight beside it."""
    import threading
    names = ["u16", "u10", "c10", "u10", "u16", "c10", "u10", "u16"]
    circ = {nm: api.Circuit(files[nm][0]) for nm in set(names)}
    wits = {nm: api.read_wtns(files[nm][1]) for nm in set(names)}
    alone = {nm: circ[nm].prove(wits[nm]) for nm in circ}
    blind = {2: (7, 9), 5: (123456789, 987654321)}
    try:
        api.set_graphs(graphs)
        with api.Server(max_inflight=3) as srv:
            tickets = []
            for k, nm in enumerate(names):
                r, s = blind.get(k, (None, None))
                tickets.append(srv.submit(circ[nm], wits[nm], r=r, s=s))
            # more requests from other host threads while those run
            extra = {}

            def client(tid):
                extra[tid] = [srv.submit(circ[nm], wits[nm]) for nm in ("u10", "u16")]

            th = [threading.Thread(target=client, args=(t,)) for t in range(3)]
            for t in th:
                t.start()
            for t in th:
                t.join()
            for k, nm in enumerate(names):
                proof, lat = srv.wait(tickets[k])
                assert lat > 0
                if k in blind:
                    z, w = files[nm]
                    r, s = blind[k]
                    assert np.array_equal(proof, oracle.prove(blob(z), blob(w), r=r, s=s)), k
                else:
                    assert np.array_equal(proof, alone[nm]), (k, nm)
            for tid, ts in extra.items():
                for t, nm in zip(ts, ("u10", "u16")):
                    assert np.array_equal(srv.wait(t)[0], alone[nm]), (tid, nm)
            st = srv.stats()
            assert st["completed"] == len(names) + 6 and st["failed"] == 0
            assert 1 <= st["peak_inflight"] <= 3
    finally:
        api.set_graphs(False)


def test_server_admission_by_free_memory(api, files):
    """With a reserve larger than the device, a request is admitted only when
    nothing else runs: one proof in flight at a time, all of them correct."""
    z, w = files["u16"]
    c = api.Circuit(z)
    wit = api.read_wtns(w)
    ref = c.prove(wit)
    with api.Server(max_inflight=4, reserve_bytes=1 << 50) as srv:
        ts = [srv.submit(c, wit) for _ in range(4)]
        for t in ts:
            assert np.array_equal(srv.wait(t)[0], ref)
        st = srv.stats()
    assert st["peak_inflight"] == 1 and st["completed"] == 4


def test_server_errors(api, files):
    from zyklop_b200 import ZkError
    z, w = files["u10"]
    c = api.Circuit(z)
    wit = api.read_wtns(w)
    with api.Server(max_inflight=2) as srv:
        bad = srv.submit(c, wit[:5])
        good = srv.submit(c, wit)
        with pytest.raises(ZkError) as e:
            srv.wait(bad)
        assert e.value.code == 6
        assert np.array_equal(srv.wait(good)[0], c.prove(wit))
        with pytest.raises(ZkError) as e:
            srv.wait(good)  # released
        assert e.value.code == 1
        assert srv.stats()["failed"] == 1


def test_server_cancel_queued(api, files):
    """Requests still queued are dropped with ZK_ECANCELED; the rest finish
    with the right proof."""
    from zyklop_b200 import ZkError
    z, w = files["u16"]
    c = api.Circuit(z)
    wit = api.read_wtns(w)
    ref = c.prove(wit)
    with api.Server(max_inflight=1) as srv:
        ts = [srv.submit(c, wit) for _ in range(12)]
        n = srv.cancel_queued()
        ok = cancelled = 0
        for t in ts:
            try:
                assert np.array_equal(srv.wait(t)[0], ref)
                ok += 1
            except ZkError as e:
                assert e.code == 10
                cancelled += 1
        assert cancelled == n and ok + cancelled == 12


def test_twiddle_growth_in_fresh_contexts(api, oracle, files):
    """Loading a small circuit and then a larger one grows the context's
    twiddle tables; proofs of both must stay exact in every fresh context."""
    from zyklop_b200._lib import check, lib
    L = lib()
    want = {nm: oracle.prove(blob(files[nm][0]), blob(files[nm][1])) for nm in ("c10", "u16")}
    for _ in range(4):
        ctx = ctypes.c_void_p()
        check(L.zk_ctx_create(0, ctypes.byref(ctx)))
        try:
            circ = {nm: api.Circuit(files[nm][0], ctx=ctx) for nm in ("c10", "u16")}
            for nm, c in circ.items():
                assert np.array_equal(c.prove(api.read_wtns(files[nm][1])), want[nm]), nm
                c.close()
        finally:
            check(L.zk_ctx_destroy(ctx))


def test_server_admits_small_circuits_first(api, files):
    """Policy 1 admits the smallest queued circuit next (aging aside), so a
    small proof queued behind large ones finishes before them; policy 0
    keeps arrival order.  Results are unchanged either way."""
    import time
    big, small = api.Circuit(files["u16"][0]), api.Circuit(files["u10"][0])
    wb, ws = api.read_wtns(files["u16"][1]), api.read_wtns(files["u10"][1])
    ref_b, ref_s = big.prove(wb), small.prove(ws)
    for policy in (1, 0):
        with api.Server(max_inflight=1) as srv:
            srv.set_policy(policy, max_wait_ms=60000)
            jobs = [(big, wb, ref_b)] * 4 + [(small, ws, ref_s)]
            sub = []
            for c, w, ref in jobs:
                sub.append((time.perf_counter(), srv.submit(c, w), ref))
            done = []
            for t0, tk, ref in sub:
                p, lat = srv.wait(tk)
                assert np.array_equal(p, ref)
                done.append(t0 + lat / 1e3)
        if policy == 1:
            assert done[4] < done[3]
        else:
            assert done[4] > done[3]


@pytest.mark.parametrize("group", [3, 16])
def test_fused_batch_matches_single_proofs(api, oracle, files, group):
    """Fused groups (multi-instance MSM chains over several proofs) give,
    job for job, the single-proof results: mixed circuits and table sizes,
    several groups with alternating workspaces, blinded and unblinded."""
    names = ["u10", "c10", "u16", "u10", "c10", "c10", "u16", "u10", "c10", "u10", "c10", "u16",
             "u10"]
    circ = {}
    for nm in ("u10", "c10", "u16"):
        circ[nm] = api.Circuit(files[nm][0])
    circ["u10"].precompute(10, 9)   # u10 and c10 share table bits (one group key) ...
    circ["c10"].precompute(10, 9)
    circ["u16"].precompute(12, 11)  # ... u16 forms its own
    wits = {nm: api.read_wtns(files[nm][1]) for nm in circ}
    single = {nm: circ[nm].prove(wits[nm]) for nm in circ}
    try:
        api.set_batch_mode(api.BATCH_FUSED, group)
        proofs = api.prove_batch([circ[nm] for nm in names], [wits[nm] for nm in names])
        for k, nm in enumerate(names):
            assert np.array_equal(proofs[k], single[nm]), (k, nm)
        rs = [5 + 3 * k for k in range(5)]
        ss = [7 + 11 * k for k in range(5)]
        sub = names[:5]
        bp = api.prove_batch([circ[nm] for nm in sub], [wits[nm] for nm in sub], rs=rs, ss=ss)
        for k, nm in enumerate(sub):
            z, w = files[nm]
            assert np.array_equal(bp[k], oracle.prove(blob(z), blob(w), r=rs[k], s=ss[k])), (k, nm)
        # device witnesses
        dw = [api.to_device(wits[nm]) for nm in names[:4]]
        from zyklop_b200._lib import check, lib
        handles = (ctypes.c_void_p * 4)(*[circ[nm].handle.value for nm in names[:4]])
        wp = (ctypes.c_void_p * 4)(*[t.data_ptr() for t in dw])
        nw = (ctypes.c_size_t * 4)(*[t.numel() // 4 for t in dw])
        out = np.zeros((4, 32), np.uint64)
        check(lib().zk_prove_batch(None, 4, handles, wp, nw, 1, None, None,
                                   out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), 1))
        for k, nm in enumerate(names[:4]):
            assert np.array_equal(out[k], single[nm]), (k, nm)
    finally:
        api.set_batch_mode(api.BATCH_AUTO, 16)
    for c in circ.values():
        c.close()


def test_fused_batch_needs_tables(api, files):
    from zyklop_b200 import ZkError
    c = api.Circuit(files["u10"][0])
    wit = api.read_wtns(files["u10"][1])
    try:
        api.set_batch_mode(api.BATCH_FUSED, 8)
        with pytest.raises(ZkError) as e:
            api.prove_batch([c], [wit])
        assert e.value.code == 1
    finally:
        api.set_batch_mode(api.BATCH_AUTO, 16)
    assert np.array_equal(api.prove_batch([c], [wit])[0], c.prove(wit))


def test_fused_group_at_the_instance_limit(api, files):
    """32 unblinded jobs in one fused group: the A/C chain holds 64 instances,
    the multi-instance maximum; every proof equals the single proof."""
    c = api.Circuit(files["u10"][0])
    c.precompute(10, 9)
    wit = api.read_wtns(files["u10"][1])
    single = c.prove(wit)
    try:
        api.set_batch_mode(api.BATCH_FUSED, 64)
        proofs = api.prove_batch([c] * 32, [wit] * 32)
        assert all(np.array_equal(p, single) for p in proofs)
        # 33 jobs: a second group of one
        proofs = api.prove_batch([c] * 33, [wit] * 33)
        assert all(np.array_equal(p, single) for p in proofs)
    finally:
        api.set_batch_mode(api.BATCH_AUTO, 16)
    c.close()


@pytest.mark.parametrize("c_c,c_h", [(8, 8), (7, 8)])
def test_c_and_h_msms_share_a_reduction_only_with_equal_windows(api, oracle, files, c_c, c_h):
    """pi_C adds the C and H MSMs, so a proof lets C's buckets go into H's
    reduction when both run with the same window bits.  The C MSM takes the
    witness's (circom-like: skewed) tuned settings and H the uniform ones;
    importing different window bits for the two must turn the sharing off.
    Proofs stay exact either way, one-shot and resident (windowed)."""
    from zyklop_b200._lib import check, lib
    L = lib()
    z, w = files["c10"]
    want = oracle.prove(blob(z), blob(w))
    ctx = ctypes.c_void_p()
    check(L.zk_ctx_create(0, ctypes.byref(ctx)))
    try:
        api.tune_import(f"msm 1 10 1 0 {c_c} 16 16 4\nmsm 1 10 0 0 {c_h} 16 16 4\n", ctx=ctx)
        assert np.array_equal(api.prove_files(z, w, ctx=ctx), want)
        c = api.Circuit(z, ctx=ctx)
        wit = api.read_wtns(w)
        assert np.array_equal(c.prove(wit), want)
        assert np.array_equal(c.prove(wit), want)
        c.close()
    finally:
        check(L.zk_ctx_destroy(ctx))


def test_fused_groups_replay_captured_graphs(api, oracle, files):
    """With graphs on, each fused group's device pipeline is captured the
    first time and replayed when the same group comes again: every replay
    gives the single-proof results, also after another group composition
    was captured in between, and blinded groups stay exact."""
    circ = {nm: api.Circuit(files[nm][0]) for nm in ("u10", "c10", "u16")}
    circ["u10"].precompute(10, 9)
    circ["c10"].precompute(10, 9)
    circ["u16"].precompute(12, 11)
    wits = {nm: api.read_wtns(files[nm][1]) for nm in circ}
    single = {nm: circ[nm].prove(wits[nm]) for nm in circ}
    a = ["u10", "c10", "u16", "c10", "u10"]
    b = ["u16", "u16", "c10"]
    try:
        api.set_batch_mode(api.BATCH_FUSED, 16)
        api.set_graphs(True)
        for names in (a, a, b, a, b):
            proofs = api.prove_batch([circ[nm] for nm in names], [wits[nm] for nm in names])
            for k, nm in enumerate(names):
                assert np.array_equal(proofs[k], single[nm]), (names, k, nm)
        rs, ss = [3, 5, 7], [11, 13, 17]
        for _ in range(2):
            bp = api.prove_batch([circ[nm] for nm in b], [wits[nm] for nm in b], rs=rs, ss=ss)
            for k, nm in enumerate(b):
                z, w = files[nm]
                assert np.array_equal(bp[k], oracle.prove(blob(z), blob(w), r=rs[k], s=ss[k]))
    finally:
        api.set_graphs(False)
        api.set_batch_mode(api.BATCH_AUTO, 16)
    for c in circ.values():
        c.close()
