#!/usr/bin/env python
"""Groth16 (BN254) proving throughput on B200.

One step = one Groth16 proof of a seeded synthetic circuit with 2^20
constraints (config-0 circuit shape: 2 nonzeros per A/B row, 8 public
inputs, uniform witness), produced by libzyklop_b200.so.

  value  proofs/s with the circuit resident in HBM and the witness already on
         the device (zk_prove_device), CUDA events on the context stream,
         max over ranks;
  e2e    proofs/s through the reference-facing one-shot call
         zk_groth16_prove_files(zkey, wtns) -- the drop-in for the reference's
         groth16Prove -- which reads both files from the page cache and
         uploads the CRS, matrices and witness inside the timed region;
  roofline  the dominant kernel (MSM bucket accumulation) against the
         measured IMAD throughput of the device;
  cpu_baseline  the CPU oracle (C + OpenMP, every host thread) proving the
         same circuit once.

--impl reference runs the reference's own sm_100a build (oracle/_ref,
compiled from the reference sources) through its groth16Prove on the same
files, and the same primitive sweep through its msm_g1 / msm_g2_device / ntt /
computeHPoly; it writes its proofs and primitive results to the work
directory, and this arm checks its own against them bit for bit
(parity_vs_reference).  All inputs are written by zyklop_b200/bin/zk_synth in
a child process, so the reference process never loads this library.  With
torchrun, every rank proves independently (replicas; the prover is
single-GPU by design).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--log-domain L]
"""
import argparse
import contextlib
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "groth16_proofs_per_s"
UNIT = "proofs/s"
# algorithmic Fp multiplications per MSM point (bucket accumulation with the
# reference's 16-window, 7M+4S mixed-add decomposition) and IMAD-class ops per
# Fp multiplication (8x8 limb products lo+hi for a*b and m*p, plus m).  Both
# are work conventions: the kernels issue 232 IMAD-class ops per Fp product
# (Karatsuba) and 560 per Fp2 product (two reductions), so a fraction of the
# carry-chain probe counted this way can exceed the issued one.
FP_MULTS_PER_POINT = {"accum_g1": 176.0, "accum_g2": 528.0}
IMAD_PER_FP_MULT = 264.0
# what the fixed-base accumulation issues per sorted record (one mixed XYZZ
# add): G1 6 products x 232 + 2 squares x (72 + 136) + one shared-reduction
# difference of products (2 x 96 + 136); G2 8 Fp2 products x 560 + 2 Fp2
# squares x 2 x 232
ISSUED_IMAD_PER_RECORD = {"accum_g1": 6 * 232 + 2 * (72 + 136) + 2 * 96 + 136,
                          "accum_g2": 8 * 560 + 2 * 2 * 232}


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["mine", "reference"], default="mine")
    p.add_argument("--log-domain", type=int, default=20)
    p.add_argument("--witness", choices=["uniform", "circom"], default="uniform")
    p.add_argument("--e2e-steps", type=int, default=0, help="default: min(steps, 5)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--table-c", default="0,0", help="fixed-base window bits G1,G2 (0 = default)")
    p.add_argument("--workdir", default=os.environ.get("ZK_BENCH_DIR", "/tmp/zyklop_bench"))
    p.add_argument("--batch-proofs", type=int, default=64, help="0 skips the batched section")
    p.add_argument("--batch-inflight", type=int, default=8)
    p.add_argument("--batch-group", type=int, default=16)
    p.add_argument("--no-autotune", action="store_true",
                   help="skip the autotuner (default settings for every size)")
    p.add_argument("--serve-seconds", type=float, default=60.0, help="0 skips serving")
    p.add_argument("--serve-seconds-fair", type=float, default=20.0)
    p.add_argument("--serve-rate", type=float, default=200.0)
    p.add_argument("--serve-logs", default="16,19,21,23")
    p.add_argument("--serve-inflight", type=int, default=3,
                   help="proofs the server keeps on the GPU (3: best p99 measured; 2 lowers p50)")
    p.add_argument("--prim-g1", default="18,20,22,24", help="G1 MSM sizes (log2); empty skips")
    p.add_argument("--prim-g2", default="18,20")
    p.add_argument("--prim-ntt", default="16,18,20,22,24")
    p.add_argument("--prim-hpoly", default="16,20,22", help="H pipeline (coset INTT/NTT) sizes")
    p.add_argument("--config2-log", type=int, default=22,
                   help="single proof, circom-like witness, 1-4 nonzeros per row; 0 skips")
    p.add_argument("--config2-steps", type=int, default=10)
    p.add_argument("--parity-only", action="store_true",
                   help="(--impl reference) write the reference outputs without timing")
    p.add_argument("--no-parity", action="store_true",
                   help="skip the comparison with the reference build's outputs")
    return p.parse_args()


# ------------------------------------------------------------ distributed
class Dist:
    """One process per GPU (torchrun env).  NCCL on GPUs; gloo when CUDA is
    absent (the host-side logic runs and is tested on CPU that way)."""

    def __init__(self, backend=None):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.cuda = False
        if self.world > 1:
            import datetime
            import torch
            import torch.distributed as dist
            self.cuda = torch.cuda.is_available()
            backend = backend or ("nccl" if self.cuda else "gloo")
            self.cuda = backend == "nccl"
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
            self.pg = dist

    def barrier(self):
        if self.pg:
            import torch
            if self.cuda:
                self.pg.barrier(device_ids=[self.local])
                torch.cuda.synchronize()
            else:
                self.pg.barrier()

    def max(self, x):
        if not self.pg:
            return x
        import torch
        t = torch.tensor([float(x)], device="cuda" if self.cuda else "cpu")
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(device)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.3)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=10)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, mx, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
                power.append(float(f[3]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "power_w_max": max(power) if power else None, "samples": len(sm),
                "reasons": sorted(reasons)}


@contextlib.contextmanager
def silenced():
    """Silence fd 1 / 2 (the reference prover prints progress on both)."""
    sys.stdout.flush()
    sys.stderr.flush()
    saved = os.dup(1), os.dup(2)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    os.dup2(devnull, 2)
    try:
        yield
    finally:
        os.dup2(saved[0], 1)
        os.dup2(saved[1], 2)
        os.close(devnull)
        os.close(saved[0])
        os.close(saved[1])


# ------------------------------------------------------------- workload
SYNTH = os.path.join(ROOT, "zyklop_b200", "bin", "zk_synth")


def run_synth(*argv):
    """zk_synth in a child process (this process never loads the library for
    input generation, so the reference arm maps only the reference build)."""
    r = subprocess.run([SYNTH, *[str(a) for a in argv]], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"zk_synth {' '.join(map(str, argv))} failed: {r.stderr.strip()}")


def synth_cached(args, dist, lg, witness, seed):
    """Seeded synthetic circuit + witness files, generated once per workdir.
    uniform: 2 nonzeros per A/B row; circom: 1-4 nonzeros per row and the
    circom-like witness mix (55% bits, 15% below 2^64, 30% uniform)."""
    tag = f"l{lg}_{witness}_s{seed}"
    d = os.path.join(args.workdir, tag)
    z, w = os.path.join(d, "circuit.zkey"), os.path.join(d, "witness.wtns")
    done = os.path.join(d, "ok")
    if dist.rank == 0 and not os.path.exists(done):
        os.makedirs(d, exist_ok=True)
        run_synth("circuit", z, w, lg, witness, seed)
        open(done, "w").write("ok\n")
    dist.barrier()
    return z, w


def circuit_files(args, dist):
    return synth_cached(args, dist, args.log_domain, args.witness, 1)


def zkey_bytes(z, sections):
    data = open(z, "rb").read(12)
    total = 0
    with open(z, "rb") as f:
        f.seek(8)
        ns = int.from_bytes(f.read(4), "little")
        for _ in range(ns):
            t = int.from_bytes(f.read(4), "little")
            s = int.from_bytes(f.read(8), "little")
            if t in sections:
                total += s
            f.seek(s, 1)
    return total


def config(args, n_vars, domain):
    return {"workload": f"groth16_prove_2^{args.log_domain}",
            "constraints": domain - 9, "domain": domain, "n_vars": n_vars, "n_public": 8,
            "circuit": "seeded synthetic R1CS, 2 nnz per A/B row (config-0 shape)",
            "witness": args.witness, "proof": "unblinded (reference-compatible)",
            "l2": "inputs larger than L2: ~0.6 GB of CRS points and matrices read per proof",
            "parallelism": f"replicas{args.gpus}"}


def wtns_n_vars(w):
    with open(w, "rb") as f:
        return int.from_bytes(f.read(64)[60:64], "little")


def cpu_baseline(z, w):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import _oracle
    orc = _oracle.load()
    zb, wb = open(z, "rb").read(), open(w, "rb").read()
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    orc.prove(zb, wb, threads=threads)
    t = time.perf_counter() - t0
    return {"value": 1.0 / t, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": "one full proof of the same circuit by the CPU oracle (C, OpenMP; "
                      f"{t:.1f} s)"}


# ------------------------------------------------------------------ mine
def traffic_per_point():
    """DRAM bytes per point of one accumulation launch (ncu summary)."""
    out = {}
    path = os.path.join(ROOT, "profiles", "traffic_per_point.txt")
    if os.path.exists(path):
        for line in open(path):
            f = line.split()
            if len(f) == 2 and not line.startswith("#"):
                out[f[0]] = float(f[1])
    return out


def roofline_of(kind, rec, peak, step_ms, records_per_point=None, peak_variants=None,
                headline="convention"):
    """IMAD-class ops of the accumulation kernels of `kind` over their
    measured event time, against the measured carry-chain IMAD peak.
    `convention` counts the fixed algorithmic work per point (the reference's
    16-window decomposition, 11 or 33 products per window, 264 ops per
    product); with the fixed-base window count known (records_per_point),
    `issued` counts what the kernel issues (records x ops per record), which
    is less.  headline picks which of the two `achieved` / `frac` repeat.
    `peak_variants` gives the headline rate against each measured or nominal
    integer-pipe rate."""
    kms, kl, ku = rec
    if not kl or kms <= 0:
        return None
    conv = ku * FP_MULTS_PER_POINT[kind] * IMAD_PER_FP_MULT / (kms / 1e3) / 1e12
    per_point = traffic_per_point().get(kind)
    r = {"bound": "imad", "kernel": f"k_msm_accum0 ({kind})", "achieved": conv,
         "peak": peak, "unit": "TIOP/s", "frac": conv / peak, "work": "convention",
         "traffic": per_point * ku / kl if per_point else None,
         "peak_source": "zk_imad_probe (measured carry-chain IMAD throughput)",
         "avg_launch_ms": kms / kl, "launches": int(kl),
         "convention": {"achieved": conv, "frac": conv / peak,
                        "per_point": f"{FP_MULTS_PER_POINT[kind]:.0f} Fp products x "
                                     f"{IMAD_PER_FP_MULT:.0f} ops"}}
    if step_ms:
        r["share_of_step"] = kms / step_ms
    if records_per_point:
        ia = ku * records_per_point * ISSUED_IMAD_PER_RECORD[kind] / (kms / 1e3) / 1e12
        r["issued"] = {"records_per_point": records_per_point,
                       "imad_per_record": ISSUED_IMAD_PER_RECORD[kind],
                       "achieved": ia, "frac": ia / peak}
        if headline == "issued":
            r["achieved"], r["frac"], r["work"] = ia, ia / peak, "issued"
    if peak_variants:
        r["peak_variants"] = {k: {"peak": v, "frac": r["achieved"] / v}
                              for k, v in peak_variants.items() if v}
    return r


def int_peaks(L, ctx, sm_mhz):
    """The integer-pipe rates the roofline is read against (TIOP/s): the two
    measured probes and the nominal 64 IMAD / clock / SM at the sampled SM
    clock."""
    from zyklop_b200._lib import check
    out = {}
    for kind, name in ((0, "carry_chain_probe"), (1, "independent_mad_probe")):
        v = ctypes.c_double()
        check(L.zk_int_probe(ctx, kind, ctypes.byref(v)))
        out[name] = v.value
    import torch
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    if sm_mhz:
        out["nominal_64_per_clk_per_sm"] = 64.0 * sms * sm_mhz * 1e6 / 1e12
    return out


def table_windows(args, tuned, group):
    """Windows (records per point) of the fixed-base tables the resident
    proof uses: --table-c, else the tuned window bits, else the default."""
    from zyklop_b200.api import table_c_default
    c = int(args.table_c.split(",")[group - 1])
    if c <= 0 and isinstance(tuned, list):
        for t in tuned:
            f = t.split()
            if len(f) == 5 and f[0] == "table" and f[1] == str(group) and f[2] == str(args.log_domain):
                c = int(f[4])
    if c <= 0:
        c = table_c_default(args.log_domain)
    return 254 // c + 1


def run_mine(args, dist):
    import torch
    torch.cuda.set_device(dist.local)
    from zyklop_b200 import api
    from zyklop_b200._lib import Profile, check, lib
    L = lib()
    z, w = circuit_files(args, dist)
    ctx = ctypes.c_void_p()
    check(L.zk_ctx_create(dist.local, ctypes.byref(ctx)))
    stream = torch.cuda.current_stream()
    check(L.zk_ctx_set_stream(ctx, ctypes.c_void_p(stream.cuda_stream)))
    t_tune = time.perf_counter()
    tuned = autotune_sizes(args, api, ctx, [args.log_domain],
                           api.UNIFORM if args.witness == "uniform" else api.SKEWED)
    t_tune = time.perf_counter() - t_tune
    circuit = api.Circuit(z, ctx=ctx)
    circuit.prove(api.read_wtns(w))  # detects the witness distribution
    t_pre = time.perf_counter()
    tc = [int(x) for x in args.table_c.split(",")]
    circuit.precompute(tc[0], tc[1])  # fixed-base window tables for the resident CRS
    t_pre = time.perf_counter() - t_pre
    wit = api.read_wtns(w)
    dwit = api.to_device(wit)
    n = wit.shape[0]
    peak = ctypes.c_double()
    check(L.zk_imad_probe(ctx, ctypes.byref(peak)))
    proof = np.zeros(32, np.uint64)
    pp = proof.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))

    def step():
        check(L.zk_prove_device(circuit.handle, api.ptr(dwit), n, None, None, pp))

    for _ in range(args.warmup):
        step()
    reference_proof = proof.copy()
    torch.cuda.synchronize()
    check(L.zk_ctx_set_profiling(ctx, 1))
    prof = Profile()
    check(L.zk_ctx_profile(ctx, ctypes.byref(prof)))  # clear
    lc0 = ctypes.c_uint64()
    check(L.zk_launch_count(ctypes.byref(lc0)))
    clocks = ClockSampler(dist.local)
    dist.barrier()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(args.steps):
        step()
    end.record(stream)
    torch.cuda.synchronize()
    dist.barrier()
    clk = clocks.stop()
    ms = dist.max(start.elapsed_time(end))
    lc1 = ctypes.c_uint64()
    check(L.zk_launch_count(ctypes.byref(lc1)))
    check(L.zk_ctx_profile(ctx, ctypes.byref(prof)))
    check(L.zk_ctx_set_profiling(ctx, 0))
    assert np.array_equal(proof, reference_proof), "proofs changed between steps"
    value = args.gpus * args.steps / (ms / 1e3)

    # roofline of the dominant kernel kind, from the timed region (the five
    # MSM streams of a proof overlap, so each launch's event time includes
    # time shared with the other streams)
    kinds = {k: (prof.ms[i], prof.launches[i], prof.units[i]) for i, k in enumerate(Profile.KINDS)}
    dom = max(FP_MULTS_PER_POINT, key=lambda k: kinds[k][0])
    # issued work assumes every window of every point makes a record: true for
    # uniform scalars, not for circom-like witnesses (zero digits are skipped)
    wins = ({"accum_g1": table_windows(args, tuned, 1), "accum_g2": table_windows(args, tuned, 2)}
            if args.witness == "uniform" else {"accum_g1": None, "accum_g2": None})
    variants = int_peaks(L, ctx, clk.get("sm_mhz"))
    roofline = roofline_of(dom, kinds[dom], peak.value, ms, wins[dom], variants)
    other = {k: {"ms_per_step": v[0] / args.steps, "launches": int(v[1])} for k, v in kinds.items()}

    # the same kernels with a proof's MSMs back to back on one stream (an
    # extra, untimed pass): event times are then the kernels' own durations
    check(L.zk_ctx_set_prove_streams(ctx, 1))
    step()
    torch.cuda.synchronize()
    check(L.zk_ctx_set_profiling(ctx, 1))
    check(L.zk_ctx_profile(ctx, ctypes.byref(prof)))  # clear
    for _ in range(min(args.steps, 3)):
        step()
    torch.cuda.synchronize()
    check(L.zk_ctx_profile(ctx, ctypes.byref(prof)))
    check(L.zk_ctx_set_profiling(ctx, 0))
    check(L.zk_ctx_set_prove_streams(ctx, 0))
    assert np.array_equal(proof, reference_proof), "proofs changed with one MSM stream"
    skinds = {k: (prof.ms[i], prof.launches[i], prof.units[i]) for i, k in enumerate(Profile.KINDS)}
    # alone on one stream the fixed-base kernels issue less than the
    # convention counts (which would read above 1): issued is the headline
    roofline_serial = {k: roofline_of(k, skinds[k], peak.value, None, wins[k], variants,
                                      headline="issued" if wins[k] else "convention")
                       for k in FP_MULTS_PER_POINT}

    # e2e through the one-shot host-buffer entry point
    e2e_steps = args.e2e_steps or min(args.steps, 5)
    h2d = zkey_bytes(z, {4, 5, 6, 7, 8, 9}) + os.path.getsize(w)
    W1, W2 = 17, 17  # windows of the windowed MSMs at 2^20 (16-bit windows)
    d2h = 3 * 2 * 128 * W1 + 2 * 256 * W2  # (U, A) pairs per window: A, C, H and B2
    check(L.zk_groth16_prove_files(ctx, z.encode(), w.encode(), pp))  # warm the page cache
    assert np.array_equal(proof, reference_proof)
    dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        check(L.zk_groth16_prove_files(ctx, z.encode(), w.encode(), pp))
    e1.record(stream)
    torch.cuda.synchronize()
    ems = dist.max(e0.elapsed_time(e1))
    # resident circuit, host witness (the serving path)
    r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    r0.record(stream)
    for _ in range(e2e_steps):
        check(L.zk_prove(circuit.handle, wit.ctypes.data_as(ctypes.c_void_p), n, None, None, pp))
    r1.record(stream)
    torch.cuda.synchronize()
    rms = dist.max(r0.elapsed_time(r1))

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32 limbs (exact Fr/Fp arithmetic)",
        "data": "synthetic (seeded circuit, CRS and witness)",
        "config": config(args, circuit.n_vars, circuit.domain),
        "setup": {"resident_crs": "zkey uploaded once; fixed-base window tables built once "
                                  f"({t_pre:.2f} s, zk_circuit_precompute)",
                  "autotuned": tuned, "autotune_s": round(t_tune, 1)},
        "e2e": {"value": args.gpus * e2e_steps / (ems / 1e3), "unit": UNIT,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "call": "zk_groth16_prove_files (zkey + wtns files -> proof)"},
        "e2e_resident": {"value": args.gpus * e2e_steps / (rms / 1e3), "unit": UNIT,
                         "h2d_bytes_per_step": 32 * n,
                         "d2h_bytes_per_step": 3 * 2 * 128 + 2 * 256,  # one (U, A) per MSM
                         "call": "zk_prove (resident circuit, host witness)"},
        "roofline": roofline,
        "roofline_serial_msm": roofline_serial,
        "kernels": other,
        "clocks": clk,
        "gpu_launches": int(lc1.value - lc0.value),
    }
    circuit.close()
    line["_proof"] = reference_proof.tobytes().hex()
    return line, (z, w), ctx


def run_config2(args, dist, ctx, L):
    """Config 2: one proof of a 2^22-constraint circuit with 1-4 nonzeros per
    A/B row and a circom-like witness.  value: resident circuit with tuned
    fixed-base tables and a device witness (CUDA events on the context
    stream); e2e: the drop-in one-shot call on the files."""
    import torch
    from zyklop_b200 import api
    from zyklop_b200._lib import check
    lg = args.config2_log
    z, w = synth_cached(args, dist, lg, "circom", 2)
    t_tune = time.perf_counter()
    tuned = autotune_sizes(args, api, ctx, [lg], api.SKEWED)
    t_tune = time.perf_counter() - t_tune
    circuit = api.Circuit(z, ctx=ctx)
    wit = api.read_wtns(w)
    circuit.prove(wit)  # detects the witness distribution
    t_pre = time.perf_counter()
    circuit.precompute(0, 0)
    t_pre = time.perf_counter() - t_pre
    dwit = api.to_device(wit)
    n = wit.shape[0]
    proof = np.zeros(32, np.uint64)
    pp = proof.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
    stream = torch.cuda.current_stream()

    def step():
        check(L.zk_prove_device(circuit.handle, api.ptr(dwit), n, None, None, pp))

    for _ in range(2):
        step()
    first = proof.copy()
    clocks = ClockSampler(dist.local)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.config2_steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = dist.max(e0.elapsed_time(e1))
    assert np.array_equal(proof, first), "config-2 proofs changed between steps"
    circuit.close()
    e_steps = 3
    check(L.zk_groth16_prove_files(ctx, z.encode(), w.encode(), pp))  # warm the page cache
    assert np.array_equal(proof, first)
    e0.record(stream)
    for _ in range(e_steps):
        check(L.zk_groth16_prove_files(ctx, z.encode(), w.encode(), pp))
    e1.record(stream)
    torch.cuda.synchronize()
    ems = dist.max(e0.elapsed_time(e1))
    assert np.array_equal(proof, first), "one-shot config-2 proof differs from the resident one"
    return {
        "workload": f"groth16_prove_2^{lg}_circom",
        "config": {"constraints": (1 << lg) - 9, "domain": 1 << lg, "n_vars": wtns_n_vars(w),
                   "n_public": 8, "circuit": "seeded synthetic R1CS, 1-4 nnz per A/B row",
                   "witness": "circom-like (55% in {0,1}, 15% below 2^64, 30% uniform)",
                   "proof": "unblinded (reference-compatible)"},
        "value": args.gpus * args.config2_steps / (ms / 1e3), "unit": UNIT,
        "steps": args.config2_steps, "ms_per_step": ms / args.config2_steps,
        "e2e": {"value": args.gpus * e_steps / (ems / 1e3), "unit": UNIT, "steps": e_steps,
                "h2d_bytes_per_step": zkey_bytes(z, {4, 5, 7, 8, 9}) + os.path.getsize(w),
                "d2h_bytes_per_step": 3 * 2 * 128 * 17 + 2 * 256 * 17,
                "call": "zk_groth16_prove_files (zkey + wtns files -> proof)"},
        "setup": {"autotuned": tuned, "autotune_s": round(t_tune, 1),
                  "tables_s": round(t_pre, 2)},
        "clocks": clk,
        "_proof": first.tobytes().hex(),
    }


# -------------------------------------------------------------- primitives
def hbm_peak():
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def prim_inputs(args, group, log_max, seed):
    """Points k_i * G (device, SoA; written by zk_synth in a child process)
    and uniform scalars below 2^252 (numpy, seeded) for the sweep."""
    import torch
    d = os.path.join(args.workdir, "prims")
    os.makedirs(d, exist_ok=True)
    fx = os.path.join(d, f"g{group}_l{log_max}_s{seed}_x.bin")
    fy = os.path.join(d, f"g{group}_l{log_max}_s{seed}_y.bin")
    if not (os.path.exists(fx) and os.path.exists(fy)):
        run_synth("points", group, log_max, seed, fx, fy)
    px = torch.from_numpy(np.fromfile(fx, dtype=np.int64)).cuda()
    py = torch.from_numpy(np.fromfile(fy, dtype=np.int64)).cuda()
    return px, py, torch.from_numpy(seeded_fr(1 << log_max, seed).view(np.int64)).cuda()


def seeded_fr(n, seed, top_bits=60):
    """n x 4 u64 values below 2^(192 + top_bits) from a seeded numpy stream."""
    rng = np.random.default_rng(seed)
    s = rng.integers(0, 2**63, size=(n, 4), dtype=np.uint64) * np.uint64(2) + \
        rng.integers(0, 2, size=(n, 4), dtype=np.uint64)
    s[:, 3] &= np.uint64((1 << top_bits) - 1)
    return s


PRIM_REPS = 3  # timed calls per primitive size (0: one untimed call, for parity only)


def time_calls(fn, reps=None):
    import torch
    reps = PRIM_REPS if reps is None else min(reps, PRIM_REPS)
    fn()
    torch.cuda.synchronize()
    if reps == 0:
        return float("nan")
    ts = []
    for _ in range(reps):
        t = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        ts.append(time.perf_counter() - t)
    return float(np.median(ts))


def digest(t):
    """sha256 of a device buffer's bytes (compares large outputs across arms)."""
    import hashlib
    return hashlib.sha256(t.cpu().numpy().tobytes()).hexdigest()[:32]


def run_primitives(args, msm_fns, ntt_fn, hpoly_fn, imad_peak):
    """Config-1 sweep: G1 MSM at 2^18..2^24 and G2 MSM at 2^18, 2^20 (uniform
    scalars, points k_i G), Fr NTT and INTT at 2^16..2^24, and the H pipeline
    (three coset INTT / NTT pairs) at a few sizes.  msm_fns[g](px, py, sc, n)
    returns the result as hex; ntt_fn(buf, log_n, inverse) and
    hpoly_fn(a, b, c, log_n, h) run in place on device buffers.  Returns the
    timings and, under "outputs", every result (MSM points as hex, NTT / H
    outputs as sha256 digests) for the parity check between arms."""
    import torch
    out = {"g1_msm": {}, "g2_msm": {}, "ntt": {}, "intt": {}, "hpoly": {}}
    outputs = {"g1_msm": {}, "g2_msm": {}, "ntt": {}, "intt": {}, "hpoly": {}}
    peak_hbm, hbm_src = hbm_peak()
    for g, logs in ((1, [int(x) for x in args.prim_g1.split(",") if x]),
                    (2, [int(x) for x in args.prim_g2.split(",") if x])):
        if not logs:
            continue
        px, py, sc = prim_inputs(args, g, max(logs), 40 + g)
        for lg in logs:
            n = 1 << lg
            res = {}
            t = time_calls(lambda: res.__setitem__("r", msm_fns[g](px, py, sc, n)))
            per_point = FP_MULTS_PER_POINT["accum_g1" if g == 1 else "accum_g2"]
            r = {"ms": t * 1e3, "points_per_s": n / t}
            if imad_peak:
                r["imad_frac"] = n * per_point * IMAD_PER_FP_MULT / t / 1e12 / imad_peak
            out[f"g{g}_msm"][f"2^{lg}"] = r
            outputs[f"g{g}_msm"][f"2^{lg}"] = res["r"]
        del px, py, sc
        torch.cuda.empty_cache()
    for lg in [int(x) for x in args.prim_ntt.split(",") if x]:
        n = 1 << lg
        src = torch.from_numpy(seeded_fr(n, 500 + lg, 58).view(np.int64)).cuda()
        for inverse, key in ((False, "ntt"), (True, "intt")):
            buf = src.clone()
            t = time_calls(lambda: ntt_fn(buf, lg, inverse), reps=3)
            # parity: one transform of the seeded input
            buf.copy_(src)
            ntt_fn(buf, lg, inverse)
            torch.cuda.synchronize()
            outputs[key][f"2^{lg}"] = digest(buf)
            r = {"ms": t * 1e3, "gb_per_s": 64 * n / t / 1e9, "hbm_frac": 64 * n / t / 1e9 / peak_hbm}
            if imad_peak:  # one twiddle product per butterfly: (n / 2) log2 n products
                r["imad_frac"] = (n // 2) * lg * IMAD_PER_FP_MULT / t / 1e12 / imad_peak
            out[key][f"2^{lg}"] = r
            del buf
        del src
    for lg in [int(x) for x in args.prim_hpoly.split(",") if x]:
        if hpoly_fn is None:
            break
        n = 1 << lg
        a0 = torch.from_numpy(seeded_fr(n, 700 + lg, 58).view(np.int64)).cuda()
        b0 = torch.from_numpy(seeded_fr(n, 800 + lg, 58).view(np.int64)).cuda()
        a, b = a0.clone(), b0.clone()
        c, h = torch.empty_like(a0), torch.empty_like(a0)

        def once():
            a.copy_(a0)
            b.copy_(b0)
            hpoly_fn(a, b, c, lg, h)
        t = time_calls(once)
        outputs["hpoly"][f"2^{lg}"] = digest(h)
        # 3 INTT + 3 NTT (64 B per element each) + pointwise / coset / h passes
        out["hpoly"][f"2^{lg}"] = {"ms": t * 1e3, "elements_per_s": n / t,
                                   "transforms": "3 coset INTT/NTT pairs + glue"}
        del a0, b0, a, b, c, h
        torch.cuda.empty_cache()
    out["conventions"] = (f"MSM work {FP_MULTS_PER_POINT['accum_g1']:.0f} (G1) / "
                          f"{FP_MULTS_PER_POINT['accum_g2']:.0f} (G2) Fp products per point x "
                          f"{IMAD_PER_FP_MULT:.0f} IMAD-class ops against the measured IMAD "
                          f"probe; NTT bytes 64 per element against HBM {peak_hbm:.0f} GB/s "
                          f"({hbm_src}) and (n/2) log2 n products against the IMAD probe; "
                          "wall time of the API call, inputs resident (the H pipeline call "
                          "includes copying its two inputs back in)")
    out["outputs"] = outputs
    return out


def mine_primitives(args, ctx, L, imad_peak):
    from zyklop_b200 import api
    from zyklop_b200._lib import check
    res = np.zeros(16, np.uint64)
    inf = ctypes.c_int()

    def msm(fn, width):
        def call(px, py, sc, n):
            check(fn(ctx, api.ptr(px), api.ptr(py), api.ptr(sc), n,
                     res.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), ctypes.byref(inf)))
            return res[:width].tobytes().hex()
        return call

    def ntt(buf, lg, inverse):
        check(L.zk_ntt(ctx, api.ptr(buf), lg, 1 if inverse else 0))

    def hpoly(a, b, c, lg, h):
        check(L.zk_hpoly(ctx, api.ptr(a), api.ptr(b), lg, api.ptr(h)))

    out = run_primitives(args, {1: msm(L.zk_msm_g1, 8), 2: msm(L.zk_msm_g2, 16)}, ntt, hpoly,
                         imad_peak)
    out["calls"] = ("zk_msm_g1 / zk_msm_g2 (windowed, autotuned where tuned), zk_ntt (forward and "
                    "inverse), zk_hpoly")
    return out


def cpu_msm_baseline(lg=18):
    """The oracle's G1 MSM (C, OpenMP, all host threads) on 2^lg points k_i G
    (made on the GPU) with uniform scalars."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import _oracle
    from zyklop_b200 import api
    orc = _oracle.load()
    rng = np.random.default_rng(7)
    n = 1 << lg
    k = rng.integers(0, 2**63, size=(n, 4), dtype=np.uint64)
    k[:, 3] &= np.uint64((1 << 60) - 1)
    px, py = api.mul_generator(1, k)
    s = rng.integers(0, 2**63, size=(n, 4), dtype=np.uint64)
    s[:, 3] &= np.uint64((1 << 60) - 1)
    threads = os.cpu_count() or 1
    t = time.perf_counter()
    orc.msm_g1(px, py, s, threads=threads)
    t = time.perf_counter() - t
    return {"value": n / t, "unit": "points/s", "cores": threads, "kind": "port",
            "sample": f"one 2^{lg}-point G1 MSM by the CPU oracle (C, OpenMP; {t:.2f} s)"}


# -------------------------------------------------------------- autotuning
def autotune_sizes(args, api, ctx, logs, witness_dist, max_table_bytes=16 << 30, table_upto=21):
    """Fixed-base table window bits and MSM settings for circuits of 2^lg
    constraints: witness MSMs with the witness distribution, H with uniform
    scalars.  Table sizes are searched up to 2^table_upto points (larger
    ones keep the default window bits).  Returns the tuned entries."""
    if args.no_autotune:
        return "defaults"
    from zyklop_b200.api import table_c_default
    for lg in logs:
        for g in (1, 2):
            if lg <= table_upto:
                tc = api.autotune_table_c(g, lg, witness_dist, max_table_bytes=max_table_bytes,
                                          ctx=ctx)["table_c"]
            else:
                tc = table_c_default(lg)
            api.autotune_msm(g, lg, witness_dist, fixed_c=tc, ctx=ctx)
            if g == 1 and witness_dist != api.UNIFORM:
                api.autotune_msm(g, lg, api.UNIFORM, fixed_c=tc, ctx=ctx)
    return api.tune_export(ctx=ctx).strip().splitlines()


# --------------------------------------------------------------- batched
def pct(xs, q):
    return float(np.percentile(np.asarray(xs, dtype=np.float64), q)) if len(xs) else None


def config3_sizes(n_circuits=8, seed=3):
    """Circuit sizes (log2) of the batched workload: log-uniform in
    [2^14, 2^20] with both ends present (the first two circuits are 2^14 and
    2^20, the others drawn)."""
    rng = np.random.default_rng(seed)
    return [14, 20] + [int(round(x)) for x in rng.uniform(14, 20, n_circuits - 2)]


def run_batched(args, dist, ctx, L, logs=None, n_proofs=None, seed=3, label="config3"):
    """Independent proofs over seeded circuits (circom-like witnesses, 1-4
    nonzeros per row), all circuits resident with fixed-base tables:
    zk_prove_batch (in-flight pipelines with CUDA-graph replay, and fused
    groups over multi-instance MSM chains) against the same proofs one at a
    time through zk_prove, and through the one-shot file call.  Default:
    config 3, 64 proofs over 8 circuits of log-uniform size in [2^14, 2^20]."""
    import torch
    from zyklop_b200 import api
    from zyklop_b200._lib import check
    rng = np.random.default_rng(seed)
    logs = logs or config3_sizes()
    n_proofs = n_proofs or args.batch_proofs
    jobs = [int(j) for j in rng.integers(0, len(logs), n_proofs)]
    files = [synth_cached(args, dist, lg, "circom", 100 + k) for k, lg in enumerate(logs)]
    t_tune = time.perf_counter()
    tuned = autotune_sizes(args, api, ctx, sorted(set(logs)), api.SKEWED)
    t_tune = time.perf_counter() - t_tune
    circuits = [api.Circuit(z, ctx=ctx) for z, _ in files]
    wits = [api.read_wtns(w) for _, w in files]
    for c, w in zip(circuits, wits):
        c.prove(w)  # detects the witness distribution (keys the tuned settings)
        c.precompute(0, 0)
    stream = torch.cuda.current_stream()
    proof = np.zeros(32, np.uint64)
    pp = proof.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))

    def plain_once():
        lat, out = [], []
        for j in jobs:
            t = time.perf_counter()
            check(L.zk_prove(circuits[j].handle, wits[j].ctypes.data_as(ctypes.c_void_p),
                             wits[j].shape[0], None, None, pp))
            lat.append((time.perf_counter() - t) * 1e3)
            out.append(proof.copy())
        return lat, out

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return r, e0.elapsed_time(e1)

    plain_once()  # warm-up: workspaces sized, tables resident
    (lat, plain_proofs), plain_ms = timed(plain_once)
    run = lambda: api.prove_batch([circuits[j] for j in jobs], [wits[j] for j in jobs],
                                  inflight=args.batch_inflight, ctx=ctx)
    modes = {}
    # in-flight pipelines with CUDA-graph replay
    api.set_batch_mode(api.BATCH_INFLIGHT, ctx=ctx)
    api.set_graphs(True, ctx=ctx)
    run()  # warm-up: graph capture per (workspace, circuit)
    proofs_inflight, modes["inflight"] = timed(run)
    api.set_graphs(False, ctx=ctx)
    # fused groups (multi-instance MSM chains, one persistent H launch per
    # group), enqueued directly and replayed from captured group graphs
    api.set_batch_mode(api.BATCH_FUSED, args.batch_group, ctx=ctx)
    run()  # warm-up: both group workspaces sized
    proofs_fused, modes["fused"] = timed(run)
    api.set_graphs(True, ctx=ctx)
    run()  # warm-up: one graph captured per group
    proofs_fused_g, modes["fused_graphs"] = timed(run)
    api.set_graphs(False, ctx=ctx)
    api.set_batch_mode(api.BATCH_AUTO, ctx=ctx)
    for got in (proofs_inflight, proofs_fused, proofs_fused_g):
        assert all(np.array_equal(a, b) for a, b in zip(plain_proofs, got)), \
            "batched proofs differ from one-at-a-time proofs"
    best = min(modes, key=modes.get)
    batch_ms = modes[best]

    def files_once():
        for j in jobs:
            check(L.zk_groth16_prove_files(ctx, files[j][0].encode(), files[j][1].encode(), pp))
    _, files_ms = timed(files_once)
    for c in circuits:
        c.close()
    n = len(jobs)
    return {
        "workload": f"{label}: {n} proofs, {len(logs)} circuits of 2^{min(logs)}..2^{max(logs)} "
                    f"constraints (sizes {sorted(logs)}), circom-like witnesses",
        "batched_proofs_per_s": n / (batch_ms / 1e3),
        "plain_proofs_per_s": n / (plain_ms / 1e3),
        "speedup_vs_plain": plain_ms / batch_ms,
        "plain_files_proofs_per_s": n / (files_ms / 1e3),
        "speedup_vs_plain_files": files_ms / batch_ms,
        "plain_latency_ms": {"p50": pct(lat, 50), "p99": pct(lat, 99)},
        "batched_call": f"zk_prove_batch, {best.replace('_', ' with ')} mode",
        "batched_modes_proofs_per_s": {
            f"inflight ({args.batch_inflight} in flight, CUDA graphs)": n / (modes["inflight"] / 1e3),
            f"fused (groups of {args.batch_group})": n / (modes["fused"] / 1e3),
            f"fused (groups of {args.batch_group}, CUDA graphs)": n / (modes["fused_graphs"] / 1e3)},
        "autotuned": tuned, "autotune_s": round(t_tune, 1),
        "plain_call": "zk_prove one at a time (same resident circuits and tables)",
        "plain_files_call": "zk_groth16_prove_files one at a time (zkey loaded per proof, "
                            "like the reference's groth16Prove)",
        "bit_exact": True,
    }


# --------------------------------------------------------------- serving
def run_serving(args, dist, ctx, L):
    """Seeded Poisson request stream over 4 resident circuits of 2^16, 2^19,
    2^21 and 2^23 constraints (mixed 50/25/15/10) through the continuous-
    batching server (zk_server_*): latency from submit to proof, sustained
    proofs/s.  The offered rate is first the configured one (above capacity:
    the queue grows and what is still queued at the end is dropped), then 80%
    of the sustained rate measured there."""
    import queue as _queue
    from zyklop_b200 import api
    from zyklop_b200 import ZkError
    logs = [int(x) for x in args.serve_logs.split(",")]
    mix = [0.5, 0.25, 0.15, 0.10]
    files = [synth_cached(args, dist, lg, "circom", 200 + k) for k, lg in enumerate(logs)]
    t_tune = time.perf_counter()
    tuned = autotune_sizes(args, api, ctx, logs, api.SKEWED)
    t_tune = time.perf_counter() - t_tune
    circuits = [api.Circuit(z, ctx=ctx) for z, _ in files]
    wits = [api.read_wtns(w) for _, w in files]
    t = time.perf_counter()
    for c, w in zip(circuits, wits):
        c.prove(w)  # detects the witness distribution (keys the tuned settings)
        c.precompute(0, 0)
    t_pre = time.perf_counter() - t
    alone = [c.prove(w) for c, w in zip(circuits, wits)]  # the reference answer per circuit

    def leg(rate, seconds, seed):
        rng = np.random.default_rng(seed)
        srv = api.Server(max_inflight=args.serve_inflight, ctx=ctx)
        tq = _queue.Queue()
        lat, done, bad, dropped = [], [0], [0], [0]

        def waiter():
            while True:
                item = tq.get()
                if item is None:
                    return
                tk, k = item
                try:
                    p, ms = srv.wait(tk)
                    lat.append((k, ms))
                    done[0] += 1
                    if not np.array_equal(p, alone[k]):
                        bad[0] += 1
                except ZkError as e:
                    if e.code == 10:
                        dropped[0] += 1
                    else:
                        raise

        th = threading.Thread(target=waiter)
        th.start()
        t0 = time.perf_counter()
        at, sent = 0.0, 0
        while True:
            at += rng.exponential(1.0 / rate)
            if at >= seconds:
                break
            k = int(rng.choice(4, p=mix))
            while time.perf_counter() - t0 < at:
                time.sleep(0.0002)
            tq.put((srv.submit(circuits[k], wits[k]), k))
            sent += 1
        window = time.perf_counter() - t0
        srv.cancel_queued()
        tq.put(None)
        th.join()
        st = srv.stats()
        srv.close()
        return {"offered_req_per_s": rate, "seconds": round(window, 2), "submitted": sent,
                "completed": done[0], "dropped_unstarted": dropped[0],
                "sustained_proofs_per_s": done[0] / (time.perf_counter() - t0),
                "latency_ms": {"p50": pct([m for _, m in lat], 50),
                               "p99": pct([m for _, m in lat], 99)},
                "latency_ms_by_size": {
                    f"2^{logs[q]}": {"n": sum(1 for k, _ in lat if k == q),
                                     "p50": pct([m for k, m in lat if k == q], 50),
                                     "p99": pct([m for k, m in lat if k == q], 99)}
                    for q in range(4)},
                "peak_inflight": st["peak_inflight"], "admission_waits": st["admission_waits"],
                "mismatches": bad[0]}

    leg(min(args.serve_rate, 50.0), 2.0, 7)  # warm-up: workspaces grown
    over = leg(args.serve_rate, args.serve_seconds, 11)
    fair = leg(0.8 * over["sustained_proofs_per_s"], args.serve_seconds_fair, 13)
    for c in circuits:
        c.close()
    assert over["mismatches"] == 0 and fair["mismatches"] == 0, "served proof differs"
    return {"workload": f"Poisson requests over circuits 2^{logs[0]}/2^{logs[1]}/2^{logs[2]}/"
                        f"2^{logs[3]} mixed 50/25/15/10, circom-like witnesses, resident CRS "
                        f"with fixed-base tables (built in {t_pre:.1f} s)",
            "server": f"zk_server, up to {args.serve_inflight} proofs in flight, "
                      "admission by free device memory, smallest circuit first with aging",
            "autotuned": tuned, "autotune_s": round(t_tune, 1),
            "at_offered_rate": over, "at_80pct_of_sustained": fair, "bit_exact": True}


# ------------------------------------------------------------- reference
def reference_prove_lib():
    lib_path = os.path.join(ROOT, "oracle", "_ref", "libzkref_prove.so")
    if not os.path.exists(lib_path):
        return None
    L = ctypes.CDLL(lib_path)
    L.zkref_prove_files.argtypes = [ctypes.c_char_p, ctypes.c_char_p,
                                    ctypes.POINTER(ctypes.c_uint64)]
    return L


def reference_proofs(L, z, w, steps, warmup, stream):
    """groth16Prove of the reference build on (z, w): `warmup` untimed and
    `steps` timed proofs (CUDA events on the current stream around host
    calls that synchronize).  Returns (ms, proof)."""
    import torch
    proof = np.zeros(32, np.uint64)
    pp = proof.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
    with silenced():
        for _ in range(max(warmup, 1 if steps == 0 else 0)):
            L.zkref_prove_files(z.encode(), w.encode(), pp)
    torch.cuda.synchronize()
    if steps == 0:
        return None, proof
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with silenced():
        start.record(stream)
        for _ in range(steps):
            L.zkref_prove_files(z.encode(), w.encode(), pp)
        end.record(stream)
        torch.cuda.synchronize()
    return start.elapsed_time(end), proof


def ref_outputs_path(args):
    return os.path.join(args.workdir, "ref_outputs.json")


def run_reference(args, dist):
    """The reference arm: its groth16Prove on the config-0 circuit (timed
    steps), on the config-2 circuit (a few timed steps), and its primitive
    sweep; every result goes to ref_outputs.json in the work directory."""
    import torch
    torch.cuda.set_device(dist.local)
    L = reference_prove_lib()
    if L is None:
        return {"impl": "reference", "unavailable":
                "reference sm_100a build missing (oracle/_ref; make -C oracle/refbuild)"}
    z, w = circuit_files(args, dist)
    stream = torch.cuda.current_stream()
    record = {"workdir_inputs": {"config0": [z, w]}}
    if args.parity_only:
        _, proof = reference_proofs(L, z, w, 0, 1, stream)
        record["proof_2^%d" % args.log_domain] = proof.tobytes().hex()
        if args.config2_log:
            z2, w2 = synth_cached(args, dist, args.config2_log, "circom", 2)
            _, p2 = reference_proofs(L, z2, w2, 0, 1, stream)
            record["proof_2^%d" % args.config2_log] = p2.tobytes().hex()
        global PRIM_REPS
        PRIM_REPS = 0
        prims = reference_primitives(args)
        record["primitives"] = prims["outputs"] if prims else {}
        json.dump(record, open(ref_outputs_path(args), "w"))
        return None
    clocks = ClockSampler(dist.local)
    dist.barrier()
    ms, proof = reference_proofs(L, z, w, args.steps, args.warmup, stream)
    dist.barrier()
    clk = clocks.stop()
    ms = dist.max(ms)
    value = args.gpus * args.steps / (ms / 1e3)
    record["proof_2^%d" % args.log_domain] = proof.tobytes().hex()
    record["value"] = value
    config2 = None
    if args.config2_log:
        z2, w2 = synth_cached(args, dist, args.config2_log, "circom", 2)
        k2 = max(1, min(args.steps, 3))
        ms2, p2 = reference_proofs(L, z2, w2, k2, 1, stream)
        record["proof_2^%d" % args.config2_log] = p2.tobytes().hex()
        config2 = {"workload": f"groth16_prove_2^{args.config2_log}_circom",
                   "value": k2 / (ms2 / 1e3), "unit": UNIT, "steps": k2,
                   "ms_per_step": ms2 / k2,
                   "call": "groth16Prove (zkey + wtns files -> proof), every step a full proof"}
        record["config2_value"] = config2["value"]
    prims = reference_primitives(args)
    if prims:
        record["primitives"] = prims["outputs"]
    json.dump(record, open(ref_outputs_path(args), "w"))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64 limbs (exact Fr/Fp arithmetic)",
        "data": "synthetic (seeded circuit, CRS and witness)",
        "config": config(args, wtns_n_vars(w), 1 << args.log_domain),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 8, "kind": "reference",
                         "sample": "the reference's own sm_100a build (groth16Prove from "
                                   "zkey/wtns files; GPU kernels + 8 OpenMP host threads), "
                                   "every step a full proof"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "clocks": clk,
        "config2": config2,
        "primitives": prims,
        "inputs": "written by zyklop_b200/bin/zk_synth in a child process; this process loads "
                  "only the reference build (oracle/_ref)",
    }
    return line


def reference_outputs(args):
    """The reference build's results on this run's inputs: ref_outputs.json
    as the reference arm left it in the work directory, else made now by the
    reference build in a child process (bench.py --impl reference
    --parity-only).  Returns (outputs, source)."""
    path = ref_outputs_path(args)
    want = ["proof_2^%d" % args.log_domain] + (
        ["proof_2^%d" % args.config2_log] if args.config2_log else [])
    if os.path.exists(path):
        rec = json.load(open(path))
        if all(k in rec for k in want):
            return rec, "the reference arm's outputs (ref_outputs.json, same inputs)"
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--parity-only",
           "--workdir", args.workdir, "--log-domain", str(args.log_domain),
           "--config2-log", str(args.config2_log), "--prim-g1", args.prim_g1,
           "--prim-g2", args.prim_g2, "--prim-ntt", args.prim_ntt,
           "--prim-hpoly", args.prim_hpoly]
    env = dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    r = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=1200)
    if r.returncode != 0 or not os.path.exists(path):
        return None, "reference build failed: " + r.stderr.strip()[-300:]
    return json.load(open(path)), "the reference build run in a child process (--parity-only)"


def parity_report(mine, ref, source):
    """Bit-equality of this arm's results with the reference build's, per
    item; None where the reference has no result for it."""
    if ref is None:
        return {"checked": False, "source": source}
    out = {"source": source}
    ok = True
    for k, v in mine.items():
        if isinstance(v, dict):
            sub = {}
            for kk, vv in v.items():
                theirs = ref.get("primitives", {}).get(k, {}).get(kk)
                sub[kk] = None if theirs is None else theirs == vv
                ok = ok and sub[kk] is not False
            out[k] = sub
        else:
            theirs = ref.get(k)
            out[k] = None if theirs is None else theirs == v
            ok = ok and out[k] is not False
    out["all_equal"] = ok
    return out


def reference_primitives(args):
    """The same config-1 sweep through the reference build's own primitives
    (msm_g1, msm_g2_device, ntt, computeHPoly) on device buffers."""
    path = os.path.join(ROOT, "oracle", "_ref", "libzkref_prims.so")
    ipath = os.path.join(ROOT, "oracle", "_ref", "libzkref_inter.so")
    if not os.path.exists(path) or not (args.prim_g1 or args.prim_g2 or args.prim_ntt):
        return None
    u64p = ctypes.POINTER(ctypes.c_uint64)
    L = ctypes.CDLL(path)
    for name in ("zkref_msm_g1_device", "zkref_msm_g2_device"):
        fn = getattr(L, name)
        fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, u64p]
        fn.restype = ctypes.c_int
    L.zkref_ntt_device.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    L.zkref_ntt_device.restype = ctypes.c_int
    hp = None
    if os.path.exists(ipath):
        IL = ctypes.CDLL(ipath)
        if hasattr(IL, "zkref_hpoly_device"):
            hp = IL.zkref_hpoly_device
            hp.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int, ctypes.c_void_p]
            hp.restype = ctypes.c_int
    out = np.zeros(16, np.uint64)

    def msm(fn, width):
        def call(px, py, sc, n):
            with silenced():
                fn(ctypes.c_void_p(px.data_ptr()), ctypes.c_void_p(py.data_ptr()),
                   ctypes.c_void_p(sc.data_ptr()), n, out.ctypes.data_as(u64p))
            return out[:width].tobytes().hex()
        return call

    def ntt(buf, lg, inverse):
        with silenced():
            L.zkref_ntt_device(ctypes.c_void_p(buf.data_ptr()), lg, 1 if inverse else 0)

    def hpoly(a, b, c, lg, h):
        with silenced():
            hp(*[ctypes.c_void_p(t.data_ptr()) for t in (a, b, c)], lg, ctypes.c_void_p(h.data_ptr()))

    r = run_primitives(args, {1: msm(L.zkref_msm_g1_device, 8), 2: msm(L.zkref_msm_g2_device, 16)},
                       ntt, hpoly if hp else None, None)
    r["calls"] = ("the reference's msm_g1, msm_g2_device, ntt (oracle/_ref/libzkref_prims.so) and "
                  "computeHPoly (oracle/_ref/libzkref_inter.so); each call includes the "
                  "reference's own nttPrepare / nttDestroy")
    return r


def lib_handle():
    from zyklop_b200._lib import lib
    return lib()


def main():
    args = parse_args()
    if args.impl == "reference":
        # rank 0 alone runs the reference; other ranks exit without work and
        # no process group is formed (so nothing waits on them)
        if int(os.environ.get("RANK", "0")) != 0:
            return
        os.environ["WORLD_SIZE"] = "1"
        dist = Dist()
        line = run_reference(args, dist)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    dist = Dist()
    try:
        line, files, ctx = run_mine(args, dist)
        mine_out = {"proof_2^%d" % args.log_domain: line.pop("_proof")}
        if dist.world == 1 and args.config2_log:
            c2 = run_config2(args, dist, ctx, lib_handle())
            mine_out["proof_2^%d" % args.config2_log] = c2.pop("_proof")
            line["config2"] = c2
        if dist.world == 1 and args.batch_proofs > 0:
            line["batched"] = run_batched(args, dist, ctx, lib_handle())
            # the same comparison at 2^20 alone: 16 proofs over two 2^20 circuits
            line["batched"]["at_2^20"] = run_batched(args, dist, ctx, lib_handle(), logs=[20, 20],
                                                     n_proofs=16, seed=5, label="2^20 only")
        if dist.world == 1 and args.serve_seconds > 0:
            line["serving"] = run_serving(args, dist, ctx, lib_handle())
        if dist.world == 1 and (args.prim_g1 or args.prim_g2 or args.prim_ntt):
            line["primitives"] = mine_primitives(args, ctx, lib_handle(),
                                                 line["roofline"]["peak"])
            mine_out.update(line["primitives"].pop("outputs"))
            if not args.no_cpu_baseline:
                cb = cpu_msm_baseline()
                if cb:
                    line["primitives"]["cpu_baseline_g1_msm"] = cb
        lib_handle().zk_ctx_destroy(ctx)
        if dist.rank == 0 and args.gpus == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(*files)
        if dist.rank == 0 and dist.world == 1 and not args.no_parity:
            ref, source = reference_outputs(args)
            line["parity_vs_reference"] = parity_report(mine_out, ref, source)
            if ref and "config2" in line and "config2_value" in ref:
                line["config2"]["reference_value"] = ref["config2_value"]
        if dist.rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
