"""The C++ drop-in boundary (include/groth16.h over libzyklop_b200.so).

CPU: a caller written against the reference's C++ API (tests/cxx/
groth16_caller.cpp, the flow of the reference CLI src/main.cu:115-171)
compiles against include/groth16.h and links to the library, and the API
structs have the reference's sizes and field offsets (include/groth16.cuh:
69-98; checked against the reference header itself when its sources are
present).  GPU: the same program proves a circuit, and its proof.json and
calldata equal the reference build's.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CALLER = os.path.join(ROOT, "tests", "cxx", "groth16_caller.cpp")
LIBDIR = os.path.join(ROOT, "zyklop_b200")
REFERENCE = os.environ.get("ZK_REFERENCE_DIR", "/root/reference")

LAYOUT_PROBE = r"""
#include <cstddef>
#include <cstdio>
#include HEADER
int main() {
  std::printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(Groth16Proof),
              offsetof(Groth16Proof, pi_B), offsetof(Groth16Proof, pi_C),
              sizeof(Groth16ZkeyHeader), offsetof(Groth16ZkeyHeader, log_domain),
              offsetof(Groth16ZkeyHeader, prime), sizeof(Groth16CoefEntry),
              offsetof(Groth16CoefEntry, constraint), offsetof(Groth16CoefEntry, signal),
              offsetof(Groth16CoefEntry, value), alignof(Groth16CoefEntry));
  return 0;
}
"""


def build_caller(out_dir):
    exe = os.path.join(out_dir, "groth16_caller")
    subprocess.run(["g++", "-O1", "-std=c++17", "-Wall", "-I", os.path.join(ROOT, "include"),
                    CALLER, "-o", exe, "-L", LIBDIR, "-lzyklop_b200",
                    f"-Wl,-rpath,{LIBDIR}"], check=True, capture_output=True, text=True)
    return exe


def layout(out_dir, compiler, header, extra=()):
    src = os.path.join(out_dir, f"probe_{compiler}.cpp")
    exe = os.path.join(out_dir, f"probe_{compiler}")
    open(src, "w").write(LAYOUT_PROBE.replace("HEADER", f'"{header}"'))
    cmd = [compiler, "-std=c++17", *extra, src, "-o", exe]
    if compiler == "nvcc":
        cmd = [compiler, "-std=c++17", "-x", "cu", *extra, src, "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()


def test_caller_compiles_links_and_runs_without_arguments(tmp_path):
    if not os.path.exists(os.path.join(LIBDIR, "libzyklop_b200.so")):
        pytest.skip("library not built")
    exe = build_caller(str(tmp_path))
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "Usage" in r.stderr
    assert r.stdout.startswith("sizeof Groth16Proof 256 Groth16ZkeyHeader 56 Groth16CoefEntry 48")


def test_struct_layouts_match_reference_header(tmp_path):
    mine = layout(str(tmp_path), "g++", os.path.join(ROOT, "include", "groth16.h"))
    # 256-byte proof; header fields up to the prime; a 48-byte coefficient entry
    assert mine == ["256", "64", "192", "56", "16", "24", "48", "4", "8", "16", "8"]
    ref_header = os.path.join(REFERENCE, "include", "groth16.cuh")
    if not os.path.exists(ref_header):
        pytest.skip("reference sources not present")
    theirs = layout(str(tmp_path), "nvcc", ref_header,
                    ["-I", os.path.join(REFERENCE, "include")])
    assert mine == theirs


@pytest.mark.gpu
def test_caller_output_matches_reference(tmp_path):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from zyklop_b200 import api
    import _ref
    z, w = tmp_path / "c.zkey", tmp_path / "c.wtns"
    api.synth_circuit(z, w, 12, n_public=8, n_private_inputs=8, nnz=(1, 4), witness="circom",
                      seed=31)
    exe = build_caller(str(tmp_path))
    r = subprocess.run([exe, str(z), str(w), str(tmp_path / "p.json"), str(tmp_path / "cd.hex")],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "header 4096 " in r.stdout
    proof = api.prove_files(z, w)
    calldata = bytes.fromhex(open(tmp_path / "cd.hex").read().strip())
    assert calldata == bytes(api.proof_to_calldata(proof))
    assert open(tmp_path / "p.json").read() == api.proof_to_json(proof) + "\n"
    L = _ref.prove_lib()
    if L is None:
        pytest.skip("reference sm_100a build (oracle/_ref) not present")
    theirs = np.zeros(32, np.uint64)
    u64p = ctypes.POINTER(ctypes.c_uint64)
    assert L.zkref_prove_files(str(z).encode(), str(w).encode(), theirs.ctypes.data_as(u64p)) == 0
    assert np.array_equal(proof, theirs)
    buf = ctypes.create_string_buffer(4096)
    L.zkref_proof_json(theirs.ctypes.data_as(u64p), buf, 4096)
    assert open(tmp_path / "p.json").read() == buf.value.decode() + "\n"
    cd = (ctypes.c_uint8 * 256)()
    L.zkref_proof_calldata(theirs.ctypes.data_as(u64p), cd, 256)
    assert calldata == bytes(cd)
