"""bench.py's multi-rank host logic on CPU: world_size 2 over gloo.

Each rank proves independently (replicas), so the only cross-rank steps are
the barriers around the timed region and the max over ranks of the measured
time; the reference arm runs on rank 0 alone and the other ranks exit
without work."""
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import os, sys
sys.path.insert(0, os.environ["ZK_ROOT"])
import bench
d = bench.Dist(backend="gloo")
assert d.world == 2 and d.pg is not None and not d.cuda
d.barrier()
m = d.max(10.0 + 5.0 * d.rank)
assert m == 15.0, m
d.barrier()
d.close()
print("rank", d.rank, "ok", flush=True)
"""


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_barrier_and_max_over_gloo():
    port = str(free_port())
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2",
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=port, ZK_ROOT=ROOT,
                   CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True))
    outs = [p.communicate(timeout=240)[0] for p in procs]
    for rank, (p, out) in enumerate(zip(procs, outs)):
        assert p.returncode == 0, out
        assert f"rank {rank} ok" in out


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
               MASTER_PORT=str(free_port()), CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2"], env=env, capture_output=True, text=True, timeout=240)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
